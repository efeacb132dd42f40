// radio_kernels.cuh — launch-side declarations shared by the host library.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "radio_device.cuh"

struct c8r_lepton_transport_record;
struct c8r_counters;
struct c8r_track_columns;

namespace c8r {

// Device-side counters of one event (the layout of RadioCounters).
struct alignas(8) DeviceCounters {
  unsigned long long coreas_contributions;
  unsigned long long zhs_contributions;
  unsigned long long zhs_subtracks;
  unsigned long long valid_tracks;
  unsigned long long fixed_point_overflows;
  double weighted_segment_count;
  double track_length_m;
  double weighted_track_length_m;
  double electron_weighted_track_length_m;
  double positron_weighted_track_length_m;
  double signed_charge_weighted_track_length_m;
  double energy_weighted_track_length_gev_m;
  double maximum_segment_length_m;
  double weighted_direction_change_rad;
  double weighted_direction_change_squared_rad2;
  double weighted_beta_deficit_track_length_m;
  double weighted_time_residual_s;
  double maximum_direction_change_rad;
  double signed_charge_weighted_direction_change[3];
  double weighted_track_length_by_kinetic_energy_m[15];
};
static_assert(sizeof(DeviceCounters) == 288, "RadioCounters layout");

// One event of a projection launch: its tracks (SoA, `stride` doubles per
// row), observers, traces and counters.  Algorithm 0 = CoREAS field,
// algorithm 1 = ZHS potential.  Trace rows are [X | Y | Z] of total_bins each.
struct EventPlan {
  const double* tracks;
  uint64_t stride;
  const unsigned long long* valid_tracks;  // device: tracks written by ingest
  const ObserverCache* observers[2];
  uint32_t observer_count[2];
  unsigned long long* fixed[2];  // int64 fixed-point traces (deterministic)
  double* floating[2];           // FP64 traces (floating mode)
  uint64_t total_bins[2];
  Propagation propagation;
  DeviceCounters* counters;
  uint64_t first_item;           // work-list offset of this event (in its algorithm's list)
  uint32_t chunk_size;           // tracks per work item
  uint32_t chunks;
  uint32_t window;               // shared-memory bins per item (<= kernel window)
  uint64_t first_track;          // chunk c covers first_track + c * chunk_size onwards,
  uint64_t last_track;           // clipped to [.., last_track) and the valid tracks
  uint32_t precomputed;          // tracks carry their source terms (every observer shares
                                 // one destination row; see IngestTerms)
  uint32_t pad_;
};

// Source terms written at ingest: when every observer of an event shares one
// destination row (always in a homogeneous medium), each track record gets
// the propagation terms of its start, end and two midpoints for that row,
// and the windowed kernels read them instead of looking them up per pair.
struct IngestTerms {
  int32_t enabled;
  int32_t pad_;
  Propagation propagation;
  Destination destination;
};
// The destination row shared by all `count` observers, if they share one.
bool shared_destination(ObserverCache const* observers, std::size_t count, Destination& out);

// Persistent windowed launch over a work list of (event, chunk, algorithm,
// observer) items drawn from an atomic counter.  Passed as a __grid_constant__
// kernel parameter (no host-to-device copy; graph-capturable).
constexpr int kMaxEventsPerLaunch = 64;
// Pairs a batched launch takes beyond its first event (its two-pass ZHS
// storage stays near 8% of them).
constexpr uint64_t kMaxPairsPerLaunch = 4000000000ull;
constexpr int kPlanEntries = kMaxEventsPerLaunch + 1;  // + the short-chunk tail of the last event
constexpr int kWindowThreads = 640;  // upper bound (and default) of the windowed block size
// Where the first pass of a two-pass ZHS launch left a work item's deferred
// pairs: `count` entries from `begin` of CTA `cta`'s list; `redo` when the
// second pass projects the item in full (its window could not be shown free
// of overflow, its trace was longer than the window, or the CTA's list was
// full).
struct ItemState {
  uint32_t cta, begin, count, redo;
};

struct WorkPlan {
  EventPlan events[kPlanEntries];
  int32_t algorithm;        // 0: CoREAS items, 1: ZHS items
  uint32_t event_count;
  uint32_t window;          // shared-memory bins per CTA (max over events)
  uint64_t total_items;
  unsigned int* next_item;  // zeroed before each launch
  // Each CTA's list of the deferred pairs of its current item,
  // `deferred_stride` entries from deferred + blockIdx.x * deferred_stride
  // (at least the longest chunk of the plan; deferred_list_stride below).
  unsigned int* deferred;
  uint32_t deferred_stride;
  // Items run again with checked window adds (the unchecked run's bound did
  // not hold); counted when not null.
  unsigned long long* reruns;
  // Items the first pass of two handed to the second; counted when not null.
  unsigned long long* handbacks;
  // Two-pass ZHS (fixed point), when item_state is set: the first pass runs
  // the track loop alone and keeps each CTA's deferred pairs of all its items
  // in its list (`deferred`), the second drains them item by item and
  // projects in full the items the first handed back, with its own lists
  // (`drain_deferred`, deferred_stride entries a CTA) and work counter.
  // The drain needs more registers than the track loop, so the track loop
  // runs larger CTAs on its own (attach_deferred sets these).  The first
  // pass's lists hold `deferred_capacity` entries a CTA.
  ItemState* item_state;
  unsigned int* drain_deferred;
  unsigned int* drain_next_item;
  uint32_t deferred_capacity;
};

// A work item spans at most kMaxChunkTracks tracks: a deferred-list entry is
// the pair's track offset in the item (its low 30 bits) and two bits of the
// track loop's decision (CoREAS: the near-Cherenkov branch and its order).
constexpr uint32_t kMaxChunkTracks = 1u << 30;
constexpr unsigned kDeferredHintShift = 30;
constexpr unsigned kDeferredOffsetMask = (1u << kDeferredHintShift) - 1u;

// Entries per CTA of a launch's deferred lists: the plan's longest chunk.
inline uint32_t deferred_list_stride(WorkPlan const& plan) {
  uint32_t stride = 0;
  for (uint32_t e = 0; e < plan.event_count; ++e)
    if (plan.events[e].chunk_size > stride) stride = plan.events[e].chunk_size;
  return stride;
}

// Pairs a launch of `plan` covers at most (its items' chunks at full length).
inline uint64_t plan_pairs(WorkPlan const& plan) {
  uint64_t pairs = 0;
  for (uint32_t e = 0; e < plan.event_count; ++e) {
    EventPlan const& ev = plan.events[e];
    pairs += static_cast<uint64_t>(ev.chunks) * ev.chunk_size * ev.observer_count[plan.algorithm];
  }
  return pairs;
}

// First-pass list entries a CTA of a two-pass launch holds: the deferred
// pairs of all its items, sized for 8% of its share of the launch's pairs
// (ZHS defers 3% on the 1e7 x 160 workload) and at least one chunk; an item
// past the end is handed back to the second pass (correct, slower).
constexpr double kTwoPassDeferredShare = 0.08;
// Launches whose two-pass storage would pass 2^30 words (4 GiB) run one pass.
constexpr uint64_t kTwoPassMaxWords = 1ull << 30;

inline uint64_t pass1_capacity(WorkPlan const& plan, uint64_t ctas) {
  uint64_t const share = static_cast<uint64_t>(kTwoPassDeferredShare * static_cast<double>(plan_pairs(plan)) /
                                               static_cast<double>(ctas > 0 ? ctas : 1)) + 1;
  uint64_t const capacity = share > plan.deferred_stride ? share : plan.deferred_stride;
  return capacity < 0xffffffffull ? capacity : 0xffffffffull;
}

inline uint64_t two_pass_words(WorkPlan const& plan, uint64_t ctas) {
  return ctas * pass1_capacity(plan, ctas) + ctas * plan.deferred_stride +
         plan.total_items * (sizeof(ItemState) / sizeof(unsigned)) + 1;
}

// ZHS launches in fixed point run in two passes when their storage fits.
inline bool two_pass(WorkPlan const& plan, uint64_t ctas, bool fixed) {
  return fixed && plan.algorithm == 1 && two_pass_words(plan, ctas) <= kTwoPassMaxWords;
}

// 32-bit words of deferred-list storage a launch of `plan` (deferred_stride
// and total_items set) over `ctas` CTAs needs: its CTAs' lists, and for two
// passes the first pass's longer lists, the second pass's lists, the items'
// states and its work counter.
inline uint64_t deferred_words(WorkPlan const& plan, uint64_t ctas, bool fixed) {
  if (!two_pass(plan, ctas, fixed)) return ctas * plan.deferred_stride;
  return two_pass_words(plan, ctas);
}

// Points the plan's deferred-list storage into `words` (deferred_words of it).
inline void attach_deferred(WorkPlan& plan, unsigned* words, uint64_t ctas, bool fixed) {
  plan.deferred = words;
  plan.item_state = nullptr;
  plan.drain_deferred = nullptr;
  plan.drain_next_item = nullptr;
  plan.deferred_capacity = plan.deferred_stride;
  if (!two_pass(plan, ctas, fixed)) return;
  uint64_t const first = ctas * pass1_capacity(plan, ctas);
  plan.deferred_capacity = static_cast<uint32_t>(pass1_capacity(plan, ctas));
  plan.drain_deferred = words + first;
  plan.item_state = reinterpret_cast<ItemState*>(words + first + ctas * plan.deferred_stride);
  plan.drain_next_item = reinterpret_cast<unsigned*>(plan.item_state + plan.total_items);
}

// Appends the (chunk, observer) work items of `ev` for plan.algorithm to
// `plan` (first_item, event_count and total_items follow).  With `fine_tail`
// and a free event slot, the last chunks go in as a second entry of chunks a
// quarter as long (at least 8192 tracks), about two items for each of the
// `ctas` persistent CTAs: the launch then ends on short items instead of one
// CTA finishing a long item while the others wait.  Every track stays in
// exactly one item.  Returns the number of items appended.
inline uint64_t append_work(WorkPlan& plan, EventPlan ev, uint64_t ctas, bool fine_tail) {
  constexpr uint64_t kSplit = 4, kMinTailChunk = 8192;
  uint64_t const per = ev.observer_count[plan.algorithm];
  if (per == 0 || ev.chunks == 0 || plan.event_count >= kPlanEntries) return 0;
  uint64_t const big = ev.chunk_size;
  // whole track tiles, so that short items start on a tile as long ones do
  uint64_t const small = track_capacity((big + kSplit - 1) / kSplit > kMinTailChunk ? (big + kSplit - 1) / kSplit
                                                                                    : kMinTailChunk);
  uint64_t head = ev.chunks;
  if (fine_tail && plan.event_count + 2 <= kPlanEntries && small < big) {
    uint64_t const short_items = (2 * ctas + per - 1) / per;
    uint64_t const replaced = (short_items * small + big - 1) / big;  // long chunks they cover
    head = replaced >= ev.chunks ? 0 : ev.chunks - replaced;
  }
  uint64_t const before = plan.total_items;
  if (head > 0) {
    EventPlan e = ev;
    e.chunks = static_cast<uint32_t>(head);
    e.first_item = plan.total_items;
    plan.events[plan.event_count++] = e;
    plan.total_items += head * per;
  }
  if (head < ev.chunks) {
    uint64_t const stop = ev.first_track + ev.chunks * big;
    EventPlan e = ev;
    e.first_track = ev.first_track + head * big;
    e.last_track = stop < ev.last_track ? stop : ev.last_track;
    e.chunk_size = static_cast<uint32_t>(small);
    e.chunks = static_cast<uint32_t>(((ev.chunks - head) * big + small - 1) / small);
    e.first_item = plan.total_items;
    plan.events[plan.event_count++] = e;
    plan.total_items += static_cast<uint64_t>(e.chunks) * per;
  }
  return plan.total_items - before;
}

enum class Precision : int { kFP64 = 0, kMixed = 1 };

// Record ingest: LeptonTransportRecord AoS -> compacted SoA kinematics
// (make_radio_track_kinematics + record_track).  `slot` receives the number of
// valid tracks written.
cudaError_t launch_ingest(const c8r_lepton_transport_record* records, uint64_t count,
                          double* tracks, uint64_t stride, unsigned long long* slot,
                          DeviceCounters* counters, bool diagnostics, IngestTerms const& terms,
                          cudaStream_t stream);

// The same ingest from a structure-of-arrays view of the steps.
cudaError_t launch_ingest_columns(c8r_track_columns const& columns, uint64_t count, double* tracks,
                                  uint64_t stride, unsigned long long* slot, DeviceCounters* counters,
                                  bool diagnostics, IngestTerms const& terms, cudaStream_t stream);

// Direct pair kernel: one thread per (track, observer) pair, global atomics.
// The valid-track count is read on the device; `track_bound` (the record
// count) bounds the grid on the host.
cudaError_t launch_direct(EventPlan const& event, uint64_t track_bound, bool coreas, bool zhs,
                          bool fixed, Precision precision, cudaStream_t stream);

// The reference's large-batch tile shape: 256-thread CTAs over tiles of 8
// tracks x 32 observers staged in shared memory, one thread per pair, global
// atomics (RadioTileProjection, RadioAccumulator.inl:13-85).
cudaError_t launch_tiled(EventPlan const& event, uint64_t track_bound, bool coreas, bool zhs,
                         bool fixed, Precision precision, cudaStream_t stream);

// Persistent windowed kernel.  `ctas` persistent CTAs of `threads` threads.
// The plan needs plan.deferred with ctas * deferred_stride entries and
// deferred_stride >= deferred_list_stride(plan) (else cudaErrorInvalidValue).
cudaError_t launch_windowed(WorkPlan const& plan, bool fixed, Precision precision, int ctas,
                            int threads, cudaStream_t stream);
// Largest window (bins) that fits the opt-in shared memory of this device.
int windowed_max_bins(int device);
// Resident CTAs per SM of the windowed kernel for a window and block size.
int windowed_ctas_per_sm(int window, int threads, bool fixed, Precision precision);

// The precision study's kernel (precision_study.cu): one thread per pair,
// arrival-time arithmetic in FP64, compensated double-FP32 or FP32,
// amplitudes in FP32.
enum class TimeArithmetic : int { kDouble = 0, kDoubleFloat = 1, kFloat = 2 };
cudaError_t launch_study(EventPlan const& event, uint64_t track_bound, bool coreas, bool zhs,
                         bool fixed, TimeArithmetic arithmetic, cudaStream_t stream);

// Output step: decoded CoREAS fields, or ZHS fields -(A[i+1] - A[i]) fs,
// added into `out` (fixed traces when `fixed` is non-null, else `floating`).
cudaError_t launch_output(const long long* fixed, const double* floating, double* out, uint64_t total_bins,
                          const ObserverCache* observers, const double* factors, uint32_t observer_count,
                          uint64_t max_bins, bool differentiate, cudaStream_t stream);

// Fixed-point decode on the device: out[r*bins + i] = in[r*bins + i] * factor(observer).
cudaError_t launch_decode(const long long* fixed, double* out, uint64_t total_bins,
                          const uint64_t* observer_offsets, const double* factors,
                          uint32_t observer_count, uint64_t max_bins, cudaStream_t stream);

}  // namespace c8r
