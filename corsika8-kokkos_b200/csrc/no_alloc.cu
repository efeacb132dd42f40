// no_alloc.cu — c8r_accumulate_device_no_alloc: the record ingest and the
// windowed projection with every piece of device scratch (packed track
// kinematics, observer constants, refractivity table, the launches'
// deferred-pair lists, valid-track slot, work counter, fallback counters) in
// one file-scope static device array, so that a call allocates no device
// memory.
//
// Who needs it: a transport code that has handed the whole of HBM to its own
// pool (a Kokkos memory pool, a particle stack sized to the card) cannot get
// memory from cudaMalloc when it projects tracks, and a caller that drives
// several streams cannot afford cudaMalloc/cudaFree, which synchronise the
// device.  Such a caller owns its inputs and outputs and passes them in; the
// scratch lives in this library's module instead.
//
// The array costs kScratchBytes on every GPU that loads this library's module,
// held until the process exits.  Every call on a device shares it, and it
// keeps the last call's contents: each call clears what must start at zero
// (slot, work counter, fallback counters) and overwrites the rest before
// reading it.  Two calls that overlap on the GPU (different streams, or
// different host threads without ordering) race on the array: order them on
// one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/c8radio.h"
#include "host_setup.hpp"
#include "radio_kernels.cuh"

namespace c8r {
void set_global_error(char const* message);  // accumulator.cu
}

namespace {

using c8r::DeviceCounters;
using c8r::ObserverCache;

constexpr std::size_t kScratchBytes = C8R_NO_ALLOC_SCRATCH_BYTES;
constexpr std::size_t kMaxObservers = C8R_NO_ALLOC_MAX_OBSERVERS;
constexpr std::size_t kMaxTableEntries = C8R_NO_ALLOC_MAX_TABLE_ENTRIES;
constexpr std::size_t kTrackBytes = c8r::kTrackDoubles * sizeof(double);

// Scratch layout (byte offsets, each a multiple of 256).
constexpr std::size_t kCountersOffset = 0;
constexpr std::size_t kSlotOffset = 512;
constexpr std::size_t kNextItemOffset = 768;
constexpr std::size_t kTableOffset = 1024;
constexpr std::size_t kObserversOffset = kTableOffset + kMaxTableEntries * sizeof(double2);
// the launches' per-CTA deferred-pair lists (track offsets in the chunk)
constexpr std::size_t kDeferredOffset = kObserversOffset + kMaxObservers * sizeof(ObserverCache);
constexpr std::size_t kDeferredEntries = std::size_t(2) << 20;
constexpr std::size_t kTracksOffset = kDeferredOffset + kDeferredEntries * sizeof(unsigned);
// whole tiles of the track workspace layout (c8r::track_column)
constexpr std::size_t kTrackCapacity =
    (kScratchBytes - kTracksOffset) / kTrackBytes / c8r::kTrackTile * c8r::kTrackTile;
static_assert(sizeof(DeviceCounters) <= kSlotOffset - kCountersOffset, "scratch layout");
static_assert(kObserversOffset % 256 == 0 && kDeferredOffset % 256 == 0 && kTracksOffset % 256 == 0,
              "scratch alignment");
static_assert(kTrackCapacity >= 65536, "scratch too small for a useful track chunk");

constexpr int kMaxDevices = 64;

struct DeviceSetup {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of the array on this device
  int sms = 0;
  int max_window = 0;
};

std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

void check(cudaError_t err, char const* what) {
  if (err != cudaSuccess)
    throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(err));
}

}  // namespace

// The scratch itself.  In host code this name is only a stand-in for the
// symbol: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_no_alloc_scratch[kScratchBytes];

namespace {

// Once per device, with that device current: the array's device address
// (this loads the module on the device if nothing has yet), SM count and the
// largest shared-memory window of the windowed kernel.
DeviceSetup const& setup_current_device() {
  int device = 0;
  check(cudaGetDevice(&device), "cudaGetDevice");
  if (device < 0 || device >= kMaxDevices) throw std::out_of_range("radio device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup& s = g_setup[device];
  if (!s.ready) {
    void* address = nullptr;
    check(cudaGetSymbolAddress(&address, g_no_alloc_scratch), "cudaGetSymbolAddress(radio scratch)");
    check(cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    s.max_window = c8r::windowed_max_bins(device);
    if (s.max_window <= 0) throw std::runtime_error("windowed radio kernel does not fit on this device");
    s.scratch = static_cast<unsigned char*>(address);
    s.ready = true;
  }
  return s;
}

// Host data reaches the scratch array as the by-value parameter of a copy
// kernel: the launch copies its parameters when it is queued, so the call
// neither waits for earlier work on `stream` nor depends on the kind of host
// memory the caller's arrays are in (a cudaMemcpyAsync from pageable memory
// would synchronise, and one from pinned memory would read it later).
constexpr std::size_t kUploadBytes = 16384;
struct UploadBlock {
  uint4 words[kUploadBytes / sizeof(uint4)];
};

__global__ void upload_kernel(const __grid_constant__ UploadBlock block, uint4* __restrict__ out,
                              uint32_t words) {
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) out[i] = block.words[i];
}

// Queues a copy of `bytes` (a multiple of 16, at most kUploadBytes) from the
// host block to device address `out` (16-byte aligned).
void upload(UploadBlock const& block, void* out, std::size_t bytes, cudaStream_t stream) {
  uint32_t const words = static_cast<uint32_t>(bytes / sizeof(uint4));
  upload_kernel<<<1, 256, 0, stream>>>(block, static_cast<uint4*>(out), words);
  check(cudaGetLastError(), "radio scratch upload");
}

// Whether every observer seen shares one destination row (the ingest then
// writes each track's source terms).
struct SharedDestination {
  bool any = false, shared = true;
  c8r::Destination row{};
  void see(ObserverCache const& o) {
    c8r::Destination d{};
    if (!c8r::shared_destination(&o, 1, d)) return;
    if (!any) {
      row = d;
      any = true;
    } else {
      ObserverCache pair[2] = {o, o};
      pair[1].dest_height = row.height;
      pair[1].dest_index = row.index;
      pair[1].dest_n = row.n;
      pair[1].dest_integral = row.integral;
      shared = shared && c8r::shared_destination(pair, 2, d);
    }
  }
};

// The accumulator's per-observer constants (make_observer_cache), built a
// block at a time on the host and uploaded by value.
void upload_observers(c8r_config const& config, int algorithm, ObserverCache* device_out,
                      std::size_t& bins, SharedDestination& destination, cudaStream_t stream) {
  static_assert(sizeof(ObserverCache) % sizeof(uint4) == 0, "observer constants in 16-byte words");
  c8r_observer_snapshot const* snapshots = algorithm == 0 ? config.coreas_observers : config.zhs_observers;
  std::size_t const count = algorithm == 0 ? config.coreas_observer_count : config.zhs_observer_count;
  auto const& p = config.propagation;
  bool const homogeneous = p.homogeneous_refractive_index > 0.;
  bool const fixed = config.deterministic != 0;
  double const limit = config.fixed_point_field_limit_v_per_m;
  constexpr std::size_t kBlock = kUploadBytes / sizeof(ObserverCache);
  UploadBlock block;
  std::size_t offset = 0;
  for (std::size_t first = 0; first < count; first += kBlock) {
    std::size_t const n = std::min(kBlock, count - first);
    for (std::size_t k = 0; k < n; ++k) {
      c8r_observer_snapshot const& s = snapshots[first + k];
      ObserverCache const cache = c8r::make_observer_cache(
          s, algorithm, homogeneous, p.minimum_height_m, p.inverse_step_per_m,
          [&](uint64_t i) { return make_double2(p.refractivity[i], p.integrated_refractivity[i]); },
          fixed, limit, config.count_samples != 0, offset);
      destination.see(cache);
      std::memcpy(reinterpret_cast<unsigned char*>(block.words) + k * sizeof(ObserverCache), &cache,
                  sizeof cache);
      offset += static_cast<std::size_t>(s.number_of_bins);
    }
    upload(block, device_out + first, n * sizeof(ObserverCache), stream);
  }
  bins = offset;
}

// The {n-1, integral} table interleaved from the caller's two arrays.
void upload_table(c8r_propagation_snapshot const& p, double2* device_out, cudaStream_t stream) {
  constexpr std::size_t kBlock = kUploadBytes / sizeof(double2);
  UploadBlock block;
  auto* entries = reinterpret_cast<double2*>(block.words);
  for (std::size_t first = 0; first < p.table_size; first += kBlock) {
    std::size_t const n = std::min<std::size_t>(kBlock, p.table_size - first);
    for (std::size_t k = 0; k < n; ++k)
      entries[k] = make_double2(p.refractivity[first + k], p.integrated_refractivity[first + k]);
    upload(block, device_out + first, n * sizeof(double2), stream);
  }
}

void accumulate_no_alloc(c8r_config const& config, c8r_lepton_transport_record const* records,
                         std::size_t count, std::size_t extent, void* coreas_traces,
                         void* zhs_traces, c8r_counters* counters, cudaStream_t stream) {
  if (!config.enabled) return;
  if (c8r_config_validate(&config) != C8R_OK) throw std::invalid_argument(c8r_last_global_error());
  if (count > extent) throw std::out_of_range("radio track count exceeds input view");
  if (count != 0 && records == nullptr) throw std::invalid_argument("null device radio track input");
  if (config.precision > C8R_PRECISION_MIXED)
    throw std::invalid_argument("no-alloc radio call takes FP64 or mixed precision");
  bool const on[2] = {config.coreas_enabled != 0, config.zhs_enabled != 0};
  std::size_t const observers[2] = {on[0] ? config.coreas_observer_count : 0,
                                    on[1] ? config.zhs_observer_count : 0};
  // size limits of the static scratch, checked before any CUDA call
  if (observers[0] + observers[1] > kMaxObservers)
    throw std::length_error("no-alloc radio call: more than " + std::to_string(kMaxObservers) +
                            " observers (CoREAS + ZHS) do not fit its static scratch");
  bool const homogeneous = config.propagation.homogeneous_refractive_index > 0.;
  if (!homogeneous && config.propagation.table_size > kMaxTableEntries)
    throw std::length_error("no-alloc radio call: refractivity table of more than " +
                            std::to_string(kMaxTableEntries) + " entries does not fit its static scratch");
  if ((on[0] && observers[0] && coreas_traces == nullptr) || (on[1] && observers[1] && zhs_traces == nullptr))
    throw std::invalid_argument("null device radio trace output");

  // nothing to project: no device work at all
  if (count == 0 || observers[0] + observers[1] == 0) return;

  DeviceSetup const& dev = setup_current_device();
  unsigned char* const base = dev.scratch;
  auto* const fallback_counters = reinterpret_cast<DeviceCounters*>(base + kCountersOffset);
  auto* const slot = reinterpret_cast<unsigned long long*>(base + kSlotOffset);
  auto* const next_item = reinterpret_cast<unsigned*>(base + kNextItemOffset);
  auto* const table = reinterpret_cast<double2*>(base + kTableOffset);
  auto* const caches = reinterpret_cast<ObserverCache*>(base + kObserversOffset);
  auto* const tracks = reinterpret_cast<double*>(base + kTracksOffset);
  auto* const deferred = reinterpret_cast<unsigned*>(base + kDeferredOffset);
  DeviceCounters* const event_counters =
      counters ? reinterpret_cast<DeviceCounters*>(counters) : fallback_counters;
  if (!counters)
    check(cudaMemsetAsync(fallback_counters, 0, sizeof(DeviceCounters), stream), "radio scratch clear");

  // the {n-1, integral} table, interleaved straight from the caller's arrays
  c8r::Propagation prop{};
  auto const& p = config.propagation;
  prop.homogeneous = p.homogeneous_refractive_index;
  prop.min_height = p.minimum_height_m;
  prop.max_height = p.maximum_height_m;
  prop.step = p.step_m;
  prop.inv_step = p.inverse_step_per_m;
  prop.slope_n_lower = p.slope_refractivity_lower;
  prop.slope_i_lower = p.slope_integrated_refractivity_lower;
  prop.slope_n_upper = p.slope_refractivity_upper;
  prop.slope_i_upper = p.slope_integrated_refractivity_upper;
  prop.table_size = p.table_size;
  prop.refinement = config.zhs_subtrack_refinement;
  if (!homogeneous) {
    upload_table(p, table, stream);
    prop.table = table;
  }
  std::size_t bins[2] = {0, 0};
  uint64_t largest = 0;
  SharedDestination destination;
  for (int a = 0; a < 2; ++a) {
    if (!observers[a]) continue;
    upload_observers(config, a, caches + (a == 0 ? 0 : observers[0]), bins[a], destination, stream);
    c8r_observer_snapshot const* s = a == 0 ? config.coreas_observers : config.zhs_observers;
    for (std::size_t i = 0; i < observers[a]; ++i) largest = std::max<uint64_t>(largest, s[i].number_of_bins);
  }

  bool const fixed = config.deterministic != 0;
  c8r::Precision const precision =
      config.precision == C8R_PRECISION_MIXED ? c8r::Precision::kMixed : c8r::Precision::kFP64;
  uint32_t const window =
      static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(largest, dev.max_window)));
  int const threads = c8r::kWindowThreads;
  int const per_sm = c8r::windowed_ctas_per_sm(static_cast<int>(window), threads, fixed, precision);
  if (per_sm <= 0) throw std::runtime_error("windowed radio kernel does not fit on this device");

  c8r::EventPlan ev;
  std::memset(&ev, 0, sizeof ev);
  ev.tracks = tracks;
  ev.stride = kTrackCapacity;
  ev.valid_tracks = slot;
  for (int a = 0; a < 2; ++a) {
    ev.observers[a] = observers[a] ? caches + (a == 0 ? 0 : observers[0]) : nullptr;
    ev.observer_count[a] = static_cast<uint32_t>(observers[a]);
    void* const out = a == 0 ? coreas_traces : zhs_traces;
    if (fixed)
      ev.fixed[a] = static_cast<unsigned long long*>(out);
    else
      ev.floating[a] = static_cast<double*>(out);
    ev.total_bins[a] = bins[a];
  }
  ev.propagation = prop;
  ev.counters = event_counters;
  ev.window = window;
  ev.first_track = 0;
  ev.last_track = ~0ull;
  c8r::IngestTerms terms{};
  terms.enabled = destination.any && destination.shared ? 1 : 0;
  terms.propagation = prop;
  terms.destination = destination.row;
  ev.precomputed = static_cast<uint32_t>(terms.enabled);

  // records in chunks of at most kTrackCapacity: ingest into the scratch
  // kinematics, then one persistent launch per algorithm over the chunk
  for (std::size_t begin = 0; begin < count; begin += kTrackCapacity) {
    std::size_t const n = std::min(kTrackCapacity, count - begin);
    check(cudaMemsetAsync(slot, 0, sizeof(unsigned long long), stream), "radio scratch clear");
    check(c8r::launch_ingest(records + begin, n, tracks, kTrackCapacity, slot, event_counters,
                             config.track_diagnostics != 0, terms, stream),
          "radio ingest launch");
    std::size_t const ctas_total = static_cast<std::size_t>(dev.sms) * 2;
    std::size_t const per_item = observers[0] + observers[1];
    std::size_t const target = std::max<std::size_t>(1, (16 * ctas_total + per_item - 1) / per_item);
    // a chunk no longer than one CTA's share of the deferred lists
    std::size_t const list_share = kDeferredEntries / (static_cast<std::size_t>(per_sm) * dev.sms);
    std::size_t const chunk =
        std::min(list_share, std::max<std::size_t>(8192, (n + target - 1) / target));
    ev.chunk_size = static_cast<uint32_t>(chunk);
    ev.chunks = static_cast<uint32_t>((n + chunk - 1) / chunk);
    for (int a = 0; a < 2; ++a) {
      if (!observers[a]) continue;
      c8r::WorkPlan plan;
      std::memset(&plan, 0, sizeof plan);
      plan.events[0] = ev;
      plan.algorithm = a;
      plan.event_count = 1;
      plan.window = window;
      plan.total_items = static_cast<uint64_t>(ev.chunks) * observers[a];
      plan.next_item = next_item;
      uint64_t ctas = static_cast<uint64_t>(per_sm) * dev.sms;
      if (ctas > plan.total_items) ctas = plan.total_items;
      plan.deferred = deferred;
      plan.deferred_stride = static_cast<uint32_t>(chunk);
      check(cudaMemsetAsync(next_item, 0, sizeof(unsigned), stream), "radio scratch clear");
      check(c8r::launch_windowed(plan, fixed, precision, static_cast<int>(ctas), threads, stream),
            "radio windowed launch");
    }
  }
}

}  // namespace

extern "C" int c8r_accumulate_device_no_alloc(const c8r_config* config,
                                              const c8r_lepton_transport_record* records,
                                              size_t count, size_t extent, void* coreas_traces,
                                              void* zhs_traces, c8r_counters* counters,
                                              void* stream) {
  try {
    if (!config) throw std::invalid_argument("null radio config");
    accumulate_no_alloc(*config, records, count, extent, coreas_traces, zhs_traces, counters,
                        static_cast<cudaStream_t>(stream));
    return C8R_OK;
  } catch (std::invalid_argument const& e) {
    c8r::set_global_error(e.what());
    return C8R_INVALID_ARGUMENT;
  } catch (std::out_of_range const& e) {
    c8r::set_global_error(e.what());
    return C8R_OUT_OF_RANGE;
  } catch (std::length_error const& e) {
    c8r::set_global_error(e.what());
    return C8R_LENGTH_ERROR;
  } catch (std::runtime_error const& e) {
    c8r::set_global_error(e.what());
    return C8R_CUDA_ERROR;
  } catch (...) {
    c8r::set_global_error("unknown radio failure");
    return C8R_RUNTIME_ERROR;
  }
}
