// accumulator.cu — host side of libc8radio.so: the RadioAccumulator semantics
// of corsika/detail/kokkos/radio/RadioAccumulator.inl over the sm_100a
// kernels, and the extern "C" entry points declared in include/c8radio.h.
//
// Exceptions carry the reference's classes (std::invalid_argument,
// std::logic_error, std::out_of_range, std::runtime_error, ...) and are
// mapped to C8R_* status codes at the C boundary.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <map>
#include <limits>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/c8radio.h"
#include "host_setup.hpp"
#include "radio_kernels.cuh"
#include "status.hpp"

namespace c8r {
namespace {

constexpr std::size_t kDefaultHostBatch = 4096;   // RadioAccumulator.hpp:49
constexpr std::size_t kDirectThreshold = 16384;   // RadioAccumulator.hpp:101

void check(cudaError_t err, char const* what) {
  if (err != cudaSuccess)
    throw cuda_error(std::string(what) + ": " + cudaGetErrorString(err));
}

template <class T>
struct DeviceBuffer {
  T* ptr = nullptr;
  std::size_t count = 0;
  DeviceBuffer() = default;
  DeviceBuffer(DeviceBuffer const&) = delete;
  DeviceBuffer& operator=(DeviceBuffer const&) = delete;
  ~DeviceBuffer() { release(); }
  void allocate(std::size_t n) {
    release();
    if (n == 0) return;
    if (cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)) != cudaSuccess) {
      ptr = nullptr;
      cudaGetLastError();
      throw std::bad_alloc();
    }
    count = n;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    count = 0;
  }
  std::size_t bytes() const { return count * sizeof(T); }
  void swap(DeviceBuffer& other) noexcept {
    std::swap(ptr, other.ptr);
    std::swap(count, other.count);
  }
};

template <class T>
struct PinnedBuffer {
  T* ptr = nullptr;
  std::size_t count = 0;
  PinnedBuffer() = default;
  PinnedBuffer(PinnedBuffer const&) = delete;
  PinnedBuffer& operator=(PinnedBuffer const&) = delete;
  ~PinnedBuffer() {
    if (ptr) cudaFreeHost(ptr);
  }
  void allocate(std::size_t n) {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    count = 0;
    if (n == 0) return;
    if (cudaMallocHost(reinterpret_cast<void**>(&ptr), n * sizeof(T)) != cudaSuccess) {
      ptr = nullptr;
      cudaGetLastError();
      throw std::bad_alloc();
    }
    count = n;
  }
};

std::size_t checked_add(std::size_t a, std::size_t b) {
  if (b > std::numeric_limits<std::size_t>::max() - a)
    throw std::overflow_error("radio memory projection overflow");
  return a + b;
}
std::size_t checked_mul(std::size_t a, std::size_t b) {
  if (a != 0 && b > std::numeric_limits<std::size_t>::max() / a)
    throw std::overflow_error("radio memory projection overflow");
  return a * b;
}

// RadioAccumulator::validate, RadioAccumulator.inl:931-974.
void validate(c8r_config const& config) {
  auto const& p = config.propagation;
  if (!config.coreas_enabled && !config.zhs_enabled)
    throw std::invalid_argument("enabled radio has no algorithm");
  if (!std::isfinite(config.fixed_point_field_limit_v_per_m) ||
      !(config.fixed_point_field_limit_v_per_m > 0.))
    throw std::invalid_argument("invalid radio fixed-point limit");
  if (config.zhs_subtrack_refinement < 1 || config.zhs_subtrack_refinement > 64)
    throw std::invalid_argument("ZHS subtrack refinement must be in [1,64]");
  if (!std::isfinite(p.homogeneous_refractive_index) || p.homogeneous_refractive_index < 0.)
    throw std::invalid_argument("invalid homogeneous radio refractive index");
  bool const homogeneous = p.homogeneous_refractive_index > 0.;
  if (!homogeneous &&
      (p.table_size < 11 || p.refractivity == nullptr || p.integrated_refractivity == nullptr ||
       !std::isfinite(p.minimum_height_m) || !std::isfinite(p.maximum_height_m) ||
       !(p.maximum_height_m > p.minimum_height_m) || !std::isfinite(p.step_m) ||
       !(p.step_m > 0.) || !std::isfinite(p.inverse_step_per_m) ||
       !(p.inverse_step_per_m > 0.)))
    throw std::invalid_argument("invalid flat-atmosphere radio snapshot");
  if (config.precision < C8R_PRECISION_FP64 || config.precision > C8R_PRECISION_STUDY_FP64)
    throw std::invalid_argument("invalid radio precision");
  if (config.kernel < C8R_KERNEL_AUTO || config.kernel > C8R_KERNEL_TILED)
    throw std::invalid_argument("invalid radio kernel selection");
  if (config.count_samples && !config.deterministic)
    throw std::invalid_argument("radio sample counting needs fixed-point traces");
  auto check_observers = [&](c8r_observer_snapshot const* observers, uint64_t count) {
    if (count != 0 && observers == nullptr) throw std::invalid_argument("null radio observers");
    for (uint64_t i = 0; i < count; ++i) {
      auto const& o = observers[i];
      if (!std::isfinite(o.start_time_s) || !std::isfinite(o.duration_s) ||
          !(o.duration_s >= 0.) || !std::isfinite(o.sample_rate_hz) || !(o.sample_rate_hz > 0.) ||
          o.number_of_bins == 0)
        throw std::invalid_argument("invalid radio observer");
      double const height = (o.position_m[2] - p.minimum_height_m) * p.inverse_step_per_m;
      if (!homogeneous && (!std::isfinite(height) || height < 0. ||
                           height + 0.5 >= static_cast<double>(p.table_size)))
        throw std::invalid_argument("radio observer outside propagation table");
      for (double coordinate : o.position_m)
        if (!std::isfinite(coordinate))
          throw std::invalid_argument("radio observer position is not finite");
    }
  };
  check_observers(config.coreas_observers, config.coreas_observer_count);
  check_observers(config.zhs_observers, config.zhs_observer_count);
}

std::size_t total_bins(c8r_observer_snapshot const* observers, uint64_t count) {
  std::size_t bins = 0;
  for (uint64_t i = 0; i < count; ++i) {
    if (observers[i].number_of_bins > std::numeric_limits<std::size_t>::max() - bins)
      throw std::overflow_error("radio waveform bin overflow");
    bins += static_cast<std::size_t>(observers[i].number_of_bins);
  }
  return bins;
}

}  // namespace

// RadioAccumulator::projectedDeviceBytes, RadioAccumulator.inl:87-141 (for
// this implementation's allocations).
std::size_t projected_device_bytes(c8r_config const& config) {
  if (!config.enabled) return 0;
  validate(config);
  bool const homogeneous = config.propagation.homogeneous_refractive_index > 0.;
  std::size_t total = homogeneous ? 0 : checked_mul(config.propagation.table_size, 2 * sizeof(double));
  std::size_t const nc = config.coreas_enabled ? config.coreas_observer_count : 0;
  std::size_t const nz = config.zhs_enabled ? config.zhs_observer_count : 0;
  total = checked_add(total, checked_mul(nc + nz, sizeof(ObserverCache)));
  for (int a = 0; a < 2; ++a) {
    auto const bins = a == 0 ? total_bins(config.coreas_observers, nc)
                             : total_bins(config.zhs_observers, nz);
    auto const values = checked_mul(bins, 3);
    total = checked_add(total, checked_mul(values, sizeof(long long)));
    total = checked_add(total, checked_mul(values, sizeof(double)));  // decode buffer
  }
  total = checked_add(total, sizeof(DeviceCounters) + sizeof(unsigned long long) + 2 * sizeof(unsigned));
  total = checked_add(total, checked_mul(kDefaultHostBatch, sizeof(c8r_lepton_transport_record)));
  return total;
}

class Accumulator {
 public:
  Accumulator(c8r_config const& config, c8r_tuning const& tuning, cudaStream_t stream)
      : stream_(stream) {
    if (tuning.team_size > static_cast<uint64_t>(kWindowThreads) ||
        (tuning.team_size != 0 && tuning.team_size % 32 != 0))
      throw std::invalid_argument("radio tuning is invalid");
    enabled_ = config.enabled != 0;
    tuning_ = tuning;
    if (!enabled_) return;
    validate(config);
    // snapshot extents: every configured observer, its algorithm enabled or not
    config_bins_[0] = total_bins(config.coreas_observers, config.coreas_observer_count);
    config_bins_[1] = total_bins(config.zhs_observers, config.zhs_observer_count);
    for (std::size_t bins : config_bins_)
      if (bins > std::numeric_limits<std::size_t>::max() / 3)
        throw std::overflow_error("radio waveform bin overflow");
    check(cudaGetDevice(&device_), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_), "SM count");
    copy_config(config);
    fixed_ = config.deterministic != 0;
    precision_ = config.precision == C8R_PRECISION_MIXED ? Precision::kMixed : Precision::kFP64;
    study_ = config.precision >= C8R_PRECISION_STUDY_DOUBLE_FP32;
    if (config.precision == C8R_PRECISION_STUDY_DOUBLE_FP32) arithmetic_ = TimeArithmetic::kDoubleFloat;
    if (config.precision == C8R_PRECISION_STUDY_FP32) arithmetic_ = TimeArithmetic::kFloat;
    kernel_ = config.kernel;
    host_batch_ = tuning.batch_size ? static_cast<std::size_t>(tuning.batch_size) : kDefaultHostBatch;
    threads_ = tuning.team_size ? static_cast<int>(tuning.team_size) : kWindowThreads;
    upload_static();
    choose_ingest_terms();
    allocate_traces();
    counters_.allocate(1);
    slot_.allocate(1);
    next_item_.allocate(2);  // one work counter per algorithm
    reruns_.allocate(2);  // items re-run with checked adds, items handed to a drain pass
    staging_.allocate(host_batch_);
    for (auto& h : host_) h.allocate(host_batch_);
    for (auto& e : host_ready_) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    fuse_ = coreas_enabled_ && zhs_enabled_ && observers_share_grid();
    initialized_ = true;
    reset();
  }

  ~Accumulator() {
    if (stream_ || initialized_) cudaStreamSynchronize(stream_);
    if (copy_stream_) {
      cudaStreamSynchronize(copy_stream_);
      cudaStreamDestroy(copy_stream_);
    }
    if (side_stream_) {
      cudaStreamSynchronize(side_stream_);
      cudaStreamDestroy(side_stream_);
    }
    for (auto& e : side_events_)
      if (e) cudaEventDestroy(e);
    for (auto& e : copy_done_)
      if (e) cudaEventDestroy(e);
    for (auto& e : consumed_)
      if (e) cudaEventDestroy(e);
    for (auto& e : host_ready_)
      if (e) cudaEventDestroy(e);
    for (auto e : all_events_) cudaEventDestroy(e);
  }

  bool enabled() const { return initialized_ && enabled_; }

  // RadioAccumulator::reset, RadioAccumulator.inl:224-250.
  void reset() {
    if (!enabled()) return;
    if (host_count_ != 0) throw std::logic_error("cannot reset radio with uncommitted host tracks");
    for (int a = 0; a < 2; ++a) {
      if (fixed_traces_[a].ptr)
        check(cudaMemsetAsync(fixed_traces_[a].ptr, 0, fixed_traces_[a].bytes(), stream_), "memset");
      if (float_traces_[a].ptr)
        check(cudaMemsetAsync(float_traces_[a].ptr, 0, float_traces_[a].bytes(), stream_), "memset");
    }
    check(cudaMemsetAsync(counters_.ptr, 0, sizeof(DeviceCounters), stream_), "memset");
    check(cudaMemsetAsync(reruns_.ptr, 0, 2 * sizeof(unsigned long long), stream_), "memset");
    clear_staged();
    check(cudaStreamSynchronize(stream_), "reset fence");
    resolve_timing();
    stats_ = c8r_statistics{};
    stats_.device_bytes = device_bytes();
    stats_.track_tile_size = static_cast<uint32_t>(chunk_hint());
    stats_.observer_tile_size = static_cast<uint32_t>(window_bins_);
    downloaded_ = false;
    sealed_ = false;
  }

  // RadioAccumulator::enqueueHostLeptonTracks, RadioAccumulator.inl:252-272.
  void enqueue_host(c8r_lepton_transport_record const* records, std::size_t count) {
    if (!enabled()) throw std::logic_error("host radio tracks requested while radio is disabled");
    if (downloaded_ || sealed_) throw std::logic_error("radio already downloaded; reset before host tracks");
    if (count != 0 && records == nullptr) throw std::invalid_argument("null host radio track input");
    if (count >= host_batch_ && host_count_ == 0 && is_pinned(records)) {
      // Page-locked caller memory: DMA every batch, the last partial one
      // included, straight from it, then wait for the copies before
      // returning (the caller may reuse it).
      enqueue_pinned(records, count);
      return;
    }
    while (count != 0) {
      if (host_count_ == 0) check(cudaEventSynchronize(host_ready_[host_index_]), "staging wait");
      std::size_t const copied = std::min(count, host_batch_ - host_count_);
      std::memcpy(host_[host_index_].ptr + host_count_, records, copied * sizeof(*records));
      host_count_ += copied;
      stats_.host_tracks_enqueued += copied;
      records += copied;
      count -= copied;
      if (host_count_ == host_batch_) flush();
    }
  }

  static bool is_pinned(void const* p) {
    cudaPointerAttributes attributes{};
    if (cudaPointerGetAttributes(&attributes, p) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return attributes.type == cudaMemoryTypeHost;
  }

  // The bytes of a record the ingest reads: start.pid through start.weight
  // and end.position through end.time (with the diagnostics' energy and
  // directions), one span of 208 of the record's 752 bytes.  Host records are
  // uploaded as that span alone, a pitched copy to the same offsets of the
  // device staging records (whose other bytes the ingest never reads).
  static constexpr std::size_t kUsedBegin = offsetof(c8r_lepton_transport_record, start);
  static constexpr std::size_t kUsedEnd =
      offsetof(c8r_lepton_transport_record, end) + offsetof(c8r_particle_state, time_s) + sizeof(double);
  static_assert(offsetof(c8r_particle_state, weight) + sizeof(double) <=
                    offsetof(c8r_lepton_transport_record, end) - offsetof(c8r_lepton_transport_record, start),
                "start fields inside the span");
  static_assert(kUsedEnd - kUsedBegin == 208, "208-byte span of the 752-byte record");

  cudaError_t upload_used(c8r_lepton_transport_record* dst, c8r_lepton_transport_record const* src,
                          std::size_t n, cudaStream_t stream) {
    constexpr std::size_t kPitch = sizeof(c8r_lepton_transport_record);
    return cudaMemcpy2DAsync(reinterpret_cast<unsigned char*>(dst) + kUsedBegin, kPitch,
                             reinterpret_cast<unsigned char const*>(src) + kUsedBegin, kPitch,
                             kUsedEnd - kUsedBegin, n, cudaMemcpyHostToDevice, stream);
  }

  // Batches of host_batch_ records (the last one partial) copied from pinned
  // caller memory into a pair of device staging buffers (the copy of batch
  // k+1 overlaps the projection of batch k on the copy stream; a buffer is
  // free again once its ingest has run); returns after the last copy
  // completed.  The first batch is 1/32 of host_batch_ (at least 8192
  // records) and each next one twice as long, up to host_batch_: a copy of
  // the records' used spans takes about a third of the projection of as
  // many records (208 B at ~53 GB/s against ~11 ns on the 1e7 x 160
  // workload), so every copy but the first stays hidden behind the projection
  // of the batch before it; the first is short, and the batches few.
  void enqueue_pinned(c8r_lepton_transport_record const* records, std::size_t count) {
    if (!copy_stream_) {
      check(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking), "copy stream");
      for (auto& e : copy_done_) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
      for (auto& e : consumed_) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
      staging2_.allocate(host_batch_);
    }
    // earlier work on the accumulator stream may still read staging_
    for (auto& e : consumed_) check(cudaEventRecord(e, stream_), "event");
    std::size_t size = host_batch_ / 32 >= 8192 ? host_batch_ / 32 : std::min<std::size_t>(host_batch_, 8192);
    std::size_t offset = 0;
    for (std::size_t b = 0; offset < count; ++b) {
      std::size_t const n = std::min(count - offset, size);
      size = std::min(host_batch_, 2 * size);
      int const k = static_cast<int>(b & 1);
      c8r_lepton_transport_record* dst = k ? staging2_.ptr : staging_.ptr;
      // the staging buffer is free once the ingest that read it has run
      check(cudaStreamWaitEvent(copy_stream_, consumed_[k], 0), "wait");
      check(upload_used(dst, records + offset, n, copy_stream_), "host track upload");
      check(cudaEventRecord(copy_done_[k], copy_stream_), "event");
      check(cudaStreamWaitEvent(stream_, copy_done_[k], 0), "wait");
      stage_device(dst, n, host_batch_);
      check(cudaEventRecord(consumed_[k], stream_), "event");
      project_staged(true);
      offset += n;
      stats_.host_to_device_bytes += n * (kUsedEnd - kUsedBegin);
      ++stats_.host_track_batches;
      stats_.host_tracks_enqueued += n;
    }
    check(cudaStreamSynchronize(copy_stream_), "host track upload");
  }

  // RadioAccumulator::flushHostLeptonTracks, RadioAccumulator.inl:274-290.  The
  // staging half just filled is copied asynchronously; the other half can be
  // filled while it uploads (double buffering replaces the reference's fence).
  void flush() {
    if (host_count_ == 0) return;
    std::size_t const n = host_count_;
    check(upload_used(staging_.ptr, host_[host_index_].ptr, n, stream_), "host track upload");
    check(cudaEventRecord(host_ready_[host_index_], stream_), "event");
    host_index_ ^= 1;
    host_count_ = 0;
    accumulate_device(staging_.ptr, n, staging_.count);
    stats_.host_to_device_bytes += n * (kUsedEnd - kUsedBegin);
    ++stats_.host_track_batches;
  }

  // RadioAccumulator::accumulateLeptonTracks, RadioAccumulator.inl:292-357:
  // ingest the records and project them (with any tracks staged before).
  void accumulate_device(c8r_lepton_transport_record const* records, std::size_t count,
                         std::size_t extent) {
    if (!enabled() || count == 0) return;
    stage_device(records, count, extent);
    project_staged(true);
  }

  // B200 extension: ingest device records into the kinematics workspace,
  // after the tracks already staged, without projecting them yet.
  void stage_device(c8r_lepton_transport_record const* records, std::size_t count,
                    std::size_t extent) {
    if (!enabled() || count == 0) return;
    if (sealed_) throw std::logic_error("radio endpoint already committed; reset before new tracks");
    if (count > extent) throw std::out_of_range("radio track count exceeds input view");
    if (records == nullptr) throw std::invalid_argument("null device radio track input");
    if (staged_ > std::numeric_limits<std::size_t>::max() - count)
      throw std::length_error("radio staged track count overflow");
    ensure_capacity(staged_ + count);
    if (staged_ == 0) check(cudaMemsetAsync(slot_.ptr, 0, sizeof(unsigned long long), stream_), "memset");
    check(launch_ingest(records, count, tracks_.ptr, capacity_, slot_.ptr, counters_.ptr,
                        diagnostics_, terms_, stream_),
          "ingest launch");
    staged_ += count;
    ++stats_.track_precompute_batches;
    stats_.track_precomputed_records += count;
    stats_.maximum_track_batch = std::max<uint64_t>(stats_.maximum_track_batch, count);
    downloaded_ = false;
  }

  // The same over a structure-of-arrays view of device steps, then projected.
  void accumulate_columns(c8r_track_columns const& columns, std::size_t count) {
    if (!enabled() || count == 0) return;
    if (sealed_) throw std::logic_error("radio endpoint already committed; reset before new tracks");
    bool ok = columns.pid && columns.weight && columns.start_time_s && columns.end_time_s;
    for (int a = 0; a < 3; ++a) ok = ok && columns.start_position_m[a] && columns.end_position_m[a];
    if (diagnostics_) {
      ok = ok && columns.start_energy_gev;
      for (int a = 0; a < 3; ++a) ok = ok && columns.start_direction[a] && columns.end_direction[a];
    }
    if (!ok) throw std::invalid_argument("null device radio track column");
    if (staged_ > std::numeric_limits<std::size_t>::max() - count)
      throw std::length_error("radio staged track count overflow");
    ensure_capacity(staged_ + count);
    if (staged_ == 0) check(cudaMemsetAsync(slot_.ptr, 0, sizeof(unsigned long long), stream_), "memset");
    check(launch_ingest_columns(columns, count, tracks_.ptr, capacity_, slot_.ptr, counters_.ptr, diagnostics_,
                                terms_, stream_),
          "ingest launch");
    staged_ += count;
    ++stats_.track_precompute_batches;
    stats_.track_precomputed_records += count;
    stats_.maximum_track_batch = std::max<uint64_t>(stats_.maximum_track_batch, count);
    downloaded_ = false;
    project_staged(true);
  }

  // Projects the staged tracks of this accumulator alone; consume drops them.
  void project_staged(bool consume) {
    if (!enabled() || staged_ == 0) return;
    if (sealed_) throw std::logic_error("radio endpoint already committed; reset before new tracks");
    std::size_t const count = staged_;
    cudaEvent_t begin = nullptr, end = nullptr;
    if (timing_) {
      begin = timing_event();
      check(cudaEventRecord(begin, stream_), "event");
    }
    bool const direct = kernel_ == C8R_KERNEL_DIRECT ||
                        (kernel_ == C8R_KERNEL_AUTO && count < kDirectThreshold);
    if (study_)
      project_study(count);
    else if (kernel_ == C8R_KERNEL_TILED)
      project_tiled(count);
    else if (direct)
      project_direct(count);
    else
      project_windowed(count);
    if (timing_) {
      end = timing_event();
      check(cudaEventRecord(end, stream_), "event");
      pending_.push_back({{begin, end}, -1});
    }
    if (consume) clear_staged();
    downloaded_ = false;
  }

  void clear_staged() {
    if (staged_ == 0) return;
    check(cudaMemsetAsync(slot_.ptr, 0, sizeof(unsigned long long), stream_), "memset");
    staged_ = 0;
  }

  // Batched projection support (Batch below).
  std::size_t staged() const { return staged_; }
  cudaStream_t stream() const { return stream_; }
  bool sealed() const { return sealed_; }
  void note_batch_projection(std::size_t count, uint64_t items) {
    EventPlan const ev = make_event(count);
    uint64_t const pairs_c = count * ev.observer_count[0], pairs_z = count * ev.observer_count[1];
    stats_.track_observer_pairs += pairs_c + pairs_z;
    if (fuse_) stats_.fused_track_observer_pairs += pairs_c;
    stats_.projection_tiles += items;
    downloaded_ = false;
  }
  void set_tuning(c8r_tuning const& t) {
    if (t.team_size > static_cast<uint64_t>(kWindowThreads) || (t.team_size != 0 && t.team_size % 32 != 0))
      throw std::invalid_argument("radio tuning is invalid");
    threads_ = t.team_size ? static_cast<int>(t.team_size) : kWindowThreads;
    tuning_.team_size = t.team_size;
    tuning_.track_tile_size = t.track_tile_size;
    tuning_.observer_tile_size = t.observer_tile_size;
    stats_.track_tile_size = static_cast<uint32_t>(t.track_tile_size);
    if (enabled()) {
      choose_window();
      stats_.observer_tile_size = static_cast<uint32_t>(window_bins_);
    }
  }
  std::size_t largest_bins() const { return largest_bins_; }
  // Zeroes traces and projection counters, keeping staged tracks (autotuning).
  void zero_traces() {
    if (!enabled()) return;
    for (int a = 0; a < 2; ++a) {
      if (fixed_traces_[a].ptr)
        check(cudaMemsetAsync(fixed_traces_[a].ptr, 0, fixed_traces_[a].bytes(), stream_), "memset");
      if (float_traces_[a].ptr)
        check(cudaMemsetAsync(float_traces_[a].ptr, 0, float_traces_[a].bytes(), stream_), "memset");
    }
    check(cudaMemsetAsync(counters_.ptr, 0, offsetof(DeviceCounters, valid_tracks), stream_), "memset");
    check(cudaMemsetAsync(&counters_.ptr->fixed_point_overflows, 0, sizeof(unsigned long long), stream_),
          "memset");
  }

  // Sums the projection-kernel time of completed launches (blocks on them).
  void resolve_timing() {
    for (auto const& entry : pending_) {
      auto const& p = entry.first;
      check(cudaEventSynchronize(p.second), "event");
      float ms = 0.f;
      check(cudaEventElapsedTime(&ms, p.first, p.second), "event time");
      if (entry.second == 0)
        stats_.coreas_kernel_time_ms += ms;
      else if (entry.second == 1)
        stats_.zhs_kernel_time_ms += ms;
      else {
        stats_.kernel_time_ms += ms;
        ++stats_.timed_launches;
      }
      free_events_.push_back(p.first);
      free_events_.push_back(p.second);
    }
    pending_.clear();
  }

  // RadioAccumulator::download, RadioAccumulator.inl:407-439 (decode on the device).
  void download(double* coreas, double* zhs, c8r_counters* counters) {
    if (!enabled()) {
      if (counters) *counters = c8r_counters{};
      return;
    }
    if (downloaded_ || sealed_) throw std::logic_error("radio waveforms downloaded twice");
    flush();
    project_staged(true);
    DeviceCounters host{};
    fetch_counters(host);
    if (host.fixed_point_overflows != 0)
      throw std::runtime_error(
          "radio fixed-point accumulator overflowed; increase fixed_point_field_limit_V_per_m");
    for (int a = 0; a < 2; ++a) {
      double* out = a == 0 ? coreas : zhs;
      std::size_t const values = 3 * bins_[a];
      if (values == 0 || out == nullptr) continue;
      if (fixed_) {
        check(launch_decode(reinterpret_cast<long long const*>(fixed_traces_[a].ptr), decoded_[a].ptr,
                            bins_[a], decode_offsets_[a].ptr, decode_factors_[a].ptr,
                            static_cast<uint32_t>(observers_host_[a].size()), max_observer_bins_[a],
                            stream_),
              "decode launch");
        check(cudaMemcpyAsync(out, decoded_[a].ptr, values * sizeof(double), cudaMemcpyDeviceToHost,
                              stream_),
              "trace download");
      } else {
        check(cudaMemcpyAsync(out, float_traces_[a].ptr, values * sizeof(double),
                              cudaMemcpyDeviceToHost, stream_),
              "trace download");
      }
      stats_.device_to_host_bytes += values * sizeof(double);
    }
    check(cudaStreamSynchronize(stream_), "download fence");
    if (counters) std::memcpy(counters, &host, sizeof(host));
    downloaded_ = true;
  }

  // The output step on the device (RadioProcess.inl:213-223 and the observer
  // add of CorsikaOutputSink.inl:255-278): decoded CoREAS fields and
  // differentiated ZHS fields added into caller-owned device buffers, with
  // download()'s checks and sealing.
  void download_fields_device(double* coreas, double* zhs, c8r_counters* counters) {
    if (!enabled()) {
      if (counters) *counters = c8r_counters{};
      return;
    }
    if (downloaded_ || sealed_) throw std::logic_error("radio waveforms downloaded twice");
    flush();
    project_staged(true);
    DeviceCounters host{};
    fetch_counters(host);
    if (host.fixed_point_overflows != 0)
      throw std::runtime_error(
          "radio fixed-point accumulator overflowed; increase fixed_point_field_limit_V_per_m");
    for (int a = 0; a < 2; ++a) {
      double* out = a == 0 ? coreas : zhs;
      if (out == nullptr || bins_[a] == 0 || observers_host_[a].empty()) continue;
      check(launch_output(fixed_ ? reinterpret_cast<long long const*>(fixed_traces_[a].ptr) : nullptr,
                          float_traces_[a].ptr, out, bins_[a], observers_[a].ptr, decode_factors_[a].ptr,
                          static_cast<uint32_t>(observers_host_[a].size()), max_observer_bins_[a], a == 1,
                          stream_),
            "output launch");
    }
    check(cudaStreamSynchronize(stream_), "output fence");
    if (counters) std::memcpy(counters, &host, sizeof(host));
    downloaded_ = true;
  }

  // RadioAccumulator::downloadFixed, RadioAccumulator.inl:359-405: raw int64.
  void download_fixed(long long* coreas, long long* zhs, c8r_counters* counters) {
    if (!enabled() || !fixed_ || downloaded_ || sealed_)
      throw std::logic_error("fixed radio snapshot unavailable/already committed");
    flush();
    project_staged(true);
    sealed_ = true;
    DeviceCounters host{};
    fetch_counters(host);
    for (int a = 0; a < 2; ++a) {
      long long* out = a == 0 ? coreas : zhs;
      std::size_t const values = 3 * bins_[a];
      if (values == 0 || out == nullptr) continue;
      check(cudaMemcpyAsync(out, fixed_traces_[a].ptr, values * sizeof(long long),
                            cudaMemcpyDeviceToHost, stream_),
            "fixed trace download");
      stats_.device_to_host_bytes += values * sizeof(long long);
    }
    check(cudaStreamSynchronize(stream_), "download fence");
    if (counters) std::memcpy(counters, &host, sizeof(host));
    downloaded_ = true;
  }

  // RadioAccumulator::downloadFixed(shower_identity, endpoint), RadioAccumulator.inl:359-405:
  // the reference's checks in its order.  After the pending host batch is
  // flushed the identity and endpoint are checked (nothing sealed yet); then
  // the endpoint is sealed before the copies, so a failed export cannot be
  // repeated or followed by download(), and the snapshot is validated after
  // them (validate_fixed_radio: an overflowed accumulator is rejected, still
  // sealed).  Each buffer holds 3 x the bins of every configured observer of
  // its algorithm; a disabled algorithm's traces are zero, as the reference's.
  void download_fixed_snapshot(char const* identity, unsigned endpoint, long long* coreas, long long* zhs,
                               c8r_counters* counters) {
    if (!enabled() || !fixed_ || downloaded_ || sealed_)
      throw std::logic_error("fixed radio snapshot unavailable/already committed");
    flush();
    project_staged(true);
    if (identity == nullptr || identity[0] == '\0' || endpoint > 1)
      throw std::invalid_argument("invalid cooperative radio snapshot identity");
    if ((config_bins_[0] && coreas == nullptr) || (config_bins_[1] && zhs == nullptr))
      throw std::invalid_argument("null radio snapshot trace buffer");
    sealed_ = true;
    DeviceCounters host{};
    fetch_counters(host);
    for (int a = 0; a < 2; ++a) {
      long long* out = a == 0 ? coreas : zhs;
      std::size_t const values = 3 * config_bins_[a];
      if (values == 0) continue;
      if (fixed_traces_[a].ptr && bins_[a] == config_bins_[a]) {
        check(cudaMemcpyAsync(out, fixed_traces_[a].ptr, values * sizeof(long long),
                              cudaMemcpyDeviceToHost, stream_),
              "fixed trace download");
        stats_.device_to_host_bytes += values * sizeof(long long);
      } else {
        std::memset(out, 0, values * sizeof(long long));  // algorithm disabled
      }
    }
    check(cudaStreamSynchronize(stream_), "download fence");
    if (counters) std::memcpy(counters, &host, sizeof(host));
    if (host.fixed_point_overflows != 0)
      throw std::invalid_argument("invalid/overflowed cooperative fixed radio snapshot");
    downloaded_ = true;
  }

  std::size_t config_bins(int a) const { return config_bins_[a]; }

  void statistics(c8r_statistics& out) {
    resolve_timing();
    out = stats_;
  }

  std::size_t device_bytes() const {
    std::size_t total = table_.bytes() + counters_.bytes() + slot_.bytes() + next_item_.bytes() + reruns_.bytes() +
                        staging_.bytes() + staging2_.bytes() + tracks_.bytes() + deferred_[0].bytes() +
                        deferred_[1].bytes();
    for (int a = 0; a < 2; ++a)
      total += observers_[a].bytes() + fixed_traces_[a].bytes() + float_traces_[a].bytes() +
               decoded_[a].bytes() + decode_offsets_[a].bytes() + decode_factors_[a].bytes();
    return total;
  }

  std::size_t static_host_to_device_bytes() const {
    return table_.bytes() + observers_[0].bytes() + observers_[1].bytes();
  }

  // RadioAccumulator::reserveTrackCapacity / projectedTrackCapacity.
  void reserve(std::size_t count) {
    if (!enabled() || count == 0) return;
    ensure_capacity(count);
  }
  void projected_track_capacity(std::size_t count, std::size_t& retained, std::size_t& peak) const {
    std::size_t const current = device_bytes();
    retained = peak = current;
    if (!enabled() || count == 0 || count <= capacity_) return;
    if (capacity_ > std::numeric_limits<std::size_t>::max() / 2)
      throw std::length_error("radio track capacity overflow");
    std::size_t const grown = track_capacity(capacity_ == 0 ? count : std::max(count, 2 * capacity_));
    std::size_t const old_bytes = tracks_.bytes();
    std::size_t const new_bytes = checked_mul(checked_mul(grown, kTrackDoubles), sizeof(double));
    retained = current - old_bytes + new_bytes;
    peak = checked_add(current, new_bytes);
  }

  void synchronize() { check(cudaStreamSynchronize(stream_), "stream synchronize"); }

  std::size_t bins(int a) const { return bins_[a]; }
  void set_timing(bool on) { timing_ = on; }

  cudaEvent_t timing_event() {
    if (!free_events_.empty()) {
      cudaEvent_t e = free_events_.back();
      free_events_.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    check(cudaEventCreate(&e), "event");
    all_events_.push_back(e);
    return e;
  }

  // Work-plan access for the batched launcher.
  EventPlan event_plan(std::size_t count) const { return make_event(count); }
  bool fixed() const { return fixed_; }
  Precision precision() const { return precision_; }
  bool study() const { return study_; }
  int sms() const { return sms_; }
  int threads() const { return threads_; }
  uint32_t window_bins() const { return static_cast<uint32_t>(window_bins_); }

 private:
  void copy_config(c8r_config const& config) {
    coreas_enabled_ = config.coreas_enabled != 0;
    zhs_enabled_ = config.zhs_enabled != 0;
    diagnostics_ = config.track_diagnostics != 0;
    limit_ = config.fixed_point_field_limit_v_per_m;
    deterministic_ = config.deterministic != 0;
    count_samples_ = config.count_samples != 0;
    auto const& p = config.propagation;
    propagation_.homogeneous = p.homogeneous_refractive_index;
    propagation_.min_height = p.minimum_height_m;
    propagation_.max_height = p.maximum_height_m;
    propagation_.step = p.step_m;
    propagation_.inv_step = p.inverse_step_per_m;
    propagation_.slope_n_lower = p.slope_refractivity_lower;
    propagation_.slope_i_lower = p.slope_integrated_refractivity_lower;
    propagation_.slope_n_upper = p.slope_refractivity_upper;
    propagation_.slope_i_upper = p.slope_integrated_refractivity_upper;
    propagation_.table_size = p.table_size;
    propagation_.refinement = config.zhs_subtrack_refinement;
    if (p.refractivity && p.integrated_refractivity && p.table_size) {
      table_host_.resize(p.table_size);
      for (std::size_t i = 0; i < p.table_size; ++i)
        table_host_[i] = make_double2(p.refractivity[i], p.integrated_refractivity[i]);
    }
    if (coreas_enabled_)
      snapshots_[0].assign(config.coreas_observers, config.coreas_observers + config.coreas_observer_count);
    if (zhs_enabled_)
      snapshots_[1].assign(config.zhs_observers, config.zhs_observers + config.zhs_observer_count);
  }

  // RadioAccumulator::makeObservers (RadioAccumulator.inl:522-550) plus the
  // per-observer constants of propagate/add_sample, evaluated with the same
  // IEEE operations the reference performs inline.
  void make_observers(int a) {
    auto& out = observers_host_[a];
    out.clear();
    std::size_t offset = 0;
    bool const homogeneous = propagation_.homogeneous > 0.;
    for (auto const& s : snapshots_[a]) {
      out.push_back(make_observer_cache(
          s, a, homogeneous, propagation_.min_height, propagation_.inv_step,
          [&](uint64_t i) { return table_host_[i]; }, deterministic_, limit_, count_samples_, offset));
      offset += static_cast<std::size_t>(s.number_of_bins);
    }
    bins_[a] = offset;
  }

  bool observers_share_grid() const {
    auto const& c = snapshots_[0];
    auto const& z = snapshots_[1];
    if (c.size() != z.size() || c.empty()) return false;
    for (std::size_t i = 0; i < c.size(); ++i) {
      if (c[i].start_time_s != z[i].start_time_s || c[i].duration_s != z[i].duration_s ||
          c[i].sample_rate_hz != z[i].sample_rate_hz || c[i].number_of_bins != z[i].number_of_bins)
        return false;
      for (int axis = 0; axis < 3; ++axis)
        if (c[i].position_m[axis] != z[i].position_m[axis]) return false;
    }
    return true;
  }

  void upload_static() {
    if (!table_host_.empty() && propagation_.homogeneous <= 0.) {
      table_.allocate(table_host_.size());
      check(cudaMemcpy(table_.ptr, table_host_.data(), table_.bytes(), cudaMemcpyHostToDevice),
            "table upload");
    }
    propagation_.table = table_.ptr;
    std::size_t largest = 0;
    for (int a = 0; a < 2; ++a) {
      make_observers(a);
      auto const& host = observers_host_[a];
      if (!host.empty()) {
        observers_[a].allocate(host.size());
        check(cudaMemcpy(observers_[a].ptr, host.data(), observers_[a].bytes(), cudaMemcpyHostToDevice),
              "observer upload");
      }
      max_observer_bins_[a] = 0;
      std::vector<uint64_t> offsets;
      std::vector<double> factors;
      for (auto const& s : snapshots_[a]) {
        max_observer_bins_[a] = std::max<uint64_t>(max_observer_bins_[a], s.number_of_bins);
        factors.push_back(decode_factor(s, a, limit_));  // downloadSet, RadioAccumulator.inl:865-867
      }
      for (auto const& o : host) offsets.push_back(o.offset);
      offsets.push_back(bins_[a]);
      largest = std::max<std::size_t>(largest, max_observer_bins_[a]);
      if (!host.empty()) {
        decode_offsets_[a].allocate(offsets.size());
        decode_factors_[a].allocate(factors.size());
        check(cudaMemcpy(decode_offsets_[a].ptr, offsets.data(), decode_offsets_[a].bytes(),
                         cudaMemcpyHostToDevice),
              "decode upload");
        check(cudaMemcpy(decode_factors_[a].ptr, factors.data(), decode_factors_[a].bytes(),
                         cudaMemcpyHostToDevice),
              "decode upload");
      }
    }
    largest_bins_ = largest;
    choose_window();
  }

  // Shared-memory window: the longest trace, capped by the tuning's
  // observer_tile_size and by what the device's shared memory holds.
  void choose_window() {
    int const device_window = windowed_max_bins(device_);
    std::size_t window = largest_bins_;
    if (tuning_.observer_tile_size != 0) window = std::min<std::size_t>(window, tuning_.observer_tile_size);
    window_bins_ = std::min<std::size_t>(window, static_cast<std::size_t>(device_window));
    if (window_bins_ == 0) window_bins_ = 1;
  }

  // Source terms precomputed at ingest when every observer of both enabled
  // algorithms shares one destination row (always in a homogeneous medium).
  void choose_ingest_terms() {
    std::vector<ObserverCache> all;
    for (int a = 0; a < 2; ++a)
      if (a == 0 ? coreas_enabled_ : zhs_enabled_)
        all.insert(all.end(), observers_host_[a].begin(), observers_host_[a].end());
    Destination d{};
    terms_ = IngestTerms{};
    terms_.enabled = shared_destination(all.data(), all.size(), d) ? 1 : 0;
    terms_.propagation = propagation_;
    terms_.destination = d;
  }

  void allocate_traces() {
    for (int a = 0; a < 2; ++a) {
      std::size_t const values = 3 * bins_[a];
      if (values == 0) continue;
      if (fixed_) {
        fixed_traces_[a].allocate(values);
        decoded_[a].allocate(values);
      } else {
        float_traces_[a].allocate(values);
      }
    }
  }

  void ensure_capacity(std::size_t count) {
    if (capacity_ >= count) return;
    if (capacity_ > std::numeric_limits<std::size_t>::max() / 2)
      throw std::length_error("radio track capacity overflow");
    // whole tiles of the workspace layout (track_capacity)
    std::size_t const grown = track_capacity(capacity_ == 0 ? count : std::max(count, 2 * capacity_));
    DeviceBuffer<double> fresh;
    fresh.allocate(checked_mul(grown, kTrackDoubles));
    if (staged_ != 0)  // keep the tiles staged so far (capacity_ is whole tiles)
      check(cudaMemcpyAsync(fresh.ptr, tracks_.ptr, track_capacity(staged_) * kTrackDoubles * sizeof(double),
                            cudaMemcpyDeviceToDevice, stream_),
            "staged track copy");
    // earlier projections may still read the old workspace
    if (capacity_ != 0) check(cudaStreamSynchronize(stream_), "grow fence");
    tracks_.swap(fresh);
    capacity_ = grown;
    stats_.track_workspace_bytes = tracks_.bytes();
    stats_.device_bytes = device_bytes();
  }

  std::size_t chunk_hint() const { return tuning_.track_tile_size; }

  EventPlan make_event(std::size_t count) const {
    EventPlan ev;
    std::memset(&ev, 0, sizeof ev);
    ev.tracks = tracks_.ptr;
    ev.stride = capacity_;
    ev.valid_tracks = slot_.ptr;
    for (int a = 0; a < 2; ++a) {
      bool const on = a == 0 ? coreas_enabled_ : zhs_enabled_;
      ev.observers[a] = observers_[a].ptr;
      ev.observer_count[a] = on ? static_cast<uint32_t>(observers_host_[a].size()) : 0;
      ev.fixed[a] = fixed_traces_[a].ptr;
      ev.floating[a] = float_traces_[a].ptr;
      ev.total_bins[a] = bins_[a];
    }
    ev.propagation = propagation_;
    ev.counters = counters_.ptr;
    ev.window = static_cast<uint32_t>(window_bins_);
    uint32_t const per_chunk = ev.observer_count[0] + ev.observer_count[1];
    std::size_t chunk = tuning_.track_tile_size;
    if (chunk == 0) {
      // about 16 work items per CTA of each launch (one CTA per SM), at least
      // 8192 tracks each; smaller launches take chunks of an eighth of their
      // tracks up to 262144 (fewer items, so fewer window zero/flush passes:
      // the work list ends on quarter-size chunks anyway)
      std::size_t const ctas = static_cast<std::size_t>(sms_) * 2;
      std::size_t const target_chunks = std::max<std::size_t>(1, (16 * ctas + per_chunk - 1) / std::max<uint32_t>(per_chunk, 1));
      chunk = std::max<std::size_t>(8192, (count + target_chunks - 1) / target_chunks);
      chunk = std::max<std::size_t>(chunk, std::min<std::size_t>((count + 7) / 8, 262144));
      chunk = track_capacity(chunk);  // items start on a track tile
    }
    chunk = std::min<std::size_t>(chunk, kMaxChunkTracks);
    ev.chunk_size = static_cast<uint32_t>(chunk);
    ev.chunks = static_cast<uint32_t>((count + chunk - 1) / chunk);
    ev.first_track = 0;
    ev.last_track = ~0ull;
    ev.precomputed = static_cast<uint32_t>(terms_.enabled);
    return ev;
  }

  // Per-CTA deferred-pair lists of each algorithm's launch (the two launches
  // may run side by side), grown after the earlier work on stream_ (which the
  // previous ZHS launch joined) when a launch needs more.
  unsigned* deferred_lists(int algorithm, uint64_t entries) {
    DeviceBuffer<unsigned>& lists = deferred_[algorithm];
    if (lists.count < entries) {
      check(cudaStreamSynchronize(stream_), "deferred list fence");
      DeviceBuffer<unsigned> fresh;
      // a quarter more than asked: launch sizes vary, and each growth
      // synchronises the device
      fresh.allocate(entries + entries / 4);
      lists.swap(fresh);
      stats_.device_bytes = device_bytes();
    }
    return lists.ptr;
  }

  void project_direct(std::size_t count) {
    EventPlan const ev = make_event(count);
    bool const c = ev.observer_count[0] != 0, z = ev.observer_count[1] != 0;
    if (fuse_) {
      check(launch_direct(ev, count, true, true, fixed_, precision_, stream_), "direct launch");
    } else {
      if (c) check(launch_direct(ev, count, true, false, fixed_, precision_, stream_), "direct launch");
      if (z) check(launch_direct(ev, count, false, true, fixed_, precision_, stream_), "direct launch");
    }
    uint64_t const pairs_c = count * ev.observer_count[0], pairs_z = count * ev.observer_count[1];
    stats_.track_observer_pairs += pairs_c + pairs_z;
    if (fuse_) stats_.fused_track_observer_pairs += pairs_c;
    ++stats_.direct_projection_batches;
    stats_.direct_projection_records += count;
  }

  // The reference's tile shape (RadioAccumulator.inl:699-847): fused when the
  // observer grids match, else one launch per algorithm.
  void project_tiled(std::size_t count) {
    EventPlan const ev = make_event(count);
    bool const c = ev.observer_count[0] != 0, z = ev.observer_count[1] != 0;
    if (fuse_) {
      check(launch_tiled(ev, count, true, true, fixed_, precision_, stream_), "tiled launch");
    } else {
      if (c) check(launch_tiled(ev, count, true, false, fixed_, precision_, stream_), "tiled launch");
      if (z) check(launch_tiled(ev, count, false, true, fixed_, precision_, stream_), "tiled launch");
    }
    uint64_t const pairs_c = count * ev.observer_count[0], pairs_z = count * ev.observer_count[1];
    stats_.track_observer_pairs += pairs_c + pairs_z;
    if (fuse_) stats_.fused_track_observer_pairs += pairs_c;
    uint64_t const observers = std::max(ev.observer_count[0], ev.observer_count[1]);
    stats_.projection_tiles += ((count + 7) / 8) * ((observers + 31) / 32);
  }

  // The precision study's generic kernel, both algorithms in one launch.
  void project_study(std::size_t count) {
    EventPlan const ev = make_event(count);
    bool const c = ev.observer_count[0] != 0, z = ev.observer_count[1] != 0;
    check(launch_study(ev, count, c, z, fixed_, arithmetic_, stream_), "study launch");
    stats_.track_observer_pairs += count * (ev.observer_count[0] + ev.observer_count[1]);
    ++stats_.direct_projection_batches;
    stats_.direct_projection_records += count;
  }

  // One persistent launch per algorithm: each kernel instance carries one
  // algorithm's code only.  CoREAS items run on stream_ and, when both
  // algorithms are on, ZHS items on a second stream: both kernels hold one CTA
  // per SM, so ZHS CTAs start on the SMs that the CoREAS launch's last items
  // leave idle instead of after its slowest CTA.  stream_ then waits for both.
  // With kernel timing on, both run on stream_, so that each launch's events
  // bracket that launch alone.
  void project_windowed(std::size_t count) {
    EventPlan const ev = make_event(count);
    int per_sm = windowed_ctas_per_sm(static_cast<int>(ev.window), threads_, fixed_, precision_);
    if (per_sm <= 0) throw cuda_error("windowed radio kernel does not fit on this device");
    bool const both = !timing_ && ev.observer_count[0] != 0 && ev.observer_count[1] != 0;
    if (both) {
      if (!side_stream_) {
        check(cudaStreamCreateWithFlags(&side_stream_, cudaStreamNonBlocking), "side stream");
        for (auto& e : side_events_) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
      }
      check(cudaEventRecord(side_events_[0], stream_), "event");
      check(cudaStreamWaitEvent(side_stream_, side_events_[0], 0), "wait");
    }
    for (int algorithm = 0; algorithm < 2; ++algorithm) {
      if (ev.observer_count[algorithm] == 0) continue;
      cudaStream_t const s = both && algorithm == 1 ? side_stream_ : stream_;
      WorkPlan plan{};
      plan.algorithm = algorithm;
      plan.window = ev.window;
      plan.next_item = next_item_.ptr + algorithm;
      plan.reruns = reruns_.ptr;
      plan.handbacks = reruns_.ptr + 1;
      uint64_t ctas = static_cast<uint64_t>(per_sm) * sms_;
      append_work(plan, ev, ctas, true);
      if (ctas > plan.total_items) ctas = plan.total_items;
      plan.deferred_stride = deferred_list_stride(plan);
      attach_deferred(plan, deferred_lists(algorithm, deferred_words(plan, ctas, fixed_)), ctas, fixed_);
      check(cudaMemsetAsync(plan.next_item, 0, sizeof(unsigned), s), "memset");
      cudaEvent_t b = nullptr, e = nullptr;
      if (timing_) {
        b = timing_event();
        check(cudaEventRecord(b, s), "event");
      }
      check(launch_windowed(plan, fixed_, precision_, static_cast<int>(ctas), threads_, s),
            "windowed launch");
      if (timing_) {
        e = timing_event();
        check(cudaEventRecord(e, s), "event");
        pending_.push_back({{b, e}, algorithm});
      }
      stats_.projection_tiles += plan.total_items;
    }
    if (both) {
      check(cudaEventRecord(side_events_[1], side_stream_), "event");
      check(cudaStreamWaitEvent(stream_, side_events_[1], 0), "wait");
    }
    uint64_t const pairs_c = count * ev.observer_count[0];
    uint64_t const pairs_z = count * ev.observer_count[1];
    stats_.track_observer_pairs += pairs_c + pairs_z;
    if (fuse_) stats_.fused_track_observer_pairs += pairs_c;
  }

  void fetch_counters(DeviceCounters& host) {
    check(cudaMemcpyAsync(&host, counters_.ptr, sizeof(host), cudaMemcpyDeviceToHost, stream_),
          "counter download");
    check(cudaMemcpyAsync(&stats_.window_reruns, reruns_.ptr, sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, stream_),
          "counter download");
    check(cudaMemcpyAsync(&stats_.window_handbacks, reruns_.ptr + 1, sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, stream_),
          "counter download");
    check(cudaStreamSynchronize(stream_), "counter fence");
    stats_.lepton_tracks = host.valid_tracks;
    stats_.coreas_contributions = host.coreas_contributions;
    stats_.zhs_contributions = host.zhs_contributions;
    stats_.zhs_subtracks = host.zhs_subtracks;
    stats_.fixed_point_overflows = host.fixed_point_overflows;
    std::memcpy(&stats_.counters, &host, sizeof(host));
    stats_.device_to_host_bytes += sizeof(host);
  }

  cudaStream_t stream_ = nullptr;
  int device_ = 0;
  int sms_ = 148;
  int threads_ = 384;
  bool enabled_ = false;
  bool initialized_ = false;
  bool coreas_enabled_ = false, zhs_enabled_ = false, diagnostics_ = false;
  bool fixed_ = true, deterministic_ = true, fuse_ = false, count_samples_ = false;
  bool downloaded_ = false, sealed_ = false, timing_ = false;
  int kernel_ = C8R_KERNEL_AUTO;
  Precision precision_ = Precision::kFP64;
  bool study_ = false;
  TimeArithmetic arithmetic_ = TimeArithmetic::kDouble;
  double limit_ = 1.;
  c8r_tuning tuning_{};
  Propagation propagation_{};
  IngestTerms terms_{};  // source terms written at ingest (enabled: shared destination row)
  std::vector<double2> table_host_;
  std::vector<c8r_observer_snapshot> snapshots_[2];
  std::vector<ObserverCache> observers_host_[2];
  std::size_t bins_[2] = {0, 0};
  std::size_t config_bins_[2] = {0, 0};  // all configured observers (snapshot extents)
  uint64_t max_observer_bins_[2] = {0, 0};
  std::size_t window_bins_ = 0;
  std::size_t largest_bins_ = 0;  // longest trace of the configured observers
  DeviceBuffer<double2> table_;
  DeviceBuffer<ObserverCache> observers_[2];
  DeviceBuffer<unsigned long long> fixed_traces_[2];
  DeviceBuffer<double> float_traces_[2];
  DeviceBuffer<double> decoded_[2];
  DeviceBuffer<uint64_t> decode_offsets_[2];
  DeviceBuffer<double> decode_factors_[2];
  DeviceBuffer<DeviceCounters> counters_;
  DeviceBuffer<unsigned long long> slot_;
  DeviceBuffer<unsigned> next_item_;
  DeviceBuffer<unsigned long long> reruns_;  // windowed items re-run with checked adds, handed back
  DeviceBuffer<unsigned> deferred_[2];  // per-CTA deferred-pair lists, by algorithm
  DeviceBuffer<double> tracks_;
  std::size_t capacity_ = 0;
  std::size_t staged_ = 0;  // records ingested since the last projection (upper bound of tracks)
  DeviceBuffer<c8r_lepton_transport_record> staging_, staging2_;
  cudaStream_t copy_stream_ = nullptr;
  cudaEvent_t copy_done_[2] = {nullptr, nullptr};
  cudaEvent_t consumed_[2] = {nullptr, nullptr};
  cudaStream_t side_stream_ = nullptr;               // ZHS launches beside CoREAS
  cudaEvent_t side_events_[2] = {nullptr, nullptr};  // tracks ingested, ZHS done
  PinnedBuffer<c8r_lepton_transport_record> host_[2];
  cudaEvent_t host_ready_[2] = {nullptr, nullptr};
  // (begin, end) event pairs; tag -1 = a whole accumulate's projection,
  // 0 / 1 = the windowed CoREAS / ZHS launch inside it
  std::vector<std::pair<std::pair<cudaEvent_t, cudaEvent_t>, int>> pending_;
  std::vector<cudaEvent_t> free_events_, all_events_;
  int host_index_ = 0;
  std::size_t host_count_ = 0;
  std::size_t host_batch_ = kDefaultHostBatch;
  c8r_statistics stats_{};
};


// Batched projection (many showers per launch): the staged tracks of many
// accumulators projected by one persistent launch per algorithm (up to
// kMaxEventsPerLaunch events a launch), optionally replayed from a CUDA graph
// captured per distinct launch plan.
class Batch {
 public:
  explicit Batch(cudaStream_t stream) : stream_(stream) {
    next_item_.allocate(1);
  }
  ~Batch() {
    if (stream_) cudaStreamSynchronize(stream_);
    for (auto& g : graphs_) {
      cudaGraphExecDestroy(g.second.exec);
      cudaGraphDestroy(g.second.graph);
    }
  }

  void project(Accumulator* const* events, std::size_t n, int flags) {
    auto plans = plan(events, n);
    if (plans.launches.empty()) return;
    bool const graph = (flags & C8R_BATCH_GRAPH) != 0;
    if (graph) {
      if (stream_ == nullptr)
        throw std::invalid_argument("graph replay needs a non-default CUDA stream");
      std::string key(reinterpret_cast<char const*>(plans.launches.data()),
                      plans.launches.size() * sizeof(Launch));
      auto it = graphs_.find(key);
      if (it == graphs_.end()) {
        Graph g{};
        check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "graph capture");
        try {
          enqueue(plans);
        } catch (...) {
          cudaGraph_t discard = nullptr;
          cudaStreamEndCapture(stream_, &discard);
          if (discard) cudaGraphDestroy(discard);
          throw;
        }
        check(cudaStreamEndCapture(stream_, &g.graph), "graph capture");
        check(cudaGraphInstantiate(&g.exec, g.graph, 0), "graph instantiate");
        it = graphs_.emplace(std::move(key), g).first;
        ++captures_;
      }
      check(cudaGraphLaunch(it->second.exec, stream_), "graph launch");
    } else {
      enqueue(plans);
    }
    for (std::size_t i = 0; i < n; ++i) {
      if (!events[i]->enabled() || events[i]->staged() == 0) continue;
      events[i]->note_batch_projection(events[i]->staged(), plans.items[i]);
      if (!(flags & C8R_BATCH_KEEP_STAGED)) events[i]->clear_staged();
    }
  }

  // Sweeps the tile space of the windowed kernel on the staged events, keeps
  // the fastest, and zeroes the traces it wrote.  The kernel's tile is one
  // antenna's window per CTA, a stage of `team_size` track segments (one per
  // thread) and work items of `track_tile_size` tracks; the sweep takes team
  // size {256, 384, 512, 640} x tracks per item {auto, 32768, 131072, 524288}
  // with the whole trace as window, then, at the best pair, bin windows of
  // {2048, 1024, 512} shorter than the longest trace (bins past a window go
  // to checked global atomics).
  c8r_tuning autotune(Accumulator* const* events, std::size_t n, int repetitions, double& best_ms) {
    static constexpr uint64_t kTeams[] = {256, 384, 512, 640};
    static constexpr uint64_t kChunks[] = {0, 32768, 131072, 524288};
    static constexpr uint64_t kWindows[] = {2048, 1024, 512};
    c8r_tuning best{};
    best_ms = -1.;
    cudaEvent_t a = nullptr, b = nullptr;
    check(cudaEventCreate(&a), "event");
    check(cudaEventCreate(&b), "event");
    auto trial = [&](c8r_tuning const& t) {
      for (std::size_t i = 0; i < n; ++i) events[i]->set_tuning(t);
      project(events, n, C8R_BATCH_KEEP_STAGED);  // warm
      check(cudaEventRecord(a, stream_), "event");
      for (int r = 0; r < repetitions; ++r) project(events, n, C8R_BATCH_KEEP_STAGED);
      check(cudaEventRecord(b, stream_), "event");
      check(cudaEventSynchronize(b), "event");
      float ms = 0.f;
      check(cudaEventElapsedTime(&ms, a, b), "event time");
      double const per = ms / repetitions;
      if (best_ms < 0. || per < best_ms) {
        best_ms = per;
        best = t;
      }
    };
    for (uint64_t team : kTeams) {
      for (uint64_t chunk : kChunks) {
        c8r_tuning t{};
        t.team_size = team;
        t.track_tile_size = chunk;
        trial(t);
      }
    }
    std::size_t longest = 0;
    for (std::size_t i = 0; i < n; ++i) longest = std::max(longest, events[i]->largest_bins());
    c8r_tuning const pair = best;
    for (uint64_t window : kWindows) {
      if (window >= longest) continue;
      c8r_tuning t = pair;
      t.observer_tile_size = window;
      trial(t);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (std::size_t i = 0; i < n; ++i) {
      events[i]->set_tuning(best);
      events[i]->zero_traces();
    }
    return best;
  }

  uint64_t captures() const { return captures_; }

 private:
  struct Launch {
    WorkPlan plan;
    int ctas;
    int threads;
  };
  struct Plans {
    std::vector<Launch> launches;
    std::vector<uint64_t> items;  // work items per event
    bool fixed = true;
    Precision precision = Precision::kFP64;
  };
  struct Graph {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
  };

  Plans plan(Accumulator* const* events, std::size_t n) {
    Plans out;
    out.items.assign(n, 0);
    std::vector<std::pair<std::size_t, EventPlan>> active;
    bool fixed = true;
    Precision precision = Precision::kFP64;
    int threads = 0;
    uint32_t window = 1;
    for (std::size_t i = 0; i < n; ++i) {
      Accumulator* e = events[i];
      if (e == nullptr) throw std::invalid_argument("null radio accumulator in batch");
      if (!e->enabled() || e->staged() == 0) continue;
      if (e->sealed()) throw std::logic_error("radio endpoint already committed; reset before new tracks");
      if (e->stream() != stream_) throw std::invalid_argument("batched accumulators must share the batch stream");
      if (e->study()) throw std::invalid_argument("precision-study accumulators cannot be batched");
      EventPlan ev = e->event_plan(e->staged());
      if (active.empty()) {
        fixed = e->fixed();
        precision = e->precision();
        threads = e->threads();
      } else if (e->fixed() != fixed || e->precision() != precision) {
        throw std::invalid_argument("batched accumulators must share precision and trace mode");
      }
      window = std::max(window, ev.window);
      active.push_back({i, ev});
    }
    if (active.empty()) return out;
    out.fixed = fixed;
    out.precision = precision;
    int device = 0, sms = 0;
    check(cudaGetDevice(&device), "device");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    int const per_sm = windowed_ctas_per_sm(static_cast<int>(window), threads, fixed, precision);
    if (per_sm <= 0) throw cuda_error("windowed radio kernel does not fit on this device");
    for (int algorithm = 0; algorithm < 2; ++algorithm) {
      for (std::size_t first = 0; first < active.size();) {
        Launch l;
        std::memset(&l, 0, sizeof l);  // zero padding: the launch bytes key the graph cache
        l.plan.algorithm = algorithm;
        l.plan.window = window;
        l.plan.next_item = next_item_.ptr;
        l.threads = threads;
        uint64_t ctas = static_cast<uint64_t>(per_sm) * sms;
        // the events of this launch; the last one ends the work list on short items
        // at most kMaxEventsPerLaunch events and, for two-pass (fixed-point
        // ZHS) launches, past the first event kMaxPairsPerLaunch pairs: their
        // first pass's lists grow with the launch's pairs
        std::vector<std::size_t> members;
        std::size_t j = first;
        uint64_t pairs = 0;
        for (; j < active.size() && members.size() < static_cast<std::size_t>(kMaxEventsPerLaunch); ++j) {
          EventPlan const& e = active[j].second;
          if (e.observer_count[algorithm] == 0) continue;
          uint64_t const p = static_cast<uint64_t>(e.chunks) * e.chunk_size * e.observer_count[algorithm];
          if (algorithm == 1 && fixed && !members.empty() && pairs + p > kMaxPairsPerLaunch) break;
          members.push_back(j);
          pairs += p;
        }
        first = j;
        if (members.empty()) continue;
        for (std::size_t m = 0; m < members.size(); ++m)
          out.items[active[members[m]].first] +=
              append_work(l.plan, active[members[m]].second, ctas, m + 1 == members.size());
        uint64_t const items = l.plan.total_items;
        if (ctas > items) ctas = items;
        l.plan.deferred_stride = deferred_list_stride(l.plan);
        l.ctas = static_cast<int>(ctas);
        out.launches.push_back(l);
      }
    }
    // one list storage for every launch (they run one after the other), sized
    // for the largest before any launch points into it: growing it between
    // launches would leave the earlier ones on the freed storage
    uint64_t words = 0;
    for (auto const& l : out.launches)
      words = std::max(words, deferred_words(l.plan, static_cast<uint64_t>(l.ctas), fixed));
    unsigned* const storage = deferred_lists(words);
    for (auto& l : out.launches) attach_deferred(l.plan, storage, static_cast<uint64_t>(l.ctas), fixed);
    return out;
  }

  void enqueue(Plans const& plans) {
    for (auto const& l : plans.launches) {
      check(cudaMemsetAsync(next_item_.ptr, 0, sizeof(unsigned), stream_), "memset");
      check(launch_windowed(l.plan, plans.fixed, plans.precision, l.ctas, l.threads, stream_),
            "batched windowed launch");
    }
  }

  cudaStream_t stream_ = nullptr;
  // The launches' per-CTA deferred-pair lists (the launches run one after the
  // other), grown after the batch stream's earlier work when a plan needs
  // more; captured graphs that name the old lists are dropped.
  unsigned* deferred_lists(uint64_t entries) {
    if (deferred_.count < entries) {
      check(cudaStreamSynchronize(stream_), "deferred list fence");
      for (auto& g : graphs_) {
        cudaGraphExecDestroy(g.second.exec);
        cudaGraphDestroy(g.second.graph);
      }
      graphs_.clear();
      DeviceBuffer<unsigned> fresh;
      fresh.allocate(entries + entries / 4);  // a quarter more: each growth synchronises
      deferred_.swap(fresh);
    }
    return deferred_.ptr;
  }

  DeviceBuffer<unsigned> next_item_;
  DeviceBuffer<unsigned> deferred_;
  std::map<std::string, Graph> graphs_;
  uint64_t captures_ = 0;
};

}  // namespace c8r

// ============================================================== C boundary
struct c8r_accumulator {
  c8r::Accumulator* impl = nullptr;
  std::string error;
};

struct c8r_batch {
  c8r::Batch* impl = nullptr;
  std::string error;
};

namespace {

thread_local std::string g_last_error;

using c8r::guarded;

int with_handle(c8r_accumulator const* h, std::string* error_slot, bool need) {
  (void)error_slot;
  if (h == nullptr || (need && h->impl == nullptr)) {
    g_last_error = "null radio accumulator handle";
    return C8R_INVALID_ARGUMENT;
  }
  return C8R_OK;
}

}  // namespace

namespace c8r {
// Error text of entry points defined in other files (c8r_last_global_error).
void set_global_error(char const* message) { g_last_error = message; }
}  // namespace c8r

extern "C" {

// Part of the tuning cache's key: raised whenever the kernels' launch shapes
// change, so that a tile tuned for earlier kernels is not applied to these.
const char* c8r_version(void) { return "c8radio-b200 1.1 (sm_100a)"; }

const char* c8r_last_error(const c8r_accumulator* handle) {
  if (handle == nullptr) return g_last_error.c_str();
  return handle->error.c_str();
}

const char* c8r_last_global_error(void) { return g_last_error.c_str(); }

int c8r_config_validate(const c8r_config* config) {
  return guarded(&g_last_error, [&] {
    if (!config) throw std::invalid_argument("null radio config");
    c8r::validate(*config);
  });
}

int c8r_projected_device_bytes(const c8r_config* config, size_t* bytes) {
  return guarded(&g_last_error, [&] {
    if (!config || !bytes) throw std::invalid_argument("null argument");
    *bytes = c8r::projected_device_bytes(*config);
  });
}

int c8r_create(const c8r_config* config, const c8r_tuning* tuning, void* stream,
               c8r_accumulator** handle) {
  return guarded(&g_last_error, [&] {
    if (!config || !handle) throw std::invalid_argument("null argument");
    *handle = nullptr;
    c8r_tuning const t = tuning ? *tuning : c8r_tuning{};
    auto* h = new c8r_accumulator;
    try {
      h->impl = new c8r::Accumulator(*config, t, static_cast<cudaStream_t>(stream));
    } catch (...) {
      delete h;
      throw;
    }
    *handle = h;
  });
}

void c8r_destroy(c8r_accumulator* handle) {
  if (!handle) return;
  delete handle->impl;
  delete handle;
}

int c8r_enabled(const c8r_accumulator* handle, int* enabled) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  if (!enabled) return C8R_INVALID_ARGUMENT;
  *enabled = handle->impl->enabled() ? 1 : 0;
  return C8R_OK;
}

int c8r_reset(c8r_accumulator* handle) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] { handle->impl->reset(); });
}

int c8r_enqueue_host(c8r_accumulator* handle, const c8r_lepton_transport_record* records,
                     size_t count) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] { handle->impl->enqueue_host(records, count); });
}

int c8r_flush(c8r_accumulator* handle) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] { handle->impl->flush(); });
}

int c8r_accumulate_device(c8r_accumulator* handle, const c8r_lepton_transport_record* records,
                          size_t count, size_t extent) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error,
                 [&] { handle->impl->accumulate_device(records, count, extent); });
}

int c8r_download(c8r_accumulator* handle, double* coreas_xyz, double* zhs_xyz,
                 c8r_counters* counters) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] { handle->impl->download(coreas_xyz, zhs_xyz, counters); });
}

int c8r_download_fixed(c8r_accumulator* handle, long long* coreas_xyz, long long* zhs_xyz,
                       c8r_counters* counters) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error,
                 [&] { handle->impl->download_fixed(coreas_xyz, zhs_xyz, counters); });
}

int c8r_download_fixed_snapshot(c8r_accumulator* handle, const char* shower_identity, uint32_t endpoint,
                                long long* coreas_xyz, long long* zhs_xyz, c8r_counters* counters) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] {
    handle->impl->download_fixed_snapshot(shower_identity, endpoint, coreas_xyz, zhs_xyz, counters);
  });
}

int c8r_snapshot_bins(const c8r_accumulator* handle, size_t* coreas_bins, size_t* zhs_bins) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  if (coreas_bins) *coreas_bins = handle->impl->config_bins(0);
  if (zhs_bins) *zhs_bins = handle->impl->config_bins(1);
  return C8R_OK;
}

int c8r_accumulate_columns(c8r_accumulator* handle, const c8r_track_columns* columns, size_t count) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] {
    if (!columns) throw std::invalid_argument("null radio track columns");
    handle->impl->accumulate_columns(*columns, count);
  });
}

int c8r_download_fields_device(c8r_accumulator* handle, double* coreas_field_xyz, double* zhs_field_xyz,
                               c8r_counters* counters) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error,
                 [&] { handle->impl->download_fields_device(coreas_field_xyz, zhs_field_xyz, counters); });
}

// merge_fixed_accumulators (FixedAccumulatorMerge.inl:12-29) without the layout
// labels: every bin checked before any is written.
int c8r_merge_fixed(long long* destination, const long long* source, size_t count) {
  return guarded(&g_last_error, [&] {
    if (count && (!destination || !source)) throw std::invalid_argument("null argument");
    for (size_t i = 0; i < count; ++i) {
      long long const x = destination[i], y = source[i];
      if ((y > 0 && x > std::numeric_limits<long long>::max() - y) ||
          (y < 0 && x < std::numeric_limits<long long>::min() - y))
        throw std::overflow_error("cooperative fixed-point accumulation overflow");
    }
    for (size_t i = 0; i < count; ++i) destination[i] += source[i];
  });
}

int c8r_total_bins(const c8r_accumulator* handle, size_t* coreas_bins, size_t* zhs_bins) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  if (coreas_bins) *coreas_bins = handle->impl->bins(0);
  if (zhs_bins) *zhs_bins = handle->impl->bins(1);
  return C8R_OK;
}

int c8r_get_statistics(const c8r_accumulator* handle, c8r_statistics* statistics) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  if (!statistics) return C8R_INVALID_ARGUMENT;
  auto* h = const_cast<c8r_accumulator*>(handle);
  return guarded(&h->error, [&] { h->impl->statistics(*statistics); });
}

int c8r_device_bytes(const c8r_accumulator* handle, size_t* bytes) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  if (!bytes) return C8R_INVALID_ARGUMENT;
  *bytes = handle->impl->device_bytes();
  return C8R_OK;
}

int c8r_static_host_to_device_bytes(const c8r_accumulator* handle, size_t* bytes) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  if (!bytes) return C8R_INVALID_ARGUMENT;
  *bytes = handle->impl->static_host_to_device_bytes();
  return C8R_OK;
}

int c8r_reserve(c8r_accumulator* handle, size_t count) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] { handle->impl->reserve(count); });
}

int c8r_projected_track_capacity(const c8r_accumulator* handle, size_t count,
                                 size_t* retained_bytes, size_t* transient_peak_bytes) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  std::size_t r = 0, p = 0;
  int const status = guarded(const_cast<std::string*>(&handle->error),
                             [&] { handle->impl->projected_track_capacity(count, r, p); });
  if (retained_bytes) *retained_bytes = r;
  if (transient_peak_bytes) *transient_peak_bytes = p;
  return status;
}

int c8r_set_kernel_timing(c8r_accumulator* handle, int enabled) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  handle->impl->set_timing(enabled != 0);
  return C8R_OK;
}

int c8r_stage_device(c8r_accumulator* handle, const c8r_lepton_transport_record* records,
                     size_t count, size_t extent) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] { handle->impl->stage_device(records, count, extent); });
}

int c8r_project_staged(c8r_accumulator* handle) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] { handle->impl->project_staged(true); });
}

int c8r_set_tuning(c8r_accumulator* handle, const c8r_tuning* tuning) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  if (!tuning) return C8R_INVALID_ARGUMENT;
  return guarded(&handle->error, [&] { handle->impl->set_tuning(*tuning); });
}

int c8r_batch_create(void* stream, c8r_batch** batch) {
  return guarded(&g_last_error, [&] {
    if (!batch) throw std::invalid_argument("null argument");
    auto* b = new c8r_batch;
    try {
      b->impl = new c8r::Batch(static_cast<cudaStream_t>(stream));
    } catch (...) {
      delete b;
      throw;
    }
    *batch = b;
  });
}

void c8r_batch_destroy(c8r_batch* batch) {
  if (!batch) return;
  delete batch->impl;
  delete batch;
}

const char* c8r_batch_last_error(const c8r_batch* batch) {
  return batch ? batch->error.c_str() : g_last_error.c_str();
}

static std::vector<c8r::Accumulator*> unwrap(c8r_accumulator* const* events, size_t count) {
  if (count != 0 && events == nullptr) throw std::invalid_argument("null radio accumulator list");
  std::vector<c8r::Accumulator*> out(count);
  for (size_t i = 0; i < count; ++i) {
    if (events[i] == nullptr || events[i]->impl == nullptr)
      throw std::invalid_argument("null radio accumulator in batch");
    out[i] = events[i]->impl;
  }
  return out;
}

int c8r_batch_project(c8r_batch* batch, c8r_accumulator* const* events, size_t count, int flags) {
  if (!batch || !batch->impl) return C8R_INVALID_ARGUMENT;
  return guarded(&batch->error, [&] {
    auto list = unwrap(events, count);
    batch->impl->project(list.data(), list.size(), flags);
  });
}

int c8r_batch_autotune(c8r_batch* batch, c8r_accumulator* const* events, size_t count,
                       int repetitions, c8r_tuning* best, double* best_ms) {
  if (!batch || !batch->impl) return C8R_INVALID_ARGUMENT;
  return guarded(&batch->error, [&] {
    auto list = unwrap(events, count);
    double ms = 0.;
    c8r_tuning const t = batch->impl->autotune(list.data(), list.size(), repetitions > 0 ? repetitions : 1, ms);
    if (best) *best = t;
    if (best_ms) *best_ms = ms;
  });
}

int c8r_batch_graph_captures(const c8r_batch* batch, unsigned long long* captures) {
  if (!batch || !batch->impl || !captures) return C8R_INVALID_ARGUMENT;
  *captures = batch->impl->captures();
  return C8R_OK;
}

int c8r_synchronize(c8r_accumulator* handle) {
  if (int s = with_handle(handle, nullptr, true)) return s;
  return guarded(&handle->error, [&] { handle->impl->synchronize(); });
}

}  // extern "C"
