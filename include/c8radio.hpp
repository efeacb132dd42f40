// c8radio.hpp — header-only C++17 shim over the C ABI of libc8radio.so.
//
// Restores the class, method names and exception classes of the reference's
// corsika::kokkos::radio::RadioAccumulator
// (corsika/kokkos/radio/RadioAccumulator.hpp:35-237), its cooperative export
// (FixedRadioSnapshot.hpp:18-24, CooperativeRadioMerge.hpp:45-66) and the
// IRadioBackend contract (corsika/kokkos/radio/IRadioBackend.hpp:29-41), so a
// host caller switches by changing the include and the namespace.  The B200
// library does the work; this header only converts types and status codes.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "c8radio.h"

namespace c8radio {

using LeptonTransportRecord = c8r_lepton_transport_record;
using RadioObserverSnapshot = c8r_observer_snapshot;
using RadioCounters = c8r_counters;
using RadioStatistics = c8r_statistics;

// The reference's execution-space instance maps to a CUDA stream: a
// Kokkos::Cuda instance passes exec.cuda_stream().  One accumulator works on
// the stream it was initialized with (the reference's one-owner, one-instance
// contract, IRadioBackend.hpp:27); a call given another non-default stream is
// rejected with std::invalid_argument.
struct CudaExecution {
  void* stream_{};
  CudaExecution() = default;
  CudaExecution(void* stream) : stream_(stream) {}  // NOLINT: implicit, as the reference's exec
};

// corsika/kokkos/scheduling/CooperativeEndpoint.hpp
enum class CooperativeEndpoint : unsigned { Cuda = C8R_ENDPOINT_CUDA, OpenMP = C8R_ENDPOINT_OPENMP };

// corsika/kokkos/radio/FlatAtmosphereRadioSnapshot.hpp:20-36
struct FlatAtmosphereRadioSnapshot {
  double homogeneousRefractiveIndex_{};
  double minimumHeightM_{};
  double maximumHeightM_{};
  double stepM_{};
  double inverseStepPerM_{};
  double slopeRefractivityLower_{};
  double slopeIntegratedRefractivityLower_{};
  double slopeRefractivityUpper_{};
  double slopeIntegratedRefractivityUpper_{};
  std::vector<double> refractivity_{};
  std::vector<double> integratedRefractivity_{};
};

// corsika/kokkos/radio/RadioConfig.hpp:21-53 (+ B200 precision/kernel choice)
struct RadioConfig {
  bool enabled_{};
  bool coreasEnabled_{true};
  bool zhsEnabled_{true};
  bool deterministic_{true};
  double fixedPointFieldLimitVPerM_{1.};
  bool trackDiagnostics_{};
  std::uint32_t zhsSubtrackRefinement_{1};
  FlatAtmosphereRadioSnapshot propagation_{};
  std::vector<RadioObserverSnapshot> coreasObservers_{};
  std::vector<RadioObserverSnapshot> zhsObservers_{};
  int precision_{C8R_PRECISION_FP64};
  int kernel_{C8R_KERNEL_AUTO};
  bool countSamples_{};
};

// corsika/kokkos/runtime/TuningParameters.hpp:14-21
struct TuningParameters {
  std::size_t batchSize_{};
  std::size_t chunkSize_{};
  std::size_t teamSize_{};
  std::size_t trackTileSize_{};
  std::size_t observerTileSize_{};
  std::size_t deviceQueues_{1};
};

// corsika/kokkos/radio/RadioWaveform.hpp:17-21 and RadioWaveforms.hpp:19-22
struct RadioWaveform {
  std::vector<double> x_{};
  std::vector<double> y_{};
  std::vector<double> z_{};
};
struct RadioWaveforms {
  std::vector<RadioWaveform> coreas_{};
  std::vector<RadioWaveform> zhs_{};
};

// corsika/kokkos/radio/FixedRadioSnapshot.hpp:18-24: owned final integer
// waveforms of one shower endpoint (ZHS as potential), SoA [X | Y | Z] over
// every configured observer of each algorithm.
struct FixedRadioSnapshot {
  std::string showerIdentity_{};
  CooperativeEndpoint endpoint_{};
  RadioConfig config_{};
  std::vector<std::int64_t> coreas_{};
  std::vector<std::int64_t> zhs_{};
  RadioCounters counters_{};
};

struct MemoryProjection {
  std::size_t retainedBytes_{};
  std::size_t transientPeakBytes_{};
};

namespace detail {
inline void raise(int status, char const* message) {
  std::string const text = message ? message : "";
  switch (status) {
    case C8R_OK: return;
    case C8R_INVALID_ARGUMENT: throw std::invalid_argument(text);
    case C8R_LOGIC_ERROR: throw std::logic_error(text);
    case C8R_OUT_OF_RANGE: throw std::out_of_range(text);
    case C8R_LENGTH_ERROR: throw std::length_error(text);
    case C8R_OVERFLOW_ERROR: throw std::overflow_error(text);
    default: throw std::runtime_error(text);
  }
}

// The C view of a RadioConfig borrows its vectors.
inline c8r_config view(RadioConfig const& c) {
  c8r_config out{};
  out.enabled = c.enabled_;
  out.coreas_enabled = c.coreasEnabled_;
  out.zhs_enabled = c.zhsEnabled_;
  out.deterministic = c.deterministic_;
  out.fixed_point_field_limit_v_per_m = c.fixedPointFieldLimitVPerM_;
  out.track_diagnostics = c.trackDiagnostics_;
  out.zhs_subtrack_refinement = c.zhsSubtrackRefinement_;
  auto const& p = c.propagation_;
  out.propagation = {p.homogeneousRefractiveIndex_,
                     p.minimumHeightM_,
                     p.maximumHeightM_,
                     p.stepM_,
                     p.inverseStepPerM_,
                     p.slopeRefractivityLower_,
                     p.slopeIntegratedRefractivityLower_,
                     p.slopeRefractivityUpper_,
                     p.slopeIntegratedRefractivityUpper_,
                     p.refractivity_.empty() ? nullptr : p.refractivity_.data(),
                     p.integratedRefractivity_.empty() ? nullptr : p.integratedRefractivity_.data(),
                     p.refractivity_.size()};
  out.coreas_observers = c.coreasObservers_.empty() ? nullptr : c.coreasObservers_.data();
  out.coreas_observer_count = c.coreasObservers_.size();
  out.zhs_observers = c.zhsObservers_.empty() ? nullptr : c.zhsObservers_.data();
  out.zhs_observer_count = c.zhsObservers_.size();
  out.precision = c.precision_;
  out.kernel = c.kernel_;
  out.count_samples = c.countSamples_;
  return out;
}

inline std::size_t bins(std::vector<RadioObserverSnapshot> const& observers) {
  std::size_t total = 0;
  for (auto const& o : observers) total += static_cast<std::size_t>(o.number_of_bins);
  return total;
}

// One RadioWaveform per observer from SoA values (decoded with `scale(i)`).
template <class T, class Scale>
std::vector<RadioWaveform> split(std::vector<RadioObserverSnapshot> const& observers, T const* soa,
                                 Scale scale) {
  std::size_t const total = bins(observers);
  std::vector<RadioWaveform> out;
  out.reserve(observers.size());
  std::size_t offset = 0;
  for (std::size_t k = 0; k < observers.size(); ++k) {
    auto const n = static_cast<std::size_t>(observers[k].number_of_bins);
    double const f = scale(k);
    RadioWaveform w;
    w.x_.resize(n);
    w.y_.resize(n);
    w.z_.resize(n);
    for (std::size_t i = 0; i < n; ++i) {
      w.x_[i] = static_cast<double>(soa[offset + i]) * f;
      w.y_[i] = static_cast<double>(soa[total + offset + i]) * f;
      w.z_[i] = static_cast<double>(soa[2 * total + offset + i]) * f;
    }
    out.push_back(std::move(w));
    offset += n;
  }
  return out;
}

inline c8r_fixed_snapshot view(FixedRadioSnapshot const& s, c8r_config const& config) {
  c8r_fixed_snapshot out{};
  out.shower_identity = s.showerIdentity_.c_str();
  out.endpoint = static_cast<std::uint32_t>(s.endpoint_);
  out.config = &config;
  out.coreas = reinterpret_cast<long long const*>(s.coreas_.data());
  out.coreas_count = s.coreas_.size();
  out.zhs = reinterpret_cast<long long const*>(s.zhs_.data());
  out.zhs_count = s.zhs_.size();
  out.counters = s.counters_;
  return out;
}
static_assert(sizeof(std::int64_t) == sizeof(long long), "int64 traces are long long in the C ABI");
}  // namespace detail

// validate_fixed_radio (CooperativeRadioMerge.inl:142-152).
inline void validate_fixed_radio(FixedRadioSnapshot const& s) {
  auto const c = detail::view(s.config_);
  auto const v = detail::view(s, c);
  if (int status = c8r_validate_fixed_snapshot(&v)) detail::raise(status, c8r_snapshot_last_error());
}

// merge_radio_counters (CooperativeRadioMerge.inl:154-208).
inline RadioCounters merge_radio_counters(RadioCounters a, RadioCounters const& b) {
  if (int status = c8r_merge_counters(&a, &b)) detail::raise(status, c8r_snapshot_last_error());
  return a;
}

// decode_fixed_radio (CooperativeRadioMerge.inl:210-238): int64 -> V/m (CoREAS)
// and V s/m (ZHS) with limit / (2^62 factor), factor = fs for ZHS.
inline RadioWaveforms decode_fixed_radio(FixedRadioSnapshot const& s) {
  validate_fixed_radio(s);
  RadioWaveforms out;
  double const limit = s.config_.fixedPointFieldLimitVPerM_;
  constexpr double kHeadroom = 4611686018427387904.0;  // 2^62
  out.coreas_ = detail::split(s.config_.coreasObservers_, s.coreas_.data(),
                              [&](std::size_t) { return limit / (kHeadroom * 1.); });
  out.zhs_ = detail::split(s.config_.zhsObservers_, s.zhs_.data(), [&](std::size_t k) {
    return limit / (kHeadroom * s.config_.zhsObservers_[k].sample_rate_hz);
  });
  return out;
}

// RadioAccumulator with the reference's method set.  Move-only.
class RadioAccumulator {
 public:
  static constexpr std::size_t HostTrackBatchCapacity = 4096;
  static constexpr std::size_t DirectProjectionTrackThreshold = 16384;

  RadioAccumulator() = default;
  RadioAccumulator(RadioAccumulator const&) = delete;
  RadioAccumulator& operator=(RadioAccumulator const&) = delete;
  RadioAccumulator(RadioAccumulator&& other) noexcept { swap(other); }
  RadioAccumulator& operator=(RadioAccumulator&& other) noexcept {
    swap(other);
    return *this;
  }
  ~RadioAccumulator() { c8r_destroy(handle_); }

  static std::size_t projectedDeviceBytes(RadioConfig const& requested) {
    auto const c = detail::view(requested);
    std::size_t bytes = 0;
    int const status = c8r_projected_device_bytes(&c, &bytes);
    if (status != C8R_OK) detail::raise(status, c8r_last_global_error());
    return bytes;
  }

  void initialize(RadioConfig const& requested, TuningParameters const& tuning = {},
                  CudaExecution const& execution = {}) {
    if (initialized_) throw std::logic_error("radio accumulator already initialized");
    config_ = requested;
    stream_ = execution.stream_;
    auto const c = detail::view(config_);
    c8r_tuning const t{tuning.batchSize_,       tuning.chunkSize_,        tuning.teamSize_,
                       tuning.trackTileSize_,   tuning.observerTileSize_, tuning.deviceQueues_};
    int const status = c8r_create(&c, &t, stream_, &handle_);
    if (status != C8R_OK) detail::raise(status, c8r_last_global_error());
    initialized_ = true;
  }

  bool enabled() const noexcept {
    int on = 0;
    return handle_ && c8r_enabled(handle_, &on) == C8R_OK && on;
  }

  void reset(CudaExecution const& execution = {}) {
    same(execution);
    check(c8r_reset(handle_));
  }

  // Copies before returning (RadioAccumulator.hpp:110-115).
  void enqueueHostLeptonTracks(LeptonTransportRecord const* records, std::size_t count,
                               CudaExecution const& execution = {}) {
    same(execution);
    check(c8r_enqueue_host(handle_, records, count));
  }

  void flushHostLeptonTracks(CudaExecution const& execution = {}) {
    same(execution);
    check(c8r_flush(handle_));
  }

  // `records` points to device memory holding `extent` records (the
  // reference's track_input_view_type and its extent); borrowed until the
  // queued work completes.
  void accumulateLeptonTracks(LeptonTransportRecord const* records, std::size_t count,
                              std::size_t extent, CudaExecution const& execution = {}) {
    same(execution);
    check(c8r_accumulate_device(handle_, records, count, extent));
  }

  // Cooperative end-of-shower export (RadioAccumulator.hpp:123-127): the raw
  // int64 traces, no conversion or differentiation.
  FixedRadioSnapshot downloadFixed(std::string const& shower_identity, CooperativeEndpoint endpoint,
                                   CudaExecution const& execution = {}) {
    same(execution);
    if (!handle_) throw std::logic_error("fixed radio snapshot unavailable/already committed");
    FixedRadioSnapshot out;
    std::size_t cb = 0, zb = 0;
    check(c8r_snapshot_bins(handle_, &cb, &zb));
    out.coreas_.resize(3 * cb);
    out.zhs_.resize(3 * zb);
    check(c8r_download_fixed_snapshot(handle_, shower_identity.c_str(), static_cast<std::uint32_t>(endpoint),
                                      reinterpret_cast<long long*>(out.coreas_.data()),
                                      reinterpret_cast<long long*>(out.zhs_.data()), &out.counters_));
    out.showerIdentity_ = shower_identity;
    out.endpoint_ = endpoint;
    out.config_ = config_;
    return out;
  }

  RadioWaveforms download(CudaExecution const& execution = {}) {
    same(execution);
    RadioWaveforms out;
    if (!enabled()) return out;
    std::size_t cb = 0, zb = 0;
    check(c8r_total_bins(handle_, &cb, &zb));
    std::vector<double> coreas(3 * cb), zhs(3 * zb);
    check(c8r_download(handle_, coreas.empty() ? nullptr : coreas.data(),
                       zhs.empty() ? nullptr : zhs.data(), nullptr));
    auto one = [](std::size_t) { return 1.; };
    if (config_.coreasEnabled_) out.coreas_ = detail::split(config_.coreasObservers_, coreas.data(), one);
    if (config_.zhsEnabled_) out.zhs_ = detail::split(config_.zhsObservers_, zhs.data(), one);
    return out;
  }

  RadioStatistics statistics() const {
    RadioStatistics s{};
    check(c8r_get_statistics(handle_, &s));
    return s;
  }

  std::size_t deviceBytes() const {
    std::size_t b = 0;
    if (handle_) check(c8r_device_bytes(handle_, &b));
    return b;
  }

  std::size_t staticHostToDeviceBytes() const {
    std::size_t b = 0;
    if (handle_) check(c8r_static_host_to_device_bytes(handle_, &b));
    return b;
  }

  void reserveTrackCapacity(std::size_t count, CudaExecution const& execution = {}) {
    same(execution);
    check(c8r_reserve(handle_, count));
  }

  MemoryProjection projectedTrackCapacity(std::size_t count) const {
    MemoryProjection m;
    check(c8r_projected_track_capacity(handle_, count, &m.retainedBytes_, &m.transientPeakBytes_));
    return m;
  }

  c8r_accumulator* native_handle() const noexcept { return handle_; }

 private:
  void check(int status) const {
    if (status != C8R_OK) detail::raise(status, c8r_last_error(handle_));
  }
  void same(CudaExecution const& execution) const {
    if (execution.stream_ != nullptr && execution.stream_ != stream_)
      throw std::invalid_argument("radio accumulator works on the execution instance it was initialized with");
  }
  void swap(RadioAccumulator& other) noexcept {
    std::swap(handle_, other.handle_);
    std::swap(config_, other.config_);
    std::swap(stream_, other.stream_);
    std::swap(initialized_, other.initialized_);
  }

  c8r_accumulator* handle_ = nullptr;
  RadioConfig config_{};
  void* stream_ = nullptr;
  bool initialized_ = false;
};

// CooperativeRadioMerge (CooperativeRadioMerge.hpp:53-65): accepts both
// endpoint snapshots of one shower once; rejects mismatch and overflow
// without changing what it holds.  Move-only.
class CooperativeRadioMerge {
 public:
  CooperativeRadioMerge(std::string identity, RadioConfig config)
      : identity_(std::move(identity)), config_(std::move(config)) {
    auto const c = detail::view(config_);
    if (int status = c8r_cooperative_merge_create(identity_.c_str(), &c, &merge_))
      detail::raise(status, c8r_snapshot_last_error());
  }
  CooperativeRadioMerge(CooperativeRadioMerge const&) = delete;
  CooperativeRadioMerge& operator=(CooperativeRadioMerge const&) = delete;
  CooperativeRadioMerge(CooperativeRadioMerge&& other) noexcept
      : identity_(std::move(other.identity_)), config_(std::move(other.config_)), merge_(other.merge_) {
    other.merge_ = nullptr;
  }
  ~CooperativeRadioMerge() { c8r_cooperative_merge_destroy(merge_); }

  void commit(FixedRadioSnapshot const& input) {
    auto const c = detail::view(input.config_);
    auto const v = detail::view(input, c);
    if (int status = c8r_cooperative_merge_commit(merge_, &v))
      detail::raise(status, c8r_cooperative_merge_last_error(merge_));
  }

  FixedRadioSnapshot take() {
    FixedRadioSnapshot out;
    out.showerIdentity_ = identity_;
    out.config_ = config_;
    out.coreas_.resize(3 * detail::bins(config_.coreasObservers_));
    out.zhs_.resize(3 * detail::bins(config_.zhsObservers_));
    std::uint32_t endpoint = 0;
    if (int status = c8r_cooperative_merge_take(merge_, reinterpret_cast<long long*>(out.coreas_.data()),
                                                reinterpret_cast<long long*>(out.zhs_.data()),
                                                &out.counters_, &endpoint))
      detail::raise(status, c8r_cooperative_merge_last_error(merge_));
    out.endpoint_ = static_cast<CooperativeEndpoint>(endpoint);
    return out;
  }

 private:
  std::string identity_;
  RadioConfig config_;
  c8r_cooperative_merge* merge_ = nullptr;
};

// IRadioBackend (IRadioBackend.hpp:29-41): host dispatch contract.
class IRadioBackend {
 public:
  virtual ~IRadioBackend() = default;
  virtual bool gpuRadioEnabled() const noexcept = 0;
  virtual void enqueueRadioTracks(LeptonTransportRecord const* records, std::size_t count) = 0;
  virtual RadioWaveforms downloadRadioWaveforms() = 0;
};

// An IRadioBackend that owns a B200 accumulator.
class B200RadioBackend final : public IRadioBackend {
 public:
  explicit B200RadioBackend(RadioConfig const& config, TuningParameters const& tuning = {},
                            CudaExecution const& execution = {}) {
    accumulator_.initialize(config, tuning, execution);
  }
  bool gpuRadioEnabled() const noexcept override { return accumulator_.enabled(); }
  void enqueueRadioTracks(LeptonTransportRecord const* records, std::size_t count) override {
    accumulator_.enqueueHostLeptonTracks(records, count);
  }
  RadioWaveforms downloadRadioWaveforms() override { return accumulator_.download(); }
  RadioAccumulator& accumulator() noexcept { return accumulator_; }

 private:
  RadioAccumulator accumulator_;
};

}  // namespace c8radio
