// c8radio.hpp — header-only C++17 shim over the C ABI of libc8radio.so.
//
// Restores the class, method names and exception classes of the reference's
// corsika::kokkos::radio::RadioAccumulator
// (corsika/kokkos/radio/RadioAccumulator.hpp:35-237) and the IRadioBackend
// contract (corsika/kokkos/radio/IRadioBackend.hpp:29-41), so a host caller
// switches by changing the include and the namespace.  The B200 library does
// the work; this header only converts types and status codes.
#pragma once

#include <cstddef>
#include <cstdint>
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

// Int64 traces of downloadFixed (FixedRadioSnapshot.hpp:18-24, without the
// cooperative identity fields).
struct FixedRadioSnapshot {
  std::vector<long long> coreas_{};
  std::vector<long long> zhs_{};
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

inline std::vector<RadioWaveform> split(std::vector<RadioObserverSnapshot> const& observers,
                                        std::vector<double> const& soa) {
  std::size_t total = 0;
  for (auto const& o : observers) total += static_cast<std::size_t>(o.number_of_bins);
  std::vector<RadioWaveform> out;
  out.reserve(observers.size());
  std::size_t offset = 0;
  for (auto const& o : observers) {
    auto const n = static_cast<std::size_t>(o.number_of_bins);
    RadioWaveform w;
    w.x_.assign(soa.begin() + offset, soa.begin() + offset + n);
    w.y_.assign(soa.begin() + total + offset, soa.begin() + total + offset + n);
    w.z_.assign(soa.begin() + 2 * total + offset, soa.begin() + 2 * total + offset + n);
    out.push_back(std::move(w));
    offset += n;
  }
  return out;
}
}  // namespace detail

// RadioAccumulator with the reference's method set.  `stream` is a
// cudaStream_t (nullptr = legacy default stream); the reference's Kokkos
// execution instance maps to it.  Move-only.
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
                  void* stream = nullptr) {
    if (handle_) throw std::logic_error("radio accumulator already initialized");
    config_ = requested;
    auto const c = detail::view(config_);
    c8r_tuning const t{tuning.batchSize_,       tuning.chunkSize_,        tuning.teamSize_,
                       tuning.trackTileSize_,   tuning.observerTileSize_, tuning.deviceQueues_};
    int const status = c8r_create(&c, &t, stream, &handle_);
    if (status != C8R_OK) detail::raise(status, c8r_last_global_error());
  }

  bool enabled() const noexcept {
    int on = 0;
    return handle_ && c8r_enabled(handle_, &on) == C8R_OK && on;
  }

  void reset() { check(c8r_reset(handle_)); }

  void enqueueHostLeptonTracks(LeptonTransportRecord const* records, std::size_t count) {
    check(c8r_enqueue_host(handle_, records, count));
  }

  void flushHostLeptonTracks() { check(c8r_flush(handle_)); }

  // `records` points to device memory holding `extent` records.
  void accumulateLeptonTracks(LeptonTransportRecord const* records, std::size_t count,
                              std::size_t extent) {
    check(c8r_accumulate_device(handle_, records, count, extent));
  }

  RadioWaveforms download() {
    RadioWaveforms out;
    if (!enabled()) return out;
    std::size_t cb = 0, zb = 0;
    check(c8r_total_bins(handle_, &cb, &zb));
    std::vector<double> coreas(3 * cb), zhs(3 * zb);
    check(c8r_download(handle_, coreas.empty() ? nullptr : coreas.data(),
                       zhs.empty() ? nullptr : zhs.data(), nullptr));
    if (config_.coreasEnabled_) out.coreas_ = detail::split(config_.coreasObservers_, coreas);
    if (config_.zhsEnabled_) out.zhs_ = detail::split(config_.zhsObservers_, zhs);
    return out;
  }

  FixedRadioSnapshot downloadFixed() {
    std::size_t cb = 0, zb = 0;
    check(c8r_total_bins(handle_, &cb, &zb));
    FixedRadioSnapshot out;
    out.coreas_.resize(3 * cb);
    out.zhs_.resize(3 * zb);
    check(c8r_download_fixed(handle_, out.coreas_.empty() ? nullptr : out.coreas_.data(),
                             out.zhs_.empty() ? nullptr : out.zhs_.data(), &out.counters_));
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

  void reserveTrackCapacity(std::size_t count) { check(c8r_reserve(handle_, count)); }

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
  void swap(RadioAccumulator& other) noexcept {
    std::swap(handle_, other.handle_);
    std::swap(config_, other.config_);
  }

  c8r_accumulator* handle_ = nullptr;
  RadioConfig config_{};
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
                            void* stream = nullptr) {
    accumulator_.initialize(config, tuning, stream);
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
