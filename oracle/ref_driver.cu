/*
 * ref_driver.cu — TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into
 * oracle/_ref/libc8ref.so from the reference's own, unmodified sources
 * (corsika/kokkos/radio/algorithms/RadioProjection.hpp and its .inl), which
 * compile in the host pass of nvcc without Kokkos once an atomics policy is
 * supplied.  This is the reference's production FP64 projection run on the
 * host cores; it pins the C restatement and serves as the timed CPU
 * baseline.  Only the driver loop below is written here: a per-thread
 * private trace row and a checked merge, as the reference's OpenMP backend
 * does (corsika/detail/kokkos/radio/RadioAccumulator.inl:718-791,
 * RadioAccumulatorOperations.inl:48-60).
 */
#include <corsika/kokkos/radio/algorithms/RadioProjection.hpp>

#include <cstddef>
#include <cstring>
#include <vector>
#include <omp.h>

#include "../include/c8radio.h"

namespace cr = corsika::kokkos::radio;
namespace ck = corsika::kokkos;

static_assert(sizeof(ck::LeptonTransportRecord) == sizeof(c8r_lepton_transport_record),
              "record layout");
static_assert(offsetof(ck::LeptonTransportRecord, start_) ==
                  offsetof(c8r_lepton_transport_record, start),
              "record layout");
static_assert(offsetof(ck::LeptonTransportRecord, end_) ==
                  offsetof(c8r_lepton_transport_record, end),
              "record layout");
static_assert(sizeof(cr::RadioCounters) == sizeof(c8r_counters), "counter layout");

namespace {
  /* Plain (single-owner) operations with the reference's previous-value
   * contract: every worker writes only its private row and counters. */
  struct PrivateOperations {
    __host__ __device__ static long long add(long long* address, long long value) {
      auto* storage = reinterpret_cast<unsigned long long*>(address);
      auto previous = *storage;
      *storage = previous + static_cast<unsigned long long>(value);
      return static_cast<long long>(previous);
    }
    __host__ __device__ static unsigned long long add(unsigned long long* address,
                                                      unsigned long long value) {
      auto previous = *address;
      *address = previous + value;
      return previous;
    }
    __host__ __device__ static double add(double* address, double value) {
      auto previous = *address;
      *address = previous + value;
      return previous;
    }
    __host__ __device__ static void maximum(double* address, double value) {
      if (value > *address) *address = value;
    }
  };

  cr::RadioPropagationView propagation_view(c8r_config const& c) {
    cr::RadioPropagationView p{};
    auto const& s = c.propagation;
    p.homogeneousRefractiveIndex_ = s.homogeneous_refractive_index;
    p.minimumHeightM_ = s.minimum_height_m;
    p.maximumHeightM_ = s.maximum_height_m;
    p.stepM_ = s.step_m;
    p.inverseStepPerM_ = s.inverse_step_per_m;
    p.slopeRefractivityLower_ = s.slope_refractivity_lower;
    p.slopeIntegratedRefractivityLower_ = s.slope_integrated_refractivity_lower;
    p.slopeRefractivityUpper_ = s.slope_refractivity_upper;
    p.slopeIntegratedRefractivityUpper_ = s.slope_integrated_refractivity_upper;
    p.refractivity_ = s.refractivity;
    p.integratedRefractivity_ = s.integrated_refractivity;
    p.tableSize_ = s.table_size;
    p.zhsSubtrackRefinement_ = c.zhs_subtrack_refinement;
    return p;
  }

  /* The observer conversion of RadioAccumulator::makeObservers
   * (RadioAccumulator.inl:522-550), which lives in Kokkos-only code. */
  std::vector<cr::RadioObserverView> observer_views(c8r_observer_snapshot const* in,
                                                    std::size_t n, bool potential,
                                                    bool deterministic, double limit,
                                                    std::size_t& total) {
    std::vector<cr::RadioObserverView> out(n);
    total = 0;
    for (std::size_t i = 0; i < n; ++i) {
      auto& o = out[i];
      for (int a = 0; a < 3; ++a) o.positionM_[a] = in[i].position_m[a];
      o.startTimeS_ = in[i].start_time_s;
      o.durationS_ = in[i].duration_s;
      o.sampleRateHz_ = in[i].sample_rate_hz;
      auto factor = potential ? in[i].sample_rate_hz : 1.;
      o.fixedPointScale_ = deterministic ? cr::FixedPointHeadroom * factor / limit : 1.;
      o.inverseFixedPointScale_ = 1. / o.fixedPointScale_;
      o.numberOfBins_ = in[i].number_of_bins;
      o.waveformOffset_ = total;
      total += in[i].number_of_bins;
    }
    return out;
  }

  void merge(cr::RadioCounters& a, cr::RadioCounters const& b) {
    a.coreasContributions_ += b.coreasContributions_;
    a.zhsContributions_ += b.zhsContributions_;
    a.zhsSubtracks_ += b.zhsSubtracks_;
    a.validTracks_ += b.validTracks_;
    a.fixedPointOverflows_ += b.fixedPointOverflows_;
    a.weightedSegmentCount_ += b.weightedSegmentCount_;
    a.trackLengthM_ += b.trackLengthM_;
    a.weightedTrackLengthM_ += b.weightedTrackLengthM_;
    a.electronWeightedTrackLengthM_ += b.electronWeightedTrackLengthM_;
    a.positronWeightedTrackLengthM_ += b.positronWeightedTrackLengthM_;
    a.signedChargeWeightedTrackLengthM_ += b.signedChargeWeightedTrackLengthM_;
    a.energyWeightedTrackLengthGeVM_ += b.energyWeightedTrackLengthGeVM_;
    PrivateOperations::maximum(&a.maximumSegmentLengthM_, b.maximumSegmentLengthM_);
    a.weightedDirectionChangeRad_ += b.weightedDirectionChangeRad_;
    a.weightedDirectionChangeSquaredRad2_ += b.weightedDirectionChangeSquaredRad2_;
    a.weightedBetaDeficitTrackLengthM_ += b.weightedBetaDeficitTrackLengthM_;
    a.weightedTimeResidualS_ += b.weightedTimeResidualS_;
    PrivateOperations::maximum(&a.maximumDirectionChangeRad_, b.maximumDirectionChangeRad_);
    for (int i = 0; i < 3; ++i)
      a.signedChargeWeightedDirectionChange_[i] += b.signedChargeWeightedDirectionChange_[i];
    for (int i = 0; i < 15; ++i)
      a.weightedTrackLengthByKineticEnergyM_[i] += b.weightedTrackLengthByKineticEnergyM_[i];
  }
} // namespace

extern "C" {

/* Same contract as c8o_project in radio_oracle.h. */
int c8ref_project(c8r_config const* config, c8r_lepton_transport_record const* records,
                  std::size_t count, long long* coreas_fixed, long long* zhs_fixed,
                  double* coreas_floating, double* zhs_floating, c8r_counters* counters,
                  int threads) {
  if (!config || !counters || (count && !records)) return 1;
  bool const deterministic = config->deterministic != 0;
  std::size_t coreas_bins = 0, zhs_bins = 0;
  auto coreas = observer_views(config->coreas_observers,
                               config->coreas_enabled ? config->coreas_observer_count : 0,
                               false, deterministic, config->fixed_point_field_limit_v_per_m,
                               coreas_bins);
  auto zhs = observer_views(config->zhs_observers,
                            config->zhs_enabled ? config->zhs_observer_count : 0, true,
                            deterministic, config->fixed_point_field_limit_v_per_m, zhs_bins);
  auto const propagation = propagation_view(*config);
  if (threads <= 0) threads = 1;
  std::size_t const cv = 3 * coreas_bins, zv = 3 * zhs_bins;
  std::vector<long long> cfix, zfix;
  std::vector<double> cflt, zflt;
  if (deterministic) {
    cfix.assign(static_cast<std::size_t>(threads) * cv, 0);
    zfix.assign(static_cast<std::size_t>(threads) * zv, 0);
  } else {
    cflt.assign(static_cast<std::size_t>(threads) * cv, 0.);
    zflt.assign(static_cast<std::size_t>(threads) * zv, 0.);
  }
  std::vector<cr::RadioCounters> local(static_cast<std::size_t>(threads));
  bool const diagnostics = config->track_diagnostics != 0;
  auto const* input = reinterpret_cast<ck::LeptonTransportRecord const*>(records);

#pragma omp parallel num_threads(threads)
  {
    int const slot = omp_get_thread_num();
    cr::RadioWaveformView cw{}, zw{};
    if (deterministic) {
      auto* c = cfix.data() + slot * cv;
      auto* z = zfix.data() + slot * zv;
      cw.fixedX_ = c, cw.fixedY_ = c + coreas_bins, cw.fixedZ_ = c + 2 * coreas_bins;
      zw.fixedX_ = z, zw.fixedY_ = z + zhs_bins, zw.fixedZ_ = z + 2 * zhs_bins;
    } else {
      auto* c = cflt.data() + slot * cv;
      auto* z = zflt.data() + slot * zv;
      cw.floatingX_ = c, cw.floatingY_ = c + coreas_bins, cw.floatingZ_ = c + 2 * coreas_bins;
      zw.floatingX_ = z, zw.floatingY_ = z + zhs_bins, zw.floatingZ_ = z + 2 * zhs_bins;
    }
    auto* counter = &local[slot];
    std::size_t const observers = coreas.size() > zhs.size() ? coreas.size() : zhs.size();
#pragma omp for schedule(dynamic, 64)
    for (long long i = 0; i < static_cast<long long>(count); ++i) {
      cr::RadioTrackKinematics track{};
      if (!cr::record_track<PrivateOperations>(input[i], &track, counter, diagnostics))
        continue;
      for (std::size_t o = 0; o < observers; ++o) {
        if (o < coreas.size())
          cr::accumulate_co_reas<PrivateOperations>(track, propagation, coreas[o], cw, counter);
        if (o < zhs.size())
          cr::accumulate_zhs<PrivateOperations>(track, propagation, zhs[o], zw, counter);
      }
    }
  }

  unsigned long long merge_overflows = 0;
  auto fold = [&](std::vector<long long> const& rows, std::size_t values, long long* out) {
    for (std::size_t v = 0; v < values; ++v) {
      long long sum = out ? out[v] : 0;
      for (int s = 0; s < threads; ++s)
        if (!cr::checked_radio_atomic_add<PrivateOperations>(&sum, rows[s * values + v]))
          ++merge_overflows;
      if (out) out[v] = sum;
    }
  };
  auto fold_float = [&](std::vector<double> const& rows, std::size_t values, double* out) {
    for (std::size_t v = 0; v < values; ++v) {
      double sum = out ? out[v] : 0.;
      for (int s = 0; s < threads; ++s) sum += rows[s * values + v];
      if (out) out[v] = sum;
    }
  };
  if (deterministic) {
    fold(cfix, cv, coreas_fixed);
    fold(zfix, zv, zhs_fixed);
  } else {
    fold_float(cflt, cv, coreas_floating);
    fold_float(zflt, zv, zhs_floating);
  }
  auto* total = reinterpret_cast<cr::RadioCounters*>(counters);
  for (auto const& l : local) merge(*total, l);
  total->fixedPointOverflows_ += merge_overflows;
  return 0;
}

/* Primitive known-answer hooks (testRadioProjection.cpp:133-307). */
void c8ref_propagate(c8r_config const* config, double const source[3],
                     double const observer_position[3], double out[7]) {
  auto const p = propagation_view(*config);
  cr::RadioObserverView o{};
  for (int a = 0; a < 3; ++a) o.positionM_[a] = observer_position[a];
  auto const path = cr::propagate(p, {source[0], source[1], source[2]}, o);
  out[0] = path.propagationTimeS_;
  out[1] = path.refractiveIndexSource_;
  out[2] = path.refractiveIndexDestination_;
  out[3] = path.distanceM_;
  out[4] = path.emit_.x_;
  out[5] = path.emit_.y_;
  out[6] = path.emit_.z_;
}

double c8ref_doppler(double index, double const beta[3], double const emit[3]) {
  return cr::co_reas_doppler(index, {beta[0], beta[1], beta[2]}, {emit[0], emit[1], emit[2]});
}

double c8ref_nearest_bin(double x) { return cr::observer_nearest_bin(x); }

void c8ref_separate(double* start, double* end, double resolution, int signed_order) {
  cr::separate_same_bin_endpoints(*start, *end, resolution, signed_order != 0);
}

/* One add_sample on a single observer whose fixed (scale != 0) or floating
 * rows the caller provides; returns the contribution counter increment. */
unsigned long long c8ref_add_sample(double start, double duration, double rate,
                                    unsigned long long bins, int potential, double time,
                                    double const value[3], double scale, long long* fixed,
                                    double* floating, unsigned long long* overflows) {
  cr::RadioObserverView o{};
  o.startTimeS_ = start;
  o.durationS_ = duration;
  o.sampleRateHz_ = rate;
  o.numberOfBins_ = bins;
  o.fixedPointScale_ = scale;
  cr::RadioWaveformView w{};
  if (fixed) {
    w.fixedX_ = fixed, w.fixedY_ = fixed + bins, w.fixedZ_ = fixed + 2 * bins;
  } else {
    w.floatingX_ = floating, w.floatingY_ = floating + bins, w.floatingZ_ = floating + 2 * bins;
  }
  cr::RadioCounters counters{};
  unsigned long long contributions = 0;
  cr::RadioVector v{value[0], value[1], value[2]};
  if (potential)
    cr::add_sample<PrivateOperations, true>(o, w, time, v, &contributions, &counters);
  else
    cr::add_sample<PrivateOperations, false>(o, w, time, v, &contributions, &counters);
  *overflows += counters.fixedPointOverflows_;
  return contributions;
}

int c8ref_checked_add(long long* address, long long increment) {
  return cr::checked_radio_atomic_add<PrivateOperations>(address, increment) ? 1 : 0;
}

int c8ref_add_fixed_point(long long* address, double contribution, double scale) {
  return cr::add_radio_fixed_point<PrivateOperations>(address, contribution, scale) ? 1 : 0;
}

} // extern "C"
