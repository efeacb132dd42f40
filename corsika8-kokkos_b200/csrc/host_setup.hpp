// host_setup.hpp — host-side set-up shared by the accumulator, the
// no-allocation entry point and the server: the per-observer constants of
// RadioAccumulator::makeObservers (corsika/detail/kokkos/radio/RadioAccumulator.inl:522-550)
// plus those the projection evaluates inline, with the same IEEE operations
// (this file is compiled with -ffp-contract=off).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>

#include "../../include/c8radio.h"
#include "radio_device.cuh"

namespace c8r {

// `table_at(i)` returns {refractivity[i], integratedRefractivity[i]}.
template <class TableAt>
ObserverCache make_observer_cache(c8r_observer_snapshot const& s, int algorithm, bool homogeneous,
                                  double minimum_height, double inverse_step, TableAt table_at,
                                  bool deterministic, double limit, bool count_samples,
                                  std::size_t offset) {
  ObserverCache o;
  std::memset(&o, 0, sizeof o);
  o.px = s.position_m[0];
  o.py = s.position_m[1];
  o.pz = s.position_m[2];
  o.start_time = s.start_time_s;
  o.end_time = s.start_time_s + s.duration_s;               // RadioProjection.inl:273
  o.sample_rate = s.sample_rate_hz;
  o.resolution = 1. / s.sample_rate_hz;                     // :374, :396
  o.wavelength = kSpeedOfLight / s.sample_rate_hz;          // :492
  double const factor = algorithm == 1 ? s.sample_rate_hz : 1.;
  o.fixed_scale = deterministic ? kHeadroom * factor / limit : 1.;  // RadioAccumulator.inl:537-540
  o.fixed_scale_f = static_cast<float>(o.fixed_scale);
  o.count_samples = count_samples ? 1u : 0u;
  o.bins_d = static_cast<double>(s.number_of_bins);
  o.bins = s.number_of_bins;
  o.offset = offset;
  if (!homogeneous) {  // destination bin of propagate, RadioProjection.inl:184-192
    o.dest_height = (s.position_m[2] - minimum_height) * inverse_step;
    o.dest_index = static_cast<uint64_t>(o.dest_height + 0.5);
    auto const entry = table_at(o.dest_index);
    o.dest_n = entry.x + 1.;
    o.dest_integral = entry.y;
  }
  return o;
}

// Decode factor of downloadSet (RadioAccumulator.inl:865-867): fixed value x
// this = V/m (CoREAS) or V*s/m (ZHS).
inline double decode_factor(c8r_observer_snapshot const& s, int algorithm, double limit) {
  double const factor = algorithm == 1 ? s.sample_rate_hz : 1.;
  return limit / (kHeadroom * factor);
}

}  // namespace c8r
