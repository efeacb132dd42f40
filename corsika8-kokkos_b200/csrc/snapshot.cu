// snapshot.cu — the cooperative fixed-point export of a shower endpoint, on
// the host: validation of a snapshot, the checked counter merge and the
// two-endpoint merge object, as corsika/detail/kokkos/radio/CooperativeRadioMerge.inl
// defines them (validate_fixed_radio :142-152, merge_radio_counters :154-208,
// CooperativeRadioMerge :240-277) over plain C views (c8r_fixed_snapshot).
// The export itself (RadioAccumulator::downloadFixed) is
// c8r_download_fixed_snapshot in accumulator.cu.
//
// Messages and exception classes are the reference's, so the C++ shim throws
// what a reference caller already catches.
#include <cmath>
#include <cstddef>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/c8radio.h"
#include "status.hpp"

namespace {

thread_local std::string g_error;

// radio_bins (CooperativeRadioMerge.inl:125-140): total bins, every observer
// checked.
std::size_t radio_bins(c8r_observer_snapshot const* observers, uint64_t count) {
  if (count != 0 && observers == nullptr) throw std::invalid_argument("invalid cooperative radio observer layout");
  std::size_t n = 0;
  for (uint64_t i = 0; i < count; ++i) {
    auto const& o = observers[i];
    if (!o.number_of_bins || o.number_of_bins > std::numeric_limits<std::size_t>::max() / 3 - n ||
        !std::isfinite(o.sample_rate_hz) || o.sample_rate_hz <= 0. || !std::isfinite(o.start_time_s) ||
        !std::isfinite(o.duration_s) || o.duration_s < 0.)
      throw std::invalid_argument("invalid cooperative radio observer layout");
    for (double x : o.position_m)
      if (!std::isfinite(x)) throw std::invalid_argument("nonfinite cooperative radio observer");
    n += static_cast<std::size_t>(o.number_of_bins);
  }
  return n;
}

// validate_fixed_radio (CooperativeRadioMerge.inl:142-152).
void validate_snapshot(c8r_fixed_snapshot const& s) {
  if (s.config == nullptr) throw std::invalid_argument("invalid/overflowed cooperative fixed radio snapshot");
  c8r_config const& c = *s.config;
  if (s.shower_identity == nullptr || s.shower_identity[0] == '\0' || !c.enabled || !c.deterministic ||
      (!c.coreas_enabled && !c.zhs_enabled) || !std::isfinite(c.fixed_point_field_limit_v_per_m) ||
      c.fixed_point_field_limit_v_per_m <= 0. || s.endpoint > 1 || s.counters.fixed_point_overflows)
    throw std::invalid_argument("invalid/overflowed cooperative fixed radio snapshot");
  if (s.coreas_count != 3 * radio_bins(c.coreas_observers, c.coreas_observer_count) ||
      s.zhs_count != 3 * radio_bins(c.zhs_observers, c.zhs_observer_count))
    throw std::invalid_argument("cooperative radio snapshot extent mismatch");
  if ((s.coreas_count && s.coreas == nullptr) || (s.zhs_count && s.zhs == nullptr))
    throw std::invalid_argument("cooperative radio snapshot extent mismatch");
}

// merge_radio_counters (CooperativeRadioMerge.inl:154-208): returns a + b, or
// throws std::overflow_error before anything is changed.
c8r_counters merge_counters(c8r_counters a, c8r_counters const& b) {
  auto add = [](unsigned long long x, unsigned long long y) {
    if (y > std::numeric_limits<unsigned long long>::max() - x)
      throw std::overflow_error("cooperative radio counter overflow");
    return x + y;
  };
  a.coreas_contributions = add(a.coreas_contributions, b.coreas_contributions);
  a.zhs_contributions = add(a.zhs_contributions, b.zhs_contributions);
  a.zhs_subtracks = add(a.zhs_subtracks, b.zhs_subtracks);
  a.valid_tracks = add(a.valid_tracks, b.valid_tracks);
  a.fixed_point_overflows = add(a.fixed_point_overflows, b.fixed_point_overflows);
  auto sum = [](double x, double y) {
    double const z = x + y;
    if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z))
      throw std::overflow_error("nonfinite cooperative radio diagnostics");
    return z;
  };
  a.weighted_segment_count = sum(a.weighted_segment_count, b.weighted_segment_count);
  a.track_length_m = sum(a.track_length_m, b.track_length_m);
  a.weighted_track_length_m = sum(a.weighted_track_length_m, b.weighted_track_length_m);
  a.electron_weighted_track_length_m = sum(a.electron_weighted_track_length_m, b.electron_weighted_track_length_m);
  a.positron_weighted_track_length_m = sum(a.positron_weighted_track_length_m, b.positron_weighted_track_length_m);
  a.signed_charge_weighted_track_length_m =
      sum(a.signed_charge_weighted_track_length_m, b.signed_charge_weighted_track_length_m);
  a.energy_weighted_track_length_gev_m =
      sum(a.energy_weighted_track_length_gev_m, b.energy_weighted_track_length_gev_m);
  a.weighted_direction_change_rad = sum(a.weighted_direction_change_rad, b.weighted_direction_change_rad);
  a.weighted_direction_change_squared_rad2 =
      sum(a.weighted_direction_change_squared_rad2, b.weighted_direction_change_squared_rad2);
  a.weighted_beta_deficit_track_length_m =
      sum(a.weighted_beta_deficit_track_length_m, b.weighted_beta_deficit_track_length_m);
  a.weighted_time_residual_s = sum(a.weighted_time_residual_s, b.weighted_time_residual_s);
  for (int i = 0; i < 3; ++i)
    a.signed_charge_weighted_direction_change[i] =
        sum(a.signed_charge_weighted_direction_change[i], b.signed_charge_weighted_direction_change[i]);
  for (int i = 0; i < 15; ++i)
    a.weighted_track_length_by_kinetic_energy_m[i] =
        sum(a.weighted_track_length_by_kinetic_energy_m[i], b.weighted_track_length_by_kinetic_energy_m[i]);
  // maxima are not additive: finite inputs, the larger kept
  for (double x : {a.maximum_segment_length_m, b.maximum_segment_length_m, a.maximum_direction_change_rad,
                   b.maximum_direction_change_rad})
    if (!std::isfinite(x)) throw std::overflow_error("nonfinite cooperative radio maximum");
  a.maximum_segment_length_m = std::max(a.maximum_segment_length_m, b.maximum_segment_length_m);
  a.maximum_direction_change_rad = std::max(a.maximum_direction_change_rad, b.maximum_direction_change_rad);
  return a;
}

// A deep copy of a c8r_config (its observer and table arrays owned).
struct OwnedConfig {
  c8r_config config{};
  std::vector<c8r_observer_snapshot> coreas, zhs;
  std::vector<double> refractivity, integrated;

  explicit OwnedConfig(c8r_config const& c) : config(c) {
    auto const& p = c.propagation;
    if (p.table_size) {
      if (p.refractivity == nullptr || p.integrated_refractivity == nullptr)
        throw std::invalid_argument("invalid flat-atmosphere radio snapshot");
      refractivity.assign(p.refractivity, p.refractivity + p.table_size);
      integrated.assign(p.integrated_refractivity, p.integrated_refractivity + p.table_size);
    }
    if (c.coreas_observer_count && c.coreas_observers == nullptr) throw std::invalid_argument("null radio observers");
    if (c.zhs_observer_count && c.zhs_observers == nullptr) throw std::invalid_argument("null radio observers");
    coreas.assign(c.coreas_observers, c.coreas_observers + c.coreas_observer_count);
    zhs.assign(c.zhs_observers, c.zhs_observers + c.zhs_observer_count);
    config.propagation.refractivity = refractivity.empty() ? nullptr : refractivity.data();
    config.propagation.integrated_refractivity = integrated.empty() ? nullptr : integrated.data();
    config.coreas_observers = coreas.empty() ? nullptr : coreas.data();
    config.zhs_observers = zhs.empty() ? nullptr : zhs.data();
  }
};

// same_observers (CooperativeRadioMerge.inl:79-91).
bool same_observers(c8r_observer_snapshot const* a, uint64_t na, c8r_observer_snapshot const* b, uint64_t nb) {
  if (na != nb) return false;
  for (uint64_t i = 0; i < na; ++i) {
    for (int d = 0; d < 3; ++d)
      if (a[i].position_m[d] != b[i].position_m[d]) return false;
    if (a[i].start_time_s != b[i].start_time_s || a[i].duration_s != b[i].duration_s ||
        a[i].sample_rate_hz != b[i].sample_rate_hz || a[i].number_of_bins != b[i].number_of_bins)
      return false;
  }
  return true;
}

bool same_table(double const* a, double const* b, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i)
    if (a[i] != b[i]) return false;
  return true;
}

// same_radio_physics (CooperativeRadioMerge.inl:93-123).  Of the B200
// extensions, count_samples changes what a trace holds (sample counts), so
// it must agree; precision and kernel do not change the units.
bool same_physics(c8r_config const& a, c8r_config const& b) {
  if (!!a.enabled != !!b.enabled || !!a.coreas_enabled != !!b.coreas_enabled ||
      !!a.zhs_enabled != !!b.zhs_enabled || !!a.deterministic != !!b.deterministic ||
      a.fixed_point_field_limit_v_per_m != b.fixed_point_field_limit_v_per_m ||
      a.zhs_subtrack_refinement != b.zhs_subtrack_refinement ||
      !!a.track_diagnostics != !!b.track_diagnostics || !!a.count_samples != !!b.count_samples)
    return false;
  auto const& p = a.propagation;
  auto const& q = b.propagation;
  if (p.homogeneous_refractive_index != q.homogeneous_refractive_index ||
      p.minimum_height_m != q.minimum_height_m || p.maximum_height_m != q.maximum_height_m ||
      p.step_m != q.step_m || p.inverse_step_per_m != q.inverse_step_per_m ||
      p.slope_refractivity_lower != q.slope_refractivity_lower ||
      p.slope_refractivity_upper != q.slope_refractivity_upper ||
      p.slope_integrated_refractivity_lower != q.slope_integrated_refractivity_lower ||
      p.slope_integrated_refractivity_upper != q.slope_integrated_refractivity_upper ||
      p.table_size != q.table_size)
    return false;
  if (p.table_size && (p.refractivity == nullptr || q.refractivity == nullptr ||
                       p.integrated_refractivity == nullptr || q.integrated_refractivity == nullptr))
    return false;
  if (!same_table(p.refractivity, q.refractivity, p.table_size) ||
      !same_table(p.integrated_refractivity, q.integrated_refractivity, p.table_size))
    return false;
  return same_observers(a.coreas_observers, a.coreas_observer_count, b.coreas_observers, b.coreas_observer_count) &&
         same_observers(a.zhs_observers, a.zhs_observer_count, b.zhs_observers, b.zhs_observer_count);
}

// merge_fixed_accumulators (FixedAccumulatorMerge.inl:12-29): every bin
// checked before any is written.
void preflight(std::vector<long long> const& destination, long long const* source, std::size_t count) {
  if (destination.size() != count) throw std::invalid_argument("incompatible fixed-point accumulators");
  for (std::size_t i = 0; i < count; ++i) {
    long long const x = destination[i], y = source[i];
    if ((y > 0 && x > std::numeric_limits<long long>::max() - y) ||
        (y < 0 && x < std::numeric_limits<long long>::min() - y))
      throw std::overflow_error("cooperative fixed-point accumulation overflow");
  }
}

}  // namespace

// CooperativeRadioMerge (CooperativeRadioMerge.hpp:53-65): accepts each
// endpoint's snapshot once and keeps their checked sum.
struct c8r_cooperative_merge {
  std::string identity;
  OwnedConfig config;
  std::vector<long long> coreas, zhs;
  c8r_counters counters{};
  unsigned endpoint = 0;  // endpoint of the first commit (the merged snapshot's)
  unsigned seen = 0;
  bool finished = false;
  std::string error;

  c8r_cooperative_merge(char const* id, c8r_config const& c) : identity(id ? id : ""), config(c) {
    if (identity.empty()) throw std::invalid_argument("empty cooperative shower identity");
  }

  // CooperativeRadioMerge::commit (CooperativeRadioMerge.inl:248-270): all
  // checks and the whole merge before any state changes.
  void commit(c8r_fixed_snapshot const& input) {
    if (finished) throw std::logic_error("cooperative radio output already taken");
    validate_snapshot(input);
    unsigned const bit = 1u << input.endpoint;
    if ((seen & bit) || identity != input.shower_identity || !same_physics(*input.config, config.config))
      throw std::invalid_argument("duplicate/incompatible cooperative radio commit");
    if (seen == 0) {
      coreas.assign(input.coreas, input.coreas + input.coreas_count);
      zhs.assign(input.zhs, input.zhs + input.zhs_count);
      counters = input.counters;
      endpoint = input.endpoint;
    } else {
      preflight(coreas, input.coreas, input.coreas_count);
      preflight(zhs, input.zhs, input.zhs_count);
      c8r_counters const merged = merge_counters(counters, input.counters);
      for (std::size_t i = 0; i < input.coreas_count; ++i) coreas[i] += input.coreas[i];
      for (std::size_t i = 0; i < input.zhs_count; ++i) zhs[i] += input.zhs[i];
      counters = merged;
    }
    seen |= bit;
  }

  // CooperativeRadioMerge::take (CooperativeRadioMerge.inl:272-277).
  void take(long long* coreas_out, long long* zhs_out, c8r_counters* counters_out, uint32_t* endpoint_out) {
    if (seen != 3 || finished) throw std::logic_error("cooperative radio endpoints not complete/already taken");
    if ((!coreas.empty() && coreas_out == nullptr) || (!zhs.empty() && zhs_out == nullptr))
      throw std::invalid_argument("null radio snapshot trace buffer");
    finished = true;
    if (!coreas.empty()) std::memcpy(coreas_out, coreas.data(), coreas.size() * sizeof(long long));
    if (!zhs.empty()) std::memcpy(zhs_out, zhs.data(), zhs.size() * sizeof(long long));
    if (counters_out) *counters_out = counters;
    if (endpoint_out) *endpoint_out = endpoint;
    std::vector<long long>().swap(coreas);
    std::vector<long long>().swap(zhs);
  }
};

extern "C" {

int c8r_validate_fixed_snapshot(const c8r_fixed_snapshot* snapshot) {
  return c8r::guarded(&g_error, [&] {
    if (!snapshot) throw std::invalid_argument("null radio snapshot");
    validate_snapshot(*snapshot);
  });
}

int c8r_merge_counters(c8r_counters* destination, const c8r_counters* source) {
  return c8r::guarded(&g_error, [&] {
    if (!destination || !source) throw std::invalid_argument("null argument");
    *destination = merge_counters(*destination, *source);
  });
}

const char* c8r_snapshot_last_error(void) { return g_error.c_str(); }

int c8r_cooperative_merge_create(const char* shower_identity, const c8r_config* config,
                                 c8r_cooperative_merge** merge) {
  return c8r::guarded(&g_error, [&] {
    if (!config || !merge) throw std::invalid_argument("null argument");
    *merge = nullptr;
    *merge = new c8r_cooperative_merge(shower_identity, *config);
  });
}

void c8r_cooperative_merge_destroy(c8r_cooperative_merge* merge) { delete merge; }

const char* c8r_cooperative_merge_last_error(const c8r_cooperative_merge* merge) {
  return merge ? merge->error.c_str() : g_error.c_str();
}

int c8r_cooperative_merge_commit(c8r_cooperative_merge* merge, const c8r_fixed_snapshot* snapshot) {
  if (!merge) {
    g_error = "null cooperative radio merge";
    return C8R_INVALID_ARGUMENT;
  }
  return c8r::guarded(&merge->error, [&] {
    if (!snapshot) throw std::invalid_argument("null radio snapshot");
    merge->commit(*snapshot);
  });
}

int c8r_cooperative_merge_take(c8r_cooperative_merge* merge, long long* coreas_xyz, long long* zhs_xyz,
                               c8r_counters* counters, uint32_t* endpoint) {
  if (!merge) {
    g_error = "null cooperative radio merge";
    return C8R_INVALID_ARGUMENT;
  }
  return c8r::guarded(&merge->error, [&] { merge->take(coreas_xyz, zhs_xyz, counters, endpoint); });
}

}  // extern "C"
