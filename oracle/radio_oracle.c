/*
 * radio_oracle.c — TEST INFRASTRUCTURE ONLY: the checker, never the product.
 *
 * Plain C99 restatement of the CORSIKA8-kokkos radio projection, following
 * corsika/detail/kokkos/radio/algorithms/RadioProjection.inl operation for
 * operation (same association order, no FMA contraction: build with
 * -ffp-contract=off), and the accumulator semantics of
 * corsika/detail/kokkos/radio/RadioAccumulator.inl.  Parity is pinned
 * against the reference's own projection code (oracle/_ref) and the known
 * answers of tests/kokkos/radio/testRadioProjection.cpp.
 *
 * One deliberate choice: co_reas_doppler's exact-zero recovery follows the
 * reference's DEVICE branch (FMA-compensated dot, RadioProjection.inl:123-141)
 * rather than its host long-double branch (:117-122), because the product
 * this oracle checks is the device path.  Both give -2^-60 on the
 * reference's known-answer case (testRadioProjection.cpp:204,224).
 */
#include "radio_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* corsika/kokkos/ScalarPhysicalConstants.hpp:18-20 and
 * corsika/kokkos/radio/RadioProjectionData.hpp:21-37. */
static const double kSpeedOfLight = 299792458.;
static const double kElementaryCharge = 1.6021766208e-19;
static const double kVacuumPermittivity = 8.8541878128e-12;
static const double kPi = 3.141592653589793238462643383279502884;
static const double kCoreasThreshold = 1.e-3;
static const double kHeadroom = 4611686018427387904.0;      /* 2^62 */
static const double kSignedLimit = 9223372036854775808.0;   /* 2^63 */
/* corsika/kokkos/em/algorithms/TransportMass.hpp:20 */
static const double kElectronMassGeV = 5.109989e-4;

static double em_constant(void) {
  /* 1 / (4 pi eps0 c), evaluated left to right as the reference's constexpr. */
  return 1. / (4. * kPi * kVacuumPermittivity * kSpeedOfLight);
}

/* static_cast<int>(double) as x86-64 executes it (cvttsd2si): values outside
 * the int range and NaN become INT_MIN.  The reference relies on this cast for
 * ZHS bin spans (RadioProjection.inl:457) and subtrack counts (:502). */
static int x86_int(double value) {
  if (!(value > -2147483649.0 && value < 2147483648.0)) return INT_MIN;
  return (int)value;
}

/* static_cast<long long>(double) as x86-64 executes it (64-bit cvttsd2si). */
static long long x86_ll(double value) {
  if (!(value >= -9223372036854775808.0 && value < 9223372036854775808.0)) return LLONG_MIN;
  return (long long)value;
}

static double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

static void cross3(const double a[3], const double b[3], double out[3]) {
  double r0 = a[1] * b[2] - a[2] * b[1];
  double r1 = a[2] * b[0] - a[0] * b[2];
  double r2 = a[0] * b[1] - a[1] * b[0];
  out[0] = r0;
  out[1] = r1;
  out[2] = r2;
}

/* RadioProjection.inl:75-82: floor plus a fractional >= 0.5 test. */
double c8o_nearest_bin(double scaled_time) {
  double integral = floor(scaled_time);
  return integral + (scaled_time - integral >= 0.5 ? 1. : 0.);
}

/* RadioProjection.inl:113-143 (device branch for the exact-zero case). */
double c8o_doppler(double index, const double beta[3], const double emit[3]) {
  double ordinary = 1. - index * dot3(beta, emit);
  if (ordinary != 0.) return ordinary;
  double px = beta[0] * emit[0];
  double py = beta[1] * emit[1];
  double pz = beta[2] * emit[2];
  double ex = fma(beta[0], emit[0], -px);
  double ey = fma(beta[1], emit[1], -py);
  double ez = fma(beta[2], emit[2], -pz);
  double xy = px + py;
  double xy_virtual = xy - px;
  double xy_error = (px - (xy - xy_virtual)) + (py - xy_virtual);
  double xyz = xy + pz;
  double xyz_virtual = xyz - xy;
  double xyz_error = (xy - (xyz - xyz_virtual)) + (pz - xyz_virtual);
  double low = ex + ey + ez + xy_error + xyz_error;
  double product = index * xyz;
  double product_error = fma(index, xyz, -product) + index * low;
  return (1. - product) - product_error;
}

/* RadioProjection.inl:145-168 (make_radio_track_kinematics). */
int c8o_make_track(const c8r_lepton_transport_record* record, c8o_track* track) {
  int32_t pid = record->start.pid;
  if (!(pid == 11 || pid == -11)) return 0;
  for (int axis = 0; axis < 3; ++axis) {
    track->start[axis] = record->start.position_m[axis];
    track->end[axis] = record->end.position_m[axis];
  }
  track->start_time_s = record->start.time_s;
  track->end_time_s = record->end.time_s;
  track->duration_s = track->end_time_s - track->start_time_s;
  for (int axis = 0; axis < 3; ++axis)
    track->displacement[axis] = track->end[axis] - track->start[axis];
  track->track_length_m = sqrt(dot3(track->displacement, track->displacement));
  if (!(track->duration_s > 0.) || !(track->track_length_m > 0.)) return 0;
  double denominator = kSpeedOfLight * track->duration_s;
  for (int axis = 0; axis < 3; ++axis) track->beta[axis] = track->displacement[axis] / denominator;
  track->beta_module = track->track_length_m / (kSpeedOfLight * track->duration_s);
  double charge = pid == 11 ? -kElementaryCharge : kElementaryCharge;
  track->constant = charge * em_constant() * record->start.weight;
  track->valid = 1;
  return 1;
}

/* RadioProjection.inl:170-238 (propagate): straight ray, nearest table bin,
 * edge extrapolation and the shadowed indices at/below the lower edge. */
void c8o_propagate(const c8o_propagation* table, const double source[3],
                   const c8o_observer* observer, c8o_path* path) {
  double displacement[3];
  for (int axis = 0; axis < 3; ++axis)
    displacement[axis] = observer->position_m[axis] - source[axis];
  double distance = sqrt(dot3(displacement, displacement));
  for (int axis = 0; axis < 3; ++axis) path->emit[axis] = displacement[axis] / distance;
  path->distance_m = distance;
  if (table->homogeneous_refractive_index > 0.) {
    double index = table->homogeneous_refractive_index;
    path->propagation_time_s = index * distance / kSpeedOfLight;
    path->refractive_index_source = index;
    path->refractive_index_destination = index;
    return;
  }
  double source_height = (source[2] - table->minimum_height_m) * table->inverse_step_per_m;
  double destination_height =
      (observer->position_m[2] - table->minimum_height_m) * table->inverse_step_per_m;
  uint64_t last = table->table_size - 1;
  uint64_t destination_index = (uint64_t)(destination_height + 0.5);
  double n_source = 1.;
  double integrated_source = 1.;
  double n_destination = table->refractivity[destination_index] + 1.;
  double integrated_destination = table->integrated_refractivity[destination_index];
  double height = 1.;
  if (source_height + 0.5 >= (double)last) {
    n_source = table->refractivity[last] +
               table->slope_refractivity_upper *
                   fabs((source[2] - table->maximum_height_m) * table->inverse_step_per_m) +
               1.;
    integrated_source = table->integrated_refractivity[last] +
                        table->slope_integrated_refractivity_upper *
                            fabs(table->maximum_height_m - source[2]);
    height = source_height - destination_height;
  } else if (source_height + 0.5 < (double)last && source_height > 0.) {
    uint64_t source_index = (uint64_t)(source_height + 0.5);
    n_source = table->refractivity[source_index] + 1.;
    integrated_source = table->integrated_refractivity[source_index];
    height = (double)((int64_t)source_index - (int64_t)destination_index) * table->step_m;
    if (height == 0.) height = 1.;
  } else if (source_height == 0.) {
    n_source = 1.;
    n_destination = 1.;
    integrated_source = table->integrated_refractivity[0];
    height = destination_height - source_height;
  } else {
    n_source = table->refractivity[0] + table->slope_refractivity_lower * fabs(source_height) + 1.;
    integrated_source = table->integrated_refractivity[0] +
                        table->slope_integrated_refractivity_lower * fabs(source_height);
    n_destination = 1.;
    height = destination_height - fabs(source_height);
  }
  path->propagation_time_s =
      (1. + (integrated_source - integrated_destination) / height) * distance / kSpeedOfLight;
  path->refractive_index_source = n_source;
  path->refractive_index_destination = n_destination;
}

/* RadioProjection.inl:246-251: two's-complement add, overflow from previous. */
int c8o_checked_add(long long* address, long long increment) {
  long long previous = *address;
  *address = (long long)((unsigned long long)previous + (unsigned long long)increment);
  return !((increment > 0 && previous > LLONG_MAX - increment) ||
           (increment < 0 && previous < LLONG_MIN - increment));
}

/* Diagnostic sample-count mode of c8o_project: every in-range sample adds 1. */
static int count_mode = 0;

/* RadioProjection.inl:254-260. */
int c8o_add_fixed_point(long long* address, double contribution, double scale) {
  if (count_mode) return c8o_checked_add(address, 1);
  double scaled = contribution * scale;
  if (!isfinite(scaled) || fabs(scaled) >= kSignedLimit) return 0;
  return c8o_checked_add(address, (long long)rint(scaled));
}

/* RadioProjection.inl:263-301 (add_sample): CoREAS fields are time gated,
 * ZHS potentials are not; nearest bin; fixed or floating rows. */
void c8o_add_sample(const c8o_observer* observer, const c8o_waveforms* waveforms,
                    double time_s, const double contribution[3],
                    unsigned long long* contribution_counter, c8r_counters* counters,
                    int vector_potential) {
  if (!vector_potential) {
    if (time_s < observer->start_time_s ||
        time_s > observer->start_time_s + observer->duration_s)
      return;
  }
  double bin_value =
      c8o_nearest_bin((time_s - observer->start_time_s) * observer->sample_rate_hz);
  if (!(bin_value >= 0. && bin_value < (double)observer->number_of_bins)) return;
  uint64_t bin = (uint64_t)bin_value;
  if (bin >= observer->number_of_bins) return;
  uint64_t offset = observer->waveform_offset + bin;
  if (waveforms->fixed[0] != NULL) {
    int valid_x = c8o_add_fixed_point(waveforms->fixed[0] + offset, contribution[0],
                                      observer->fixed_point_scale);
    int valid_y = c8o_add_fixed_point(waveforms->fixed[1] + offset, contribution[1],
                                      observer->fixed_point_scale);
    int valid_z = c8o_add_fixed_point(waveforms->fixed[2] + offset, contribution[2],
                                      observer->fixed_point_scale);
    if (!(valid_x && valid_y && valid_z)) {
      counters->fixed_point_overflows += 1ULL;
      return;
    }
  } else {
    waveforms->floating[0][offset] += contribution[0];
    waveforms->floating[1][offset] += contribution[1];
    waveforms->floating[2][offset] += contribution[2];
  }
  *contribution_counter += 1ULL;
}

/* RadioProjection.inl:303-336. */
void c8o_separate_same_bin_endpoints(double* start_time, double* end_time,
                                     double grid_resolution, int signed_order) {
  long long start_bin = x86_ll(c8o_nearest_bin(*start_time / grid_resolution));
  long long end_bin = x86_ll(c8o_nearest_bin(*end_time / grid_resolution));
  if (start_bin != end_bin) return;
  double start_fraction = *start_time / grid_resolution - floor(*start_time / grid_resolution);
  double end_fraction = *end_time / grid_resolution - floor(*end_time / grid_resolution);
  int forward = !signed_order || *end_time >= *start_time;
  if (forward) {
    if (start_fraction >= 0.5 && end_fraction >= 0.5)
      *start_time -= grid_resolution;
    else if (start_fraction < 0.5 && end_fraction < 0.5)
      *end_time += grid_resolution;
    else if (end_fraction >= 1. - start_fraction)
      *end_time += grid_resolution;
    else
      *start_time -= grid_resolution;
  } else {
    if (start_fraction >= 0.5 && end_fraction >= 0.5)
      *end_time -= grid_resolution;
    else if (start_fraction < 0.5 && end_fraction < 0.5)
      *start_time += grid_resolution;
    else if (start_fraction >= 1. - end_fraction)
      *start_time += grid_resolution;
    else
      *end_time -= grid_resolution;
  }
}

static void scale3(const double a[3], double value, double out[3]) {
  out[0] = a[0] * value;
  out[1] = a[1] * value;
  out[2] = a[2] * value;
}

/* transverse_endpoint, RadioProjection.inl:240-243: k x (k x beta). */
static void transverse(const double emit[3], const double beta[3], double out[3]) {
  double inner[3];
  cross3(emit, beta, inner);
  cross3(emit, inner, out);
}

/* RadioProjection.inl:339-409 (accumulate_co_reas). */
void c8o_accumulate_coreas(const c8o_track* track, const c8o_propagation* propagation,
                           const c8o_observer* observer, const c8o_waveforms* waveforms,
                           c8r_counters* counters) {
  c8o_path path_start, path_end;
  c8o_propagate(propagation, track->start, observer, &path_start);
  c8o_propagate(propagation, track->end, observer, &path_end);
  double pre_doppler = c8o_doppler(path_start.refractive_index_source, track->beta, path_start.emit);
  double post_doppler = c8o_doppler(path_end.refractive_index_source, track->beta, path_end.emit);
  double start_receive = track->start_time_s + path_start.propagation_time_s;
  double end_receive = track->end_time_s + path_end.propagation_time_s;
  double fs = observer->sample_rate_hz;
  double field_start[3], field_end[3], t[3];

  if (path_start.refractive_index_destination > 1. &&
      (fabs(pre_doppler) < kCoreasThreshold || fabs(post_doppler) < kCoreasThreshold)) {
    double midpoint[3];
    for (int axis = 0; axis < 3; ++axis)
      midpoint[axis] = (track->start[axis] + track->end[axis]) * 0.5;
    double middle_time = (track->start_time_s + track->end_time_s) * 0.5;
    c8o_path path_middle;
    c8o_propagate(propagation, midpoint, observer, &path_middle);
    double middle_receive = middle_time + path_middle.propagation_time_s;
    double middle_doppler =
        c8o_doppler(path_middle.refractive_index_source, track->beta, path_middle.emit);
    transverse(path_middle.emit, track->beta, t);
    scale3(t, track->constant * fs / (middle_doppler * path_middle.distance_m), field_start);
    scale3(field_start, -1., field_end);
    double delta_time =
        track->track_length_m / (kSpeedOfLight * track->beta_module) * fabs(middle_doppler);
    if (start_receive < end_receive) {
      start_receive = middle_receive - 0.5 * delta_time;
      end_receive = middle_receive + 0.5 * delta_time;
    } else {
      start_receive = middle_receive + 0.5 * delta_time;
      end_receive = middle_receive - 0.5 * delta_time;
    }
    double grid_resolution = 1. / fs;
    delta_time = end_receive - start_receive;
    if (fabs(delta_time) < grid_resolution) {
      double scale = fabs(delta_time / grid_resolution);
      scale3(field_start, scale, field_start);
      scale3(field_end, scale, field_end);
      c8o_separate_same_bin_endpoints(&start_receive, &end_receive, grid_resolution, 1);
    }
    c8o_add_sample(observer, waveforms, start_receive, field_start,
                   &counters->coreas_contributions, counters, 0);
    c8o_add_sample(observer, waveforms, end_receive, field_end,
                   &counters->coreas_contributions, counters, 0);
    return;
  }

  transverse(path_start.emit, track->beta, t);
  scale3(t, track->constant * fs / (pre_doppler * path_start.distance_m), field_start);
  transverse(path_end.emit, track->beta, t);
  scale3(t, -track->constant * fs / (post_doppler * path_end.distance_m), field_end);
  if (pre_doppler < 1.e-9 || post_doppler < 1.e-9) {
    double grid_resolution = 1. / fs;
    double delta_time = end_receive - start_receive;
    if (fabs(delta_time) < grid_resolution) {
      double scale = fabs(delta_time / grid_resolution);
      scale3(field_start, scale, field_start);
      scale3(field_end, scale, field_end);
      c8o_separate_same_bin_endpoints(&start_receive, &end_receive, grid_resolution, 0);
    }
  }
  c8o_add_sample(observer, waveforms, start_receive, field_start,
                 &counters->coreas_contributions, counters, 0);
  c8o_add_sample(observer, waveforms, end_receive, field_end,
                 &counters->coreas_contributions, counters, 0);
}

/* RadioProjection.inl:412-480 (accumulate_zhs_segment). */
static void zhs_segment(const double point1[3], const double point2[3], double time1,
                        double time2, const double beta[3], double constant,
                        const c8o_propagation* propagation, const c8o_observer* observer,
                        const c8o_waveforms* waveforms, c8r_counters* counters,
                        int subdivided) {
  double midpoint[3];
  for (int axis = 0; axis < 3; ++axis) midpoint[axis] = (point1[axis] + point2[axis]) * 0.5;
  c8o_path path;
  c8o_propagate(propagation, midpoint, observer, &path);
  double n_source = path.refractive_index_source;
  double beta_times_k = dot3(beta, path.emit);
  double middle_time = (time1 + time2) * 0.5;
  double detection_time1 =
      time1 + path.propagation_time_s - n_source * beta_times_k * (time1 - middle_time);
  double detection_time2 =
      time2 + path.propagation_time_s - n_source * beta_times_k * (time2 - middle_time);
  double sign = 1.;
  if (detection_time1 > detection_time2) {
    detection_time1 =
        time2 + path.propagation_time_s - n_source * beta_times_k * (time2 - middle_time);
    detection_time2 =
        time1 + path.propagation_time_s - n_source * beta_times_k * (time1 - middle_time);
    sign = -1.;
  }
  double fs = observer->sample_rate_hz;
  double start_bin = floor((detection_time1 - observer->start_time_s) * fs + 0.5);
  double end_bin = floor((detection_time2 - observer->start_time_s) * fs + 0.5);
  double inner[3], beta_perpendicular[3], potential[3];
  cross3(beta, path.emit, inner);
  cross3(path.emit, inner, beta_perpendicular);
  double denominator = 1. - n_source * beta_times_k;

  if (start_bin == end_bin) {
    if (fabs(denominator) > 1.e-15) {
      double fraction = fabs(detection_time2 * fs - detection_time1 * fs);
      scale3(beta_perpendicular,
             sign * constant * fraction / (denominator * path.distance_m), potential);
    } else {
      double fraction = (time2 - time1) * fs;
      scale3(beta_perpendicular, sign * constant * fraction / path.distance_m, potential);
    }
    c8o_add_sample(observer, waveforms, detection_time2, potential,
                   &counters->zhs_contributions, counters, 1);
    return;
  }
  int number_of_bins = x86_int(end_bin - start_bin);
  double fraction = fabs(start_bin + 0.5 - (detection_time1 - observer->start_time_s) * fs);
  scale3(beta_perpendicular, sign * constant * fraction / (denominator * path.distance_m),
         potential);
  c8o_add_sample(observer, waveforms, detection_time1, potential,
                 &counters->zhs_contributions, counters, 1);
  for (int index = 1; index < number_of_bins; ++index) {
    scale3(beta_perpendicular,
           (subdivided ? 1. : sign) * constant / (denominator * path.distance_m), potential);
    c8o_add_sample(observer, waveforms, detection_time1 + (double)index / fs, potential,
                   &counters->zhs_contributions, counters, 1);
  }
  fraction = fabs((detection_time2 - observer->start_time_s) * fs + 0.5 - end_bin);
  scale3(beta_perpendicular, sign * constant * fraction / (denominator * path.distance_m),
         potential);
  c8o_add_sample(observer, waveforms, detection_time2, potential,
                 &counters->zhs_contributions, counters, 1);
}

/* RadioProjection.inl:483-529 (accumulate_zhs): Fraunhofer subdivision. */
void c8o_accumulate_zhs(const c8o_track* track, const c8o_propagation* propagation,
                        const c8o_observer* observer, const c8o_waveforms* waveforms,
                        c8r_counters* counters) {
  double midpoint[3];
  for (int axis = 0; axis < 3; ++axis)
    midpoint[axis] = (track->start[axis] + track->end[axis]) * 0.5;
  c8o_path middle_path;
  c8o_propagate(propagation, midpoint, observer, &middle_path);
  double u_times_k = dot3(track->beta, middle_path.emit) / track->beta_module;
  double sin_theta_squared = 1. - u_times_k * u_times_k;
  double wavelength = kSpeedOfLight / observer->sample_rate_hz;
  double fraunhofer = sin_theta_squared * track->track_length_m * track->track_length_m /
                      middle_path.distance_m / wavelength * 2. * kPi;
  double subtrack_divisor = 1.;
  int number_of_subtracks = 1;
  if (fraunhofer > 1.) {
    subtrack_divisor = sqrt(fraunhofer) + 1.;
    number_of_subtracks = x86_int(ceil(subtrack_divisor));
  }
  counters->zhs_subtracks += (unsigned long long)(long long)number_of_subtracks;
  double spatial_step[3], refined_spatial_step[3];
  for (int axis = 0; axis < 3; ++axis) spatial_step[axis] = track->displacement[axis] / subtrack_divisor;
  double time_step = track->duration_s / subtrack_divisor;
  int refinement = (int)propagation->zhs_subtrack_refinement;
  for (int axis = 0; axis < 3; ++axis)
    refined_spatial_step[axis] = spatial_step[axis] / (double)refinement;
  double refined_time_step = time_step / (double)refinement;
  double point1[3] = {track->start[0], track->start[1], track->start[2]};
  double time1 = track->start_time_s;
  int subdivided = number_of_subtracks > 1 || refinement > 1;
  for (int index = 0; index < number_of_subtracks; ++index) {
    for (int refined_index = 0; refined_index < refinement; ++refined_index) {
      double point2[3];
      for (int axis = 0; axis < 3; ++axis) point2[axis] = point1[axis] + refined_spatial_step[axis];
      double time2 = time1 + refined_time_step;
      zhs_segment(point1, point2, time1, time2, track->beta, track->constant, propagation,
                  observer, waveforms, counters, subdivided);
      memcpy(point1, point2, sizeof point1);
      time1 = time2;
    }
  }
  if (refinement > 1)
    counters->zhs_subtracks +=
        (unsigned long long)(long long)(number_of_subtracks * (refinement - 1));
}

/* RadioProjection.inl:531-538. */
size_t c8o_diagnostic_energy_bin(double kinetic_energy_gev) {
  static const double upper_edges[14] = {1.e-3, 2.e-3, 5.e-3, 1.e-2, 2.e-2, 5.e-2, 1.e-1,
                                         2.e-1, 5.e-1, 1.,    2.,    5.,    10.,   100.};
  size_t index = 0;
  while (index < 14 && kinetic_energy_gev > upper_edges[index]) ++index;
  return index;
}

static void max_into(double* address, double value) {
  if (value > *address) *address = value;
}

/* RadioProjection.inl:541-611 (record_track with optional diagnostics). */
int c8o_record_track(const c8r_lepton_transport_record* record, c8o_track* output,
                     c8r_counters* counters, int collect_diagnostics) {
  c8o_track track;
  memset(&track, 0, sizeof track);
  if (!c8o_make_track(record, &track)) {
    if (output != NULL) memset(output, 0, sizeof *output);
    return 0;
  }
  if (output != NULL) *output = track;
  counters->valid_tracks += 1ULL;
  if (!collect_diagnostics) return 1;
  double length_m = track.track_length_m;
  double weight = record->start.weight;
  double kinetic = record->start.energy_gev - kElectronMassGeV;
  if (!isfinite(length_m) || !(length_m > 0.) || !isfinite(weight) || weight < 0. ||
      !isfinite(kinetic) || kinetic < 0.)
    return 1;
  double weighted_length = weight * length_m;
  counters->weighted_segment_count += weight;
  counters->track_length_m += length_m;
  counters->weighted_track_length_m += weighted_length;
  counters->energy_weighted_track_length_gev_m += weighted_length * kinetic;
  max_into(&counters->maximum_segment_length_m, length_m);
  if (record->start.pid == 11) {
    counters->electron_weighted_track_length_m += weighted_length;
    counters->signed_charge_weighted_track_length_m += -weighted_length;
  } else {
    counters->positron_weighted_track_length_m += weighted_length;
    counters->signed_charge_weighted_track_length_m += weighted_length;
  }
  counters->weighted_track_length_by_kinetic_energy_m[c8o_diagnostic_energy_bin(kinetic)] +=
      weighted_length;
  double direction_dot = 0.;
  double delta[3];
  for (int axis = 0; axis < 3; ++axis) {
    double pre = record->start.direction[axis];
    double post = record->end.direction[axis];
    direction_dot += pre * post;
    delta[axis] = post - pre;
  }
  /* radio_min(1, radio_max(-1, dot)) with the reference's comparison order,
   * which lets a NaN through (RadioProjection.inl:67-73, :591-592). */
  double clamped = -1. > direction_dot ? -1. : direction_dot;
  clamped = 1. < clamped ? 1. : clamped;
  double change = acos(clamped);
  double residual = track.duration_s - length_m / kSpeedOfLight;
  counters->weighted_direction_change_rad += weight * change;
  counters->weighted_direction_change_squared_rad2 += weight * change * change;
  counters->weighted_beta_deficit_track_length_m += weighted_length * (1. - track.beta_module);
  counters->weighted_time_residual_s += weight * residual;
  max_into(&counters->maximum_direction_change_rad, change);
  double charge_sign = record->start.pid == 11 ? -1. : 1.;
  for (int axis = 0; axis < 3; ++axis)
    counters->signed_charge_weighted_direction_change[axis] += charge_sign * weight * delta[axis];
  return 1;
}

/* RadioAccumulator.inl:522-550 (makeObservers). */
uint64_t c8o_make_observers(const c8r_observer_snapshot* input, size_t count,
                            int zhs_potential, int deterministic, double field_limit,
                            c8o_observer* output) {
  uint64_t total = 0;
  for (size_t i = 0; i < count; ++i) {
    c8o_observer* o = &output[i];
    memset(o, 0, sizeof *o);
    for (int axis = 0; axis < 3; ++axis) o->position_m[axis] = input[i].position_m[axis];
    o->start_time_s = input[i].start_time_s;
    o->duration_s = input[i].duration_s;
    o->sample_rate_hz = input[i].sample_rate_hz;
    double factor = zhs_potential ? input[i].sample_rate_hz : 1.;
    o->fixed_point_scale = deterministic ? kHeadroom * factor / field_limit : 1.;
    o->inverse_fixed_point_scale = 1. / o->fixed_point_scale;
    o->number_of_bins = input[i].number_of_bins;
    o->waveform_offset = total;
    total += input[i].number_of_bins;
  }
  return total;
}

static void merge_counters(c8r_counters* into, const c8r_counters* from) {
  into->coreas_contributions += from->coreas_contributions;
  into->zhs_contributions += from->zhs_contributions;
  into->zhs_subtracks += from->zhs_subtracks;
  into->valid_tracks += from->valid_tracks;
  into->fixed_point_overflows += from->fixed_point_overflows;
  into->weighted_segment_count += from->weighted_segment_count;
  into->track_length_m += from->track_length_m;
  into->weighted_track_length_m += from->weighted_track_length_m;
  into->electron_weighted_track_length_m += from->electron_weighted_track_length_m;
  into->positron_weighted_track_length_m += from->positron_weighted_track_length_m;
  into->signed_charge_weighted_track_length_m += from->signed_charge_weighted_track_length_m;
  into->energy_weighted_track_length_gev_m += from->energy_weighted_track_length_gev_m;
  max_into(&into->maximum_segment_length_m, from->maximum_segment_length_m);
  into->weighted_direction_change_rad += from->weighted_direction_change_rad;
  into->weighted_direction_change_squared_rad2 += from->weighted_direction_change_squared_rad2;
  into->weighted_beta_deficit_track_length_m += from->weighted_beta_deficit_track_length_m;
  into->weighted_time_residual_s += from->weighted_time_residual_s;
  max_into(&into->maximum_direction_change_rad, from->maximum_direction_change_rad);
  for (int i = 0; i < 3; ++i)
    into->signed_charge_weighted_direction_change[i] +=
        from->signed_charge_weighted_direction_change[i];
  for (int i = 0; i < 15; ++i)
    into->weighted_track_length_by_kinetic_energy_m[i] +=
        from->weighted_track_length_by_kinetic_energy_m[i];
}

int c8o_project(const c8r_config* config, const c8r_lepton_transport_record* records,
                size_t count, long long* coreas_fixed, long long* zhs_fixed,
                double* coreas_floating, double* zhs_floating, c8r_counters* counters,
                int threads) {
  if (config == NULL || counters == NULL || (count != 0 && records == NULL)) return 1;
  int deterministic = config->deterministic != 0;
  size_t n_coreas = config->coreas_enabled ? (size_t)config->coreas_observer_count : 0;
  size_t n_zhs = config->zhs_enabled ? (size_t)config->zhs_observer_count : 0;
  c8o_observer* coreas = calloc(n_coreas ? n_coreas : 1, sizeof *coreas);
  c8o_observer* zhs = calloc(n_zhs ? n_zhs : 1, sizeof *zhs);
  if (!coreas || !zhs) return 8;
  uint64_t coreas_bins = c8o_make_observers(config->coreas_observers, n_coreas, 0, deterministic,
                                            config->fixed_point_field_limit_v_per_m, coreas);
  uint64_t zhs_bins = c8o_make_observers(config->zhs_observers, n_zhs, 1, deterministic,
                                         config->fixed_point_field_limit_v_per_m, zhs);
  c8o_propagation propagation;
  memset(&propagation, 0, sizeof propagation);
  const c8r_propagation_snapshot* p = &config->propagation;
  propagation.homogeneous_refractive_index = p->homogeneous_refractive_index;
  propagation.minimum_height_m = p->minimum_height_m;
  propagation.maximum_height_m = p->maximum_height_m;
  propagation.step_m = p->step_m;
  propagation.inverse_step_per_m = p->inverse_step_per_m;
  propagation.slope_refractivity_lower = p->slope_refractivity_lower;
  propagation.slope_integrated_refractivity_lower = p->slope_integrated_refractivity_lower;
  propagation.slope_refractivity_upper = p->slope_refractivity_upper;
  propagation.slope_integrated_refractivity_upper = p->slope_integrated_refractivity_upper;
  propagation.refractivity = p->refractivity;
  propagation.integrated_refractivity = p->integrated_refractivity;
  propagation.table_size = p->table_size;
  propagation.zhs_subtrack_refinement = config->zhs_subtrack_refinement;

  count_mode = config->count_samples != 0;
  if (threads <= 0) threads = 1;
#ifndef _OPENMP
  threads = 1;
#endif
  size_t coreas_values = 3 * (size_t)coreas_bins, zhs_values = 3 * (size_t)zhs_bins;
  size_t row_bytes = deterministic ? sizeof(long long) : sizeof(double);
  unsigned char* coreas_rows = calloc((size_t)threads * (coreas_values ? coreas_values : 1), row_bytes);
  unsigned char* zhs_rows = calloc((size_t)threads * (zhs_values ? zhs_values : 1), row_bytes);
  c8r_counters* thread_counters = calloc((size_t)threads, sizeof(c8r_counters));
  if (!coreas_rows || !zhs_rows || !thread_counters) {
    free(coreas);
    free(zhs);
    free(coreas_rows);
    free(zhs_rows);
    free(thread_counters);
    return 8;
  }
  int diagnostics = config->track_diagnostics != 0;

#ifdef _OPENMP
#pragma omp parallel num_threads(threads)
#endif
  {
    int slot = 0;
#ifdef _OPENMP
    slot = omp_get_thread_num();
#endif
    c8o_waveforms coreas_w, zhs_w;
    memset(&coreas_w, 0, sizeof coreas_w);
    memset(&zhs_w, 0, sizeof zhs_w);
    for (int axis = 0; axis < 3; ++axis) {
      if (deterministic) {
        long long* c = (long long*)coreas_rows + (size_t)slot * coreas_values;
        long long* z = (long long*)zhs_rows + (size_t)slot * zhs_values;
        coreas_w.fixed[axis] = c + axis * coreas_bins;
        zhs_w.fixed[axis] = z + axis * zhs_bins;
      } else {
        double* c = (double*)coreas_rows + (size_t)slot * coreas_values;
        double* z = (double*)zhs_rows + (size_t)slot * zhs_values;
        coreas_w.floating[axis] = c + axis * coreas_bins;
        zhs_w.floating[axis] = z + axis * zhs_bins;
      }
    }
    c8r_counters* local = &thread_counters[slot];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
    for (long long i = 0; i < (long long)count; ++i) {
      c8o_track track;
      if (!c8o_record_track(&records[i], &track, local, diagnostics)) continue;
      size_t observers = n_coreas > n_zhs ? n_coreas : n_zhs;
      for (size_t o = 0; o < observers; ++o) {
        if (o < n_coreas) c8o_accumulate_coreas(&track, &propagation, &coreas[o], &coreas_w, local);
        if (o < n_zhs) c8o_accumulate_zhs(&track, &propagation, &zhs[o], &zhs_w, local);
      }
    }
  }

  /* Merge of private rows, RadioAccumulatorOperations.inl:48-60. */
  unsigned long long merge_overflows = 0;
  for (int algorithm = 0; algorithm < 2; ++algorithm) {
    size_t values = algorithm ? zhs_values : coreas_values;
    unsigned char* rows = algorithm ? zhs_rows : coreas_rows;
    for (size_t v = 0; v < values; ++v) {
      if (deterministic) {
        long long* out = algorithm ? zhs_fixed : coreas_fixed;
        long long sum = out ? out[v] : 0;
        for (int s = 0; s < threads; ++s)
          if (!c8o_checked_add(&sum, ((long long*)rows)[(size_t)s * values + v])) ++merge_overflows;
        if (out) out[v] = sum;
      } else {
        double* out = algorithm ? zhs_floating : coreas_floating;
        double sum = out ? out[v] : 0.;
        for (int s = 0; s < threads; ++s) sum += ((double*)rows)[(size_t)s * values + v];
        if (out) out[v] = sum;
      }
    }
  }
  for (int s = 0; s < threads; ++s) merge_counters(counters, &thread_counters[s]);
  counters->fixed_point_overflows += merge_overflows;
  free(coreas);
  free(zhs);
  free(coreas_rows);
  free(zhs_rows);
  free(thread_counters);
  count_mode = 0;
  return 0;
}
