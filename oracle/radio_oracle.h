/*
 * radio_oracle.h — TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 * CPU restatement of the CORSIKA8-kokkos radio projection (CoREAS endpoint
 * field + ZHS vector potential, fixed-point or floating traces).  Used by the
 * tests, the smoke check and the bench's CPU baseline leg as the checker.
 * Parity of this restatement is pinned against the reference's own
 * projection code compiled into oracle/_ref and against the known answers of
 * the reference's tests (tests/kokkos/radio/testRadioProjection.cpp).
 */
#ifndef C8RADIO_ORACLE_H
#define C8RADIO_ORACLE_H

#include <stddef.h>
#include <stdint.h>
#include "../include/c8radio.h"

#ifdef __cplusplus
extern "C" {
#endif

/* RadioObserverView, corsika/kokkos/radio/RadioProjectionData.hpp:39-48 (80 B). */
typedef struct c8o_observer {
  double position_m[3];
  double start_time_s;
  double duration_s;
  double sample_rate_hz;
  double fixed_point_scale;
  double inverse_fixed_point_scale;
  uint64_t number_of_bins;
  uint64_t waveform_offset;
} c8o_observer;

/* RadioPropagationView, RadioProjectionData.hpp:50-64 (104 B). */
typedef struct c8o_propagation {
  double homogeneous_refractive_index;
  double minimum_height_m;
  double maximum_height_m;
  double step_m;
  double inverse_step_per_m;
  double slope_refractivity_lower;
  double slope_integrated_refractivity_lower;
  double slope_refractivity_upper;
  double slope_integrated_refractivity_upper;
  const double* refractivity;
  const double* integrated_refractivity;
  uint64_t table_size;
  uint32_t zhs_subtrack_refinement;
  uint32_t pad_;
} c8o_propagation;

/* RadioWaveformView, RadioProjectionData.hpp:66-73: SoA X|Y|Z rows. */
typedef struct c8o_waveforms {
  double* floating[3];
  long long* fixed[3];
} c8o_waveforms;

/* RadioSignalPath, RadioProjectionData.hpp:104-110. */
typedef struct c8o_path {
  double propagation_time_s;
  double refractive_index_source;
  double refractive_index_destination;
  double distance_m;
  double emit[3];
} c8o_path;

/* RadioTrackKinematics, RadioProjectionData.hpp:112-124 (152 B). */
typedef struct c8o_track {
  double start[3];
  double end[3];
  double displacement[3];
  double beta[3];
  double start_time_s;
  double end_time_s;
  double duration_s;
  double track_length_m;
  double beta_module;
  double constant;
  uint32_t valid;
  uint32_t pad_;
} c8o_track;

double c8o_nearest_bin(double scaled_time);
double c8o_doppler(double index, const double beta[3], const double emit[3]);
int c8o_make_track(const c8r_lepton_transport_record* record, c8o_track* track);
void c8o_propagate(const c8o_propagation* table, const double source[3],
                   const c8o_observer* observer, c8o_path* path);
int c8o_checked_add(long long* address, long long increment);
int c8o_add_fixed_point(long long* address, double contribution, double scale);
void c8o_add_sample(const c8o_observer* observer, const c8o_waveforms* waveforms,
                    double time_s, const double contribution[3],
                    unsigned long long* contribution_counter, c8r_counters* counters,
                    int vector_potential);
void c8o_separate_same_bin_endpoints(double* start_time, double* end_time,
                                     double grid_resolution, int signed_order);
void c8o_accumulate_coreas(const c8o_track* track, const c8o_propagation* propagation,
                           const c8o_observer* observer, const c8o_waveforms* waveforms,
                           c8r_counters* counters);
void c8o_accumulate_zhs(const c8o_track* track, const c8o_propagation* propagation,
                        const c8o_observer* observer, const c8o_waveforms* waveforms,
                        c8r_counters* counters);
size_t c8o_diagnostic_energy_bin(double kinetic_energy_gev);
int c8o_record_track(const c8r_lepton_transport_record* record, c8o_track* output,
                     c8r_counters* counters, int collect_diagnostics);

/* Observer views as RadioAccumulator::makeObservers builds them
 * (RadioAccumulator.inl:522-550).  Returns the total bin count. */
uint64_t c8o_make_observers(const c8r_observer_snapshot* input, size_t count,
                            int zhs_potential, int deterministic, double field_limit,
                            c8o_observer* output);

/* Whole accumulation of one batch: the pair loop of RadioAccumulator::project
 * with one private trace row per worker and a checked merge
 * (RadioAccumulator.inl:718-791, RadioAccumulatorOperations.inl:48-60).
 * Traces are SoA [X|Y|Z] of 3*total_bins values per algorithm; fixed traces
 * are used when config->deterministic, else floating.  Outputs are ADDED to.
 * counters are added to (tracks, contributions, subtracks, overflows, and the
 * diagnostics when config->track_diagnostics).  threads <= 0 uses one. */
int c8o_project(const c8r_config* config, const c8r_lepton_transport_record* records,
                size_t count, long long* coreas_fixed, long long* zhs_fixed,
                double* coreas_floating, double* zhs_floating, c8r_counters* counters,
                int threads);

#ifdef __cplusplus
}
#endif

#endif
