/*
 * c8radio.h — C ABI of the B200 radio projection library (libc8radio.so).
 *
 * Drop-in boundary for the CORSIKA8-kokkos radio hot path: CoREAS endpoint
 * fields and ZHS vector potentials of every electron/positron track segment
 * at every antenna, binned into antenna time traces.  The entry points below
 * replace the member functions of corsika::kokkos::radio::RadioAccumulator
 * (corsika/kokkos/radio/RadioAccumulator.hpp:59-145) behind IRadioBackend
 * (corsika/kokkos/radio/IRadioBackend.hpp:29-41).  Every function returns a
 * C8R_* status; the C++ shim c8radio.hpp turns these back into the
 * reference's exception classes.
 *
 * Plain C, plain pointers and sizes.  The record, observer, propagation and
 * counter structs keep the reference's byte layouts so device producers and
 * host callers need no conversion.
 */
#ifndef C8RADIO_H
#define C8RADIO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (one per reference exception class) -------------------- */
enum {
  C8R_OK = 0,
  C8R_INVALID_ARGUMENT = 1, /* std::invalid_argument */
  C8R_LOGIC_ERROR = 2,      /* std::logic_error */
  C8R_OUT_OF_RANGE = 3,     /* std::out_of_range */
  C8R_RUNTIME_ERROR = 4,    /* std::runtime_error (fixed-point overflow) */
  C8R_LENGTH_ERROR = 5,     /* std::length_error */
  C8R_OVERFLOW_ERROR = 6,   /* std::overflow_error */
  C8R_CUDA_ERROR = 7,       /* CUDA runtime failure (message holds the CUDA string) */
  C8R_BAD_ALLOC = 8,        /* device or pinned host allocation failed */
  C8R_TIMEOUT = 9           /* server: not admitted / not complete within the timeout */
};

/* ---- record layout: corsika/kokkos/data/ParticleState.hpp:24-44 ----------- */
typedef struct c8r_particle_state {
  int32_t pid;           /* signed PDG id: 11 e-, -11 e+ */
  int32_t medium_id;
  uint32_t generation;
  uint32_t reserved;
  double energy_gev;     /* total energy */
  double position_m[3];
  double direction[3];
  double time_s;
  double weight;
  uint64_t history_id;
  uint64_t parent_history_id;
  uint64_t step_id;
  int32_t environment_node;
  int32_t pad_[3];
} c8r_particle_state; /* 128 bytes (alignas(16) in the reference) */

/* corsika/kokkos/em/LeptonTransportRecord.hpp:38-70 (752 bytes).  Only start
 * and end are read by radio projection; the leading InteractionRecord (320 B)
 * and the trailing transport fields (176 B) are carried opaque. */
typedef struct c8r_lepton_transport_record {
  unsigned char interaction[320];
  c8r_particle_state start;
  c8r_particle_state end;
  unsigned char transport[176];
} c8r_lepton_transport_record;

/* ---- configuration: corsika/kokkos/radio/RadioObserverSnapshot.hpp:17-23 -- */
typedef struct c8r_observer_snapshot {
  double position_m[3];
  double start_time_s;
  double duration_s;
  double sample_rate_hz;
  uint64_t number_of_bins;
} c8r_observer_snapshot;

/* corsika/kokkos/radio/FlatAtmosphereRadioSnapshot.hpp:20-36; the two tables
 * are borrowed host arrays of table_size doubles (copied by c8r_create). */
typedef struct c8r_propagation_snapshot {
  double homogeneous_refractive_index; /* >0 selects n R / c, no table */
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
} c8r_propagation_snapshot;

/* Arithmetic of the projection kernels. */
enum {
  C8R_PRECISION_FP64 = 0,  /* every expression in FP64, operation for operation as
                              the reference: the plain drop-in */
  C8R_PRECISION_MIXED = 1, /* arrival times, distances, emission directions and
                              1 - n beta.k in FP64 (bin indices and branches are
                              identical); field and potential amplitudes in FP32 */
  /* Precision study (one thread per pair, accumulate and download only): the
     arrival-time, distance, direction and 1 - n beta.k arithmetic in ... */
  C8R_PRECISION_STUDY_DOUBLE_FP32 = 2, /* compensated double-FP32 (hi + lo floats) */
  C8R_PRECISION_STUDY_FP32 = 3,        /* plain FP32 (bins may differ) */
  C8R_PRECISION_STUDY_FP64 = 4         /* FP64 through the same generic kernel (its check) */
};

/* Kernel family used by accumulate. */
enum {
  C8R_KERNEL_AUTO = 0,     /* windowed when the trace window fits, else direct */
  C8R_KERNEL_DIRECT = 1,   /* one thread per (track, antenna) pair, global 64-bit
                              atomics per sample: the reference's launch shape */
  C8R_KERNEL_WINDOWED = 2, /* CTA owns one antenna's trace in shared memory for a
                              chunk of tracks; flushed with checked global atomics */
  C8R_KERNEL_TILED = 3     /* the reference's large-batch shape (RadioTileProjection,
                              RadioAccumulator.inl:13-85): 256-thread CTAs over tiles
                              of 8 tracks x 32 observers staged in shared memory, one
                              thread per pair, global 64-bit atomics per sample (the
                              reference itself projects batches below 16384 tracks
                              with the direct shape) */
};

/* corsika/kokkos/radio/RadioConfig.hpp:21-53 */
typedef struct c8r_config {
  int32_t enabled;
  int32_t coreas_enabled;
  int32_t zhs_enabled;
  int32_t deterministic;      /* 1: int64 fixed-point traces (production default) */
  double fixed_point_field_limit_v_per_m;
  int32_t track_diagnostics;
  uint32_t zhs_subtrack_refinement; /* [1, 64] */
  c8r_propagation_snapshot propagation;
  const c8r_observer_snapshot* coreas_observers;
  uint64_t coreas_observer_count;
  const c8r_observer_snapshot* zhs_observers;
  uint64_t zhs_observer_count;
  /* B200 extensions (zero keeps the defaults). */
  int32_t precision;          /* C8R_PRECISION_* */
  int32_t kernel;             /* C8R_KERNEL_* */
  int32_t count_samples;      /* diagnostic: each in-range sample adds 1 to every
                                 component instead of its amplitude (fixed-point
                                 mode only); traces then count samples per bin */
  int32_t reserved_;
} c8r_config;

/* corsika/kokkos/runtime/TuningParameters.hpp:14-21; zero keeps defaults.
 * track_tile_size = tracks per windowed CTA chunk, observer_tile_size = bins
 * per shared-memory window, team_size = threads per CoREAS CTA (a team below
 * the default 640 also caps the ZHS CTAs, which otherwise take the largest
 * block of their pass and amplitude type: 384 to 768 threads). */
typedef struct c8r_tuning {
  uint64_t batch_size;
  uint64_t chunk_size;
  uint64_t team_size;
  uint64_t track_tile_size;
  uint64_t observer_tile_size;
  uint64_t device_queues;
} c8r_tuning;

/* corsika/kokkos/radio/RadioProjectionData.hpp:75-96 (288 bytes). */
typedef struct c8r_counters {
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
} c8r_counters;

/* corsika/kokkos/radio/RadioStatistics.hpp:17-63 (the fields this path fills). */
typedef struct c8r_statistics {
  uint64_t lepton_tracks;
  uint64_t track_observer_pairs;
  uint64_t fused_track_observer_pairs;
  uint64_t coreas_contributions;
  uint64_t zhs_contributions;
  uint64_t zhs_subtracks;
  uint64_t fixed_point_overflows;
  uint64_t device_bytes;
  uint64_t host_to_device_bytes;
  uint64_t host_tracks_enqueued;
  uint64_t host_track_batches;
  uint64_t device_to_host_bytes;
  uint64_t track_precompute_batches;
  uint64_t track_precomputed_records;
  uint64_t direct_projection_batches;
  uint64_t direct_projection_records;
  uint64_t projection_tiles;
  uint64_t track_workspace_bytes;
  uint64_t maximum_track_batch;
  uint32_t track_tile_size;
  uint32_t observer_tile_size;
  double kernel_time_ms;      /* CUDA-event time of projection kernels (timing on) */
  uint64_t timed_launches;    /* accumulate calls included in kernel_time_ms */
  double coreas_kernel_time_ms; /* windowed CoREAS launches alone (timing on) */
  double zhs_kernel_time_ms;    /* windowed ZHS launches alone (timing on) */
  c8r_counters counters;      /* last downloaded device counters */
  uint64_t window_reruns;     /* windowed work items projected again with checked adds
                                 (their unchecked run could not exclude an overflow);
                                 read with the counters at download */
  uint64_t window_handbacks;  /* ZHS work items the track-loop pass of a two-pass launch
                                 handed to the drain pass to project in full (trace past
                                 the window, window bound not shown, or its deferred
                                 pairs past its CTA's list); read at download */
} c8r_statistics;

/* Measured device rates used as roofline denominators (c8r_probe_peaks). */
typedef struct c8r_peaks {
  double fp64_flops;            /* FP64 FMA stream, 2 FLOP per FMA */
  double fp32_flops;            /* FP32 FMA stream, 2 FLOP per FMA */
  double shared_atomics_per_s;  /* 64-bit shared-memory atomic adds, distinct addresses */
  double global_atomics_per_s;  /* 64-bit global atomic adds over 128 MiB */
} c8r_peaks;

typedef struct c8r_accumulator c8r_accumulator;

/* Library identity and error text. */
const char* c8r_version(void);
/* Message of the last failing call on this handle (never NULL). */
const char* c8r_last_error(const c8r_accumulator* handle);
/* Message of the last failing call that had no handle (create, validate). */
const char* c8r_last_global_error(void);

/* RadioAccumulator::validate (RadioAccumulator.inl:931-974). */
int c8r_config_validate(const c8r_config* config);
/* RadioAccumulator::projectedDeviceBytes (RadioAccumulator.inl:87-141). */
int c8r_projected_device_bytes(const c8r_config* config, size_t* bytes);

/* RadioAccumulator::initialize (RadioAccumulator.inl:143-217).  stream is a
 * cudaStream_t (NULL = legacy default stream); all work is ordered on it. */
int c8r_create(const c8r_config* config, const c8r_tuning* tuning, void* stream,
               c8r_accumulator** handle);
/* Releases device memory after completing queued work.  NULL is ignored. */
void c8r_destroy(c8r_accumulator* handle);

/* RadioAccumulator::enabled (RadioAccumulator.inl:219-222). */
int c8r_enabled(const c8r_accumulator* handle, int* enabled);
/* RadioAccumulator::reset (RadioAccumulator.inl:224-250). */
int c8r_reset(c8r_accumulator* handle);
/* RadioAccumulator::enqueueHostLeptonTracks (RadioAccumulator.inl:252-272):
 * copies before returning; full batches (tuning batch_size, default 4096
 * records) are flushed.  Page-locked input is copied by DMA straight into
 * device staging (the call returns once those copies completed). */
int c8r_enqueue_host(c8r_accumulator* handle, const c8r_lepton_transport_record* records,
                     size_t count);
/* RadioAccumulator::flushHostLeptonTracks (RadioAccumulator.inl:274-290). */
int c8r_flush(c8r_accumulator* handle);
/* RadioAccumulator::accumulateLeptonTracks (RadioAccumulator.inl:292-357):
 * records is DEVICE memory holding extent records, borrowed until the
 * queued work completes; count > extent is C8R_OUT_OF_RANGE. */
int c8r_accumulate_device(c8r_accumulator* handle,
                          const c8r_lepton_transport_record* records, size_t count,
                          size_t extent);
/* RadioAccumulator::download (RadioAccumulator.inl:407-439).  Writes decoded
 * traces in the reference's SoA order [X: all bins | Y | Z] per algorithm
 * (RadioAccumulator.inl:570-589); each buffer holds 3 * total_bins doubles and
 * may be NULL when the algorithm has no observers.  counters may be NULL. */
int c8r_download(c8r_accumulator* handle, double* coreas_xyz, double* zhs_xyz,
                 c8r_counters* counters);
/* RadioAccumulator::downloadFixed (RadioAccumulator.inl:359-405): raw int64
 * fixed-point traces, same layout; requires deterministic mode. */
int c8r_download_fixed(c8r_accumulator* handle, long long* coreas_xyz, long long* zhs_xyz,
                       c8r_counters* counters);
/* Total bins (sum over observers) of each algorithm's traces. */
int c8r_total_bins(const c8r_accumulator* handle, size_t* coreas_bins, size_t* zhs_bins);

/* RadioAccumulator::statistics / deviceBytes / staticHostToDeviceBytes. */
int c8r_get_statistics(const c8r_accumulator* handle, c8r_statistics* statistics);
int c8r_device_bytes(const c8r_accumulator* handle, size_t* bytes);
int c8r_static_host_to_device_bytes(const c8r_accumulator* handle, size_t* bytes);
/* RadioAccumulator::reserveTrackCapacity / projectedTrackCapacity
 * (RadioAccumulator.inl:478-508). */
int c8r_reserve(c8r_accumulator* handle, size_t count);
int c8r_projected_track_capacity(const c8r_accumulator* handle, size_t count,
                                 size_t* retained_bytes, size_t* transient_peak_bytes);
/* B200 extension: when enabled, each accumulate records CUDA events around
 * its projection kernels (no host synchronisation); c8r_get_statistics sums
 * the elapsed times of completed launches into kernel_time_ms.  The CoREAS
 * and ZHS launches then run one after the other on the accumulator's stream
 * (otherwise the ZHS launch runs beside the CoREAS one on a second stream). */
int c8r_set_kernel_timing(c8r_accumulator* handle, int enabled);
/* B200 extension, no reference counterpart: measures the rates of c8r_peaks
 * on the current device (a few milliseconds of probe kernels). */
int c8r_probe_peaks(c8r_peaks* peaks);
/* Blocks until all work queued on the accumulator's stream has completed. */
int c8r_synchronize(c8r_accumulator* handle);

/* ---- B200 extensions: staging and batched projection ---------------------
 * No reference counterpart: the reference projects every accumulateLeptonTracks
 * batch on its own (RadioAccumulator.inl:292-357).  Here ingest and projection
 * can be separated so that many events share one persistent launch. */

/* Ingests device records into the accumulator's kinematics workspace after
 * the tracks already staged, without projecting them (same checks as
 * c8r_accumulate_device).  download/download_fixed project staged tracks. */
int c8r_stage_device(c8r_accumulator* handle, const c8r_lepton_transport_record* records,
                     size_t count, size_t extent);
/* Projects and drops this accumulator's staged tracks. */
int c8r_project_staged(c8r_accumulator* handle);
/* Changes team_size (threads per windowed CTA) and track_tile_size (tracks per
 * work item, 0 = automatic) of an accumulator. */
int c8r_set_tuning(c8r_accumulator* handle, const c8r_tuning* tuning);

typedef struct c8r_batch c8r_batch;
enum {
  C8R_BATCH_GRAPH = 1,       /* replay a CUDA graph captured per distinct launch plan */
  C8R_BATCH_KEEP_STAGED = 2  /* keep the staged tracks after projecting them */
};
/* A batch projects the staged tracks of several accumulators (one shower each,
 * same stream, precision and trace mode) with one persistent launch per
 * algorithm for up to 64 events; graph replay needs a non-default stream. */
int c8r_batch_create(void* stream, c8r_batch** batch);
void c8r_batch_destroy(c8r_batch* batch);
const char* c8r_batch_last_error(const c8r_batch* batch);
int c8r_batch_project(c8r_batch* batch, c8r_accumulator* const* events, size_t count, int flags);
/* Sweeps the windowed kernel's tile space on the staged events (repetitions
 * timed runs each): team size (track segments per stage) {256,384,512,640} x
 * tracks per item {auto,32768,131072,524288} with the whole trace as bin
 * window, then bin windows {2048,1024,512} shorter than the longest trace at
 * the best pair (one antenna per CTA).  Applies the fastest to every event,
 * zeroes the traces the sweep wrote and returns it (observer_tile_size 0:
 * the whole trace). */
int c8r_batch_autotune(c8r_batch* batch, c8r_accumulator* const* events, size_t count,
                       int repetitions, c8r_tuning* best, double* best_ms);
int c8r_batch_graph_captures(const c8r_batch* batch, unsigned long long* captures);

/* ---- Tuning cache -----------------------------------------------------------
 * In the manner of the reference's c8-kokkos-tuning-v1 cache
 * (corsika/kokkos/runtime/TuningCache.hpp:16-47): the autotuner's choice
 * persisted as key=value lines ("c8radio-b200-tuning-v1"), keyed by the
 * current device (name, compute capability, multiprocessors), driver and
 * runtime versions, this library's version and a caller-chosen one-line
 * workload label.  load sets *matched = 1 and *tuning (team_size,
 * track_tile_size, observer_tile_size) only when the file exists and every
 * key field equals the current one; a missing or non-matching file gives
 * *matched = 0 (C8R_RUNTIME_ERROR when require_match), a malformed one
 * C8R_RUNTIME_ERROR.  store writes a temporary file and renames it. */
int c8r_tuning_cache_load(const char* path, const char* workload, int require_match, c8r_tuning* tuning,
                          int* matched);
int c8r_tuning_cache_store(const char* path, const char* workload, const c8r_tuning* tuning);
const char* c8r_tuning_cache_last_error(void);

/* ---- Producer-side input: track steps as columns ----------------------------
 * No counterpart in the reference, which reads the 752-byte records
 * (LeptonCascade.inl:81-83).  A producer that keeps its steps as a structure
 * of arrays passes one device array per field radio reads, and skips writing
 * and reading the records: the ingest reads about 100 bytes a track, in
 * coalesced columns.  Same kinematics, bit for bit, as from records.  The
 * direction and start-energy columns are read only with track_diagnostics. */
typedef struct c8r_track_columns {
  const int32_t* pid;               /* start state's PDG id (11, -11; others skipped) */
  const double* weight;             /* start state's weight */
  const double* start_time_s;
  const double* end_time_s;
  const double* start_energy_gev;   /* total energy (diagnostics) */
  const double* start_position_m[3];
  const double* end_position_m[3];
  const double* start_direction[3]; /* diagnostics */
  const double* end_direction[3];   /* diagnostics */
} c8r_track_columns;
/* accumulateLeptonTracks over columns: count steps, stream ordered. */
int c8r_accumulate_columns(c8r_accumulator* handle, const c8r_track_columns* columns, size_t count);

/* ---- Output step on the device ----------------------------------------------
 * RadioProcess.inl:213-223 and CorsikaOutputSink.inl:255-278: like c8r_download,
 * but the decoded CoREAS fields (V/m, rows [X | Y | Z] of the CoREAS total bins)
 * and the ZHS fields E_i = -(A_{i+1} - A_i) fs at the bin midpoints (V/m, one
 * sample fewer per observer: rows of zhs total bins - zhs observers) are ADDED
 * into caller-owned device buffers, so the waveforms of many showers sum on the
 * device before one copy to the host.  Seals the accumulator as download does. */
int c8r_download_fields_device(c8r_accumulator* handle, double* coreas_field_xyz, double* zhs_field_xyz,
                               c8r_counters* counters);
/* merge_fixed_accumulators (FixedAccumulatorMerge.inl:12-29), the core of
 * CooperativeRadioMerge::commit (CooperativeRadioMerge.inl:180-202):
 * destination += source for int64 fixed-point snapshots of one layout, every
 * bin checked first; C8R_OVERFLOW_ERROR (nothing written) on overflow. */
int c8r_merge_fixed(long long* destination, const long long* source, size_t count);

/* ---- Cooperative fixed-point export ------------------------------------------
 * corsika/kokkos/scheduling/CooperativeEndpoint.hpp: the two endpoints that
 * may each project part of one shower. */
enum {
  C8R_ENDPOINT_CUDA = 0,
  C8R_ENDPOINT_OPENMP = 1
};
/* FixedRadioSnapshot (corsika/kokkos/radio/FixedRadioSnapshot.hpp:18-24) as a
 * view over caller-owned arrays: the final int64 traces of one endpoint of one
 * shower (ZHS as potential), in the accumulator's SoA order.  Each trace array
 * holds 3 x the bins of EVERY observer the config lists for its algorithm
 * (c8r_snapshot_bins), zero for a disabled algorithm. */
typedef struct c8r_fixed_snapshot {
  const char* shower_identity;  /* NUL-terminated, non-empty */
  uint32_t endpoint;            /* C8R_ENDPOINT_* */
  uint32_t reserved_;
  const c8r_config* config;     /* the config the endpoint was created with */
  const long long* coreas;
  size_t coreas_count;          /* 3 x CoREAS bins */
  const long long* zhs;
  size_t zhs_count;             /* 3 x ZHS bins */
  c8r_counters counters;
} c8r_fixed_snapshot;
/* RadioAccumulator::downloadFixed(shower_identity, endpoint)
 * (RadioAccumulator.inl:359-405): flushes the pending host batch, checks the
 * identity and endpoint (C8R_INVALID_ARGUMENT, nothing sealed), seals the
 * accumulator, copies the int64 traces and counters, then validates them
 * (validate_fixed_radio: an overflowed accumulator gives C8R_INVALID_ARGUMENT
 * and stays sealed).  C8R_LOGIC_ERROR when disabled, not deterministic,
 * already downloaded or sealed.  Buffers sized by c8r_snapshot_bins. */
int c8r_download_fixed_snapshot(c8r_accumulator* handle, const char* shower_identity, uint32_t endpoint,
                                long long* coreas_xyz, long long* zhs_xyz, c8r_counters* counters);
/* Bins of every configured observer of each algorithm (snapshot extents / 3). */
int c8r_snapshot_bins(const c8r_accumulator* handle, size_t* coreas_bins, size_t* zhs_bins);
/* validate_fixed_radio (CooperativeRadioMerge.inl:142-152). */
int c8r_validate_fixed_snapshot(const c8r_fixed_snapshot* snapshot);
/* merge_radio_counters (CooperativeRadioMerge.inl:154-208): destination +=
 * source; C8R_OVERFLOW_ERROR (destination unchanged) when an integer counter
 * would wrap or a diagnostic sum or maximum is not finite. */
int c8r_merge_counters(c8r_counters* destination, const c8r_counters* source);
/* Message of the last failing snapshot call of this thread without a merge. */
const char* c8r_snapshot_last_error(void);
/* CooperativeRadioMerge (CooperativeRadioMerge.hpp:53-65, .inl:240-277): one
 * shower's identity and config (deep-copied at creation).  commit accepts each
 * endpoint's snapshot once; it rejects an invalid snapshot, a second commit of
 * an endpoint, another identity or a config of different physics
 * (C8R_INVALID_ARGUMENT), an int64 bin or counter overflow of the sum
 * (C8R_OVERFLOW_ERROR) and any commit after take (C8R_LOGIC_ERROR); a rejected
 * commit changes nothing.  take writes the merged traces (sized like a
 * snapshot of the config), counters and the first commit's endpoint once both
 * endpoints are in; otherwise, or a second time, C8R_LOGIC_ERROR. */
typedef struct c8r_cooperative_merge c8r_cooperative_merge;
int c8r_cooperative_merge_create(const char* shower_identity, const c8r_config* config,
                                 c8r_cooperative_merge** merge);
void c8r_cooperative_merge_destroy(c8r_cooperative_merge* merge);
const char* c8r_cooperative_merge_last_error(const c8r_cooperative_merge* merge);
int c8r_cooperative_merge_commit(c8r_cooperative_merge* merge, const c8r_fixed_snapshot* snapshot);
int c8r_cooperative_merge_take(c8r_cooperative_merge* merge, long long* coreas_xyz, long long* zhs_xyz,
                               c8r_counters* counters, uint32_t* endpoint);

/* ---- Track spool, version 1: completed host tracks on disk ----------------
 * corsika/kokkos/radio/RadioTrackSpoolFormat.hpp:24-29 and
 * RadioTrackSpool{Reader,Writer}.hpp: a 32-byte header ("C8_RADIO_TRACKS\0",
 * version 1, record size 140, record count, all ones until completed) and
 * one 140-byte little-endian record per track.  Failures return
 * C8R_RUNTIME_ERROR with c8r_last_global_error() set, as the reference throws
 * std::runtime_error. */
typedef struct c8r_track_segment { /* corsika::radio::RadioTrackSegment */
  int32_t pdg;                     /* 11 or -11 */
  double start_position_m[3];
  double end_position_m[3];
  double start_direction[3];
  double end_direction[3];
  double start_time_s;
  double end_time_s;
  double start_kinetic_energy_gev;
  double end_kinetic_energy_gev;
  double weight;
} c8r_track_segment;
typedef struct c8r_spool_writer c8r_spool_writer;
typedef struct c8r_spool_reader c8r_spool_reader;
/* RadioTrackSpoolWriter (RadioTrackSpoolWriter.inl:11-45): refuses an existing
 * path; append validates each track; only complete() publishes the count. */
int c8r_spool_writer_create(const char* path, c8r_spool_writer** writer);
int c8r_spool_append(c8r_spool_writer* writer, const c8r_track_segment* tracks, size_t count);
int c8r_spool_complete(c8r_spool_writer* writer);
int c8r_spool_writer_count(const c8r_spool_writer* writer, uint64_t* count);
void c8r_spool_writer_destroy(c8r_spool_writer* writer);
/* RadioTrackSpoolReader (RadioTrackSpoolReader.inl:11-47): validates magic,
 * version, record size, completion and file length; reads at most `maximum`
 * (1..65536) tracks per call, each validated. */
int c8r_spool_reader_open(const char* path, c8r_spool_reader** reader, uint64_t* count);
int c8r_spool_read(c8r_spool_reader* reader, c8r_track_segment* tracks, size_t maximum, size_t* read);
int c8r_spool_reader_state(const c8r_spool_reader* reader, uint64_t* consumed, int* finished);
void c8r_spool_reader_destroy(c8r_spool_reader* reader);
/* make_host_radio_record (HostRadioRecord.inl:11-31): total energy = kinetic + m_e. */
int c8r_track_records(const c8r_track_segment* tracks, size_t count, c8r_lepton_transport_record* records);
/* Replays every remaining track of a spool into an accumulator as host tracks
 * (c8r_enqueue_host), read in batches of `batch` (1..65536). */
int c8r_spool_replay(c8r_spool_reader* reader, c8r_accumulator* accumulator, size_t batch);

/* ---- Serving: many showers in flight on one GPU ---------------------------
 * No reference counterpart (the reference runs one shower per accumulator).
 * A server reserves one HBM arena of budget_bytes at creation and admits
 * events against it.  An admitted event keeps its observer constants,
 * refractivity table, traces and counters resident; its tracks are ingested
 * into kinematics blocks of block_tracks tracks taken from the arena and
 * handed back once projected, so an event of any size needs only a few
 * blocks at a time.  A scheduler thread projects in rounds: each round is one
 * persistent windowed launch per algorithm over slices of every ready event
 * (about round_pairs track-antenna pairs, shared evenly among the events), so
 * events that arrive while others are on the GPU join the next round.  Each
 * event's traces are the same, bit for bit in fixed-point mode, as those of an
 * accumulator that projects it alone.  All calls are thread-safe. */
typedef struct c8r_server c8r_server;
typedef struct c8r_server_options {
  uint64_t budget_bytes; /* HBM arena reserved at creation (events, blocks) */
  uint64_t block_tracks; /* tracks per kinematics block; 0 = 1048576 */
  uint64_t chunk_tracks; /* tracks per work item; 0 = 131072 (divides block_tracks, at most 2^30) */
  uint64_t round_pairs;  /* track-observer pairs per round; 0 = 1e9 */
  uint32_t team_size;    /* threads per windowed CTA; 0 = 640 (ZHS CTAs: 384 to 768) */
  uint32_t reserved_[7];
} c8r_server_options;
typedef struct c8r_server_event_info {
  uint64_t records;            /* records added */
  uint64_t coreas_observers, zhs_observers;
  uint64_t rounds;             /* rounds that projected part of the event */
  double open_s, admitted_s, closed_s, completed_s;  /* server clock (s since creation) */
} c8r_server_event_info;
typedef struct c8r_server_stats {
  uint64_t rounds, launches, events_admitted, events_completed, blocks_allocated;
  uint64_t arena_bytes, arena_used_bytes, arena_peak_bytes;
  uint64_t work_items;         /* (chunk, antenna) items launched */
} c8r_server_stats;

int c8r_server_create(const c8r_server_options* options, c8r_server** server);
void c8r_server_destroy(c8r_server* server);
const char* c8r_server_last_error(const c8r_server* server);
/* Admits an event: waits up to timeout_ms (< 0: no limit) until its resident
 * part and one kinematics block fit the arena (C8R_TIMEOUT otherwise). */
int c8r_server_open(c8r_server* server, const c8r_config* config, int timeout_ms, uint64_t* event);
/* Ingests device records on `stream` (ordered with the producer, like
 * c8r_accumulate_device); waits for a free block when its block is full. */
int c8r_server_add_device(c8r_server* server, uint64_t event, const c8r_lepton_transport_record* records,
                          size_t count, size_t extent, void* stream);
/* No more tracks: the event completes once all its tracks are projected. */
int c8r_server_close(c8r_server* server, uint64_t event);
/* C8R_OK once the event is complete, C8R_TIMEOUT after timeout_ms (< 0: no limit). */
int c8r_server_wait(c8r_server* server, uint64_t event, int timeout_ms);
/* Copies a complete event's traces to host memory (fixed-point as
 * c8r_download_fixed, or decoded as c8r_download) and releases the event. */
int c8r_server_fetch_fixed(c8r_server* server, uint64_t event, long long* coreas_xyz, long long* zhs_xyz,
                           c8r_counters* counters, c8r_server_event_info* info);
int c8r_server_fetch(c8r_server* server, uint64_t event, double* coreas_xyz, double* zhs_xyz,
                     c8r_counters* counters, c8r_server_event_info* info);
int c8r_server_get_stats(const c8r_server* server, c8r_server_stats* stats);

/* ---- Accumulate without allocating device memory ---------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they project tracks: a transport code that has given all of HBM
 * to its own pool allocator (a Kokkos memory pool, a particle stack sized to
 * the card), or one that drives several streams and cannot accept the device
 * synchronisation of cudaMalloc/cudaFree.
 *
 * Ingests `count` device records (count <= extent) and adds their CoREAS
 * field and ZHS potential into CALLER-OWNED device traces, with the
 * accumulator's trace layout and units: rows [X | Y | Z] of the algorithm's
 * total bins, observers in config order; long long fixed-point values when
 * config->deterministic (as c8r_download_fixed returns them), else double.
 * `counters` is a device c8r_counters added into, or NULL.  Fixed-point
 * overflows are reported only through counters->fixed_point_overflows (the
 * call itself does not wait for the GPU): a caller that passes NULL gives up
 * overflow detection.  The caller zeroes traces and counters before its
 * first call; later calls add to them, as c8r_accumulate_device does.
 * config->kernel is ignored (always the windowed projection).  Every host
 * array of the config (observers, refractivity tables) has been read when
 * the call returns: observer constants and the table travel to the device as
 * kernel parameters, so the call does not wait for earlier work on `stream`
 * whatever memory those arrays are in.  The work itself is queued on
 * `stream`.  A call with count == 0 does nothing on the device.
 *
 * Scratch: one static device array of C8R_NO_ALLOC_SCRATCH_BYTES per GPU that
 * loads this library's module, held until the process exits.  The call calls
 * no cudaMalloc, cudaFree or other allocating routine.  Its first call on a
 * device sets up that device (looks up the array's address, loading the
 * module there if needed): make that first call before any stream capture.
 * All calls on a device share the array, so calls that overlap on the GPU
 * race: keep them ordered on one stream.  Records are processed in chunks
 * that fit the array, so `count` has no limit; more than
 * C8R_NO_ALLOC_MAX_OBSERVERS observers (CoREAS + ZHS) or a refractivity table
 * of more than C8R_NO_ALLOC_MAX_TABLE_ENTRIES entries is rejected with
 * C8R_LENGTH_ERROR before any device work. */
#define C8R_NO_ALLOC_SCRATCH_BYTES (32u << 20)
#define C8R_NO_ALLOC_MAX_OBSERVERS 2048u
#define C8R_NO_ALLOC_MAX_TABLE_ENTRIES 131072u
int c8r_accumulate_device_no_alloc(const c8r_config* config,
                                   const c8r_lepton_transport_record* records, size_t count,
                                   size_t extent, void* coreas_traces, void* zhs_traces,
                                   c8r_counters* counters, void* stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* C8RADIO_H */
