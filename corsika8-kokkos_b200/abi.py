"""ctypes mirror of include/c8radio.h and the numpy record layout.

Every struct here has the byte layout of its C declaration, which in turn has
the layout of the corresponding CORSIKA8-kokkos type (LeptonTransportRecord,
RadioObserverSnapshot, FlatAtmosphereRadioSnapshot, RadioConfig,
TuningParameters, RadioCounters, RadioStatistics).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

# corsika/kokkos/data/ParticleState.hpp:24-44 (128 bytes)
PARTICLE_STATE = np.dtype(
    [
        ("pid", "<i4"),
        ("medium_id", "<i4"),
        ("generation", "<u4"),
        ("reserved", "<u4"),
        ("energy_gev", "<f8"),
        ("position_m", "<f8", (3,)),
        ("direction", "<f8", (3,)),
        ("time_s", "<f8"),
        ("weight", "<f8"),
        ("history_id", "<u8"),
        ("parent_history_id", "<u8"),
        ("step_id", "<u8"),
        ("environment_node", "<i4"),
        ("pad_", "<i4", (3,)),
    ],
    align=False,
)
assert PARTICLE_STATE.itemsize == 128

# corsika/kokkos/em/LeptonTransportRecord.hpp:38-70 (752 bytes)
LEPTON_RECORD = np.dtype(
    [
        ("interaction", "u1", (320,)),
        ("start", PARTICLE_STATE),
        ("end", PARTICLE_STATE),
        ("transport", "u1", (176,)),
    ]
)
assert LEPTON_RECORD.itemsize == 752

# RadioObserverSnapshot (56 bytes)
OBSERVER = np.dtype(
    [
        ("position_m", "<f8", (3,)),
        ("start_time_s", "<f8"),
        ("duration_s", "<f8"),
        ("sample_rate_hz", "<f8"),
        ("number_of_bins", "<u8"),
    ]
)
assert OBSERVER.itemsize == 56

C8R_OK = 0
C8R_INVALID_ARGUMENT = 1
C8R_LOGIC_ERROR = 2
C8R_OUT_OF_RANGE = 3
C8R_RUNTIME_ERROR = 4
C8R_LENGTH_ERROR = 5
C8R_OVERFLOW_ERROR = 6
C8R_CUDA_ERROR = 7
C8R_BAD_ALLOC = 8
C8R_TIMEOUT = 9

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_STUDY_DOUBLE_FP32 = 2
PRECISION_STUDY_FP32 = 3
PRECISION_STUDY_FP64 = 4
KERNEL_AUTO = 0
KERNEL_DIRECT = 1
KERNEL_WINDOWED = 2
KERNEL_TILED = 3
BATCH_GRAPH = 1
BATCH_KEEP_STAGED = 2


class ObserverSnapshot(C.Structure):
    _fields_ = [
        ("position_m", C.c_double * 3),
        ("start_time_s", C.c_double),
        ("duration_s", C.c_double),
        ("sample_rate_hz", C.c_double),
        ("number_of_bins", C.c_uint64),
    ]


class PropagationSnapshot(C.Structure):
    _fields_ = [
        ("homogeneous_refractive_index", C.c_double),
        ("minimum_height_m", C.c_double),
        ("maximum_height_m", C.c_double),
        ("step_m", C.c_double),
        ("inverse_step_per_m", C.c_double),
        ("slope_refractivity_lower", C.c_double),
        ("slope_integrated_refractivity_lower", C.c_double),
        ("slope_refractivity_upper", C.c_double),
        ("slope_integrated_refractivity_upper", C.c_double),
        ("refractivity", C.POINTER(C.c_double)),
        ("integrated_refractivity", C.POINTER(C.c_double)),
        ("table_size", C.c_uint64),
    ]


class Config(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32),
        ("coreas_enabled", C.c_int32),
        ("zhs_enabled", C.c_int32),
        ("deterministic", C.c_int32),
        ("fixed_point_field_limit_v_per_m", C.c_double),
        ("track_diagnostics", C.c_int32),
        ("zhs_subtrack_refinement", C.c_uint32),
        ("propagation", PropagationSnapshot),
        ("coreas_observers", C.c_void_p),
        ("coreas_observer_count", C.c_uint64),
        ("zhs_observers", C.c_void_p),
        ("zhs_observer_count", C.c_uint64),
        ("precision", C.c_int32),
        ("kernel", C.c_int32),
        ("count_samples", C.c_int32),
        ("reserved_", C.c_int32),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("batch_size", C.c_uint64),
        ("chunk_size", C.c_uint64),
        ("team_size", C.c_uint64),
        ("track_tile_size", C.c_uint64),
        ("observer_tile_size", C.c_uint64),
        ("device_queues", C.c_uint64),
    ]


COUNTER_FIELDS = [
    ("coreas_contributions", C.c_ulonglong),
    ("zhs_contributions", C.c_ulonglong),
    ("zhs_subtracks", C.c_ulonglong),
    ("valid_tracks", C.c_ulonglong),
    ("fixed_point_overflows", C.c_ulonglong),
    ("weighted_segment_count", C.c_double),
    ("track_length_m", C.c_double),
    ("weighted_track_length_m", C.c_double),
    ("electron_weighted_track_length_m", C.c_double),
    ("positron_weighted_track_length_m", C.c_double),
    ("signed_charge_weighted_track_length_m", C.c_double),
    ("energy_weighted_track_length_gev_m", C.c_double),
    ("maximum_segment_length_m", C.c_double),
    ("weighted_direction_change_rad", C.c_double),
    ("weighted_direction_change_squared_rad2", C.c_double),
    ("weighted_beta_deficit_track_length_m", C.c_double),
    ("weighted_time_residual_s", C.c_double),
    ("maximum_direction_change_rad", C.c_double),
    ("signed_charge_weighted_direction_change", C.c_double * 3),
    ("weighted_track_length_by_kinetic_energy_m", C.c_double * 15),
]


class Counters(C.Structure):
    _fields_ = COUNTER_FIELDS

    def as_dict(self) -> dict:
        out = {}
        for name, kind in COUNTER_FIELDS:
            value = getattr(self, name)
            out[name] = list(value) if isinstance(value, C.Array) else value
        return out


assert C.sizeof(Counters) == 288


class Statistics(C.Structure):
    _fields_ = [
        ("lepton_tracks", C.c_uint64),
        ("track_observer_pairs", C.c_uint64),
        ("fused_track_observer_pairs", C.c_uint64),
        ("coreas_contributions", C.c_uint64),
        ("zhs_contributions", C.c_uint64),
        ("zhs_subtracks", C.c_uint64),
        ("fixed_point_overflows", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("host_to_device_bytes", C.c_uint64),
        ("host_tracks_enqueued", C.c_uint64),
        ("host_track_batches", C.c_uint64),
        ("device_to_host_bytes", C.c_uint64),
        ("track_precompute_batches", C.c_uint64),
        ("track_precomputed_records", C.c_uint64),
        ("direct_projection_batches", C.c_uint64),
        ("direct_projection_records", C.c_uint64),
        ("projection_tiles", C.c_uint64),
        ("track_workspace_bytes", C.c_uint64),
        ("maximum_track_batch", C.c_uint64),
        ("track_tile_size", C.c_uint32),
        ("observer_tile_size", C.c_uint32),
        ("kernel_time_ms", C.c_double),
        ("timed_launches", C.c_uint64),
        ("coreas_kernel_time_ms", C.c_double),
        ("zhs_kernel_time_ms", C.c_double),
        ("counters", Counters),
        ("window_reruns", C.c_uint64),
        ("window_handbacks", C.c_uint64),
    ]


class Peaks(C.Structure):
    _fields_ = [("fp64_flops", C.c_double), ("fp32_flops", C.c_double),
                ("shared_atomics_per_s", C.c_double), ("global_atomics_per_s", C.c_double)]


# Exported symbols of libc8radio.so and their prototypes.
TRACK_SEGMENT = np.dtype([
    ("pdg", np.int32), ("start_position_m", np.float64, 3), ("end_position_m", np.float64, 3),
    ("start_direction", np.float64, 3), ("end_direction", np.float64, 3), ("start_time_s", np.float64),
    ("end_time_s", np.float64), ("start_kinetic_energy_gev", np.float64),
    ("end_kinetic_energy_gev", np.float64), ("weight", np.float64)], align=True)
assert TRACK_SEGMENT.itemsize == 144


class TrackColumns(C.Structure):
    _fields_ = [("pid", C.c_void_p), ("weight", C.c_void_p), ("start_time_s", C.c_void_p),
                ("end_time_s", C.c_void_p), ("start_energy_gev", C.c_void_p),
                ("start_position_m", C.c_void_p * 3), ("end_position_m", C.c_void_p * 3),
                ("start_direction", C.c_void_p * 3), ("end_direction", C.c_void_p * 3)]


class FixedSnapshot(C.Structure):
    """c8r_fixed_snapshot: a view of one endpoint's FixedRadioSnapshot."""
    _fields_ = [
        ("shower_identity", C.c_char_p),
        ("endpoint", C.c_uint32),
        ("reserved_", C.c_uint32),
        ("config", C.POINTER(Config)),
        ("coreas", C.c_void_p),
        ("coreas_count", C.c_size_t),
        ("zhs", C.c_void_p),
        ("zhs_count", C.c_size_t),
        ("counters", Counters),
    ]


ENDPOINT_CUDA = 0
ENDPOINT_OPENMP = 1


class ServerOptions(C.Structure):
    _fields_ = [
        ("budget_bytes", C.c_uint64),
        ("block_tracks", C.c_uint64),
        ("chunk_tracks", C.c_uint64),
        ("round_pairs", C.c_uint64),
        ("team_size", C.c_uint32),
        ("reserved_", C.c_uint32 * 7),
    ]


class ServerEventInfo(C.Structure):
    _fields_ = [
        ("records", C.c_uint64),
        ("coreas_observers", C.c_uint64),
        ("zhs_observers", C.c_uint64),
        ("rounds", C.c_uint64),
        ("open_s", C.c_double),
        ("admitted_s", C.c_double),
        ("closed_s", C.c_double),
        ("completed_s", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [(name, C.c_uint64) for name in (
        "rounds", "launches", "events_admitted", "events_completed", "blocks_allocated",
        "arena_bytes", "arena_used_bytes", "arena_peak_bytes", "work_items")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


PROTOTYPES = {
    "c8r_version": (C.c_char_p, []),
    "c8r_last_error": (C.c_char_p, [C.c_void_p]),
    "c8r_last_global_error": (C.c_char_p, []),
    "c8r_config_validate": (C.c_int, [C.POINTER(Config)]),
    "c8r_projected_device_bytes": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_size_t)]),
    "c8r_create": (C.c_int, [C.POINTER(Config), C.POINTER(Tuning), C.c_void_p, C.POINTER(C.c_void_p)]),
    "c8r_destroy": (None, [C.c_void_p]),
    "c8r_enabled": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "c8r_reset": (C.c_int, [C.c_void_p]),
    "c8r_enqueue_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "c8r_flush": (C.c_int, [C.c_void_p]),
    "c8r_accumulate_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t]),
    "c8r_download": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Counters)]),
    "c8r_download_fixed": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Counters)]),
    "c8r_total_bins": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "c8r_get_statistics": (C.c_int, [C.c_void_p, C.POINTER(Statistics)]),
    "c8r_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "c8r_static_host_to_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "c8r_reserve": (C.c_int, [C.c_void_p, C.c_size_t]),
    "c8r_projected_track_capacity": (
        C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "c8r_synchronize": (C.c_int, [C.c_void_p]),
    "c8r_set_kernel_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "c8r_probe_peaks": (C.c_int, [C.POINTER(Peaks)]),
    "c8r_stage_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t]),
    "c8r_project_staged": (C.c_int, [C.c_void_p]),
    "c8r_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    "c8r_batch_create": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "c8r_batch_destroy": (None, [C.c_void_p]),
    "c8r_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "c8r_batch_project": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_size_t, C.c_int]),
    "c8r_batch_autotune": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_size_t, C.c_int,
                                     C.POINTER(Tuning), C.POINTER(C.c_double)]),
    "c8r_batch_graph_captures": (C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong)]),
    "c8r_tuning_cache_load": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(Tuning),
                                        C.POINTER(C.c_int)]),
    "c8r_tuning_cache_store": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(Tuning)]),
    "c8r_tuning_cache_last_error": (C.c_char_p, []),
    "c8r_server_create": (C.c_int, [C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]),
    "c8r_server_destroy": (None, [C.c_void_p]),
    "c8r_server_last_error": (C.c_char_p, [C.c_void_p]),
    "c8r_server_open": (C.c_int, [C.c_void_p, C.POINTER(Config), C.c_int, C.POINTER(C.c_uint64)]),
    "c8r_server_add_device": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_size_t, C.c_size_t,
                                        C.c_void_p]),
    "c8r_server_close": (C.c_int, [C.c_void_p, C.c_uint64]),
    "c8r_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int]),
    "c8r_server_fetch_fixed": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                         C.POINTER(Counters), C.POINTER(ServerEventInfo)]),
    "c8r_server_fetch": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                   C.POINTER(Counters), C.POINTER(ServerEventInfo)]),
    "c8r_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "c8r_accumulate_columns": (C.c_int, [C.c_void_p, C.POINTER(TrackColumns), C.c_size_t]),
    "c8r_download_fields_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Counters)]),
    "c8r_merge_fixed": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "c8r_download_fixed_snapshot": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                              C.POINTER(Counters)]),
    "c8r_snapshot_bins": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "c8r_validate_fixed_snapshot": (C.c_int, [C.POINTER(FixedSnapshot)]),
    "c8r_merge_counters": (C.c_int, [C.POINTER(Counters), C.POINTER(Counters)]),
    "c8r_snapshot_last_error": (C.c_char_p, []),
    "c8r_cooperative_merge_create": (C.c_int, [C.c_char_p, C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "c8r_cooperative_merge_destroy": (None, [C.c_void_p]),
    "c8r_cooperative_merge_last_error": (C.c_char_p, [C.c_void_p]),
    "c8r_cooperative_merge_commit": (C.c_int, [C.c_void_p, C.POINTER(FixedSnapshot)]),
    "c8r_cooperative_merge_take": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Counters),
                                             C.POINTER(C.c_uint32)]),
    "c8r_spool_writer_create": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "c8r_spool_append": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "c8r_spool_complete": (C.c_int, [C.c_void_p]),
    "c8r_spool_writer_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "c8r_spool_writer_destroy": (None, [C.c_void_p]),
    "c8r_spool_reader_open": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]),
    "c8r_spool_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "c8r_spool_reader_state": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_int)]),
    "c8r_spool_reader_destroy": (None, [C.c_void_p]),
    "c8r_track_records": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p]),
    "c8r_spool_replay": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "c8r_accumulate_device_no_alloc": (C.c_int, [C.POINTER(Config), C.c_void_p, C.c_size_t, C.c_size_t,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
}


def bind(lib: C.CDLL) -> C.CDLL:
    for name, (restype, argtypes) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    return lib
