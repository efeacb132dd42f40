"""B200 radio projection (CoREAS endpoint field + ZHS vector potential).

Python view of libc8radio.so, the sm_100a drop-in for the CORSIKA8-kokkos
radio accumulator (corsika/kokkos/radio/RadioAccumulator.hpp).  Names and
argument meaning follow the reference: a RadioConfig with CoREAS and ZHS
observer snapshots and a flat-atmosphere refractivity table, a
RadioAccumulator fed LeptonTransportRecord batches from host or device
memory, and download()/download_fixed() returning the traces.  Failures raise
the Python counterparts of the reference's exception classes.

There is no CPU fallback: every call runs the CUDA library, and loading the
package without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional

import numpy as np

from . import abi
from .abi import LEPTON_RECORD, OBSERVER, PARTICLE_STATE  # noqa: F401

HERE = Path(__file__).resolve().parent
# C8R_LIBRARY selects another build of the library (A/B comparisons).
LIBRARY_PATH = Path(os.environ["C8R_LIBRARY"]).resolve() if os.environ.get("C8R_LIBRARY") else HERE / "libc8radio.so"

# ------------------------------------------------------------------ errors
class RadioError(RuntimeError):
    """Base class of radio failures reported by the C boundary."""


class InvalidArgument(RadioError, ValueError):
    """std::invalid_argument"""


class LogicError(RadioError):
    """std::logic_error"""


class OutOfRange(RadioError, IndexError):
    """std::out_of_range"""


class FixedPointOverflow(RadioError):
    """std::runtime_error raised at download when the fixed-point traces overflowed"""


class LengthError(RadioError):
    """std::length_error"""


class OverflowErrorRadio(RadioError, OverflowError):
    """std::overflow_error"""


class CudaError(RadioError):
    """CUDA runtime failure"""


class AllocationError(RadioError, MemoryError):
    """device or pinned allocation failure"""


class ServerTimeout(RadioError, TimeoutError):
    """server: not admitted / not complete within the timeout"""


_STATUS = {
    abi.C8R_INVALID_ARGUMENT: InvalidArgument,
    abi.C8R_LOGIC_ERROR: LogicError,
    abi.C8R_OUT_OF_RANGE: OutOfRange,
    abi.C8R_RUNTIME_ERROR: FixedPointOverflow,
    abi.C8R_LENGTH_ERROR: LengthError,
    abi.C8R_OVERFLOW_ERROR: OverflowErrorRadio,
    abi.C8R_CUDA_ERROR: CudaError,
    abi.C8R_BAD_ALLOC: AllocationError,
    abi.C8R_TIMEOUT: ServerTimeout,
}

_lib: Optional[C.CDLL] = None


def library() -> C.CDLL:
    """Loads libc8radio.so (building it first if sources are newer)."""
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            from . import build as _build

            _build.build()
        if not LIBRARY_PATH.exists():
            raise ImportError(f"libc8radio.so is missing at {LIBRARY_PATH}; run build.py")
        _lib = abi.bind(C.CDLL(str(LIBRARY_PATH)))
    return _lib


def _raise(status: int, message: bytes | None) -> None:
    if status == abi.C8R_OK:
        return
    text = (message or b"").decode(errors="replace")
    raise _STATUS.get(status, RadioError)(text or f"radio status {status}")


# ------------------------------------------------------------------ config
@dataclass
class FlatAtmosphereSnapshot:
    """corsika/kokkos/radio/FlatAtmosphereRadioSnapshot.hpp:20-36"""

    homogeneous_refractive_index: float = 0.0
    minimum_height_m: float = 0.0
    maximum_height_m: float = 0.0
    step_m: float = 0.0
    inverse_step_per_m: float = 0.0
    slope_refractivity_lower: float = 0.0
    slope_integrated_refractivity_lower: float = 0.0
    slope_refractivity_upper: float = 0.0
    slope_integrated_refractivity_upper: float = 0.0
    refractivity: np.ndarray = field(default_factory=lambda: np.zeros(0))
    integrated_refractivity: np.ndarray = field(default_factory=lambda: np.zeros(0))


@dataclass
class RadioConfig:
    """corsika/kokkos/radio/RadioConfig.hpp:21-53 plus the B200 precision/kernel choice."""

    enabled: bool = False
    coreas_enabled: bool = True
    zhs_enabled: bool = True
    deterministic: bool = True
    fixed_point_field_limit_v_per_m: float = 1.0
    track_diagnostics: bool = False
    zhs_subtrack_refinement: int = 1
    propagation: FlatAtmosphereSnapshot = field(default_factory=FlatAtmosphereSnapshot)
    coreas_observers: np.ndarray = field(default_factory=lambda: np.zeros(0, OBSERVER))
    zhs_observers: np.ndarray = field(default_factory=lambda: np.zeros(0, OBSERVER))
    precision: int = abi.PRECISION_FP64
    kernel: int = abi.KERNEL_AUTO
    count_samples: bool = False

    def to_c(self):
        """Returns (abi.Config, keepalive) with pointers into contiguous copies."""
        keep = []
        p = self.propagation
        n = np.ascontiguousarray(p.refractivity, dtype=np.float64)
        i = np.ascontiguousarray(p.integrated_refractivity, dtype=np.float64)
        co = np.ascontiguousarray(self.coreas_observers, dtype=OBSERVER)
        zo = np.ascontiguousarray(self.zhs_observers, dtype=OBSERVER)
        keep += [n, i, co, zo]
        dptr = C.POINTER(C.c_double)
        prop = abi.PropagationSnapshot(
            p.homogeneous_refractive_index, p.minimum_height_m, p.maximum_height_m, p.step_m,
            p.inverse_step_per_m, p.slope_refractivity_lower,
            p.slope_integrated_refractivity_lower, p.slope_refractivity_upper,
            p.slope_integrated_refractivity_upper,
            n.ctypes.data_as(dptr) if n.size else dptr(),
            i.ctypes.data_as(dptr) if i.size else dptr(),
            int(n.size),
        )
        cfg = abi.Config(
            int(self.enabled), int(self.coreas_enabled), int(self.zhs_enabled),
            int(self.deterministic), float(self.fixed_point_field_limit_v_per_m),
            int(self.track_diagnostics), int(self.zhs_subtrack_refinement), prop,
            co.ctypes.data if co.size else None, int(co.size),
            zo.ctypes.data if zo.size else None, int(zo.size),
            int(self.precision), int(self.kernel), int(self.count_samples), 0,
        )
        return cfg, keep


@dataclass
class TuningParameters:
    """corsika/kokkos/runtime/TuningParameters.hpp:14-21 (zero keeps defaults).

    batch_size: host staging batch (records); team_size: threads per windowed
    CTA; track_tile_size: tracks per windowed work item; observer_tile_size:
    shared-memory window (bins)."""

    batch_size: int = 0
    chunk_size: int = 0
    team_size: int = 0
    track_tile_size: int = 0
    observer_tile_size: int = 0
    device_queues: int = 1

    def to_c(self) -> abi.Tuning:
        return abi.Tuning(self.batch_size, self.chunk_size, self.team_size,
                          self.track_tile_size, self.observer_tile_size, self.device_queues)


def probe_peaks() -> dict:
    """FP64/FP32 FMA and 64-bit shared/global atomic rates measured on the current GPU."""
    lib = library()
    p = abi.Peaks()
    _raise(lib.c8r_probe_peaks(C.byref(p)), b"probe failed")
    return {name: getattr(p, name) for name, _ in abi.Peaks._fields_}


def tuning_cache_load(path, workload: str, require: bool = False) -> Optional[TuningParameters]:
    """The tuning stored at `path` for this device, build and workload label,
    or None when there is none that matches (c8r_tuning_cache_load)."""
    lib = library()
    t = abi.Tuning()
    matched = C.c_int()
    _raise(lib.c8r_tuning_cache_load(str(path).encode(), workload.encode(), int(require), C.byref(t),
                                     C.byref(matched)), lib.c8r_tuning_cache_last_error())
    if not matched.value:
        return None
    return TuningParameters(team_size=t.team_size, track_tile_size=t.track_tile_size,
                            observer_tile_size=t.observer_tile_size)


def tuning_cache_store(path, workload: str, tuning: TuningParameters) -> None:
    """Persists `tuning` for this device, build and workload label (c8r_tuning_cache_store)."""
    lib = library()
    t = tuning.to_c()
    _raise(lib.c8r_tuning_cache_store(str(path).encode(), workload.encode(), C.byref(t)),
           lib.c8r_tuning_cache_last_error())


def validate(config: RadioConfig) -> None:
    lib = library()
    cfg, keep = config.to_c()
    _raise(lib.c8r_config_validate(C.byref(cfg)), lib.c8r_last_global_error())


def projected_device_bytes(config: RadioConfig) -> int:
    lib = library()
    cfg, keep = config.to_c()
    out = C.c_size_t()
    _raise(lib.c8r_projected_device_bytes(C.byref(cfg), C.byref(out)), lib.c8r_last_global_error())
    return out.value


@dataclass
class RadioWaveforms:
    """corsika/kokkos/radio/RadioWaveforms.hpp:19-22: CoREAS E (V/m) and ZHS A (V s/m),
    each a (3, total_bins) array in the accumulator's SoA order; split per
    observer with `observer_traces`."""

    coreas: np.ndarray
    zhs: np.ndarray
    counters: dict


def observer_traces(traces: np.ndarray, observers: np.ndarray) -> list:
    out, offset = [], 0
    for n in observers["number_of_bins"]:
        out.append(traces[:, offset:offset + int(n)])
        offset += int(n)
    return out


class RadioAccumulator:
    """corsika::kokkos::radio::RadioAccumulator over libc8radio.so.

    stream: an integer cudaStream_t handle (e.g. torch.cuda.Stream().cuda_stream)
    or None for the legacy default stream."""

    def __init__(self, config: RadioConfig, tuning: Optional[TuningParameters] = None,
                 stream: Optional[int] = None):
        self._lib = library()
        self.config = config
        cfg, self._keep = config.to_c()
        t = (tuning or TuningParameters()).to_c()
        handle = C.c_void_p()
        status = self._lib.c8r_create(C.byref(cfg), C.byref(t), C.c_void_p(stream or 0),
                                      C.byref(handle))
        _raise(status, self._lib.c8r_last_global_error())
        self._h = handle
        cb, zb = C.c_size_t(), C.c_size_t()
        self._check(self._lib.c8r_total_bins(self._h, C.byref(cb), C.byref(zb)))
        self.coreas_bins, self.zhs_bins = cb.value, zb.value

    def _check(self, status: int) -> None:
        if status != abi.C8R_OK:
            _raise(status, self._lib.c8r_last_error(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.c8r_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # reference method set -------------------------------------------------
    def enabled(self) -> bool:
        out = C.c_int()
        self._check(self._lib.c8r_enabled(self._h, C.byref(out)))
        return bool(out.value)

    def reset(self) -> None:
        self._check(self._lib.c8r_reset(self._h))

    def enqueue_host_lepton_tracks(self, records: Optional[np.ndarray]) -> None:
        if records is None:
            self._check(self._lib.c8r_enqueue_host(self._h, None, 0))
            return
        records = np.ascontiguousarray(records, dtype=LEPTON_RECORD)
        self._check(self._lib.c8r_enqueue_host(self._h, records.ctypes.data, records.size))

    def enqueue_host_pointer(self, pointer: Optional[int], count: int) -> None:
        """Raw form of enqueueHostLeptonTracks (a NULL pointer with count > 0 is rejected)."""
        self._check(self._lib.c8r_enqueue_host(self._h, pointer, count))

    def flush_host_lepton_tracks(self) -> None:
        self._check(self._lib.c8r_flush(self._h))

    def accumulate_lepton_tracks(self, device_pointer: int, count: int,
                                 extent: Optional[int] = None) -> None:
        """accumulateLeptonTracks on records in device memory (stream ordered)."""
        self._check(self._lib.c8r_accumulate_device(
            self._h, C.c_void_p(device_pointer), count, count if extent is None else extent))

    def download(self) -> RadioWaveforms:
        coreas = np.zeros((3, self.coreas_bins), np.float64)
        zhs = np.zeros((3, self.zhs_bins), np.float64)
        counters = abi.Counters()
        self._check(self._lib.c8r_download(
            self._h, coreas.ctypes.data if coreas.size else None,
            zhs.ctypes.data if zhs.size else None, C.byref(counters)))
        return RadioWaveforms(coreas, zhs, counters.as_dict())

    def download_into(self, coreas: Optional[np.ndarray], zhs: Optional[np.ndarray]) -> dict:
        """download() into caller-owned (e.g. pinned) float64 buffers of 3*bins."""
        counters = abi.Counters()
        self._check(self._lib.c8r_download(
            self._h, None if coreas is None else coreas.ctypes.data,
            None if zhs is None else zhs.ctypes.data, C.byref(counters)))
        return counters.as_dict()

    def download_fixed(self):
        coreas = np.zeros((3, self.coreas_bins), np.int64)
        zhs = np.zeros((3, self.zhs_bins), np.int64)
        counters = abi.Counters()
        self._check(self._lib.c8r_download_fixed(
            self._h, coreas.ctypes.data if coreas.size else None,
            zhs.ctypes.data if zhs.size else None, C.byref(counters)))
        return coreas, zhs, counters.as_dict()

    def statistics(self) -> abi.Statistics:
        s = abi.Statistics()
        self._check(self._lib.c8r_get_statistics(self._h, C.byref(s)))
        return s

    def device_bytes(self) -> int:
        out = C.c_size_t()
        self._check(self._lib.c8r_device_bytes(self._h, C.byref(out)))
        return out.value

    def static_host_to_device_bytes(self) -> int:
        out = C.c_size_t()
        self._check(self._lib.c8r_static_host_to_device_bytes(self._h, C.byref(out)))
        return out.value

    def reserve_track_capacity(self, count: int) -> None:
        self._check(self._lib.c8r_reserve(self._h, count))

    def projected_track_capacity(self, count: int):
        r, p = C.c_size_t(), C.c_size_t()
        self._check(self._lib.c8r_projected_track_capacity(self._h, count, C.byref(r), C.byref(p)))
        return r.value, p.value

    def synchronize(self) -> None:
        self._check(self._lib.c8r_synchronize(self._h))

    def set_kernel_timing(self, enabled: bool) -> None:
        self._check(self._lib.c8r_set_kernel_timing(self._h, int(enabled)))

    def accumulate_columns(self, columns: dict, count: int) -> None:
        """accumulateLeptonTracks over device columns: a dict of device pointers
        ('pid', 'weight', 'start_time_s', 'end_time_s', 'start_energy_gev', and
        3-tuples 'start_position_m', 'end_position_m', 'start_direction',
        'end_direction')."""
        c = abi.TrackColumns()
        for name in ("pid", "weight", "start_time_s", "end_time_s", "start_energy_gev"):
            setattr(c, name, columns.get(name) or None)
        for name in ("start_position_m", "end_position_m", "start_direction", "end_direction"):
            values = columns.get(name) or (None, None, None)
            setattr(c, name, (C.c_void_p * 3)(*values))
        self._check(self._lib.c8r_accumulate_columns(self._h, C.byref(c), count))

    def download_fields_device(self, coreas_pointer: Optional[int], zhs_pointer: Optional[int]) -> dict:
        """Adds the decoded CoREAS fields (3 x coreas_bins doubles) and the ZHS
        fields -(A[i+1] - A[i]) fs (3 x (zhs_bins - zhs observers) doubles) into
        device buffers; returns the counters.  Seals the accumulator."""
        counters = abi.Counters()
        self._check(self._lib.c8r_download_fields_device(
            self._h, C.c_void_p(coreas_pointer or 0), C.c_void_p(zhs_pointer or 0), C.byref(counters)))
        return counters.as_dict()

    # B200 extensions: staging for batched projection -----------------------
    def stage_lepton_tracks(self, device_pointer: int, count: int,
                            extent: Optional[int] = None) -> None:
        """Ingests device records without projecting them (see RadioBatch)."""
        self._check(self._lib.c8r_stage_device(
            self._h, C.c_void_p(device_pointer), count, count if extent is None else extent))

    def project_staged(self) -> None:
        self._check(self._lib.c8r_project_staged(self._h))

    def set_tuning(self, tuning: TuningParameters) -> None:
        t = tuning.to_c()
        self._check(self._lib.c8r_set_tuning(self._h, C.byref(t)))


class RadioBatch:
    """Projects the staged tracks of several accumulators (one shower each, same
    stream, precision and trace mode) with one persistent launch per algorithm,
    optionally replayed from a captured CUDA graph (graph=True needs a
    non-default stream)."""

    def __init__(self, stream: Optional[int] = None):
        self._lib = library()
        handle = C.c_void_p()
        _raise(self._lib.c8r_batch_create(C.c_void_p(stream or 0), C.byref(handle)),
               self._lib.c8r_last_global_error())
        self._h = handle

    def _check(self, status: int) -> None:
        if status != abi.C8R_OK:
            _raise(status, self._lib.c8r_batch_last_error(self._h))

    @staticmethod
    def _handles(events):
        return (C.c_void_p * len(events))(*[e._h.value for e in events])

    def project(self, events, graph: bool = False, keep_staged: bool = False) -> None:
        flags = (abi.BATCH_GRAPH if graph else 0) | (abi.BATCH_KEEP_STAGED if keep_staged else 0)
        self._check(self._lib.c8r_batch_project(self._h, self._handles(events), len(events), flags))

    def autotune(self, events, repetitions: int = 2):
        best = abi.Tuning()
        ms = C.c_double()
        self._check(self._lib.c8r_batch_autotune(self._h, self._handles(events), len(events),
                                                 repetitions, C.byref(best), C.byref(ms)))
        return TuningParameters(best.batch_size, best.chunk_size, best.team_size,
                                best.track_tile_size, best.observer_tile_size,
                                best.device_queues), ms.value

    def graph_captures(self) -> int:
        out = C.c_ulonglong()
        self._check(self._lib.c8r_batch_graph_captures(self._h, C.byref(out)))
        return out.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.c8r_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RadioServer:
    """Many showers in flight on one GPU (c8r_server_*): events are admitted
    against an HBM budget reserved at creation, their tracks are added as
    device records, and a scheduler thread projects every ready event in
    rounds of one persistent launch per algorithm.  Thread-safe."""

    def __init__(self, budget_bytes: int, block_tracks: int = 0, chunk_tracks: int = 0,
                 round_pairs: int = 0, team_size: int = 0):
        self._lib = library()
        opts = abi.ServerOptions(budget_bytes, block_tracks, chunk_tracks, round_pairs, team_size)
        handle = C.c_void_p()
        status = self._lib.c8r_server_create(C.byref(opts), C.byref(handle))
        _raise(status, self._lib.c8r_server_last_error(None))
        self._h = handle
        self._configs = {}

    def _check(self, status: int) -> None:
        if status != abi.C8R_OK:
            _raise(status, self._lib.c8r_server_last_error(self._h))

    def open(self, config: RadioConfig, timeout_ms: int = -1) -> int:
        cfg, keep = config.to_c()
        event = C.c_uint64()
        self._check(self._lib.c8r_server_open(self._h, C.byref(cfg), timeout_ms, C.byref(event)))
        nc = int(sum(int(b) for b in config.coreas_observers["number_of_bins"])) if config.coreas_enabled else 0
        nz = int(sum(int(b) for b in config.zhs_observers["number_of_bins"])) if config.zhs_enabled else 0
        self._configs[event.value] = (nc, nz)
        return event.value

    def add_device(self, event: int, device_pointer: int, count: int, stream: Optional[int] = None,
                   extent: Optional[int] = None) -> None:
        self._check(self._lib.c8r_server_add_device(
            self._h, event, C.c_void_p(device_pointer), count, count if extent is None else extent,
            C.c_void_p(stream or 0)))

    def close_event(self, event: int) -> None:
        self._check(self._lib.c8r_server_close(self._h, event))

    def wait(self, event: int, timeout_ms: int = -1) -> None:
        self._check(self._lib.c8r_server_wait(self._h, event, timeout_ms))

    def fetch_fixed(self, event: int):
        """(coreas int64 (3, bins), zhs int64 (3, bins), counters, info); releases the event."""
        nc, nz = self._configs[event]
        coreas = np.zeros((3, nc), np.int64)
        zhs = np.zeros((3, nz), np.int64)
        counters, info = abi.Counters(), abi.ServerEventInfo()
        self._check(self._lib.c8r_server_fetch_fixed(
            self._h, event, coreas.ctypes.data if coreas.size else None,
            zhs.ctypes.data if zhs.size else None, C.byref(counters), C.byref(info)))
        del self._configs[event]
        return coreas, zhs, counters.as_dict(), info.as_dict()

    def fetch(self, event: int):
        """(RadioWaveforms decoded to V/m and V s/m, info); releases the event."""
        nc, nz = self._configs[event]
        coreas = np.zeros((3, nc), np.float64)
        zhs = np.zeros((3, nz), np.float64)
        counters, info = abi.Counters(), abi.ServerEventInfo()
        try:
            self._check(self._lib.c8r_server_fetch(
                self._h, event, coreas.ctypes.data if coreas.size else None,
                zhs.ctypes.data if zhs.size else None, C.byref(counters), C.byref(info)))
        finally:
            self._configs.pop(event, None)
        return RadioWaveforms(coreas, zhs, counters.as_dict()), info.as_dict()

    def stats(self) -> dict:
        out = abi.ServerStats()
        self._check(self._lib.c8r_server_get_stats(self._h, C.byref(out)))
        return out.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.c8r_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ------------------------------------------------------------------ spool
class SpoolWriter:
    """RadioTrackSpoolWriter (version 1): refuses an existing path; tracks are
    validated on append; only complete() publishes the record count."""

    def __init__(self, path):
        self._lib = library()
        handle = C.c_void_p()
        _raise(self._lib.c8r_spool_writer_create(str(path).encode(), C.byref(handle)),
               self._lib.c8r_last_global_error())
        self._h = handle

    def append(self, tracks: np.ndarray) -> None:
        tracks = np.ascontiguousarray(tracks, dtype=abi.TRACK_SEGMENT)
        _raise(self._lib.c8r_spool_append(self._h, tracks.ctypes.data if tracks.size else None,
                                          tracks.size), self._lib.c8r_last_global_error())

    def complete(self) -> None:
        _raise(self._lib.c8r_spool_complete(self._h), self._lib.c8r_last_global_error())

    def count(self) -> int:
        out = C.c_uint64()
        _raise(self._lib.c8r_spool_writer_count(self._h, C.byref(out)), self._lib.c8r_last_global_error())
        return out.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.c8r_spool_writer_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SpoolReader:
    """RadioTrackSpoolReader (version 1): validates the header and file length
    on open; read_batch returns at most `maximum` (1..65536) validated tracks."""

    def __init__(self, path):
        self._lib = library()
        handle, count = C.c_void_p(), C.c_uint64()
        _raise(self._lib.c8r_spool_reader_open(str(path).encode(), C.byref(handle), C.byref(count)),
               self._lib.c8r_last_global_error())
        self._h = handle
        self.count = count.value

    def read_batch(self, maximum: int = 4096) -> np.ndarray:
        out = np.zeros(max(int(maximum), 0), abi.TRACK_SEGMENT)
        n = C.c_size_t()
        _raise(self._lib.c8r_spool_read(self._h, out.ctypes.data if out.size else None, int(maximum),
                                        C.byref(n)), self._lib.c8r_last_global_error())
        return out[: n.value]

    def state(self):
        consumed, finished = C.c_uint64(), C.c_int()
        _raise(self._lib.c8r_spool_reader_state(self._h, C.byref(consumed), C.byref(finished)),
               self._lib.c8r_last_global_error())
        return consumed.value, bool(finished.value)

    def replay(self, accumulator: "RadioAccumulator", batch: int = 4096) -> None:
        """Enqueues every remaining track into the accumulator as host tracks."""
        _raise(self._lib.c8r_spool_replay(self._h, accumulator._h, int(batch)),
               self._lib.c8r_last_global_error())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.c8r_spool_reader_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def track_records(tracks: np.ndarray) -> np.ndarray:
    """make_host_radio_record for each track segment (LeptonTransportRecords)."""
    lib = library()
    tracks = np.ascontiguousarray(tracks, dtype=abi.TRACK_SEGMENT)
    out = np.zeros(tracks.size, LEPTON_RECORD)
    _raise(lib.c8r_track_records(tracks.ctypes.data if tracks.size else None, tracks.size,
                                 out.ctypes.data if out.size else None), lib.c8r_last_global_error())
    return out


def merge_fixed(destination: np.ndarray, source: np.ndarray) -> None:
    """destination += source for int64 fixed-point snapshots, every bin checked
    first (OverflowErrorRadio, nothing written, on overflow)."""
    lib = library()
    if destination.dtype != np.int64 or source.dtype != np.int64 or destination.shape != source.shape:
        raise InvalidArgument("merge_fixed takes two int64 arrays of one shape")
    if not destination.flags["C_CONTIGUOUS"]:
        raise InvalidArgument("merge_fixed destination must be contiguous")
    source = np.ascontiguousarray(source)
    _raise(lib.c8r_merge_fixed(destination.ctypes.data, source.ctypes.data, destination.size),
           lib.c8r_last_global_error())
