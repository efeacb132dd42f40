"""TEST INFRASTRUCTURE ONLY — Python binding of the CPU oracles.

Two CPU implementations of the radio projection sit behind the same call:

* ``restatement()`` — liboracle.so, the plain-C restatement in radio_oracle.c
  (built from this repository by oracle/Makefile, always available);
* ``reference()``   — _ref/libc8ref.so, the reference's own projection code
  compiled from its unmodified sources (available where it was built).

Only the tests, the smoke check and the bench's CPU-baseline leg use this
module, as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
RESTATEMENT = HERE / "liboracle.so"
REFERENCE = HERE / "_ref" / "libc8ref.so"


def build(reference_tree: str | os.PathLike | None = None) -> None:
    """Builds liboracle.so and, when a reference source tree is named (the
    argument, else the C8R_REFERENCE_TREE environment variable) and exists,
    _ref/libc8ref.so from that tree's unmodified projection sources."""
    tree = reference_tree or os.environ.get("C8R_REFERENCE_TREE")
    targets = ["oracle"]
    extra = []
    if tree and (Path(tree) / "corsika").is_dir():
        targets.append("ref")
        extra.append(f"REFERENCE={tree}")
    subprocess.run(["make", "-s", "-C", str(HERE), *targets, *extra], check=True)


class _Backend:
    def __init__(self, path: Path, prefix: str):
        self.path = path
        self.lib = C.CDLL(str(path))
        self.prefix = prefix
        fn = getattr(self.lib, f"{prefix}_project")
        fn.restype = C.c_int
        fn.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        self._project = fn

    def project(self, config, records: np.ndarray, threads: int = 1, coreas_fixed=None,
                zhs_fixed=None, coreas_floating=None, zhs_floating=None, counters=None):
        """Accumulates `records` into trace arrays ((3, bins) per algorithm,
        int64 in deterministic mode, float64 otherwise); returns
        (coreas, zhs, counters)."""
        from importlib import import_module

        abi = import_module("corsika8_kokkos_b200.abi")
        cfg, keep = config.to_c()
        nc = int(sum(int(b) for b in config.coreas_observers["number_of_bins"])) if config.coreas_enabled else 0
        nz = int(sum(int(b) for b in config.zhs_observers["number_of_bins"])) if config.zhs_enabled else 0
        if config.deterministic:
            coreas = coreas_fixed if coreas_fixed is not None else np.zeros((3, nc), np.int64)
            zhs = zhs_fixed if zhs_fixed is not None else np.zeros((3, nz), np.int64)
            args = (coreas.ctypes.data, zhs.ctypes.data, None, None)
        else:
            coreas = coreas_floating if coreas_floating is not None else np.zeros((3, nc), np.float64)
            zhs = zhs_floating if zhs_floating is not None else np.zeros((3, nz), np.float64)
            args = (None, None, coreas.ctypes.data, zhs.ctypes.data)
        counters = counters if counters is not None else abi.Counters()
        records = np.ascontiguousarray(records)
        status = self._project(C.byref(cfg), records.ctypes.data if records.size else None,
                               records.size, *args, C.byref(counters), threads)
        if status != 0:
            raise RuntimeError(f"{self.prefix}_project failed with {status}")
        return coreas, zhs, counters.as_dict()


_cache: dict = {}


def restatement() -> _Backend:
    if "o" not in _cache:
        if not RESTATEMENT.exists():
            build()
        _cache["o"] = _Backend(RESTATEMENT, "c8o")
        lib = _cache["o"].lib
        lib.c8o_nearest_bin.restype = C.c_double
        lib.c8o_nearest_bin.argtypes = [C.c_double]
        lib.c8o_doppler.restype = C.c_double
        lib.c8o_doppler.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.c8o_checked_add.restype = C.c_int
        lib.c8o_checked_add.argtypes = [C.POINTER(C.c_longlong), C.c_longlong]
        lib.c8o_add_fixed_point.restype = C.c_int
        lib.c8o_add_fixed_point.argtypes = [C.POINTER(C.c_longlong), C.c_double, C.c_double]
        lib.c8o_diagnostic_energy_bin.restype = C.c_size_t
        lib.c8o_diagnostic_energy_bin.argtypes = [C.c_double]
    return _cache["o"]


def reference_available() -> bool:
    return REFERENCE.exists()


def reference() -> _Backend:
    if "r" not in _cache:
        if not REFERENCE.exists():
            raise FileNotFoundError(f"{REFERENCE} is not built (needs the reference tree)")
        _cache["r"] = _Backend(REFERENCE, "c8ref")
        lib = _cache["r"].lib
        lib.c8ref_nearest_bin.restype = C.c_double
        lib.c8ref_nearest_bin.argtypes = [C.c_double]
        lib.c8ref_doppler.restype = C.c_double
        lib.c8ref_doppler.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.c8ref_propagate.restype = None
        lib.c8ref_propagate.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]
        lib.c8ref_separate.restype = None
        lib.c8ref_separate.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_int]
        lib.c8ref_add_sample.restype = C.c_ulonglong
        lib.c8ref_add_sample.argtypes = [C.c_double, C.c_double, C.c_double, C.c_ulonglong, C.c_int,
                                         C.c_double, C.POINTER(C.c_double), C.c_double,
                                         C.c_void_p, C.c_void_p, C.POINTER(C.c_ulonglong)]
        lib.c8ref_checked_add.restype = C.c_int
        lib.c8ref_checked_add.argtypes = [C.POINTER(C.c_longlong), C.c_longlong]
        lib.c8ref_add_fixed_point.restype = C.c_int
        lib.c8ref_add_fixed_point.argtypes = [C.POINTER(C.c_longlong), C.c_double, C.c_double]
    return _cache["r"]


def vec(values) -> C.Array:
    return (C.c_double * len(values))(*values)


# ---------------------------------------------------------------- primitives
class OracleObserver(C.Structure):
    """c8o_observer = RadioObserverView (80 bytes)."""
    _fields_ = [("position_m", C.c_double * 3), ("start_time_s", C.c_double),
                ("duration_s", C.c_double), ("sample_rate_hz", C.c_double),
                ("fixed_point_scale", C.c_double), ("inverse_fixed_point_scale", C.c_double),
                ("number_of_bins", C.c_uint64), ("waveform_offset", C.c_uint64)]


class OraclePropagation(C.Structure):
    """c8o_propagation = RadioPropagationView (104 bytes)."""
    _fields_ = [("homogeneous_refractive_index", C.c_double), ("minimum_height_m", C.c_double),
                ("maximum_height_m", C.c_double), ("step_m", C.c_double),
                ("inverse_step_per_m", C.c_double), ("slope_refractivity_lower", C.c_double),
                ("slope_integrated_refractivity_lower", C.c_double),
                ("slope_refractivity_upper", C.c_double),
                ("slope_integrated_refractivity_upper", C.c_double),
                ("refractivity", C.POINTER(C.c_double)),
                ("integrated_refractivity", C.POINTER(C.c_double)),
                ("table_size", C.c_uint64), ("zhs_subtrack_refinement", C.c_uint32),
                ("pad_", C.c_uint32)]


class OraclePath(C.Structure):
    _fields_ = [("propagation_time_s", C.c_double), ("refractive_index_source", C.c_double),
                ("refractive_index_destination", C.c_double), ("distance_m", C.c_double),
                ("emit", C.c_double * 3)]


class OracleWaveforms(C.Structure):
    _fields_ = [("floating", C.POINTER(C.c_double) * 3), ("fixed", C.POINTER(C.c_longlong) * 3)]


def _propagation_struct(snapshot, refinement=1):
    n = np.ascontiguousarray(snapshot.refractivity, dtype=np.float64)
    i = np.ascontiguousarray(snapshot.integrated_refractivity, dtype=np.float64)
    dptr = C.POINTER(C.c_double)
    p = OraclePropagation(snapshot.homogeneous_refractive_index, snapshot.minimum_height_m,
                          snapshot.maximum_height_m, snapshot.step_m, snapshot.inverse_step_per_m,
                          snapshot.slope_refractivity_lower,
                          snapshot.slope_integrated_refractivity_lower,
                          snapshot.slope_refractivity_upper,
                          snapshot.slope_integrated_refractivity_upper,
                          n.ctypes.data_as(dptr) if n.size else dptr(),
                          i.ctypes.data_as(dptr) if i.size else dptr(), int(n.size), refinement, 0)
    return p, (n, i)


def propagate_restatement(snapshot, source, observer_position):
    """c8o_propagate -> (time, n_source, n_destination, distance, kx, ky, kz)."""
    lib = restatement().lib
    lib.c8o_propagate.restype = None
    lib.c8o_propagate.argtypes = [C.POINTER(OraclePropagation), C.POINTER(C.c_double),
                                  C.POINTER(OracleObserver), C.POINTER(OraclePath)]
    p, keep = _propagation_struct(snapshot)
    o = OracleObserver()
    for a in range(3):
        o.position_m[a] = observer_position[a]
    path = OraclePath()
    lib.c8o_propagate(C.byref(p), vec(source), C.byref(o), C.byref(path))
    return (path.propagation_time_s, path.refractive_index_source,
            path.refractive_index_destination, path.distance_m, *path.emit)


def propagate_reference(config, source, observer_position):
    """The reference's propagate() on the config's propagation snapshot."""
    lib = reference().lib
    cfg, keep = config.to_c()
    out = (C.c_double * 7)()
    lib.c8ref_propagate(C.byref(cfg), vec(source), vec(observer_position), out)
    return tuple(out)


def add_sample_restatement(start, duration, rate, bins, potential, time, value, scale,
                           fixed=None, floating=None):
    """One c8o_add_sample into caller rows (3*bins); returns (contributions, overflows)."""
    from importlib import import_module

    abi = import_module("corsika8_kokkos_b200.abi")
    lib = restatement().lib
    lib.c8o_add_sample.restype = None
    lib.c8o_add_sample.argtypes = [C.POINTER(OracleObserver), C.POINTER(OracleWaveforms),
                                   C.c_double, C.POINTER(C.c_double),
                                   C.POINTER(C.c_ulonglong), C.c_void_p, C.c_int]
    o = OracleObserver()
    o.start_time_s, o.duration_s, o.sample_rate_hz = start, duration, rate
    o.number_of_bins, o.fixed_point_scale = bins, scale
    w = OracleWaveforms()
    if fixed is not None:
        base = fixed.ctypes.data
        for r in range(3):
            w.fixed[r] = C.cast(base + r * bins * 8, C.POINTER(C.c_longlong))
    else:
        base = floating.ctypes.data
        for r in range(3):
            w.floating[r] = C.cast(base + r * bins * 8, C.POINTER(C.c_double))
    counter = C.c_ulonglong(0)
    counters = abi.Counters()
    lib.c8o_add_sample(C.byref(o), C.byref(w), time, vec(value), C.byref(counter),
                       C.byref(counters), int(potential))
    return counter.value, counters.fixed_point_overflows


def add_sample_reference(start, duration, rate, bins, potential, time, value, scale,
                         fixed=None, floating=None):
    lib = reference().lib
    overflows = C.c_ulonglong(0)
    n = lib.c8ref_add_sample(start, duration, rate, bins, int(potential), time, vec(value), scale,
                             None if fixed is None else fixed.ctypes.data,
                             None if floating is None else floating.ctypes.data,
                             C.byref(overflows))
    return n, overflows.value


def separate_restatement(start, end, resolution, signed):
    lib = restatement().lib
    lib.c8o_separate_same_bin_endpoints.restype = None
    lib.c8o_separate_same_bin_endpoints.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                    C.c_double, C.c_int]
    s, e = C.c_double(start), C.c_double(end)
    lib.c8o_separate_same_bin_endpoints(C.byref(s), C.byref(e), resolution, int(signed))
    return s.value, e.value


def separate_reference(start, end, resolution, signed):
    s, e = C.c_double(start), C.c_double(end)
    reference().lib.c8ref_separate(C.byref(s), C.byref(e), resolution, int(signed))
    return s.value, e.value
