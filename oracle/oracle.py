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
REFERENCE_TREE = Path(os.environ.get("C8R_REFERENCE_TREE", "/root/reference"))


def build(reference: bool = True) -> None:
    """Builds liboracle.so and, where the reference tree exists, _ref/libc8ref.so."""
    targets = ["oracle"]
    if reference and (REFERENCE_TREE / "corsika").is_dir():
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(HERE), *targets,
                    f"REFERENCE={REFERENCE_TREE}"], check=True)


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
            build(reference=False)
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
