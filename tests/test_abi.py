"""The C ABI without a GPU: libc8radio.so loads, exports every function
include/c8radio.h declares (and the ctypes view binds each one), the structs
the ctypes view passes have the C compiler's sizes and offsets, and the
host-only entry points (validation, memory projection, error mapping) behave
as the reference's accumulator does (RadioAccumulator.inl:87-141, :931-974)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

HEADER = Path(__file__).resolve().parent.parent / "include" / "c8radio.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(c8r_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_function_is_exported_and_bound(pkg):
    names = declared_functions()
    assert len(names) >= 40
    lib = C.CDLL(str(pkg.LIBRARY_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    unbound = [n for n in names if n not in pkg.abi.PROTOTYPES]
    assert not unbound, unbound
    assert pkg.library().c8r_version().startswith(b"c8radio-b200")


LAYOUT_PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "c8radio.h"
#define S(t) printf(#t " %zu\n", sizeof(t));
#define O(t, f) printf(#t "." #f " %zu\n", offsetof(t, f));
int main(void) {
  S(c8r_particle_state) S(c8r_lepton_transport_record) S(c8r_observer_snapshot)
  S(c8r_propagation_snapshot) S(c8r_config) S(c8r_tuning) S(c8r_counters) S(c8r_statistics)
  S(c8r_server_options) S(c8r_server_event_info) S(c8r_server_stats)
  S(c8r_track_segment) S(c8r_track_columns) S(c8r_fixed_snapshot)
  O(c8r_fixed_snapshot, config) O(c8r_fixed_snapshot, counters)
  O(c8r_lepton_transport_record, start) O(c8r_lepton_transport_record, end)
  O(c8r_config, propagation) O(c8r_config, precision) O(c8r_config, count_samples)
  return 0;
}
"""


def test_struct_layouts_match_the_c_compiler(pkg, tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(LAYOUT_PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    c = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                             check=True).stdout.splitlines())
    c = {k: int(v) for k, v in c.items()}
    abi = pkg.abi
    assert c["c8r_lepton_transport_record"] == abi.LEPTON_RECORD.itemsize == 752
    assert c["c8r_lepton_transport_record.start"] == 320 and c["c8r_lepton_transport_record.end"] == 448
    assert c["c8r_observer_snapshot"] == abi.OBSERVER.itemsize == 56
    assert c["c8r_config"] == C.sizeof(abi.Config)
    assert c["c8r_config.propagation"] == abi.Config.propagation.offset
    assert c["c8r_config.precision"] == abi.Config.precision.offset
    assert c["c8r_config.count_samples"] == abi.Config.count_samples.offset
    assert c["c8r_propagation_snapshot"] == C.sizeof(abi.PropagationSnapshot)
    assert c["c8r_tuning"] == C.sizeof(abi.Tuning)
    assert c["c8r_counters"] == C.sizeof(abi.Counters) == 288
    assert c["c8r_statistics"] == C.sizeof(abi.Statistics)
    assert c["c8r_server_options"] == C.sizeof(abi.ServerOptions)
    assert c["c8r_server_event_info"] == C.sizeof(abi.ServerEventInfo)
    assert c["c8r_server_stats"] == C.sizeof(abi.ServerStats)
    assert c["c8r_track_segment"] == abi.TRACK_SEGMENT.itemsize
    assert c["c8r_track_columns"] == C.sizeof(abi.TrackColumns)
    assert c["c8r_fixed_snapshot"] == C.sizeof(abi.FixedSnapshot)
    assert c["c8r_fixed_snapshot.config"] == abi.FixedSnapshot.config.offset
    assert c["c8r_fixed_snapshot.counters"] == abi.FixedSnapshot.counters.offset


def test_validation_and_memory_projection_on_the_host(pkg, showers):
    lib = pkg.library()
    wl, _, _ = showers.workload_config("plain_c0")
    good = showers.make_config(wl)
    cfg, keep = good.to_c()
    assert lib.c8r_config_validate(C.byref(cfg)) == pkg.abi.C8R_OK
    size = C.c_size_t()
    assert lib.c8r_projected_device_bytes(C.byref(cfg), C.byref(size)) == pkg.abi.C8R_OK
    bins = 16 * 4096
    assert size.value >= 2 * 3 * bins * 16  # int64 traces + decode buffer per algorithm
    for field, value, message in (("zhs_subtrack_refinement", 0, b"refinement"),
                                  ("fixed_point_field_limit_v_per_m", -1.0, b"fixed-point limit"),
                                  ("precision", 7, b"precision")):
        bad = showers.make_config(wl)
        setattr(bad, field, value)
        cfg, keep = bad.to_c()
        assert lib.c8r_config_validate(C.byref(cfg)) == pkg.abi.C8R_INVALID_ARGUMENT
        assert message in lib.c8r_last_global_error()
    wl["observers"] = wl["observers"].copy()
    wl["observers"]["sample_rate_hz"][3] = 0.0
    cfg, keep = showers.make_config(wl).to_c()
    assert lib.c8r_config_validate(C.byref(cfg)) == pkg.abi.C8R_INVALID_ARGUMENT
    with pytest.raises(pkg.InvalidArgument):
        pkg.validate(showers.make_config(wl))


def test_null_handles_are_rejected(pkg):
    lib = pkg.library()
    assert lib.c8r_reset(None) == pkg.abi.C8R_INVALID_ARGUMENT
    assert lib.c8r_flush(None) == pkg.abi.C8R_INVALID_ARGUMENT
    assert lib.c8r_server_close(None, 1) == pkg.abi.C8R_INVALID_ARGUMENT
    assert b"null radio server" in lib.c8r_server_last_error(None)


def test_fixed_snapshot_merge_is_checked_before_writing(pkg):
    """merge_fixed_accumulators (FixedAccumulatorMerge.inl:21-28): an overflow in
    any bin leaves the destination untouched."""
    destination = np.array([1, 2 ** 62, -5, -(2 ** 62)], np.int64)
    before = destination.copy()
    with pytest.raises(pkg.OverflowErrorRadio):
        pkg.merge_fixed(destination, np.array([2, 2 ** 62, 5, 0], np.int64))
    assert np.array_equal(destination, before)
    with pytest.raises(pkg.OverflowErrorRadio):
        pkg.merge_fixed(destination, np.array([0, 0, 0, -(2 ** 62) - 1], np.int64))
    pkg.merge_fixed(destination, np.array([2, 1, 5, -(2 ** 62)], np.int64))
    assert destination.tolist() == [3, 2 ** 62 + 1, 0, -(2 ** 63)]


def test_tuning_cache_files_without_a_gpu(pkg, tmp_path):
    """The tuning cache (c8r_tuning_cache_load, in the manner of
    TuningCache.cpp:101-129): a missing file is no match, an error only when a
    match is required; a malformed file is an error either way.  Both are
    decided before the device is queried."""
    assert pkg.tuning_cache_load(tmp_path / "absent", "workload") is None
    with pytest.raises(pkg.RadioError, match="no radio tuning cache"):
        pkg.tuning_cache_load(tmp_path / "absent", "workload", require=True)
    for name, text in (("no_equals", "format=c8radio-b200-tuning-v1\nbad line\n"),
                       ("duplicate", "format=c8radio-b200-tuning-v1\nformat=x\n"),
                       ("empty_key", "=value\n")):
        path = tmp_path / name
        path.write_text(text)
        with pytest.raises(pkg.RadioError, match="tuning-cache"):
            pkg.tuning_cache_load(path, "workload")
