"""The C++ shim include/c8radio.hpp as a reference caller uses it: compiled
with g++ against libc8radio.so (tests/shim_check.cpp), it must throw the
reference's exception classes (RadioAccumulator.inl:147-430,
CooperativeRadioMerge.inl:74-277) and its cooperative export must give the
oracle's traces.

* host (no GPU): validation, validate_fixed_radio, merge_radio_counters,
  CooperativeRadioMerge commit/take (duplicate, foreign and overflowing
  commits rejected without a change) and decode_fixed_radio;
* gpu: initialize -> accumulateLeptonTracks (device records) / enqueueHostLeptonTracks
  (host records) -> downloadFixed(identity, endpoint) on two endpoints ->
  CooperativeRadioMerge -> take, equal bit for bit to the oracle on all the
  tracks; the lifecycle rejections (second export, download after export,
  tracks after export, overflow) by exception class.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CUDA = Path("/usr/local/cuda")


@pytest.fixture(scope="module")
def shim_binary(pkg, tmp_path_factory):
    pkg.library()  # built
    out = tmp_path_factory.mktemp("shim") / "shim_check"
    lib_dir = Path(pkg.LIBRARY_PATH).parent
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", str(ROOT / "include"),
           "-I", str(CUDA / "include"), str(HERE / "shim_check.cpp"), "-o", str(out),
           "-L", str(lib_dir), "-lc8radio", f"-Wl,-rpath,{lib_dir}",
           "-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    result = subprocess.run(cmd, capture_output=True, text=True)
    assert result.returncode == 0, result.stderr
    return out


def test_shim_compiles_and_throws_the_reference_exceptions_on_the_host(shim_binary):
    result = subprocess.run([str(shim_binary), "host"], capture_output=True, text=True, timeout=120)
    assert result.returncode == 0 and result.stdout.strip() == "ok", result.stdout + result.stderr


@pytest.mark.gpu
def test_shim_cooperative_export_equals_the_oracle(shim_binary, pkg, showers, oracle, tmp_path):
    wl, gen, _ = showers.workload_config("tiled_c1", bins=1024)
    observers = wl["observers"][:: 8].copy()  # 20 antennas, every radius of one arm
    records = showers.shower_records(30_000, seed=77, **gen)
    table = wl["table"]
    scalars = np.array([table["homogeneous_refractive_index"], table["minimum_height_m"],
                        table["maximum_height_m"], table["step_m"], table["inverse_step_per_m"],
                        table["slope_refractivity_lower"], table["slope_integrated_refractivity_lower"],
                        table["slope_refractivity_upper"], table["slope_integrated_refractivity_upper"],
                        1.0], np.float64)
    scalars.tofile(tmp_path / "config.bin")
    observers.tofile(tmp_path / "observers.bin")
    np.concatenate([table["refractivity"], table["integrated_refractivity"]]).astype(np.float64).tofile(
        tmp_path / "table.bin")
    records.tofile(tmp_path / "records.bin")
    result = subprocess.run([str(shim_binary), "gpu", str(tmp_path)], capture_output=True, text=True,
                            timeout=600)
    assert result.returncode == 0 and result.stdout.strip() == "ok", result.stdout + result.stderr

    config = showers.make_config(dict(wl, observers=observers))
    want_c, want_z, want_counters = oracle.restatement().project(config, records, threads=4)
    merged = np.fromfile(tmp_path / "merged.bin", dtype=np.uint8)
    values = 3 * int(observers["number_of_bins"].sum())
    traces = merged[: 2 * values * 8].view(np.int64)
    counters = pkg.abi.Counters.from_buffer_copy(merged[2 * values * 8:].tobytes()).as_dict()
    assert np.array_equal(traces[:values].reshape(3, -1), want_c)
    assert np.array_equal(traces[values:].reshape(3, -1), want_z)
    for key in ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks"):
        assert counters[key] == want_counters[key], key
    assert want_counters["coreas_contributions"] > 0
