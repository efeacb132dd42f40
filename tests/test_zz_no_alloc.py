"""c8r_accumulate_device_no_alloc: the accumulate entry point for callers that
cannot allocate device memory (a transport code whose pool allocator owns all
of HBM, or one that cannot accept the device-wide synchronisation of
cudaMalloc/cudaFree).  Its scratch is one static device array in the library,
so the caller passes only its records and its own zeroed output traces.

Its traces must equal those of the ordinary entry point
(c8r_accumulate_device + c8r_download_fixed) bit for bit, as every fixed-point
comparison in this suite does.  Two calls run back to back: the array keeps the
first call's contents, and the second call (another configuration and
precision) must not see them.  This file is named to be collected last, so the
check also holds after every other test has used the GPU, and it needs nothing
from them when run alone."""
import ctypes as C

import numpy as np
import pytest


def to_device(torch, records):
    return torch.from_numpy(np.ascontiguousarray(records).view(np.uint8).reshape(-1)).cuda()


def no_alloc_call(pkg, torch, config, records, stream=None, with_counters=True):
    """Zeroed caller-owned device outputs (int64 fixed point, or double when
    the config is not deterministic), one call on `stream` (a torch stream, or
    None for the legacy default stream), host copies back.  Without counters
    the call gets NULL and None is returned in their place."""
    lib = pkg.library()
    cfg, keep = config.to_c()
    nc = int(config.coreas_observers["number_of_bins"].sum())
    nz = int(config.zhs_observers["number_of_bins"].sum())
    dtype = torch.int64 if config.deterministic else torch.float64
    coreas = torch.zeros(3 * nc, dtype=dtype, device="cuda")
    zhs = torch.zeros(3 * nz, dtype=dtype, device="cuda")
    counters = torch.zeros(C.sizeof(pkg.abi.Counters), dtype=torch.uint8, device="cuda")
    raw = to_device(torch, records)
    torch.cuda.synchronize()  # inputs written on torch's stream before the call's stream reads them
    handle = stream.cuda_stream if stream is not None else 0
    status = lib.c8r_accumulate_device_no_alloc(
        C.byref(cfg), C.c_void_p(raw.data_ptr()), records.size, records.size,
        C.c_void_p(coreas.data_ptr()), C.c_void_p(zhs.data_ptr()),
        C.c_void_p(counters.data_ptr() if with_counters else None), C.c_void_p(handle))
    assert status == pkg.abi.C8R_OK, lib.c8r_last_global_error()
    torch.cuda.synchronize()
    host_counters = (pkg.abi.Counters.from_buffer_copy(counters.cpu().numpy().tobytes()).as_dict()
                     if with_counters else None)
    return (coreas.cpu().numpy().reshape(3, nc), zhs.cpu().numpy().reshape(3, nz), host_counters)


def ordinary_call(pkg, torch, config, records):
    acc = pkg.RadioAccumulator(config)
    raw = to_device(torch, records)
    acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
    if config.deterministic:
        out = acc.download_fixed()
    else:
        w = acc.download()
        out = (w.coreas, w.zhs, w.counters)
    acc.close()
    return out


COUNTS = ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks",
          "fixed_point_overflows")


@pytest.mark.gpu
def test_no_alloc_matches_accumulate_on_two_calls_in_a_row(pkg, showers):
    import torch

    assert torch.cuda.is_available()
    # first call: FP64, more records than one scratch chunk holds
    wl, gen, _ = showers.workload_config("plain_c0")
    first = showers.make_config(wl, precision=0, kernel=2)
    records = showers.shower_records(300_000, seed=41, **gen)
    # second call: mixed precision on a different antenna set and trace length
    wl2, gen2, _ = showers.workload_config("tiled_c1", bins=2048)
    second = showers.make_config(wl2, precision=1, kernel=2)
    records2 = showers.shower_records(60_000, seed=42, **gen2)

    for config, recs in ((first, records), (second, records2)):
        got = no_alloc_call(pkg, torch, config, recs)
        want = ordinary_call(pkg, torch, config, recs)
        assert np.array_equal(got[0], want[0]), f"{np.count_nonzero(got[0] != want[0])} CoREAS values differ"
        assert np.array_equal(got[1], want[1]), f"{np.count_nonzero(got[1] != want[1])} ZHS values differ"
        for key in COUNTS:
            assert got[2][key] == want[2][key], key
        assert got[2]["coreas_contributions"] > 0 and got[2]["zhs_contributions"] > 0


@pytest.mark.gpu
def test_no_alloc_floating_traces_null_counters_and_a_side_stream(pkg, showers):
    """FP64 floating-point traces (config.deterministic = 0), called twice in
    a row on a non-default stream, the second time without counters: the
    traces equal the ordinary entry point's within the tolerance of every
    floating comparison in this suite (FP64 atomics add in any order:
    1e-28 + 2e-12 of each algorithm's peak)."""
    import torch

    assert torch.cuda.is_available()
    wl, gen, _ = showers.workload_config("tiled_c1", bins=1024)
    config = showers.make_config(wl, precision=0, kernel=2, deterministic=False)
    records = showers.shower_records(40_000, seed=43, **gen)
    want = ordinary_call(pkg, torch, config, records)
    side = torch.cuda.Stream()
    for with_counters in (True, False):
        got = no_alloc_call(pkg, torch, config, records, stream=side, with_counters=with_counters)
        for g, w in zip(got[:2], want[:2]):
            peak = max(float(np.abs(w).max(initial=0.0)), 1e-300)
            assert np.abs(g - w).max(initial=0.0) <= 1e-28 + 2e-12 * peak
            assert np.abs(w).max() > 0
        if with_counters:
            for key in COUNTS:
                assert got[2][key] == want[2][key], key


def test_no_alloc_rejects_sizes_beyond_its_scratch(pkg, showers):
    """Rejected on the host before any device work, so this runs without a GPU."""
    lib = pkg.library()
    wl, _, _ = showers.workload_config("plain_c0")
    wl["observers"] = showers.star_antennas(8, list(np.linspace(25.0, 500.0, 129)), 1400.0, 64, 1e10)
    config = showers.make_config(wl)  # 2 x 1032 observers > 2048
    cfg, keep = config.to_c()
    status = lib.c8r_accumulate_device_no_alloc(C.byref(cfg), None, 0, 0, None, None, None, None)
    assert status == pkg.abi.C8R_LENGTH_ERROR
    assert b"2048 observers" in lib.c8r_last_global_error()

    wl, _, _ = showers.workload_config("plain_c0")
    wl["table"] = showers.flat_atmosphere_table(showers.AtmosphereModel(), 1400.0, 30000.0, 0.2)
    config = showers.make_config(wl)  # 148001 table entries > 131072
    cfg, keep = config.to_c()
    status = lib.c8r_accumulate_device_no_alloc(C.byref(cfg), None, 0, 0, None, None, None, None)
    assert status == pkg.abi.C8R_LENGTH_ERROR
    assert b"131072 entries" in lib.c8r_last_global_error()
