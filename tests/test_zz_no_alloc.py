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


def no_alloc_call(pkg, torch, config, records, stream=0):
    """Zeroed caller-owned device outputs, one call, host copies back."""
    lib = pkg.library()
    cfg, keep = config.to_c()
    nc = int(config.coreas_observers["number_of_bins"].sum())
    nz = int(config.zhs_observers["number_of_bins"].sum())
    coreas = torch.zeros(3 * nc, dtype=torch.int64, device="cuda")
    zhs = torch.zeros(3 * nz, dtype=torch.int64, device="cuda")
    counters = torch.zeros(C.sizeof(pkg.abi.Counters), dtype=torch.uint8, device="cuda")
    raw = to_device(torch, records)
    status = lib.c8r_accumulate_device_no_alloc(
        C.byref(cfg), C.c_void_p(raw.data_ptr()), records.size, records.size,
        C.c_void_p(coreas.data_ptr()), C.c_void_p(zhs.data_ptr()), C.c_void_p(counters.data_ptr()),
        C.c_void_p(stream))
    assert status == pkg.abi.C8R_OK, lib.c8r_last_global_error()
    torch.cuda.synchronize()
    host_counters = pkg.abi.Counters.from_buffer_copy(counters.cpu().numpy().tobytes()).as_dict()
    return (coreas.cpu().numpy().reshape(3, nc), zhs.cpu().numpy().reshape(3, nz), host_counters)


def ordinary_call(pkg, torch, config, records):
    acc = pkg.RadioAccumulator(config)
    raw = to_device(torch, records)
    acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
    out = acc.download_fixed()
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
