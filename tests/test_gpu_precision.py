"""The arrival-time precision study's kernel: the reference's projection with
its arrival times, distances, directions and Cherenkov denominators in FP64,
compensated double-FP32 or FP32 (amplitudes FP32).  In FP64 it must put every
sample in the reference's bin; double-FP32 keeps the bins on these workloads;
plain FP32 moves some."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WORKLOADS = [("plain_c0", 40_000, {}), ("tiled_c1", 10_000, {"bins": 2048}),
             ("ice_c2", 30_000, {"bins": 1024})]


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def records_of(showers, name, count, overrides):
    wl, gen, _ = showers.workload_config(name, **overrides)
    if gen.get("ice"):
        return wl, showers.ice_records(count, seed=31, **gen)
    return wl, showers.shower_records(count, seed=31, **gen)


def project(pkg, torch, showers, wl, records, precision, kernel, count_samples):
    config = showers.make_config(wl, precision=precision, kernel=kernel, count_samples=count_samples)
    acc = pkg.RadioAccumulator(config)
    raw = torch.from_numpy(records.view(np.uint8).reshape(-1)).cuda()
    acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
    out = acc.download_fixed() if count_samples else acc.download()
    acc.close()
    return out


def moved_samples(got, want):
    """Samples in another bin (or missing/extra) between two count traces."""
    return int(np.abs(got[0] - want[0]).sum()) // 2 + abs(int(got[0].sum()) - int(want[0].sum())) // 2


def max_rel_l2(got, want, bins):
    g, w = got.reshape(3, -1, bins), want.reshape(3, -1, bins)
    norm = np.sqrt((w ** 2).sum(axis=(0, 2)))
    ok = norm > 0
    return float((np.sqrt(((g - w) ** 2).sum(axis=(0, 2)))[ok] / norm[ok]).max(initial=0.0))


@pytest.mark.parametrize("name,count,overrides", WORKLOADS)
def test_study_kernel_in_fp64_reproduces_every_bin(pkg, showers, torch_cuda, name, count, overrides):
    wl, records = records_of(showers, name, count, overrides)
    bins = int(wl["observers"]["number_of_bins"][0])
    ref = project(pkg, torch_cuda, showers, wl, records, 0, 2, True)
    got = project(pkg, torch_cuda, showers, wl, records, pkg.abi.PRECISION_STUDY_FP64, 0, True)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    assert got[2]["zhs_subtracks"] == ref[2]["zhs_subtracks"]
    amp_ref = project(pkg, torch_cuda, showers, wl, records, 0, 2, False)
    amp = project(pkg, torch_cuda, showers, wl, records, pkg.abi.PRECISION_STUDY_FP64, 0, False)
    assert max_rel_l2(amp.coreas, amp_ref.coreas, bins) <= 1e-4
    assert max_rel_l2(amp.zhs, amp_ref.zhs, bins) <= 1e-4


def test_double_fp32_keeps_bins_and_fp32_moves_some(pkg, showers, torch_cuda):
    wl, records = records_of(showers, "ice_c2", 60_000, {"bins": 1024})
    bins = int(wl["observers"]["number_of_bins"][0])
    ref = project(pkg, torch_cuda, showers, wl, records, 0, 2, True)
    df = project(pkg, torch_cuda, showers, wl, records, pkg.abi.PRECISION_STUDY_DOUBLE_FP32, 0, True)
    total = int(ref[0][0].sum() + ref[1][0].sum())
    assert moved_samples(df[0], ref[0]) + moved_samples(df[1], ref[1]) <= 1e-6 * total
    amp_ref = project(pkg, torch_cuda, showers, wl, records, 0, 2, False)
    amp = project(pkg, torch_cuda, showers, wl, records, pkg.abi.PRECISION_STUDY_DOUBLE_FP32, 0, False)
    assert max_rel_l2(amp.coreas, amp_ref.coreas, bins) <= 1e-4
    assert max_rel_l2(amp.zhs, amp_ref.zhs, bins) <= 1e-4
    f32 = project(pkg, torch_cuda, showers, wl, records, pkg.abi.PRECISION_STUDY_FP32, 0, True)
    moved = moved_samples(f32[0], ref[0]) + moved_samples(f32[1], ref[1])
    assert 0 < moved < 0.01 * total


def test_study_precisions_are_not_served_or_batched(pkg, showers):
    wl, _, _ = showers.workload_config("plain_c0", bins=256)
    config = showers.make_config(wl, precision=pkg.abi.PRECISION_STUDY_FP32)
    server = pkg.RadioServer(budget_bytes=1 << 30)
    with pytest.raises(pkg.InvalidArgument):
        server.open(config)
    server.close()
