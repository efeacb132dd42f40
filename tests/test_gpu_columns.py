"""Producer-side input (c8r_accumulate_columns, the input half of the fused
producer path of LeptonCascade.inl:81-83): the steps as device columns (one
array per field radio reads) give the oracle's traces and counters -- bit for
bit in FP64, within 1e-4 relative L2 per trace in mixed precision with the
oracle's bins -- and the same traces as 752-byte records; the diagnostics
(FP64 sums over atomics) agree with the oracle's to rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def relative_l2_per_trace(got, want, observers):
    errors = []
    offset = 0
    for n in observers["number_of_bins"]:
        n = int(n)
        norm = np.linalg.norm(want[:, offset:offset + n])
        if norm > 0:
            errors.append(np.linalg.norm(got[:, offset:offset + n] - want[:, offset:offset + n]) / norm)
        offset += n
    return np.array(errors)


def columns_of(torch, records):
    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()
    keep = {
        "pid": dev(records["start"]["pid"].astype(np.int32)),
        "weight": dev(records["start"]["weight"]),
        "start_time_s": dev(records["start"]["time_s"]),
        "end_time_s": dev(records["end"]["time_s"]),
        "start_energy_gev": dev(records["start"]["energy_gev"]),
    }
    for state, prefix in (("start", "start"), ("end", "end")):
        keep[f"{prefix}_position_m"] = [dev(records[state]["position_m"][:, a]) for a in range(3)]
        keep[f"{prefix}_direction"] = [dev(records[state]["direction"][:, a]) for a in range(3)]
    pointers = {k: (tuple(t.data_ptr() for t in v) if isinstance(v, list) else v.data_ptr())
                for k, v in keep.items()}
    return pointers, keep


@pytest.mark.parametrize("diagnostics", [False, True])
def test_columns_equal_records(pkg, showers, diagnostics):
    import torch

    wl, gen, _ = showers.workload_config("tiled_c1", bins=2048)
    records = showers.shower_records(40_000, seed=81, **gen)
    records["start"]["pid"][::97] = 22  # photons are skipped by both paths
    config = showers.make_config(wl, precision=1, kernel=2, track_diagnostics=diagnostics)
    raw = torch.from_numpy(records.view(np.uint8).reshape(-1)).cuda()
    a = pkg.RadioAccumulator(config)
    a.accumulate_lepton_tracks(raw.data_ptr(), records.size)
    want = a.download_fixed()
    a.close()
    pointers, keep = columns_of(torch, records)
    b = pkg.RadioAccumulator(config)
    half = records.size // 2
    b.accumulate_columns(pointers, half)
    rest = {k: (tuple(p + half * (4 if k == "pid" else 8) for p in v) if isinstance(v, tuple)
                else v + half * (4 if k == "pid" else 8)) for k, v in pointers.items()}
    b.accumulate_columns(rest, records.size - half)
    got = b.download_fixed()
    b.close()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    for key in ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks"):
        assert got[2][key] == want[2][key], key
    if diagnostics:
        for key in ("track_length_m", "weighted_track_length_m", "weighted_direction_change_rad"):
            assert got[2][key] == pytest.approx(want[2][key], rel=1e-12), key
        assert got[2]["maximum_segment_length_m"] == want[2]["maximum_segment_length_m"]


def project_columns(pkg, torch, config, records):
    """Two accumulate_columns calls (the halves of the steps), then download_fixed."""
    pointers, keep = columns_of(torch, records)
    acc = pkg.RadioAccumulator(config)
    half = records.size // 2
    acc.accumulate_columns(pointers, half)
    rest = {k: (tuple(p + half * (4 if k == "pid" else 8) for p in v) if isinstance(v, tuple)
                else v + half * (4 if k == "pid" else 8)) for k, v in pointers.items()}
    acc.accumulate_columns(rest, records.size - half)
    out = acc.download_fixed()
    acc.close()
    return out


@pytest.mark.parametrize("workload,count", [("tiled_c1", 30_000), ("plain_c0", 60_000)])
def test_columns_equal_the_oracle(pkg, oracle, showers, workload, count):
    import torch

    wl, gen, _ = showers.workload_config(workload)
    records = showers.shower_records(count, seed=83, **gen)
    records["start"]["pid"][::89] = 2212  # protons are skipped by both
    exact = showers.make_config(wl, track_diagnostics=True)
    want = oracle.restatement().project(exact, records, threads=16)
    assert want[2]["coreas_contributions"] > 0 and want[2]["zhs_contributions"] > 0

    # FP64 windowed: the oracle's int64 traces and counters; diagnostics to rounding
    got = project_columns(pkg, torch, showers.make_config(wl, precision=0, kernel=2, track_diagnostics=True),
                          records)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    for key in ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks",
                "fixed_point_overflows"):
        assert got[2][key] == want[2][key], key
    for key in ("weighted_segment_count", "track_length_m", "weighted_track_length_m",
                "energy_weighted_track_length_gev_m", "weighted_direction_change_rad",
                "weighted_beta_deficit_track_length_m", "weighted_time_residual_s"):
        np.testing.assert_allclose(got[2][key], want[2][key], rtol=1e-12, atol=1e-30)
    assert got[2]["maximum_segment_length_m"] == want[2]["maximum_segment_length_m"]
    # acos on the device and in the host's libm may differ in the last place
    np.testing.assert_allclose(got[2]["maximum_direction_change_rad"], want[2]["maximum_direction_change_rad"],
                               rtol=1e-15)

    # mixed precision: 1e-4 relative L2 per trace against the oracle, same counters
    got = project_columns(pkg, torch, showers.make_config(wl, precision=1, kernel=2), records)
    scale = exact.fixed_point_field_limit_v_per_m / 2.0 ** 62
    fs = wl["observers"]["sample_rate_hz"][0]
    for key in ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks"):
        assert got[2][key] == want[2][key], key
    for a, factor in ((0, 1.0), (1, fs)):
        err = relative_l2_per_trace(got[a] * (scale / factor), want[a] * (scale / factor), wl["observers"])
        assert err.max() <= 1e-4, (a, err.max())

    # mixed precision bins: the oracle's sample-count traces, bin for bin
    counted = oracle.restatement().project(showers.make_config(wl, count_samples=True), records, threads=16)
    got = project_columns(pkg, torch, showers.make_config(wl, precision=1, kernel=2, count_samples=True),
                          records)
    assert np.array_equal(got[0], counted[0]) and np.array_equal(got[1], counted[1])
