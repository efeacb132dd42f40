"""Producer-side input: the same steps as device columns (one array per field)
or as 752-byte records give the same traces and counters, bit for bit; the
diagnostics (FP64 sums over atomics) agree to rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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
