"""Parity at the benchmarked configuration: the tiled_c1 workload at full size
(1e7 segments of the seed the benchmark uses x 160 antennas x 8192 bins),
projected through the C ABI exactly as bench.py times it -- one accumulate of
all records with the default plan (666667-track work items, the quarter-size
tail items, the ZHS launch on the side stream).

* FP64 windowed: bit for bit the oracle's int64 traces on a sample of eight
  antennas spread over arms and radii (antennas are independent, so their
  traces are those of a config holding only them), and the oracle's count of
  valid tracks;
* mixed precision: within 1e-4 relative L2 of the FP64 traces for every one of
  the 160 antennas (and of the oracle's on the sample), with the FP64 path's
  integer counters over all 160;
* bins: the mixed path's sample-count traces equal the FP64 path's for all 160
  antennas and the oracle's on the sample.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEGMENTS = 10_000_000
SEED = 1000  # bench.py's seed for rank 0
SAMPLE = (0, 29, 47, 66, 83, 101, 138, 159)  # arm * 20 + radius index


@pytest.fixture(scope="module")
def full(pkg, showers):
    import torch

    assert torch.cuda.is_available()
    wl, gen, default = showers.workload_config("tiled_c1")
    assert default == SEGMENTS and len(wl["observers"]) == 160
    assert int(wl["observers"]["number_of_bins"][0]) == 8192
    records = showers.shower_records(SEGMENTS, seed=SEED, **gen)
    device = torch.from_numpy(records.view(np.uint8).reshape(-1)).cuda()
    yield wl, records, device
    del device
    torch.cuda.empty_cache()


def project(pkg, showers, wl, records, device, **options):
    acc = pkg.RadioAccumulator(showers.make_config(wl, kernel=2, **options))
    acc.accumulate_lepton_tracks(device.data_ptr(), records.size)
    stats = acc.statistics()
    out = acc.download_fixed()
    acc.close()
    return out, stats


def antenna_columns(wl, picks):
    """Columns of the SoA trace rows that belong to the picked antennas."""
    bins = wl["observers"]["number_of_bins"].astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum(bins)])
    return np.concatenate([np.arange(offsets[a], offsets[a + 1]) for a in picks])


def relative_l2_per_trace(got, want, observers, scale):
    errors = []
    offset = 0
    for n in observers["number_of_bins"]:
        n = int(n)
        w = want[:, offset:offset + n] * scale
        norm = np.linalg.norm(w)
        if norm > 0:
            errors.append(np.linalg.norm(got[:, offset:offset + n] * scale - w) / norm)
        offset += n
    return np.array(errors)


def test_full_size_tiled_c1_parity(pkg, oracle, showers, full):
    wl, records, device = full
    picks = list(SAMPLE)
    columns = antenna_columns(wl, picks)
    sample_wl = dict(wl, observers=wl["observers"][picks])

    fp64, stats = project(pkg, showers, wl, records, device, precision=0)
    # the benchmark's plan: several long work items plus the short tail items
    assert stats.projection_tiles > 2 * 160 * 15
    want = oracle.restatement().project(showers.make_config(sample_wl), records, threads=16)
    assert np.array_equal(fp64[0][:, columns], want[0]), "FP64 CoREAS differs from the oracle"
    assert np.array_equal(fp64[1][:, columns], want[1]), "FP64 ZHS differs from the oracle"
    assert want[2]["valid_tracks"] == fp64[2]["valid_tracks"]
    assert want[2]["coreas_contributions"] > 0 and want[2]["zhs_contributions"] > 0

    mixed, _ = project(pkg, showers, wl, records, device, precision=1)
    for key in ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks",
                "fixed_point_overflows"):
        assert mixed[2][key] == fp64[2][key], key
    scale = 1.0 / 2.0 ** 62
    fs = float(wl["observers"]["sample_rate_hz"][0])
    for a, factor in ((0, 1.0), (1, fs)):
        err = relative_l2_per_trace(mixed[a], fp64[a], wl["observers"], scale / factor)
        assert err.size == 160 and err.max() <= 1e-4, (a, err.max())
        err = relative_l2_per_trace(mixed[a][:, columns], want[a], sample_wl["observers"], scale / factor)
        assert err.max() <= 1e-4, (a, err.max())

    counted_fp64, _ = project(pkg, showers, wl, records, device, precision=0, count_samples=True)
    counted_mixed, _ = project(pkg, showers, wl, records, device, precision=1, count_samples=True)
    assert np.array_equal(counted_mixed[0], counted_fp64[0]) and np.array_equal(counted_mixed[1], counted_fp64[1])
    counted = oracle.restatement().project(showers.make_config(sample_wl, count_samples=True), records, threads=16)
    assert np.array_equal(counted_mixed[0][:, columns], counted[0])
    assert np.array_equal(counted_mixed[1][:, columns], counted[1])
