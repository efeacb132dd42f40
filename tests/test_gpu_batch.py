"""Staging and batched projection (many showers, one persistent launch per
algorithm, CUDA-graph replay, autotuner): every event's fixed-point traces
equal the oracle's for that event alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def small_events(showers, count=5):
    specs = showers.batched_event_specs(events=count, seed=99, min_segments=3000,
                                        max_segments=40000, min_antennas=3, max_antennas=40,
                                        bins=1024)
    out = []
    for spec in specs:
        wl, gen = showers.event_workload(spec)
        records = showers.shower_records(spec.segments, seed=spec.seed, **gen)
        out.append((wl, records))
    return out


def device(torch, records):
    return torch.from_numpy(records.view(np.uint8).reshape(-1)).cuda()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_each_event_alone(pkg, oracle, showers, torch_cuda, precision):
    events = small_events(showers)
    stream = torch_cuda.cuda.Stream()
    accs, keep = [], []
    for wl, records in events:
        acc = pkg.RadioAccumulator(showers.make_config(wl, precision=precision, kernel=2),
                                   stream=stream.cuda_stream)
        raw = device(torch_cuda, records)
        keep.append(raw)
        half = records.size // 2
        acc.stage_lepton_tracks(raw.data_ptr(), half)
        acc.stage_lepton_tracks(raw.data_ptr() + half * records.itemsize, records.size - half)
        accs.append(acc)
    batch = pkg.RadioBatch(stream=stream.cuda_stream)
    batch.project(accs, graph=True, keep_staged=True)   # captured, replayed below
    batch.project(accs, graph=True)                     # same plan: replay, then drop staged
    assert batch.graph_captures() == 1
    for (wl, records), acc in zip(events, accs):
        coreas, zhs, counters = acc.download_fixed()
        if precision == 0:
            want = oracle.restatement().project(showers.make_config(wl), records, threads=8)
            assert np.array_equal(coreas, 2 * want[0]) and np.array_equal(zhs, 2 * want[1])
            assert counters["coreas_contributions"] == 2 * want[2]["coreas_contributions"]
            assert counters["zhs_subtracks"] == 2 * want[2]["zhs_subtracks"]
        else:
            alone = pkg.RadioAccumulator(showers.make_config(wl, precision=1, kernel=2))
            raw = device(torch_cuda, records)
            alone.accumulate_lepton_tracks(raw.data_ptr(), records.size)
            alone.accumulate_lepton_tracks(raw.data_ptr(), records.size)
            a = alone.download_fixed()
            alone.close()
            assert np.array_equal(coreas, a[0]) and np.array_equal(zhs, a[1])
        acc.close()
    batch.close()


def test_autotune_then_batch_is_exact(pkg, oracle, showers, torch_cuda):
    events = small_events(showers, count=3)
    stream = torch_cuda.cuda.Stream()
    accs, keep = [], []
    for wl, records in events:
        acc = pkg.RadioAccumulator(showers.make_config(wl, kernel=2), stream=stream.cuda_stream)
        raw = device(torch_cuda, records)
        keep.append(raw)
        acc.stage_lepton_tracks(raw.data_ptr(), records.size)
        accs.append(acc)
    batch = pkg.RadioBatch(stream=stream.cuda_stream)
    best, ms = batch.autotune(accs, repetitions=1)
    assert best.team_size in (256, 384, 512, 640) and ms > 0
    # bin windows shorter than the 1024-bin traces are part of the sweep; a
    # chosen 512-bin window sends bins past it to checked global atomics
    assert best.observer_tile_size in (0, 512)
    batch.project(accs)
    for (wl, records), acc in zip(events, accs):
        coreas, zhs, _ = acc.download_fixed()
        want = oracle.restatement().project(showers.make_config(wl), records, threads=8)
        assert np.array_equal(coreas, want[0]) and np.array_equal(zhs, want[1])
        acc.close()
    batch.close()


def test_staged_tracks_project_at_download(pkg, oracle, showers, torch_cuda):
    wl, records = small_events(showers, count=1)[0]
    acc = pkg.RadioAccumulator(showers.make_config(wl, kernel=2))
    raw = device(torch_cuda, records)
    acc.stage_lepton_tracks(raw.data_ptr(), records.size)
    coreas, zhs, counters = acc.download_fixed()
    want = oracle.restatement().project(showers.make_config(wl), records, threads=8)
    assert np.array_equal(coreas, want[0]) and np.array_equal(zhs, want[1])
    acc.close()


def test_tuning_cache_round_trip(pkg, tmp_path, torch_cuda):
    """A stored tuning loads back for the same device, build and workload
    label, and only for them (TuningCache.cpp:65-82: every key field must
    match)."""
    path = tmp_path / "radio.tuning"
    assert pkg.tuning_cache_load(path, "batched 64 events") is None
    chosen = pkg.TuningParameters(team_size=512, track_tile_size=131072, observer_tile_size=1024)
    pkg.tuning_cache_store(path, "batched 64 events", chosen)
    text = path.read_text()
    assert text.startswith("format=c8radio-b200-tuning-v1\n") and "device_name=" in text
    got = pkg.tuning_cache_load(path, "batched 64 events", require=True)
    assert (got.team_size, got.track_tile_size, got.observer_tile_size) == (512, 131072, 1024)
    assert pkg.tuning_cache_load(path, "another workload") is None
    with pytest.raises(pkg.RadioError, match="does not match"):
        pkg.tuning_cache_load(path, "another workload", require=True)
    path.write_text(text.replace("multiprocessors=", "multiprocessors=1"))
    assert pkg.tuning_cache_load(path, "batched 64 events") is None
    path.write_text(text.replace("team_size=512", "team_size=5x"))
    with pytest.raises(pkg.RadioError, match="not a count"):
        pkg.tuning_cache_load(path, "batched 64 events")
