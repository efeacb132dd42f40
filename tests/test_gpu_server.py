"""Serving (c8r_server_*): events of different sizes, antenna arrays,
precisions and media in flight together, added from several producer threads
in several batches, projected in shared rounds.  Each event's traces must be
the same in the mix as alone: bit for bit in fixed point (and equal to the
oracle for the FP64 events).  Admission waits for HBM budget."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COUNTS = ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks",
          "fixed_point_overflows")


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def device(torch, records):
    return torch.from_numpy(np.ascontiguousarray(records).view(np.uint8).reshape(-1)).cuda()


def mixed_events(showers):
    """(config, records, batches) of six events: four workloads, one empty."""
    out = []
    wl, gen, _ = showers.workload_config("plain_c0", bins=1024)
    out.append((showers.make_config(wl, precision=0, kernel=2), showers.shower_records(20000, seed=1, **gen), 1))
    wl, gen, _ = showers.workload_config("tiled_c1", bins=2048)
    out.append((showers.make_config(wl, precision=1, kernel=2), showers.shower_records(30000, seed=2, **gen), 3))
    wl, gen, _ = showers.workload_config("ice_c2", bins=1024)
    out.append((showers.make_config(wl, precision=0, kernel=2), showers.ice_records(12000, seed=3, **gen), 2))
    spec = showers.batched_event_specs(events=1, seed=5, min_segments=20000, max_segments=40000,
                                       min_antennas=20, max_antennas=40, bins=1024)[0]
    wl, gen = showers.event_workload(spec)
    out.append((showers.make_config(wl, precision=1, kernel=2),
                showers.shower_records(spec.segments, seed=spec.seed, **gen), 4))
    wl, gen, _ = showers.workload_config("plain_c0", bins=512)
    out.append((showers.make_config(wl, precision=0, kernel=2), showers.shower_records(5000, seed=6, **gen), 1))
    out.append((showers.make_config(wl, precision=0, kernel=2), showers.shower_records(0, seed=7, **gen), 0))
    return out


def alone(pkg, torch, config, records):
    acc = pkg.RadioAccumulator(config)
    if records.size:
        raw = device(torch, records)
        acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
    out = acc.download_fixed()
    acc.close()
    return out


def test_events_in_the_mix_equal_each_event_alone(pkg, oracle, showers, torch_cuda):
    torch = torch_cuda
    events = mixed_events(showers)
    raws = [device(torch, r) if r.size else None for _, r, _ in events]
    torch.cuda.synchronize()
    server = pkg.RadioServer(budget_bytes=1 << 30, block_tracks=16384, chunk_tracks=4096,
                             round_pairs=2_000_000)
    ids = [None] * len(events)
    errors = []

    def produce(k):
        try:
            config, records, batches = events[k]
            stream = torch.cuda.Stream()
            ids[k] = server.open(config)
            edges = np.linspace(0, records.size, batches + 1).astype(int) if batches else [0]
            for a, b in zip(edges[:-1], edges[1:]):
                server.add_device(ids[k], raws[k].data_ptr() + int(a) * records.itemsize, int(b - a),
                                  stream=stream.cuda_stream)
            server.close_event(ids[k])
            stream.synchronize()
        except Exception as exc:  # reported by the main thread
            errors.append(exc)

    threads = [threading.Thread(target=produce, args=(k,)) for k in range(len(events))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    results = []
    for k in range(len(events)):
        server.wait(ids[k], timeout_ms=120000)
        results.append(server.fetch_fixed(ids[k]))
    stats = server.stats()
    server.close()
    assert stats["events_completed"] == len(events)
    assert stats["rounds"] > 4 and stats["arena_used_bytes"] == 0
    for (config, records, _), (coreas, zhs, counters, info) in zip(events, results):
        want = alone(pkg, torch, config, records)
        assert np.array_equal(coreas, want[0]) and np.array_equal(zhs, want[1])
        for key in COUNTS:
            assert counters[key] == want[2][key], key
        assert info["records"] == records.size
        assert info["open_s"] <= info["admitted_s"] <= info["closed_s"] <= info["completed_s"]
        if config.precision == 0 and records.size:
            ref = oracle.restatement().project(config, records, threads=8)
            assert np.array_equal(coreas, ref[0]) and np.array_equal(zhs, ref[1])


def test_admission_waits_for_budget(pkg, showers, torch_cuda):
    torch = torch_cuda
    wl, gen, _ = showers.workload_config("plain_c0")  # 16 antennas x 4096 bins
    config = showers.make_config(wl, precision=1, kernel=2)
    first_records = showers.shower_records(40000, seed=11, **gen)
    second_records = showers.shower_records(10000, seed=12, **gen)
    raw1, raw2 = device(torch, first_records), device(torch, second_records)
    torch.cuda.synchronize()
    # resident part ~3.7 MB + one 2 MB block per event: one event fits, two do not
    server = pkg.RadioServer(budget_bytes=8 << 20, block_tracks=16384, chunk_tracks=4096)
    first = server.open(config, timeout_ms=1000)
    with pytest.raises(pkg.ServerTimeout):
        server.open(config, timeout_ms=200)
    admitted = {}

    def second_producer():
        admitted["id"] = server.open(config)  # waits until the first event is fetched
        server.add_device(admitted["id"], raw2.data_ptr(), second_records.size)
        server.close_event(admitted["id"])

    waiter = threading.Thread(target=second_producer)
    waiter.start()
    server.add_device(first, raw1.data_ptr(), first_records.size)  # blocks recycle within the budget
    server.close_event(first)
    server.wait(first, timeout_ms=60000)
    assert "id" not in admitted
    got1 = server.fetch_fixed(first)
    waiter.join(timeout=60)
    assert "id" in admitted
    server.wait(admitted["id"], timeout_ms=60000)
    got2 = server.fetch_fixed(admitted["id"])
    stats = server.stats()
    server.close()
    assert stats["arena_peak_bytes"] <= 8 << 20 and stats["blocks_allocated"] >= 4
    for got, records in ((got1, first_records), (got2, second_records)):
        want = alone(pkg, torch, config, records)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_decoded_fetch_equals_download(pkg, showers, torch_cuda):
    torch = torch_cuda
    wl, gen, _ = showers.workload_config("tiled_c1", bins=1024)
    config = showers.make_config(wl, precision=1, kernel=2)
    records = showers.shower_records(20000, seed=21, **gen)
    raw = device(torch, records)
    torch.cuda.synchronize()
    server = pkg.RadioServer(budget_bytes=1 << 30)
    event = server.open(config)
    server.add_device(event, raw.data_ptr(), records.size)
    server.close_event(event)
    waveforms, info = server.fetch(event)
    server.close()
    acc = pkg.RadioAccumulator(config)
    acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
    want = acc.download()
    acc.close()
    assert np.array_equal(waveforms.coreas, want.coreas) and np.array_equal(waveforms.zhs, want.zhs)
    assert info["rounds"] >= 1
