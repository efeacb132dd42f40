"""Two ranks over gloo on CPU: the sharding of one shower's projection
(track shards merged by an exact int64 sum, antenna shards gathered) gives the
traces of the unsharded projection bit for bit, an overflowing track-shard
merge is reported on every rank instead of wrapping, and the benchmark's
max-over-ranks reduction.  The projection itself is the oracle here (no GPU);
the host logic under test is the one bench.py and a multi-GPU caller use."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port):
    import datetime

    import torch.distributed as dist

    import __graft_entry__ as entry

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        entry.load_package()
        from corsika8_kokkos_b200 import sharding, showers

        oracle = entry.load_oracle().restatement()
        wl, gen, _ = showers.workload_config("plain_c0", bins=512)
        records = showers.shower_records(3000, seed=5, **gen)
        config = showers.make_config(wl)
        full = oracle.project(config, records, threads=2)

        begin, end = sharding.track_shard(records.size, rank, world)
        part = oracle.project(config, records[begin:end], threads=2)
        merged = sharding.merge_track_shards(part[0], part[1])
        assert np.array_equal(merged[0], full[0]) and np.array_equal(merged[1], full[1])

        observers = wl["observers"]
        a, b = sharding.antenna_shard(observers, rank, world)
        sub = dict(wl, observers=observers[a:b])
        local = oracle.project(showers.make_config(sub), records, threads=2)
        gathered = sharding.gather_antenna_shards(local[0], observers)
        assert np.array_equal(gathered, full[0])
        gathered = sharding.gather_antenna_shards(local[1], observers)
        assert np.array_equal(gathered, full[1])

        # values near the int64 limits: exact where the total fits, an error on
        # every rank where it does not (the ranks' sum is never wrapped)
        sign = 1 if rank == 0 else -1
        big = sign * np.array([[(1 << 63) - 1, -(1 << 63) + 1, -1]], dtype=np.int64)
        merged = sharding.merge_track_shards(big, -big)
        assert not merged[0].any() and not merged[1].any()
        near = np.full((1, 4), (1 << 62) - 1 + rank, dtype=np.int64)
        summed = sharding.merge_track_shards(near, -near)
        assert np.array_equal(summed[0], np.full((1, 4), (1 << 63) - 1, dtype=np.int64))
        try:
            sharding.merge_track_shards(np.full((1, 2), 1 << 62, dtype=np.int64),
                                        np.zeros((1, 2), dtype=np.int64))
        except OverflowError:
            pass
        else:
            raise AssertionError("an overflowing merge was not reported")

        assert sharding.max_over_ranks(float(rank + 1)) == float(world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_merge_exactly():
    mp.spawn(_worker, args=(2, free_port()), nprocs=2, join=True)


@pytest.mark.parametrize("world", [1, 2, 3, 7])
def test_shards_cover_everything_once(showers, world):
    from corsika8_kokkos_b200 import sharding

    ranges = [sharding.track_shard(1001, r, world) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == 1001
    assert all(ranges[i][1] == ranges[i + 1][0] for i in range(world - 1))
    observers = showers.star_antennas(8, [50.0, 150.0, 300.0], 1400.0, 256, 1e10)
    cuts = [sharding.antenna_shard(observers, r, world) for r in range(world)]
    assert cuts[0][0] == 0 and cuts[-1][1] == observers.size
    assert all(cuts[i][1] == cuts[i + 1][0] for i in range(world - 1))
