"""Spool replay on the GPU, as testRadioSpoolReplay.cpp:37-112: 2 x 4096 + 7
completed host tracks written to a spool and replayed in batches of 1, 7,
4096 and 65536 give the traces of enqueueing them directly (and the oracle's),
bit for bit, in three 4096-record host batches."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def replay_config(pkg):
    obs = np.zeros(1, pkg.OBSERVER)
    obs[0]["position_m"] = (30., 40., 0.)
    obs[0]["duration_s"] = 2.e-6
    obs[0]["sample_rate_hz"] = 1.e9
    obs[0]["number_of_bins"] = 2000
    return pkg.RadioConfig(enabled=True, deterministic=True,
                           propagation=pkg.FlatAtmosphereSnapshot(homogeneous_refractive_index=1.0003),
                           coreas_observers=obs, zhs_observers=obs)


def replay_tracks(pkg, count):
    """testRadioSpoolReplay.cpp:62-76."""
    c = 299792458.0
    t = np.zeros(count, pkg.abi.TRACK_SEGMENT)
    i = np.arange(count)
    t["pdg"] = np.where(i % 2 == 1, -11, 11)
    t["weight"] = 1.e-4 * (1 + i % 5)
    t["start_kinetic_energy_gev"] = 1. + 0.01 * (i % 7)
    t["end_kinetic_energy_gev"] = t["start_kinetic_energy_gev"]
    t["start_position_m"][:, 0] = 0.001 * (i % 37)
    t["end_position_m"][:, 0] = t["start_position_m"][:, 0] + 0.1
    t["start_direction"][:, 0] = 1.
    t["end_direction"][:, 0] = 1.
    t["start_time_s"] = 1.e-9 * (i % 17)
    t["end_time_s"] = t["start_time_s"] + 0.1 / (0.99 * c)
    return t


def test_spool_replay_in_bounded_batches_changes_nothing(pkg, oracle, tmp_path):
    count = 2 * 4096 + 7
    segments = replay_tracks(pkg, count)
    path = tmp_path / "input.bin"
    writer = pkg.SpoolWriter(path)
    writer.append(segments)
    writer.complete()
    writer.close()
    records = pkg.track_records(segments)
    config = replay_config(pkg)
    direct = pkg.RadioAccumulator(config)
    direct.enqueue_host_lepton_tracks(records)
    expected = direct.download_fixed()
    stats = direct.statistics()
    direct.close()
    assert stats.host_tracks_enqueued == count
    assert np.any(expected[0] != 0)
    want = oracle.restatement().project(config, records, threads=8)
    assert np.array_equal(expected[0], want[0]) and np.array_equal(expected[1], want[1])
    for limit in (1, 7, 4096, 65536):
        replay = pkg.RadioAccumulator(config)
        reader = pkg.SpoolReader(path)
        reader.replay(replay, batch=limit)
        assert reader.state() == (count, True)
        reader.close()
        got = replay.download_fixed()
        stats = replay.statistics()
        replay.close()
        assert np.array_equal(got[0], expected[0]) and np.array_equal(got[1], expected[1]), limit
        assert stats.host_tracks_enqueued == count and stats.lepton_tracks == count
        assert stats.host_track_batches == 3
