"""GPU parity: the sm_100a kernels through the C ABI against the oracle.

Fixed-point (deterministic) traces are compared bit for bit; floating traces
(FP64 atomics, order-dependent) within 1e-12 of each trace's peak; the mixed
path within 1e-4 relative L2 per trace with identical contribution counters.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

KERNELS = {"direct": 1, "windowed": 2, "tiled": 3}
EXACT_COUNTERS = ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks",
                  "fixed_point_overflows")


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch


def to_device(torch, records):
    return torch.from_numpy(np.ascontiguousarray(records).view(np.uint8).reshape(-1)).cuda()


def gpu_project(pkg, torch, config, records, kernel=None, tuning=None):
    if kernel is not None:
        config.kernel = kernel
    acc = pkg.RadioAccumulator(config, tuning)
    raw = to_device(torch, records) if records.size else None
    if records.size:
        acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
    if config.deterministic:
        coreas, zhs, counters = acc.download_fixed()
    else:
        w = acc.download()
        coreas, zhs, counters = w.coreas, w.zhs, w.counters
    stats = acc.statistics()
    acc.close()
    return coreas, zhs, counters, stats


def assert_same(got, want, deterministic):
    for g, w in ((got[0], want[0]), (got[1], want[1])):
        assert g.shape == w.shape
        if deterministic:
            assert np.array_equal(g, w), f"{np.count_nonzero(g != w)} of {g.size} values differ"
        else:
            peak = max(np.abs(w).max(initial=0.0), 1e-300)
            assert np.abs(g - w).max(initial=0.0) <= 1e-28 + 2e-12 * peak
    for key in EXACT_COUNTERS:
        assert got[2][key] == want[2][key], key


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_scalar_cases(pkg, oracle, torch_cuda, kernel):
    for name, config, record in cases.scalar_cases():
        for integer in (False, True):
            for mode in (1, 2, 3):
                config.deterministic = integer
                config.coreas_enabled = bool(mode & 1)
                config.zhs_enabled = bool(mode & 2)
                want = oracle.restatement().project(config, record, threads=1)
                got = gpu_project(pkg, torch_cuda, config, record, KERNELS[kernel])
                assert_same(got, want, integer)


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_homogeneous_refinement_and_invalid(pkg, oracle, torch_cuda, kernel):
    name, config, record = cases.scalar_cases()[0]
    for index in (1.0, 1.0003, 1.78):
        config.propagation.homogeneous_refractive_index = index
        config.zhs_subtrack_refinement = 3
        want = oracle.restatement().project(config, record, threads=1)
        assert_same(gpu_project(pkg, torch_cuda, config, record, KERNELS[kernel]), want, True)
    invalid = cases.invalid_records(record)
    got = gpu_project(pkg, torch_cuda, config, invalid, KERNELS[kernel])
    assert got[2]["valid_tracks"] == 0
    assert not got[0].any() and not got[1].any()


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_accumulator_grid(pkg, oracle, torch_cuda, kernel):
    for label, config, count in cases.accumulator_grid():
        records = cases.accumulator_tracks(count)
        want = oracle.restatement().project(config, records, threads=8)
        got = gpu_project(pkg, torch_cuda, config, records, KERNELS[kernel])
        assert_same(got, want, config.deterministic)
        if config.track_diagnostics:
            for key in ("weighted_segment_count", "track_length_m", "weighted_track_length_m",
                        "energy_weighted_track_length_gev_m", "maximum_segment_length_m",
                        "weighted_beta_deficit_track_length_m", "weighted_time_residual_s"):
                np.testing.assert_allclose(got[2][key], want[2][key], rtol=1e-12, atol=1e-30)
            np.testing.assert_allclose(got[2]["weighted_track_length_by_kinetic_energy_m"],
                                       want[2]["weighted_track_length_by_kinetic_energy_m"],
                                       rtol=1e-12, atol=1e-30)


def _workload_records(showers, name, count, seed):
    wl, gen, _ = showers.workload_config(name)
    if gen.get("ice"):
        return wl, showers.ice_records(count, seed=seed, **gen)
    return wl, showers.shower_records(count, seed=seed, **gen)


@pytest.mark.parametrize("name,count", [("plain_c0", 100_000), ("tiled_c1", 20_000),
                                        ("ice_c2", 50_000)])
@pytest.mark.parametrize("kernel", list(KERNELS))
def test_synthetic_showers_bit_exact(pkg, oracle, showers, torch_cuda, name, count, kernel):
    wl, records = _workload_records(showers, name, count, seed=21)
    config = showers.make_config(wl)
    want = oracle.restatement().project(config, records, threads=16)
    got = gpu_project(pkg, torch_cuda, config, records, KERNELS[kernel])
    assert_same(got, want, True)
    assert got[2]["coreas_contributions"] > 0 and got[2]["zhs_contributions"] > 0


def relative_l2_per_trace(got, want, observers):
    errors = []
    offset = 0
    for n in observers["number_of_bins"]:
        n = int(n)
        g, w = got[:, offset:offset + n], want[:, offset:offset + n]
        norm = np.linalg.norm(w)
        if norm > 0:
            errors.append(np.linalg.norm(g - w) / norm)
        offset += n
    return np.array(errors)


@pytest.mark.parametrize("name,count", [("plain_c0", 100_000), ("tiled_c1", 20_000),
                                        ("ice_c2", 50_000)])
def test_mixed_precision_within_1e4(pkg, oracle, showers, torch_cuda, name, count):
    wl, records = _workload_records(showers, name, count, seed=33)
    exact_cfg = showers.make_config(wl)
    want = oracle.restatement().project(exact_cfg, records, threads=16)
    scale = exact_cfg.fixed_point_field_limit_v_per_m / 2.0 ** 62
    fs = wl["observers"]["sample_rate_hz"][0]
    for kernel in KERNELS.values():
        mixed = showers.make_config(wl, precision=1, kernel=kernel)
        got = gpu_project(pkg, torch_cuda, mixed, records)
        for key in ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks"):
            assert got[2][key] == want[2][key], key
        for a, factor in ((0, 1.0), (1, fs)):
            err = relative_l2_per_trace(got[a] * (scale / factor), want[a] * (scale / factor),
                                        wl["observers"])
            assert err.max() <= 1e-4, (a, err.max())


@pytest.mark.parametrize("name,count", [("plain_c0", 100_000), ("tiled_c1", 20_000),
                                        ("ice_c2", 50_000)])
def test_bins_bit_exact_in_every_precision(pkg, oracle, showers, torch_cuda, name, count):
    """Sample-count traces (1 per sample per component): the multiset of bins each
    precision and kernel deposits into equals the oracle's, bin for bin."""
    wl, records = _workload_records(showers, name, count, seed=35)
    config = showers.make_config(wl, count_samples=True)
    want = oracle.restatement().project(config, records, threads=16)
    assert want[0].sum() > 0 and want[1].sum() > 0
    for precision in (0, 1):
        for kernel in KERNELS.values():
            got = gpu_project(pkg, torch_cuda, showers.make_config(
                wl, precision=precision, kernel=kernel, count_samples=True), records)
            assert np.array_equal(got[0], want[0]), (precision, kernel, "coreas")
            assert np.array_equal(got[1], want[1]), (precision, kernel, "zhs")


def test_host_enqueue_batches_match_device_path(pkg, oracle, showers, torch_cuda):
    """Bounded-batch host replay equals the device path (testRadioSpoolReplay.cpp:37-112)."""
    wl, records = _workload_records(showers, "plain_c0", 9000, seed=5)
    config = showers.make_config(wl)
    want = oracle.restatement().project(config, records, threads=8)
    for batch in (1, 7, 4096, 65536):
        acc = pkg.RadioAccumulator(config, pkg.TuningParameters(batch_size=batch))
        pieces = np.array_split(records, 5) if batch > 1 else [records[:300]]
        expected = want if batch > 1 else oracle.restatement().project(config, records[:300], threads=4)
        for piece in pieces:
            acc.enqueue_host_lepton_tracks(piece)
        coreas, zhs, counters = acc.download_fixed()
        stats = acc.statistics()
        acc.close()
        assert_same((coreas, zhs, counters), expected, True)
        assert stats.host_tracks_enqueued == sum(p.size for p in pieces)


def test_short_tail_items_and_ramped_pinned_batches(pkg, oracle, showers, torch_cuda):
    """Work lists that end on quarter-size chunks (the last large chunk split in
    four) and pinned host input copied straight from the caller's memory in
    batches doubling from 1/32 of the host batch (at least 8192 records; the
    last one partial) give the traces of one plain device launch."""
    wl, records = _workload_records(showers, "tiled_c1", 100_000, seed=41)
    want = oracle.restatement().project(showers.make_config(wl), records, threads=16)
    pinned = torch_cuda.empty(records.nbytes, dtype=torch_cuda.uint8, pin_memory=True).numpy()
    pinned[:] = records.view(np.uint8)
    host = pinned.view(pkg.LEPTON_RECORD)
    for precision in (0, 1):
        config = showers.make_config(wl, precision=precision, kernel=KERNELS["windowed"])
        plain = gpu_project(pkg, torch_cuda, config, records)
        if precision == 0:
            assert_same(plain, want, True)
        # 32768-track items: three long chunks, then four of 8192 tracks
        tiled = gpu_project(pkg, torch_cuda, config, records,
                            tuning=pkg.TuningParameters(track_tile_size=32768))
        assert_same(tiled, plain, True)
        acc = pkg.RadioAccumulator(config, pkg.TuningParameters(batch_size=65536,
                                                                track_tile_size=32768))
        acc.enqueue_host_lepton_tracks(host)
        got = acc.download_fixed()
        stats = acc.statistics()
        acc.close()
        assert_same(got, plain, True)
        # batches of 8192, then each twice as long (up to 65536), the last one partial
        sizes, size, left = [], 8192, records.size
        while left:
            sizes.append(min(size, left))
            left -= sizes[-1]
            size = min(65536, 2 * size)
        assert stats.host_track_batches == len(sizes) == 4
        assert stats.host_tracks_enqueued == records.size


def test_growing_host_batches_grow_the_deferred_lists(pkg, oracle, showers, torch_cuda):
    """Pinned host batches that grow (8192 to 131072 records; automatic chunks
    from 8192 to 16384 tracks) make the accumulator grow its per-CTA
    deferred-pair lists between launches; the traces equal the oracle's."""
    wl, records = _workload_records(showers, "plain_c0", 300_000, seed=43)
    pinned = torch_cuda.empty(records.nbytes, dtype=torch_cuda.uint8, pin_memory=True).numpy()
    pinned[:] = records.view(np.uint8)
    config = showers.make_config(wl, kernel=KERNELS["windowed"])
    acc = pkg.RadioAccumulator(config, pkg.TuningParameters(batch_size=262144))
    acc.enqueue_host_lepton_tracks(pinned.view(pkg.LEPTON_RECORD))
    got = acc.download_fixed()
    stats = acc.statistics()
    acc.close()
    want = oracle.restatement().project(config, records, threads=16)
    assert_same(got, want, True)
    assert stats.host_track_batches == 6 and stats.host_tracks_enqueued == records.size


def test_side_stream_and_serial_launches_agree(pkg, showers, torch_cuda):
    """Without kernel timing the ZHS launch runs on a second stream beside the
    CoREAS launch; with it both run on the accumulator's stream.  Fixed-point
    traces and counters are the same either way, in both precisions."""
    wl, records = _workload_records(showers, "tiled_c1", 30_000, seed=47)
    raw = to_device(torch_cuda, records)
    for precision in (0, 1):
        config = showers.make_config(wl, precision=precision, kernel=KERNELS["windowed"])
        results = []
        for timing in (False, True):
            acc = pkg.RadioAccumulator(config)
            acc.set_kernel_timing(timing)
            for _ in range(2):  # two accumulates: the second waits for the first's ZHS launch
                acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
            results.append(acc.download_fixed())
            acc.close()
        assert_same(results[0], results[1], True)


def test_lifecycle_contracts(pkg, showers, torch_cuda):
    """Rejection contracts of testRadioAccumulator.cpp:216-302."""
    wl, records = _workload_records(showers, "plain_c0", 100, seed=1)
    config = showers.make_config(wl)
    acc = pkg.RadioAccumulator(config)
    raw = to_device(torch_cuda, records)
    with pytest.raises(pkg.OutOfRange):
        acc.accumulate_lepton_tracks(raw.data_ptr(), 10, extent=5)
    with pytest.raises(pkg.InvalidArgument):
        acc.enqueue_host_pointer(None, 1)
    acc.enqueue_host_pointer(None, 0)
    acc.enqueue_host_lepton_tracks(records[:1])
    with pytest.raises(pkg.LogicError):
        acc.reset()
    first = acc.download()
    with pytest.raises(pkg.LogicError):
        acc.download()
    with pytest.raises(pkg.LogicError):
        acc.enqueue_host_lepton_tracks(records[:1])
    acc.reset()
    empty = acc.download()
    assert not empty.coreas.any() and not empty.zhs.any()
    acc.reset()
    acc.enqueue_host_lepton_tracks(records[:1])
    again = acc.download()
    assert np.array_equal(first.coreas, again.coreas) and np.array_equal(first.zhs, again.zhs)
    acc.close()
    off = pkg.RadioAccumulator(pkg.RadioConfig(enabled=False))
    assert not off.enabled()
    assert off.download().coreas.size == 0
    off.close()
    for variant in range(7):
        bad = showers.make_config(wl)
        bad.coreas_observers = bad.coreas_observers.copy()
        bad.zhs_observers = bad.zhs_observers.copy()
        if variant == 0:
            bad.coreas_enabled = bad.zhs_enabled = False
        elif variant == 1:
            bad.fixed_point_field_limit_v_per_m = 0.0
        elif variant == 2:
            bad.zhs_subtrack_refinement = 0
        elif variant == 3:
            bad.zhs_subtrack_refinement = 65
        elif variant == 4:
            bad.coreas_observers[0]["number_of_bins"] = 0
        elif variant == 5:
            bad.zhs_observers[0]["sample_rate_hz"] = -1.0
        else:
            bad.coreas_observers[0]["position_m"][0] = np.inf
        with pytest.raises(pkg.InvalidArgument):
            pkg.projected_device_bytes(bad)
        with pytest.raises(pkg.InvalidArgument):
            pkg.RadioAccumulator(bad)
    with pytest.raises(pkg.InvalidArgument):
        pkg.RadioAccumulator(config, pkg.TuningParameters(team_size=1025))


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_fixed_point_overflow_is_reported(pkg, showers, torch_cuda, kernel):
    wl, records = _workload_records(showers, "plain_c0", 3000, seed=9)
    config = showers.make_config(wl, kernel=KERNELS[kernel])
    config.fixed_point_field_limit_v_per_m = 1e-30
    acc = pkg.RadioAccumulator(config)
    raw = to_device(torch_cuda, records)
    acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
    with pytest.raises(pkg.FixedPointOverflow):
        acc.download()
    assert acc.statistics().fixed_point_overflows > 0
    acc.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_window_rerun_near_the_fixed_point_limit(pkg, oracle, showers, torch_cuda, precision):
    """A limit of 1.5x the largest |trace| value: the largest bin then holds
    2^62/1.5 > 2^61 in fixed point, so its window's bound on the sum of
    |increments| trips and that item is projected again with checked adds,
    while every final sum still fits in int64.  The traces equal those of
    256-track items (bounds far lower) and, in FP64, the oracle's."""
    wl, records = _workload_records(showers, "plain_c0", 20_000, seed=12)
    floating = showers.make_config(wl, deterministic=False)
    coreas, zhs, _ = oracle.restatement().project(floating, records, threads=8)
    fs = float(wl["observers"]["sample_rate_hz"][0])
    peak = max(np.abs(coreas).max(), fs * np.abs(zhs).max())
    config = showers.make_config(wl, precision=precision, kernel=2)
    config.fixed_point_field_limit_v_per_m = 1.5 * peak
    # one item holds every track of an antenna, so the largest bin's whole sum is in one window
    got = gpu_project(pkg, torch_cuda, config, records,
                      tuning=pkg.TuningParameters(track_tile_size=32768))
    small = gpu_project(pkg, torch_cuda, config, records,
                        tuning=pkg.TuningParameters(track_tile_size=256))
    assert np.array_equal(got[0], small[0]) and np.array_equal(got[1], small[1])
    assert got[2]["fixed_point_overflows"] == 0
    assert got[3].window_reruns >= 1  # the bound tripped: an item ran again with checked adds
    assert max(np.abs(got[0]).max(), np.abs(got[1]).max()) > 2 ** 61
    if precision == 0:
        want = oracle.restatement().project(config, records, threads=8)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def heavy_zhs_records(pkg, count, seed):
    """Slow e- (beta 0.1) moving away from an antenna at the origin, 1 km below,
    3 deg off the line of sight: each track is one undivided ZHS segment
    (Fraunhofer number ~0.3) whose detection times span about 8000 bins at
    10 GHz.  Returns (records, trace start time)."""
    from corsika8_kokkos_b200 import showers

    rng = np.random.default_rng(seed)
    c = showers.SPEED_OF_LIGHT
    beta, duration = 0.1, 727e-9
    tilt = np.radians(3.0)
    direction = np.array([np.sin(tilt), 0.0, np.cos(tilt)])
    start = np.zeros((count, 3))
    start[:, 0] = rng.uniform(-1.0, 1.0, count)
    start[:, 1] = rng.uniform(-1.0, 1.0, count)
    start[:, 2] = 1000.0
    t_start = rng.uniform(0.0, 1e-9, count)
    seg = dict(start=start, end=start + beta * c * duration * direction, t_start=t_start,
               t_end=t_start + duration, pid=np.full(count, 11, np.int32), energy_gev=np.full(count, 5.14e-4),
               direction=np.tile(direction, (count, 1)), weight=np.ones(count))
    # detection time of the first sample: midpoint travel time less n beta.k (t_mid - t_start)
    mid = 1000.0 + 0.5 * beta * c * duration * np.cos(tilt)
    first = mid / c - beta * np.cos(tilt) * 0.5 * duration
    return showers.to_records(seg), first - 5e-9


def test_window_cap_on_adds_per_thread(pkg, oracle, showers, torch_cuda):
    """The unchecked window adds rely on an FP32 sum of |increments| per
    thread, valid while a thread makes fewer than 2^22 adds in an item.  One
    item of 240000 heavy ZHS tracks (about 8000 samples each: 1.9e9 samples,
    about 5e6 a thread of a 384-thread CTA) passes the cap and must be
    projected again with checked adds; one of 100000 tracks (about 2e6 a
    thread) stays below it and must not.  Both equal the oracle bit for bit."""
    from corsika8_kokkos_b200 import FlatAtmosphereSnapshot, RadioConfig

    for count, over in ((240_000, True), (100_000, False)):
        records, start = heavy_zhs_records(pkg, count, seed=count)
        observer = np.zeros(1, pkg.abi.OBSERVER)
        observer[0]["start_time_s"] = start
        observer[0]["duration_s"] = 8191 / 1e10
        observer[0]["sample_rate_hz"] = 1e10
        observer[0]["number_of_bins"] = 8192
        config = RadioConfig(enabled=True, coreas_enabled=False, zhs_enabled=True, deterministic=True,
                             propagation=FlatAtmosphereSnapshot(homogeneous_refractive_index=1.0),
                             coreas_observers=np.zeros(0, pkg.abi.OBSERVER), zhs_observers=observer,
                             precision=0, kernel=2)
        # work items of 1M tracks: the plan ends on quarter-length items
        # (262144 tracks), so each case is one item holding every track
        got = gpu_project(pkg, torch_cuda, config, records,
                          tuning=pkg.TuningParameters(team_size=384, track_tile_size=1 << 20))
        want = oracle.restatement().project(config, records, threads=16)
        assert_same(got[:3], want, True)
        per_thread = want[2]["zhs_contributions"] / 384
        assert (per_thread > 2 ** 22) == over, per_thread
        assert (got[3].window_reruns >= 1) == over, got[3].window_reruns


@pytest.mark.parametrize("precision", [0, 1])
def test_two_pass_handback_when_the_lists_fill(pkg, oracle, showers, torch_cuda, precision):
    """Fixed-point ZHS runs the track loop and the drain as two passes.  With
    subtrack refinement 2 every ZHS pair is deferred, and with 256-track work
    items each CTA's first-pass list (one item's length here) is full after
    its first item: every later item is handed back unflushed and projected
    in full by the second pass.  The traces equal the oracle's (FP64: bit for
    bit; mixed: counters equal, traces within 1e-4), so no pair is lost or
    deposited twice."""
    wl, records = _workload_records(showers, "plain_c0", 20_000, seed=41)
    config = showers.make_config(wl, precision=precision, kernel=2)
    config.zhs_subtrack_refinement = 2
    got = gpu_project(pkg, torch_cuda, config, records, tuning=pkg.TuningParameters(track_tile_size=256))
    exact = showers.make_config(wl)
    exact.zhs_subtrack_refinement = 2
    want = oracle.restatement().project(exact, records, threads=16)
    assert got[3].window_handbacks > 0
    if precision == 0:
        assert_same(got[:3], want, True)
    else:
        for key in EXACT_COUNTERS:
            assert got[2][key] == want[2][key], key
        scale = exact.fixed_point_field_limit_v_per_m / 2.0 ** 62
        fs = wl["observers"]["sample_rate_hz"][0]
        for a, factor in ((0, 1.0), (1, fs)):
            err = relative_l2_per_trace(got[a] * (scale / factor), want[a] * (scale / factor),
                                        wl["observers"])
            assert err.max() <= 1e-4, (a, err.max())


@pytest.mark.parametrize("precision", [0, 1])
def test_traces_longer_than_the_window(pkg, oracle, showers, torch_cuda, precision):
    """20000-bin traces exceed the largest shared-memory window: the bins past
    it go to checked global atomics, and such items never take unchecked window
    adds.  FP64 traces equal the oracle's; mixed-precision bins equal FP64's."""
    wl, records = _workload_records(showers, "plain_c0", 30_000, seed=14)
    # the pulse arrives about 800 ns (bin ~8000) after each trace starts: it straddles the window edge
    wl["observers"] = showers.star_antennas(4, [40.0, 120.0], 1400.0, 20000, 1e10, pre_trigger_s=800e-9)
    count_cfg = showers.make_config(wl, precision=precision, kernel=2, count_samples=True)
    got = gpu_project(pkg, torch_cuda, count_cfg, records)
    want = oracle.restatement().project(showers.make_config(wl, count_samples=True), records, threads=8)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    # the window holds about 8600 bins on a B200 (227 KB of shared memory a block)
    width = got[3].observer_tile_size
    assert 8000 < width < 20000
    tail = got[0][0].reshape(8, 20000)[:, width:].sum() + got[1][0].reshape(8, 20000)[:, width:].sum()
    head = got[0][0].reshape(8, 20000)[:, :width].sum() + got[1][0].reshape(8, 20000)[:, :width].sum()
    assert tail > 0 and head > 0  # samples on both sides of the window edge
    if precision == 0:
        config = showers.make_config(wl, precision=0, kernel=2)
        got = gpu_project(pkg, torch_cuda, config, records)
        want = oracle.restatement().project(config, records, threads=8)
        assert_same(got, want, True)


def test_empty_and_repeated_batches(pkg, oracle, showers, torch_cuda):
    wl, records = _workload_records(showers, "plain_c0", 40_000, seed=4)
    config = showers.make_config(wl, kernel=2)
    acc = pkg.RadioAccumulator(config)
    raw = to_device(torch_cuda, records)
    acc.accumulate_lepton_tracks(raw.data_ptr(), 0)
    half = records.size // 2
    acc.accumulate_lepton_tracks(raw.data_ptr(), half)
    acc.accumulate_lepton_tracks(raw.data_ptr() + half * records.itemsize, records.size - half)
    coreas, zhs, counters = acc.download_fixed()
    acc.close()
    want = oracle.restatement().project(config, records, threads=16)
    assert_same((coreas, zhs, counters), want, True)


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_gpu_reproduces_reference_digests(pkg, torch_cuda, kernel):
    """Digests of the reference's own fixed-point output, committed in tests/golden."""
    import importlib.util
    import json
    from pathlib import Path

    here = Path(__file__).resolve().parent / "golden"
    spec = importlib.util.spec_from_file_location("make_golden", here / "make_golden.py")
    golden = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(golden)
    expected = json.loads((here / "reference_digests.json").read_text())
    for label, config, records in golden.golden_cases():
        coreas, zhs, counters, _ = gpu_project(pkg, torch_cuda, config, records, KERNELS[kernel])
        assert golden.digest(coreas, zhs) == expected[label]["sha256"], label
        for key in golden.COUNTERS:
            assert counters[key] == expected[label][key], (label, key)
