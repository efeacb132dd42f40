"""Pins the oracle (the C restatement) against the reference.

* known answers of tests/kokkos/radio/testRadioProjection.cpp:133-307 and
  tests/kokkos/radio/accumulator/testHomogeneousRadio.cpp:41-157;
* bit-for-bit equality with the reference's own projection code compiled
  from its sources (oracle/_ref) on the reference's test inputs and on
  synthetic showers;
* committed golden digests made from oracle/_ref (tests/golden).
"""
import math

import numpy as np
import pytest

import cases

INF = math.inf
NAN = math.nan
C = 299792458.0


def backends(oracle):
    out = [("restatement", oracle.restatement())]
    if oracle.reference_available():
        out.append(("reference", oracle.reference()))
    return out


def test_known_answers(oracle):
    for name, b in backends(oracle):
        lib = b.lib
        nb = getattr(lib, f"{b.prefix}_nearest_bin")
        assert nb(0.5) == 1.0
        assert nb(float.fromhex("0x1.fffffffffffffp-2")) == 0.0
        dop = getattr(lib, f"{b.prefix}_doppler")
        assert dop(1.0, oracle.vec([1.0, 2.0 ** -30, 0.0]), oracle.vec([1.0, 2.0 ** -30, 0.0])) == -(2.0 ** -60)
        assert dop(1.0, oracle.vec([1.0, 0.0, 0.0]), oracle.vec([1.0, 0.0, 0.0])) == 0.0
        checked = getattr(lib, f"{b.prefix}_checked_add")
        import ctypes as C

        v = C.c_longlong(2 ** 63 - 1)
        assert checked(C.byref(v), 1) == 0
        v = C.c_longlong(-(2 ** 63))
        assert checked(C.byref(v), -1) == 0
        fixed_point = getattr(lib, f"{b.prefix}_add_fixed_point")
        v = C.c_longlong(0)
        assert fixed_point(C.byref(v), INF, 1.0) == 0
        assert fixed_point(C.byref(v), 1.0, 2.0 ** 63) == 0
        assert fixed_point(C.byref(v), 1.5, 3.0) == 1 and v.value == 4  # rint(4.5) = 4
    lib = oracle.restatement().lib
    assert lib.c8o_diagnostic_energy_bin(0.001) == 0
    assert lib.c8o_diagnostic_energy_bin(101.0) == 14


TIMES = [-.75, -.5, math.nextafter(-.5, 0.), -.25, 0., math.nextafter(.5, 0.), .5,
         math.nextafter(.5, 1.), 4., 4.25, math.nextafter(4.5, 0.), 4.5, 4.75, -1e100, 1e100,
         -INF, INF, NAN]


def window_edges(add_sample):
    """testRadioProjection.cpp:133-231: 18 times into a 5-bin, 1 Hz, 4 s window."""
    rows = []
    for potential in (0, 1):
        floating = np.zeros(15)
        for i, t in enumerate(TIMES):
            add_sample(0.0, 4.0, 1.0, 5, potential, t, [float(1 << i), 0.0, 0.0], 1.0,
                       floating=floating)
        rows.append(floating)
    return np.concatenate(rows)


def test_window_edges(oracle):
    got = window_edges(oracle.add_sample_restatement)
    assert int(got[15]) & (1 << 3)
    assert int(got[19]) & (1 << 9)
    # CoREAS gates -0.25 out, ZHS keeps its half bins
    assert not int(got[0]) & (1 << 3)
    if oracle.reference_available():
        assert np.array_equal(got, window_edges(oracle.add_sample_reference))


def edge_table():
    n = np.array([0.0003 * math.exp(-i / 8.0) for i in range(21)])
    integral = np.cumsum(n)
    return n, integral


@pytest.mark.parametrize("index", [0.0, 1.0, 1.78])
def test_propagation_table_edges(oracle, pkg, index):
    """testRadioProjection.cpp:233-307."""
    n, integral = edge_table()
    snap = pkg.FlatAtmosphereSnapshot(index, -10.0, 10.0, 1.0, 1.0, (n[10] - n[0]) / 10.0,
                                      (integral[10] - integral[0]) / 10.0,
                                      (n[20] - n[10]) / 10.0, (integral[20] - integral[10]) / 10.0,
                                      n, integral)
    config = pkg.RadioConfig(enabled=True, propagation=snap)
    for h in (-12., -10., -9.9, -9.5, -9., 0., 9., 9.5, 10., 11., 100.):
        a = oracle.propagate_restatement(snap, (3., 4., h), (100., 0., 0.))
        if oracle.reference_available():
            b = oracle.propagate_reference(config, (3., 4., h), (100., 0., 0.))
            assert a == b, (h, a, b)
        if index > 0:
            assert a[0] == index * a[3] / C


def test_homogeneous_and_air_regression(oracle, pkg):
    """testHomogeneousRadio.cpp:41-113."""
    snap = pkg.FlatAtmosphereSnapshot(homogeneous_refractive_index=2.0)
    for p in [(0., 0., 0.), (10., 20., 30.), (-100., -200., -300.), (0., 0., 0.001), (1e5, 2e5, 3e5)]:
        t, ns, nd, *_ = oracle.propagate_restatement(snap, p, (30., 40., 0.))
        expected = 2.0 * math.hypot(math.hypot(p[0] - 30., p[1] - 40.), p[2]) / C
        assert abs(t / expected - 1.0) < 4e-15
        assert ns == 2.0 and nd == 2.0
    n = np.full(11, 0.0003)
    integral = np.array([(i + 1) * 0.0003 for i in range(11)])
    air = pkg.FlatAtmosphereSnapshot(0.0, 0.0, 10.0, 1.0, 1.0, 0, 0, 0, 0, n, integral)
    horizontal = oracle.propagate_restatement(air, (0., 0., 3.), (30., 40., 3.))
    assert horizontal[0] == 50.0 / C
    inclined = oracle.propagate_restatement(air, (0., 0., 5.), (30., 40., 3.))
    assert inclined[0] == (1. + (integral[5] - integral[3]) / 2.) * math.sqrt(2504.) / C


def test_separate_same_bin(oracle):
    if not oracle.reference_available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(5)
    for _ in range(2000):
        s, e = rng.uniform(-3, 3, 2)
        res = rng.choice([0.1, 1.0, 0.37])
        for signed in (0, 1):
            assert oracle.separate_restatement(s, e, res, signed) == \
                oracle.separate_reference(s, e, res, signed)


def _compare(oracle, config, records, exact=True):
    a = oracle.restatement().project(config, records, threads=1)
    b = oracle.reference().project(config, records, threads=1)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for key, value in b[2].items():
        if key in ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks",
                   "fixed_point_overflows"):
            assert a[2][key] == value, key
        else:
            np.testing.assert_allclose(a[2][key], value, rtol=1e-12, atol=1e-300)
    return a


def test_scalar_cases_match_reference(oracle):
    """RadioFixture.cpp cases x {float, int} x {CoREAS, ZHS, both} (testRadioProjection.cpp:26-49)."""
    if not oracle.reference_available():
        pytest.skip("reference library not built")
    all_cases = cases.scalar_cases()
    assert len(all_cases) == 14
    checked = 0
    for name, config, record in all_cases:
        for integer in (False, True):
            for mode in (1, 2, 3):
                config.deterministic = integer
                config.coreas_enabled = bool(mode & 1)
                config.zhs_enabled = bool(mode & 2)
                a = _compare(oracle, config, record)
                assert a[2]["valid_tracks"] == 1
                assert a[2]["fixed_point_overflows"] == 0
                if not mode & 1:
                    assert a[2]["coreas_contributions"] == 0
                if not mode & 2:
                    assert a[2]["zhs_contributions"] == 0
                checked += 1
    assert checked == 84


def test_homogeneous_refinement_and_invalid_records(oracle):
    if not oracle.reference_available():
        pytest.skip("reference library not built")
    name, config, record = cases.scalar_cases()[0]
    config.deterministic = True
    for index in (1.0, 1.0003, 1.78):
        config.propagation.homogeneous_refractive_index = index
        config.zhs_subtrack_refinement = 3
        _compare(oracle, config, record)
    invalid = cases.invalid_records(record)
    a = _compare(oracle, config, invalid)
    assert a[2]["valid_tracks"] == 0


def test_accumulator_grid_matches_reference(oracle):
    """testRadioAccumulator.cpp:181-214 grid, single-threaded both sides."""
    if not oracle.reference_available():
        pytest.skip("reference library not built")
    for label, config, count in cases.accumulator_grid():
        records = cases.accumulator_tracks(count)
        a = _compare(oracle, config, records)
        assert a[2]["valid_tracks"] > 0, label


@pytest.mark.parametrize("workload,count", [("plain_c0", 4000), ("tiled_c1", 600), ("ice_c2", 3000)])
def test_synthetic_showers_match_reference(oracle, showers, workload, count):
    if not oracle.reference_available():
        pytest.skip("reference library not built")
    wl, gen, _ = showers.workload_config(workload)
    if gen.get("ice"):
        records = showers.ice_records(count, seed=11, **gen)
    else:
        records = showers.shower_records(count, seed=11, **gen)
    for deterministic in (True, False):
        config = showers.make_config(wl, deterministic=deterministic)
        _compare(oracle, config, records)


def test_threaded_oracle_is_order_independent(oracle, showers):
    wl, gen, _ = showers.workload_config("plain_c0")
    records = showers.shower_records(3000, seed=2, **gen)
    config = showers.make_config(wl)
    one = oracle.restatement().project(config, records, threads=1)
    many = oracle.restatement().project(config, records, threads=8)
    assert np.array_equal(one[0], many[0]) and np.array_equal(one[1], many[1])


def test_restatement_reproduces_reference_digests(oracle):
    """The committed digests were made by the reference's own code (tests/golden/make_golden.py)."""
    import json
    from pathlib import Path

    sys_path = Path(__file__).resolve().parent / "golden"
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", sys_path / "make_golden.py")
    golden = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(golden)
    expected = json.loads((sys_path / "reference_digests.json").read_text())
    seen = 0
    for label, config, records in golden.golden_cases():
        coreas, zhs, counters = oracle.restatement().project(config, records, threads=2)
        want = expected[label]
        assert golden.digest(coreas, zhs) == want["sha256"], label
        for key in golden.COUNTERS:
            assert counters[key] == want[key], (label, key)
        seen += 1
    assert seen == len(expected) == 62
