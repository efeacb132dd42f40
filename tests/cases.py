"""Inputs of the reference's radio tests, restated for this suite.

* scalar_cases(): the 14 single-track cases of tests/kokkos/radio/RadioFixture.cpp:164-231
  (ordinary, positron_weight, fraunhofer, near_cone, lower_edge, late_track,
  window_end, edge_first/last, subbin_first/last, vacuum, table steps 0.5/1/2 m)
  on a uniform-index atmosphere table from -1 km to 2 km with three observers.
* accumulator_config()/accumulator_track(): the configuration and synthetic
  track generator of tests/kokkos/radio/accumulator/testRadioAccumulator.cpp:17-75.
* accumulator_grid(): its 15-case grid (:181-214).
"""
from __future__ import annotations

import math

import numpy as np

import __graft_entry__ as entry

pkg = entry.load_package()
from corsika8_kokkos_b200 import FlatAtmosphereSnapshot, RadioConfig  # noqa: E402
from corsika8_kokkos_b200.abi import LEPTON_RECORD, OBSERVER  # noqa: E402

C = 299792458.0
ELECTRON_MASS_GEV = 5.109989e-4


def uniform_table(index: float, lower: float, upper: float, step: float) -> FlatAtmosphereSnapshot:
    """make_radio_config on a one-node uniform-index environment (RadioFixture.cpp:92-131)."""
    minimum = lower - 1000.0
    inverse = 1.0 / step
    bins = int((upper - minimum) * inverse + 1)
    n = np.full(bins, index - 1.0)
    integral = np.cumsum(n * inverse)
    last = bins - 1
    return FlatAtmosphereSnapshot(
        0.0, minimum, upper, step, inverse,
        (n[10] - n[0]) / 10.0, (integral[10] - integral[0]) / 10.0,
        (n[last] - n[last - 10]) / 10.0, (integral[last] - integral[last - 10]) / 10.0,
        n, integral)


def _record(start, end, beta, t0, pid=11, weight=1.0):
    r = np.zeros(1, LEPTON_RECORD)
    length = math.dist(start, end)
    dt = length / (C * beta)
    direction = [(e - s) / length for s, e in zip(start, end)]
    for side, pos, t in (("start", start, t0), ("end", end, t0 + dt)):
        r[side]["pid"] = pid
        r[side]["energy_gev"] = 1.0 + ELECTRON_MASS_GEV
        r[side]["weight"] = weight
        r[side]["time_s"] = t
        r[side]["position_m"] = pos
        r[side]["direction"] = direction
    return r


def _observers(duration: float) -> np.ndarray:
    obs = np.zeros(3, OBSERVER)
    for i, (x, y) in enumerate([(100.0, 2.0), (17.0, 31.0), (1.0, 0.0)]):
        obs[i]["position_m"] = (x, y, 0.0)
        obs[i]["start_time_s"] = 0.0
        obs[i]["duration_s"] = duration
        obs[i]["sample_rate_hz"] = 1e9
        obs[i]["number_of_bins"] = int(duration * 1e9 + 1.5)  # TimeDomainObserver.inl:23
    return obs


def scalar_cases():
    """[(name, RadioConfig, record)] of RadioFixture.cpp:164-231."""
    half = 0.99 * C * 20e-9 / 2.0
    table = [
        ("ordinary", (3., 4., 100.), (4., 6., 99.), .8, 0., 2e-6, 1.0003, 11, 1.),
        ("positron_weight", (3., 4., 100.), (4., 6., 99.), .8, 0., 2e-6, 1.0003, -11, 37.),
        ("fraunhofer", (3., 4., 100.), (4., 6., 10.), .99, 0., 2e-6, 1.0003, 11, 1.),
        ("near_cone", (0., 0., 1000.), (0., 0., 990.), .999999, -3e-6, 2e-6, 1.0003, 11, 1.),
        ("lower_edge", (3., 4., -1000.), (4., 6., -1001.), .8, 0., 8e-6, 1.0003, 11, 1.),
        ("late_track", (3., 4., 100.), (4., 6., 99.), .8, 1e-3, 4e-7, 1.0003, 11, 1.),
        ("window_end", (3., 4., 10.), (8., 4., 10.), .8, 7.181319171927605e-8, 4e-7, 1.0003, 11, 1.),
        ("edge_first", (100. - half, 2., 1000.), (100. + half, 2., 1000.), .99,
         -1000. / C - 5.25e-9, 10e-9, 1., 11, 1.),
        ("edge_last", (100. - half, 2., 1000.), (100. + half, 2., 1000.), .99,
         -1000. / C - 5.75e-9, 10e-9, 1., 11, 1.),
        ("subbin_first", (100. - half / 100., 2., 1000.), (100. + half / 100., 2., 1000.), .99,
         -1000. / C - .35e-9, 10e-9, 1., 11, 1.),
        ("subbin_last", (100. - half / 100., 2., 1000.), (100. + half / 100., 2., 1000.), .99,
         -1000. / C + 10.15e-9, 10e-9, 1., 11, 1.),
        ("vacuum", (3., 4., 100.), (4., 6., 99.), .8, 0., 2e-6, 1., 11, 1.),
    ]
    out = []
    for name, s, e, beta, t0, dur, n, pid, w in table:
        steps = (1.0, 0.5, 2.0) if name == "ordinary" else (1.0,)
        for step in steps:
            obs = _observers(dur)
            cfg = RadioConfig(enabled=True, deterministic=True,
                              propagation=uniform_table(n, 0.0, 2000.0, step),
                              coreas_observers=obs, zhs_observers=obs.copy())
            out.append((f"{name}/step={step}", cfg, _record(s, e, beta, t0, pid, w)))
    # RadioFixture adds the step variants of "ordinary" after the 12 cases
    order = [c for c in out if c[0].endswith("step=1.0")] + [c for c in out if not c[0].endswith("step=1.0")]
    assert len(order) == 14
    return order


def invalid_records(base: np.ndarray) -> np.ndarray:
    """testRadioProjection.cpp:59-65: pid 22, pid 13, zero and negative duration, zero length."""
    r = np.repeat(base, 5)
    r[0]["start"]["pid"] = 22
    r[1]["start"]["pid"] = 13
    r[2]["end"]["time_s"] = r[2]["start"]["time_s"]
    r[3]["end"]["time_s"] = r[3]["start"]["time_s"] - 1.0
    r[4]["end"]["position_m"] = r[4]["start"]["position_m"]
    return r


def accumulator_config(mask: int, observers: int, separate: bool, integer: bool,
                       table: bool = False) -> RadioConfig:
    """testRadioAccumulator.cpp:17-56."""
    if table:
        n = np.array([0.0003 * math.exp(-i / 100.0) for i in range(101)])
        integral = np.zeros(101)
        for i in range(101):
            integral[i] = n[i] + (integral[i - 1] if i else 0.0)
        prop = FlatAtmosphereSnapshot(0.0, 0.0, 100.0, 1.0, 1.0,
                                      (n[10] - n[0]) / 10.0, (integral[10] - integral[0]) / 10.0,
                                      (n[100] - n[90]) / 10.0, (integral[100] - integral[90]) / 10.0,
                                      n, integral)
    else:
        prop = FlatAtmosphereSnapshot(homogeneous_refractive_index=1.0003)
    co, zo = [], []
    for i in range(observers):
        o = np.zeros(1, OBSERVER)[0]
        o["position_m"] = (30.0 + i, 40.0, 3.0)
        o["duration_s"] = 4e-6
        o["sample_rate_hz"] = 128e6
        o["number_of_bins"] = 512
        if mask & 1:
            co.append(o.copy())
        if separate:
            o["position_m"][1] += 1.0
        if mask & 2:
            zo.append(o.copy())
    return RadioConfig(enabled=True, coreas_enabled=bool(mask & 1), zhs_enabled=bool(mask & 2),
                       deterministic=integer, propagation=prop,
                       coreas_observers=np.array(co, OBSERVER), zhs_observers=np.array(zo, OBSERVER))


def accumulator_tracks(count: int) -> np.ndarray:
    """track(i), testRadioAccumulator.cpp:58-75."""
    r = np.zeros(count, LEPTON_RECORD)
    i = np.arange(count)
    s = r["start"]
    s["pid"] = np.where(i % 2 == 1, -11, 11)
    s["energy_gev"] = 1.0 + 0.01 * (i % 7)
    s["weight"] = 1e-4 * (1 + i % 5)
    s["direction"][:, 0] = 1.0
    s["position_m"][:, 0] = 0.001 * (i % 37)
    s["position_m"][:, 1] = 0.001 * (i % 23)
    s["position_m"][:, 2] = 10.0 + 0.001 * (i % 11)
    s["time_s"] = 1e-9 * (i % 17)
    r["end"] = r["start"]
    moving = i % 19 != 0
    length = 0.1 + 0.01 * (i % 7)
    e = r["end"]
    e["position_m"][moving, 0] += length[moving]
    e["time_s"][moving] += length[moving] / (0.99 * C)
    return r


def accumulator_grid():
    """[(label, config, count)] of testRadioAccumulator.cpp:181-214 (fixed-export
    and floating variants; the custom-tile variants differ only in tiling)."""
    out = []
    for mask in (1, 2, 3):
        for count in (127, 16385):
            for observers in (3, 33):
                out.append((f"mask{mask}/n{count}/obs{observers}",
                            accumulator_config(mask, observers, False, True), count))
    c = accumulator_config(3, 33, True, True, table=True)
    c.track_diagnostics = True
    c.zhs_subtrack_refinement = 3
    out.append(("table/diagnostics/refine3", c, 137))
    for integer in (False, True):
        out.append((f"separate/int{int(integer)}", accumulator_config(3, 5, True, integer), 16385))
    return out
