"""Seeded synthetic showers, antenna stars and refractivity tables.

The reference measures on no public dataset; these generators produce the
inputs of its radio path with the shapes and distributions the workloads
name: electron/positron track segments placed along a shower axis by a
Gaisser-Hillas profile through an exponential atmosphere, exponential lateral
offsets, Gaussian angular spread, exponential lengths, log-uniform kinetic
energies and a 60/40 e-/e+ mix, observed by star-shaped antenna arrays on the
ground.  Everything is drawn from numpy's PCG64 with an explicit seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .abi import LEPTON_RECORD, OBSERVER

SPEED_OF_LIGHT = 299792458.0
ELECTRON_MASS_GEV = 5.109989e-4  # corsika/kokkos/em/algorithms/TransportMass.hpp:20


@dataclass
class AtmosphereModel:
    """Exponential atmosphere rho(h) = rho0 exp(-h/H) and n(h) = 1 + N0 exp(-h/H)."""

    rho0_g_cm3: float = 1.225e-3
    scale_height_m: float = 8000.0
    refractivity_sea_level: float = 3.25e-4

    def vertical_depth(self, height_m):
        return self.rho0_g_cm3 * self.scale_height_m * 100.0 * np.exp(-np.asarray(height_m) / self.scale_height_m)

    def height_of_vertical_depth(self, depth):
        return -self.scale_height_m * np.log(np.asarray(depth) / (self.rho0_g_cm3 * self.scale_height_m * 100.0))

    def refractivity(self, height_m):
        return self.refractivity_sea_level * np.exp(-np.asarray(height_m, dtype=np.float64) / self.scale_height_m)


def flat_atmosphere_table(model: AtmosphereModel, lower_z_m: float, upper_z_m: float,
                          step_m: float = 1.0) -> dict:
    """The refractivity table of atmosphere::make_radio_config
    (corsika/detail/kokkos/radio/atmosphere/FlatAtmosphereConfig.inl:11-85):
    n - 1 sampled from (lower - 1 km) to upper in `step` increments, the
    running sum scaled by 1/step as integral, and 10-bin edge slopes."""
    if not step_m > 0:
        raise ValueError("GPU radio propagation table requires a positive step")
    minimum = lower_z_m - 1000.0
    inverse_step = 1.0 / step_m
    bins = int((upper_z_m - minimum) * inverse_step + 1)
    if bins < 11:
        raise ValueError("GPU radio propagation table requires at least eleven points")
    heights = minimum + np.arange(bins, dtype=np.float64) * step_m
    refractivity = model.refractivity(heights)
    integrated = np.cumsum(refractivity * inverse_step)
    last = bins - 1
    return dict(
        homogeneous_refractive_index=0.0,
        minimum_height_m=minimum,
        maximum_height_m=float(upper_z_m),
        step_m=float(step_m),
        inverse_step_per_m=inverse_step,
        slope_refractivity_lower=(refractivity[10] - refractivity[0]) / 10.0,
        slope_integrated_refractivity_lower=(integrated[10] - integrated[0]) / 10.0,
        slope_refractivity_upper=(refractivity[last] - refractivity[last - 10]) / 10.0,
        slope_integrated_refractivity_upper=(integrated[last] - integrated[last - 10]) / 10.0,
        refractivity=refractivity,
        integrated_refractivity=integrated,
    )


def shower_axis(zenith_deg: float, azimuth_deg: float):
    """Unit vector from the core up towards the shower origin, and two transverse unit vectors."""
    th, ph = math.radians(zenith_deg), math.radians(azimuth_deg)
    up = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
    helper = np.array([0.0, 0.0, 1.0]) if abs(up[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
    e1 = np.cross(up, helper)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(up, e1)
    return up, e1, e2


def star_antennas(arms: int, radii, ground_z_m: float, bins: int, sample_rate_hz: float,
                  zenith_deg: float = 0.0, azimuth_deg: float = 0.0,
                  pre_trigger_s: float = 50e-9) -> np.ndarray:
    """Star of `arms` x len(radii) antennas on the ground plane around the core
    (0, 0, ground).  Each trace has `bins` samples starting at the plane-front
    arrival on the axis minus `pre_trigger_s`; duration = (bins - 1)/fs so that
    C8's floor(duration fs + 1.5) gives `bins` (TimeDomainObserver.inl:23)."""
    up, _, _ = shower_axis(zenith_deg, azimuth_deg)
    direction = -up
    out = np.zeros(arms * len(radii), OBSERVER)
    core = np.array([0.0, 0.0, ground_z_m])
    k = 0
    for a in range(arms):
        phi = 2.0 * math.pi * a / arms
        for r in radii:
            pos = core + np.array([r * math.cos(phi), r * math.sin(phi), 0.0])
            arrival = float(np.dot(pos - core, direction)) / SPEED_OF_LIGHT
            out[k]["position_m"] = pos
            out[k]["start_time_s"] = arrival - pre_trigger_s
            out[k]["duration_s"] = (bins - 1) / sample_rate_hz
            out[k]["sample_rate_hz"] = sample_rate_hz
            out[k]["number_of_bins"] = bins
            k += 1
    return out


def _gaisser_hillas_depths(rng, n, xmax, lam, x_ground, x0=0.0, grid=20000):
    """Inverse-CDF samples of N(X) ~ ((X-X0)/(Xmax-X0))^((Xmax-X0)/lam) exp((Xmax-X)/lam) on [X0, x_ground]."""
    x = np.linspace(x0, x_ground, grid)
    w = (xmax - x0) / lam
    with np.errstate(divide="ignore", invalid="ignore"):
        logn = w * np.log(np.maximum((x - x0) / (xmax - x0), 1e-300)) + (xmax - x) / lam
    pdf = np.exp(logn - logn.max())
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (pdf[1:] + pdf[:-1]) * np.diff(x))])
    cdf /= cdf[-1]
    return np.interp(rng.random(n), cdf, x)


def synthetic_segments(n: int, seed: int, zenith_deg: float = 0.0, azimuth_deg: float = 0.0,
                       xmax: float = 700.0, lam: float = 70.0, ground_z_m: float = 1400.0,
                       model: AtmosphereModel | None = None, lateral_scale_m: float = 30.0,
                       angle_sigma_deg: float = 5.0, mean_length_m: float = 1.0,
                       max_length_m: float = 10.0, kinetic_min_gev: float = 1e-3,
                       kinetic_max_gev: float = 1.0, electron_fraction: float = 0.6,
                       front_curvature_m: float = 5000.0, weight: float = 1.0) -> dict:
    """Track segments of one synthetic shower as arrays (start, end, times, pid, ...).

    Positions: depth X from a Gaisser-Hillas profile along the axis through the
    exponential atmosphere (flat earth), an exponential lateral offset in the
    plane transverse to the axis.  Directions: the axis direction plus Gaussian
    transverse kicks of sigma `angle_sigma_deg`.  Start time: axis path / c
    relative to the front crossing the core, plus the curvature delay
    r^2 / (2 c R) of a spherical front of radius `front_curvature_m`."""
    model = model or AtmosphereModel()
    rng = np.random.Generator(np.random.PCG64(seed))
    up, e1, e2 = shower_axis(zenith_deg, azimuth_deg)
    cos_z = max(math.cos(math.radians(zenith_deg)), 1e-6)
    x_ground = float(model.vertical_depth(ground_z_m)) / cos_z
    depth = _gaisser_hillas_depths(rng, n, xmax, lam, x_ground)
    depth = np.maximum(depth, 1e-3)
    height = model.height_of_vertical_depth(depth * cos_z)
    s = (height - ground_z_m) / cos_z  # distance along the axis above the core
    r = rng.exponential(lateral_scale_m, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    core = np.array([0.0, 0.0, ground_z_m])
    start = (core[None, :] + s[:, None] * up[None, :] +
             (r * np.cos(phi))[:, None] * e1[None, :] + (r * np.sin(phi))[:, None] * e2[None, :])
    sigma = math.radians(angle_sigma_deg)
    kick1 = rng.normal(0.0, sigma, n)
    kick2 = rng.normal(0.0, sigma, n)
    direction = -up[None, :] + kick1[:, None] * e1[None, :] + kick2[:, None] * e2[None, :]
    direction /= np.linalg.norm(direction, axis=1)[:, None]
    length = np.minimum(rng.exponential(mean_length_m, n), max_length_m)
    log_e = rng.uniform(math.log(kinetic_min_gev), math.log(kinetic_max_gev), n)
    kinetic = np.exp(log_e)
    gamma = 1.0 + kinetic / ELECTRON_MASS_GEV
    beta = np.sqrt(1.0 - 1.0 / (gamma * gamma))
    pid = np.where(rng.random(n) < electron_fraction, 11, -11).astype(np.int32)
    end = start + length[:, None] * direction
    t_start = -s / SPEED_OF_LIGHT + r * r / (2.0 * SPEED_OF_LIGHT * front_curvature_m)
    t_end = t_start + length / (beta * SPEED_OF_LIGHT)
    return dict(start=start, end=end, t_start=t_start, t_end=t_end, pid=pid,
                energy_gev=kinetic + ELECTRON_MASS_GEV, direction=direction,
                weight=np.full(n, weight))


def to_records(seg: dict, out: np.ndarray | None = None) -> np.ndarray:
    """Packs segment arrays into LeptonTransportRecord layout (752 B each)."""
    n = seg["start"].shape[0]
    rec = np.zeros(n, LEPTON_RECORD) if out is None else out
    rec["start"]["pid"] = seg["pid"]
    rec["end"]["pid"] = seg["pid"]
    rec["start"]["energy_gev"] = seg["energy_gev"]
    rec["end"]["energy_gev"] = seg["energy_gev"]
    rec["start"]["position_m"] = seg["start"]
    rec["end"]["position_m"] = seg["end"]
    rec["start"]["direction"] = seg["direction"]
    rec["end"]["direction"] = seg["direction"]
    rec["start"]["time_s"] = seg["t_start"]
    rec["end"]["time_s"] = seg["t_end"]
    rec["start"]["weight"] = seg["weight"]
    rec["end"]["weight"] = seg["weight"]
    return rec


def shower_records(n: int, seed: int, chunk: int = 1 << 20, **kw) -> np.ndarray:
    """LeptonTransportRecords of one synthetic shower, generated in seeded chunks."""
    out = np.zeros(n, LEPTON_RECORD)
    for k, begin in enumerate(range(0, n, chunk)):
        end = min(n, begin + chunk)
        seg = synthetic_segments(end - begin, seed * 1000003 + k, **kw)
        to_records(seg, out[begin:end])
    return out


# ---------------------------------------------------------------- workloads
def workload_config(name: str, **overrides):
    """(RadioConfig kwargs, record generator kwargs, segment count) of a named workload.

    "plain_c0":   1e5 segments, vertical, 16 antennas (8 arms x 50/150 m), 4096 bins at 0.1 ns
    "tiled_c1":   1e7 segments, zenith 30, 160 antennas (8 arms x 20 radii 25..500 m), 8192 bins
    "ice_c2":     5e6 segments in uniform n = 1.78, 64 antennas on/around the Cherenkov cone
    """
    ground = 1400.0
    model = AtmosphereModel()
    if name == "plain_c0":
        segments, zenith, radii, bins = 100_000, 0.0, [50.0, 150.0], 4096
    elif name == "tiled_c1":
        segments, zenith, radii, bins = 10_000_000, 30.0, list(np.linspace(25.0, 500.0, 20)), 8192
    elif name == "ice_c2":
        return _ice_workload(**overrides)
    else:
        raise KeyError(name)
    segments = overrides.pop("segments", segments)
    bins = overrides.pop("bins", bins)
    fs = 1e10
    observers = star_antennas(8, radii, ground, bins, fs, zenith_deg=zenith)
    table = flat_atmosphere_table(model, ground, 30000.0, 1.0)
    gen = dict(zenith_deg=zenith, ground_z_m=ground, model=model)
    return dict(observers=observers, table=table, homogeneous=0.0), gen, segments


def _ice_workload(segments: int = 5_000_000, bins: int = 4096, distance_m: float = 200.0):
    """Uniform n = 1.78 (ice-like), a 50 deg zenith cascade, 64 antennas: 16 azimuths x
    {theta_c - 0.5 deg, theta_c, theta_c + 0.5 deg} at `distance_m` from shower
    maximum plus 16 on the cone at twice that distance."""
    n_index = 1.78
    zenith = 50.0
    up, e1, e2 = shower_axis(zenith, 0.0)
    direction = -up
    rho = 0.92
    xmax_depth_m = 700.0 / (rho * 100.0)
    shower_max = np.array([0.0, 0.0, 0.0])
    theta_c = math.acos(1.0 / n_index)
    fs = 1e10
    obs = []
    for ring, (offset_deg, dist) in enumerate([(-0.5, distance_m), (0.0, distance_m),
                                               (0.5, distance_m), (0.0, 2 * distance_m)]):
        theta = theta_c + math.radians(offset_deg)
        for a in range(16):
            phi = 2.0 * math.pi * a / 16
            v = (math.cos(theta) * direction + math.sin(theta) *
                 (math.cos(phi) * e1 + math.sin(phi) * e2))
            pos = shower_max + dist * v
            arrival = n_index * dist / SPEED_OF_LIGHT
            obs.append((pos, arrival - 50e-9))
    observers = np.zeros(len(obs), OBSERVER)
    for k, (pos, start) in enumerate(obs):
        observers[k]["position_m"] = pos
        observers[k]["start_time_s"] = start
        observers[k]["duration_s"] = (bins - 1) / fs
        observers[k]["sample_rate_hz"] = fs
        observers[k]["number_of_bins"] = bins
    gen = dict(ice=True, zenith_deg=zenith, xmax_depth_m=xmax_depth_m, rho=rho)
    return dict(observers=observers, table=None, homogeneous=n_index), gen, segments


def ice_records(n: int, seed: int, zenith_deg: float = 50.0, xmax_depth_m: float = 7.6,
                rho: float = 0.92, lam_g_cm2: float = 70.0, lateral_scale_m: float = 0.1,
                angle_sigma_deg: float = 5.0, mean_length_m: float = 0.05,
                max_length_m: float = 0.5, **_) -> np.ndarray:
    """Segments of a cascade in uniform ice: Gaisser-Hillas in depth rho*s around
    the shower maximum at the origin, Moliere-scale lateral spread."""
    rng = np.random.Generator(np.random.PCG64(seed))
    up, e1, e2 = shower_axis(zenith_deg, 0.0)
    direction_axis = -up
    xmax = xmax_depth_m * rho * 100.0
    depth = _gaisser_hillas_depths(rng, n, xmax, lam_g_cm2, 4.0 * xmax)
    s = depth / (rho * 100.0) - xmax_depth_m  # metres along the axis relative to max
    r = rng.exponential(lateral_scale_m, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    start = (s[:, None] * direction_axis[None, :] + (r * np.cos(phi))[:, None] * e1[None, :] +
             (r * np.sin(phi))[:, None] * e2[None, :])
    sigma = math.radians(angle_sigma_deg)
    d = (direction_axis[None, :] + rng.normal(0, sigma, n)[:, None] * e1[None, :] +
         rng.normal(0, sigma, n)[:, None] * e2[None, :])
    d /= np.linalg.norm(d, axis=1)[:, None]
    length = np.minimum(rng.exponential(mean_length_m, n), max_length_m)
    kinetic = np.exp(rng.uniform(math.log(1e-3), math.log(1.0), n))
    gamma = 1.0 + kinetic / ELECTRON_MASS_GEV
    beta = np.sqrt(1.0 - 1.0 / (gamma * gamma))
    pid = np.where(rng.random(n) < 0.6, 11, -11).astype(np.int32)
    t_start = s / SPEED_OF_LIGHT
    seg = dict(start=start, end=start + length[:, None] * d, t_start=t_start,
               t_end=t_start + length / (beta * SPEED_OF_LIGHT), pid=pid,
               energy_gev=kinetic + ELECTRON_MASS_GEV, direction=d, weight=np.ones(n))
    return to_records(seg)


def make_config(workload: dict, precision: int = 0, kernel: int = 0, deterministic: bool = True,
                coreas: bool = True, zhs: bool = True, **extra):
    """RadioConfig of a workload dict from workload_config()."""
    from . import FlatAtmosphereSnapshot, RadioConfig

    if workload["homogeneous"] > 0:
        prop = FlatAtmosphereSnapshot(homogeneous_refractive_index=workload["homogeneous"])
    else:
        prop = FlatAtmosphereSnapshot(**workload["table"])
    obs = workload["observers"]
    return RadioConfig(enabled=True, coreas_enabled=coreas, zhs_enabled=zhs,
                       deterministic=deterministic, propagation=prop,
                       coreas_observers=obs if coreas else np.zeros(0, OBSERVER),
                       zhs_observers=obs if zhs else np.zeros(0, OBSERVER),
                       precision=precision, kernel=kernel, **extra)


# ---------------------------------------------------------------- many events
@dataclass
class EventSpec:
    """One shower of a batched or served workload."""

    seed: int
    segments: int
    antennas: int
    zenith_deg: float
    xmax: float
    bins: int = 4096


def batched_event_specs(events: int = 64, seed: int = 2024, min_segments: int = 100_000,
                        max_segments: int = 20_000_000, min_antennas: int = 16,
                        max_antennas: int = 300, bins: int = 4096) -> list:
    """Events of the batched workload: segment counts log-uniform in
    [min, max], antenna stars of 16..300 antennas (8 arms), zenith uniform in
    0..60 deg, Xmax uniform in 550..850 g/cm^2, all from one seed."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(events):
        segments = int(np.exp(rng.uniform(math.log(min_segments), math.log(max_segments))))
        antennas = int(rng.integers(min_antennas, max_antennas + 1))
        out.append(EventSpec(seed=seed * 7919 + k, segments=segments, antennas=antennas,
                             zenith_deg=float(rng.uniform(0.0, 60.0)),
                             xmax=float(rng.uniform(550.0, 850.0)), bins=bins))
    return out


def event_workload(spec: EventSpec, ground_z_m: float = 1400.0):
    """(workload dict, generator kwargs) of one event: a star of 8 arms with
    ceil(antennas/8) radii spread over 25..500 m (trimmed to `antennas`),
    4096-sample traces at 0.1 ns."""
    arms = 8
    radii = list(np.linspace(25.0, 500.0, max(1, -(-spec.antennas // arms))))
    observers = star_antennas(arms, radii, ground_z_m, spec.bins, 1e10,
                              zenith_deg=spec.zenith_deg)[: spec.antennas]
    model = AtmosphereModel()
    table = flat_atmosphere_table(model, ground_z_m, 30000.0, 1.0)
    gen = dict(zenith_deg=spec.zenith_deg, xmax=spec.xmax, ground_z_m=ground_z_m, model=model)
    return dict(observers=observers, table=table, homogeneous=0.0), gen


def served_event_specs(events: int = 40, seed: int = 4242, rate_hz: float = 20.0,
                       tail_fraction: float = 0.05, tail_segments: int = 50_000_000,
                       tail_antennas: int = 300, bins: int = 4096):
    """A served stream: batched-workload events with Poisson arrivals at
    `rate_hz` and a heavy tail (round(tail_fraction x events) events, at seeded
    positions, of tail_segments x tail_antennas).  Returns (specs, arrival
    times in s from the stream start)."""
    specs = batched_event_specs(events, seed=seed, bins=bins)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    for i in rng.choice(events, int(round(tail_fraction * events)), replace=False):
        specs[int(i)].segments = tail_segments
        specs[int(i)].antennas = tail_antennas
    arrivals = np.cumsum(rng.exponential(1.0 / rate_hz, events))
    arrivals -= arrivals[0]
    return specs, arrivals


LIBRARY_ZENITHS = (0.0, 15.0, 30.0, 45.0, 60.0)
LIBRARY_XMAX = (550.0, 700.0, 850.0)


def shower_library(segments: int = 500_000, seed: int = 9090, ground_z_m: float = 1400.0) -> dict:
    """Seeded showers for replayed streams, one per (zenith, Xmax) of
    LIBRARY_ZENITHS x LIBRARY_XMAX: {(zenith, xmax): records}.  An event
    replays the library shower nearest its zenith and Xmax, cycling through it
    when the event has more segments (as a track spool is replayed)."""
    model = AtmosphereModel()
    out = {}
    for i, zenith in enumerate(LIBRARY_ZENITHS):
        for j, xmax in enumerate(LIBRARY_XMAX):
            out[(zenith, xmax)] = shower_records(segments, seed=seed + 31 * i + j, zenith_deg=zenith,
                                                 xmax=xmax, ground_z_m=ground_z_m, model=model)
    return out


def library_key(spec: EventSpec):
    zenith = min(LIBRARY_ZENITHS, key=lambda z: abs(z - spec.zenith_deg))
    xmax = min(LIBRARY_XMAX, key=lambda x: abs(x - spec.xmax))
    return zenith, xmax


def replay_slices(total: int, library_size: int):
    """(offset, count) pieces that cycle through a library shower of
    library_size records until `total` records are covered."""
    out, done, offset = [], 0, 0
    while done < total:
        n = min(total - done, library_size - offset)
        out.append((offset, n))
        done += n
        offset = (offset + n) % library_size
    return out
