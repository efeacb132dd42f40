#!/usr/bin/env python
"""Radio hot-path benchmark: CoREAS endpoint field + ZHS vector potential of
every e+/e- track segment at every antenna, binned into traces, on B200.

Workload (default): 1e7 segments of one seeded synthetic shower at zenith 30 deg
x 160 antennas (8 arms x 20 radii, 25-500 m), 8192-sample traces at 0.1 ns,
CoREAS and ZHS fused: 1.6e9 track-antenna pairs per step.  A step is one
accumulateLeptonTracks over the whole batch (record ingest + projection).

One JSON line on rank 0:
  value       pairs/s of the production path (windowed, mixed precision) with
              the records resident in HBM, device time (CUDA events), max over ranks
  e2e         the same metric through the C ABI with host records: per step
              reset + enqueueHostLeptonTracks (pinned host -> device) + download
              (decoded traces device -> host)
  roofline    FP64 roofline of the projection kernel against the FP64 FMA rate
              measured on the same GPU in this run
  cpu_baseline  the reference's own projection code on the host cores
--impl reference times that CPU implementation alone on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from datetime import timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import __graft_entry__ as entry  # noqa: E402

# Algorithmic work per unit, counted from the reference's expressions
# (RadioProjection.inl): FP64 add/sub/mul plus division/sqrt, each one FLOP.
FLOP_COREAS_PAIR = 108 + 14   # two propagations, two Doppler factors, two fields, two samples
FLOP_ZHS_SETUP = 40 + 12      # Fraunhofer midpoint propagation and subdivision
FLOP_ZHS_SUBTRACK = 79 + 7    # one segment: propagation, detection times, potential
FLOP_SAMPLE = 12 + 3          # bin, gate and three fixed-point conversions
TRACK_RECORD_BYTES = 192      # kinematics record per track (with the precomputed source terms)
# algorithmic read per track per launch: the record fields each kernel's common path loads
TRACK_BYTES = {"coreas": 160, "zhs": 128}
L2_BYTES = 126 << 20          # B200 L2

WORKLOAD_NAME = "tiled_c1"


def parse_args():
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", default=WORKLOAD_NAME)
    p.add_argument("--segments", type=int, default=0, help="override the segment count")
    p.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    p.add_argument("--kernel", choices=["windowed", "direct"], default="windowed")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--e2e-batch", type=int, default=1 << 22,
                   help="host batch (records) of the end-to-end leg")
    p.add_argument("--no-baseline", action="store_true")
    p.add_argument("--no-variants", action="store_true",
                   help="skip the FP64 windowed and plain FP64 direct comparison runs")
    p.add_argument("--baseline-segments", type=int, default=100_000)
    p.add_argument("--no-serving", action="store_true", help="skip the served-stream leg")
    p.add_argument("--serve-events", type=int, default=40)
    p.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrivals per second")
    p.add_argument("--serve-budget-gb", type=float, default=120.0)
    p.add_argument("--serve-round-pairs", type=int, default=0,
                   help="server round size in track-observer pairs (0: the server's default)")
    p.add_argument("--serve-chunk", type=int, default=0,
                   help="server tracks per work item (0: the server's default)")
    p.add_argument("--library-segments", type=int, default=500_000,
                   help="segments of each of the 15 replayed library showers")
    p.add_argument("--batched", action="store_true",
                   help="print the batched workload (64 events, one graph-replayed launch per algorithm) instead")
    p.add_argument("--batch-events", type=int, default=64)
    p.add_argument("--no-batched", action="store_true", help="skip the batched leg of the default run")
    p.add_argument("--tuning-cache", default=str(Path(tempfile.gettempdir()) / "c8radio-b200.tuning"),
                   help="tuning cache file the batched leg reads and, after autotuning, writes")
    p.add_argument("--precision-study", action="store_true",
                   help="print the arrival-time precision study of the ice workload instead")
    p.add_argument("--plain-fraction", type=int, default=8,
                   help="the plain event-by-event comparison projects 1/N of every event's segments")
    return p.parse_args()


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ workload
def build_workload(name: str, segments: int, seed: int):
    pkg = entry.load_package()
    from corsika8_kokkos_b200 import showers

    wl, gen, default_n = showers.workload_config(name)
    n = segments or default_n
    if gen.get("ice"):
        records = showers.ice_records(n, seed=seed, **gen)
    else:
        records = showers.shower_records(n, seed=seed, **gen)
    return pkg, showers, wl, records


def hbm_peak_gbs():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return json.loads(path.read_text()).get("hbm_gbs")
    return 6650.0  # fallback figure for this pool's B200s


def algorithmic_flops(pairs: int, counters: dict) -> float:
    return (pairs * (FLOP_COREAS_PAIR + FLOP_ZHS_SETUP) +
            counters["zhs_subtracks"] * FLOP_ZHS_SUBTRACK +
            (counters["coreas_contributions"] + counters["zhs_contributions"]) * FLOP_SAMPLE)


# ------------------------------------------------------------------ reference arm
def cpu_reference_rate(wl, records, showers, threads: int, steps: int = 1, warmup: int = 0):
    """Times the reference's own projection code (oracle/_ref) on the host cores,
    or the C restatement of it when the reference library is not built."""
    oracle = entry.load_oracle()
    kind = "reference" if oracle.reference_available() else "port"
    backend = oracle.reference() if kind == "reference" else oracle.restatement()
    config = showers.make_config(wl)
    pairs = records.size * len(wl["observers"])
    for _ in range(warmup):
        backend.project(config, records, threads=threads)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        backend.project(config, records, threads=threads)
        times.append(time.perf_counter() - t0)
    return pairs, times, kind


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    n = args.baseline_segments
    pkg, showers, wl, records = build_workload(args.workload, n, seed=1000)
    threads = os.cpu_count() or 1
    pairs, times, kind = cpu_reference_rate(wl, records, showers, threads, args.steps, args.warmup)
    seconds = sum(times) / len(times)
    value = pairs / seconds
    sample = (f"{n} of the workload's segments x {len(wl['observers'])} antennas "
              f"({pairs:.3g} pairs) per step, fixed-point CoREAS+ZHS")
    line = {
        "impl": "reference", "metric": "track-antenna pairs/s", "value": value,
        "unit": "pairs/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": seconds * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded shower generator)",
        "config": {"workload": args.workload, "segments": n,
                   "antennas": int(len(wl["observers"])),
                   "bins": int(wl["observers"]["number_of_bins"][0])},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def run_ours(args):
    rank, world, local = env_rank()
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    pkg, showers, wl, records = build_workload(args.workload, args.segments, seed=1000 + rank)
    from corsika8_kokkos_b200.sharding import max_over_ranks
    n = records.size
    observers = len(wl["observers"])
    pairs_per_step = n * observers
    device_records = torch.from_numpy(records.view(np.uint8).reshape(-1)).cuda()
    stream = torch.cuda.current_stream()
    precision = {"mixed": 1, "fp64": 0}[args.precision]
    kernel = {"windowed": 2, "direct": 1}[args.kernel]
    peaks = pkg.probe_peaks()

    # inputs smaller than twice the 126 MB L2: each step is timed alone, with a
    # 512 MB buffer written between steps (outside the timed windows)
    input_bytes = records.nbytes + n * TRACK_RECORD_BYTES
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda") if input_bytes < 2 * L2_BYTES else None

    def timed_run(precision, kernel, steps, warmup, timing=True):
        config = showers.make_config(wl, precision=precision, kernel=kernel)
        acc = pkg.RadioAccumulator(config, stream=stream.cuda_stream)
        ptr = device_records.data_ptr()
        for _ in range(warmup):
            acc.accumulate_lepton_tracks(ptr, n)
        acc.reset()
        acc.set_kernel_timing(timing)
        barrier()
        torch.cuda.synchronize()
        marks = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                 for _ in range(steps if flush is not None else 1)]
        with ClockSampler(local) as clocks:
            if flush is None:
                marks[0][0].record(stream)
                for _ in range(steps):
                    acc.accumulate_lepton_tracks(ptr, n)
                marks[0][1].record(stream)
            else:
                for start, end in marks:
                    flush.fill_(1)
                    start.record(stream)
                    acc.accumulate_lepton_tracks(ptr, n)
                    end.record(stream)
            torch.cuda.synchronize()
        barrier()
        ms = sum(start.elapsed_time(end) for start, end in marks) / steps
        stats = acc.statistics()
        kernel_ms = stats.kernel_time_ms / max(stats.timed_launches, 1)
        counters = acc.download().counters
        acc.close()
        return ms, kernel_ms, counters, clocks.summary(), stats

    ms, kernel_ms, counters, clocks, stats = timed_run(precision, kernel, args.steps, args.warmup)
    ms_max = max_over_ranks(ms)
    value = world * pairs_per_step / (ms_max * 1e-3)

    variants = {}
    if not args.no_variants and world == 1:
        # the FP64 windowed drop-in over the same steps as `value`; the two plain
        # FP64 shapes of the reference (one thread per pair: the direct shape it
        # uses below 16384 tracks, and its 8 x 32 tile shape above) over at most 5
        # steps each (about 1.2 s a step)
        plain_steps = min(args.steps, 5)
        for label, prec, kern, steps, warm in (("fp64_windowed", 0, 2, args.steps, args.warmup),
                                               ("fp64_direct_plain", 0, 1, plain_steps, 1),
                                               ("fp64_tiled_plain", 0, 3, plain_steps, 1)):
            if prec == precision and kern == kernel:
                continue
            vms, vkms, vcounters, vclocks, _ = timed_run(prec, kern, steps, warm)
            variants[label] = {"pairs_per_s": pairs_per_step / (vms * 1e-3), "ms_per_step": vms,
                               "kernel_ms": vkms, "steps": steps, "clocks_sm_mhz": vclocks.get("sm_mhz")}
        plain = [variants[k] for k in ("fp64_direct_plain", "fp64_tiled_plain") if k in variants]
        if plain:
            best = max(plain, key=lambda v: v["pairs_per_s"])
            variants["plain_best"] = {
                "kernel": "direct" if best is variants.get("fp64_direct_plain") else "tiled",
                "pairs_per_s": best["pairs_per_s"], "value_over_plain": value / best["pairs_per_s"]}

    # accuracy of the timed path: one accumulate of the same records in the
    # timed precision and in FP64 (the windowed FP64 path, bit-exact against
    # the oracle in the full-size parity test), fixed-point traces compared per
    # antenna trace
    accuracy = None
    if not args.no_variants and world == 1 and precision != 0:
        accuracy = trace_accuracy(pkg, showers, wl, device_records, n, precision, kernel, stream)

    # roofline of the dominant kernel (the windowed ZHS launch, two thirds of a
    # step) and of the CoREAS launch, from events on their launch stream
    per = {k: counters[k] / args.steps for k in ("zhs_subtracks", "coreas_contributions",
                                                  "zhs_contributions")}
    zhs_flops = (pairs_per_step * FLOP_ZHS_SETUP + per["zhs_subtracks"] * FLOP_ZHS_SUBTRACK +
                 per["zhs_contributions"] * FLOP_SAMPLE)
    coreas_flops = pairs_per_step * FLOP_COREAS_PAIR + per["coreas_contributions"] * FLOP_SAMPLE
    zhs_ms = stats.zhs_kernel_time_ms / args.steps
    coreas_ms = stats.coreas_kernel_time_ms / args.steps
    peak = peaks["fp64_flops"] / 1e12
    traffic, instructions = {}, {}
    traffic_file = ROOT / "profiles" / "windowed_traffic.json"
    if traffic_file.exists():
        t = json.loads(traffic_file.read_text())
        traffic = {"zhs": t["zhs_bytes_per_track"] * n, "coreas": t["coreas_bytes_per_track"] * n}
        instructions = {k: t.get(f"{k}_warp_instructions_per_pair") for k in ("zhs", "coreas")}
    # issue roofline: 4 warp instructions per clock per SM (one per scheduler)
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    issue_peak = 4 * sms * (clocks.get("sm_mhz") or 0) * 1e6

    def issue(key, ms):
        per_pair = instructions.get(key)
        if not per_pair or not ms or not issue_peak:
            return None
        achieved = per_pair * pairs_per_step / (ms * 1e-3)
        return {"warp_instructions_per_pair": per_pair, "achieved_per_s": achieved,
                "peak_per_s": issue_peak, "frac": achieved / issue_peak,
                "source": "warp instructions per pair from an ncu capture of the same kernel on a "
                          "1e6-track case of this workload; peak = 4 x SMs x the SM clock sampled "
                          "during the timed steps"}

    def roof(flops, ms, key):
        achieved = flops / (ms * 1e-3) / 1e12 if ms > 0 else None
        return {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if achieved and peak else None,
                "traffic": traffic.get(key), "kernel_ms": ms, "flop_per_launch": flops,
                "bytes_per_launch_algorithmic": TRACK_BYTES[key] * n}

    roofline = roof(zhs_flops, zhs_ms, "zhs")
    roofline.update({
        "kernel": "windowed_kernel<fixed,float,ZHS> (dominant, 62% of the step)",
        "peak_source": "FP64 FMA stream measured in this run on this GPU (c8r_probe_peaks); "
                       "of measured",
        "traffic_source": ("DRAM bytes read + written per track from an ncu capture of the same "
                           "kernel on a 1e6-track case of this workload, scaled to this launch's tracks"),
        "hbm": {"bytes_per_launch": traffic.get("zhs"),
                "achieved_gbs": (traffic.get("zhs") or 0) / (zhs_ms * 1e-3) / 1e9 if zhs_ms else None,
                "peak_gbs": hbm_peak_gbs()},
        "issue": issue("zhs", zhs_ms),
        "secondary": dict(roof(coreas_flops, coreas_ms, "coreas"),
                          kernel="windowed_kernel<fixed,float,CoREAS>", issue=issue("coreas", coreas_ms)),
        "atomics": {"shared_per_s_peak": peaks["shared_atomics_per_s"],
                    "global_per_s_peak": peaks["global_atomics_per_s"],
                    "samples_per_s": (per["coreas_contributions"] + per["zhs_contributions"]) /
                                     ((zhs_ms + coreas_ms) * 1e-3) if zhs_ms + coreas_ms else None},
    })

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(pkg, showers, wl, records, precision, kernel, stream, args, torch, barrier,
                      max_over_ranks, world)

    # the served stream runs before the CPU baseline: its latencies depend on the
    # host threads that feed it, which the baseline's worker threads would crowd
    serving = batched = None
    if rank == 0 and world == 1 and not (args.no_serving and args.no_batched):
        del device_records
        torch.cuda.empty_cache()
        library = showers.shower_library(args.library_segments)
        dev = {k: torch.from_numpy(v.view(np.uint8).reshape(-1)).cuda() for k, v in library.items()}
        if not args.no_serving:
            serving = run_serving(pkg, showers, torch, args, local, library, dev)
        if not args.no_batched:
            batched = batched_leg(pkg, showers, torch, args, library, dev, steps=3, warmup=1)
        del dev
        torch.cuda.empty_cache()

    baseline = None
    if rank == 0 and world == 1 and not args.no_baseline:
        sample = records[: args.baseline_segments]
        threads = os.cpu_count() or 1
        bpairs, btimes, kind = cpu_reference_rate(wl, sample, showers, threads, 1, 0)
        baseline = {"value": bpairs / btimes[0], "unit": "pairs/s", "cores": threads, "kind": kind,
                    "sample": f"first {sample.size} of {n} segments x {observers} antennas "
                              f"({bpairs:.3g} pairs), fixed-point CoREAS+ZHS, one pass"}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "track-antenna pairs/s", "value": value, "unit": "pairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 times / f32 amplitudes" if precision == 1 else "f64",
        "data": "synthetic (seeded shower generator, one shower per GPU)",
        "config": {"workload": args.workload, "segments": n, "antennas": observers,
                   "bins": int(wl["observers"]["number_of_bins"][0]),
                   "algorithms": "CoREAS+ZHS fused", "precision": args.precision,
                   "kernel": args.kernel, "pairs_per_step": pairs_per_step,
                   "l2": (f"inputs larger than L2 ({records.nbytes / 1e9:.2f} GB records, "
                          f"{n * TRACK_RECORD_BYTES / 1e9:.2f} GB kinematics)") if flush is None else
                         (f"L2 flushed between steps (512 MB written; inputs "
                          f"{input_bytes / 1e6:.0f} MB), steps timed alone")},
        "e2e": e2e, "roofline": roofline, "cpu_baseline": baseline,
        "clocks": clocks, "gpu_launches": 3 * args.steps,
        "counters": {k: counters[k] for k in ("valid_tracks", "coreas_contributions",
                                              "zhs_contributions", "zhs_subtracks",
                                              "fixed_point_overflows")},
        "variants": variants, "accuracy": accuracy, "peaks": peaks, "serving": serving,
        "batched": batched,
    }
    print(json.dumps(line), flush=True)


def trace_errors(got, want, observers):
    """Per antenna trace: relative L2 error and relative error of the peak
    |field| (vector magnitude over the three components) of `got` against
    `want`, both (3, total bins) fixed-point traces of one algorithm (a
    trace's decode factor is common to its bins, so the ratios need none)."""
    l2, peak = [], []
    offset = 0
    for n in observers["number_of_bins"]:
        n = int(n)
        g = got[:, offset:offset + n].astype(np.float64)
        w = want[:, offset:offset + n].astype(np.float64)
        offset += n
        norm = np.linalg.norm(w)
        if norm == 0:
            continue
        l2.append(np.linalg.norm(g - w) / norm)
        gp, wp = np.sqrt((g * g).sum(axis=0)).max(), np.sqrt((w * w).sum(axis=0)).max()
        peak.append(abs(gp - wp) / wp)
    return np.array(l2), np.array(peak)


def trace_accuracy(pkg, showers, wl, device_records, n, precision, kernel, stream):
    """Max and median per-trace relative L2 error and max peak-amplitude error
    of the timed precision against FP64 on the same records, CoREAS and ZHS."""
    traces = {}
    for label, prec in (("timed", precision), ("fp64", 0)):
        acc = pkg.RadioAccumulator(showers.make_config(wl, precision=prec, kernel=kernel),
                                   stream=stream.cuda_stream)
        acc.accumulate_lepton_tracks(device_records.data_ptr(), n)
        traces[label] = acc.download_fixed()
        acc.close()
    out = {"reference": "FP64 windowed traces of the same records (bit-exact against the oracle)"}
    worst = 0.0
    for a, name in ((0, "coreas"), (1, "zhs")):
        l2, peak = trace_errors(traces["timed"][a], traces["fp64"][a], wl["observers"])
        out[name] = {"traces": int(l2.size), "max_rel_l2": float(l2.max()), "median_rel_l2": float(np.median(l2)),
                     "max_peak_error": float(peak.max())}
        worst = max(worst, float(l2.max()))
    out["max_rel_l2_per_trace"] = worst
    out["counters_equal"] = all(traces["timed"][2][k] == traces["fp64"][2][k] for k in
                                ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks"))
    return out


# ------------------------------------------------------------------ served stream
def run_serving(pkg, showers, torch, args, local: int, library: dict, dev: dict) -> dict:
    """The served form: a Poisson stream of batched-workload events with a heavy
    tail, each event opened on a RadioServer at its arrival time by its own
    producer thread, its segments added as device records (replayed from a
    device-resident library of seeded showers), then waited for and fetched
    (fixed-point traces to host).  Latency = fetch return - scheduled arrival;
    throughput = all pairs / (last fetch - first arrival).  The stream runs
    twice: at the workload's rate (20/s, about three times what one GPU
    sustains, so its latencies are those of a queue that grows) and with the
    same events at a rate below the capacity the first run measured (0.6 of
    it: the stable regime, whose latencies are the service times).  Beside
    them, the plain FP64 drop-in (direct kernel, one accumulator per event,
    event by event) on 1/plain_fraction of every event's segments, and the
    served traces' error against the oracle on the smallest events."""
    specs, arrivals = showers.served_event_specs(events=args.serve_events, rate_hz=args.serve_rate)
    size = args.library_segments
    itemsize = next(iter(library.values())).itemsize
    configs = [showers.make_config(showers.event_workload(spec)[0], precision=1, kernel=2)
               for spec in specs]
    torch.cuda.synchronize()
    small = sorted(range(len(specs)), key=lambda k: specs[k].segments * specs[k].antennas)[:3]
    pairs = [s.segments * s.antennas for s in specs]

    overloaded, kept = serve_stream(pkg, showers, torch, args, local, specs, arrivals, configs, dev,
                                    itemsize, size, keep=small)
    stable_rate = 0.6 * overloaded["pairs_per_s"] / (sum(pairs) / len(pairs))
    stable, _ = serve_stream(pkg, showers, torch, args, local, specs, arrivals * (args.serve_rate / stable_rate),
                             configs, dev, itemsize, size, keep=())

    # plain FP64 drop-in, event by event, on a fixed fraction of each event, in
    # both of the reference's launch shapes; the comparison takes the faster
    stream = torch.cuda.current_stream()
    plain_rates = {}
    for shape, kernel in (("direct", 1), ("tiled", 3)):
        plain_pairs, plain_seconds = 0, 0.0
        for k, spec in enumerate(specs):
            count = max(1, spec.segments // args.plain_fraction)
            wl, _ = showers.event_workload(spec)
            acc = pkg.RadioAccumulator(showers.make_config(wl, precision=0, kernel=kernel),
                                       stream=stream.cuda_stream)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            base = dev[showers.library_key(spec)].data_ptr()
            for offset, n in showers.replay_slices(count, size):
                acc.accumulate_lepton_tracks(base + offset * itemsize, n)
            acc.download_fixed()
            plain_seconds += time.perf_counter() - t0
            plain_pairs += count * spec.antennas
            acc.close()
        plain_rates[shape] = plain_pairs / plain_seconds
    plain_shape = max(plain_rates, key=plain_rates.get)
    plain = plain_rates[plain_shape]

    # served (mixed precision) traces against the oracle -- the reference's FP64
    # arithmetic on the host, as the checker -- per antenna trace, on the
    # smallest events (their records rebuilt from the replayed library slices)
    worst, worst_peak = 0.0, 0.0
    traces = 0
    checker = entry.load_oracle().restatement()
    for k in small:
        wl, _ = showers.event_workload(specs[k])
        host = library[showers.library_key(specs[k])]
        records = np.concatenate([host[offset:offset + n]
                                  for offset, n in showers.replay_slices(specs[k].segments, size)])
        want = checker.project(showers.make_config(wl), records, threads=os.cpu_count() or 1)
        for got, ref in zip(kept[k], want[:2]):
            l2, peak = trace_errors(got.reshape(3, -1), ref, wl["observers"])
            traces += int(l2.size)
            if l2.size:
                worst = max(worst, float(l2.max()))
                worst_peak = max(worst_peak, float(peak.max()))
    tail = sum(1 for s in specs if s.segments == max(x.segments for x in specs))
    stable["rate_hz"] = stable_rate
    stable["rate_source"] = "0.6 x the first run's sustained pairs/s / mean pairs per event"
    return dict(overloaded, **{
        "workload": (f"served_c4: {len(specs)} events, Poisson {args.serve_rate:g}/s, segments "
                     f"log-uniform 1e5-2e7, 16-300 antennas, zenith 0-60, Xmax 550-850, "
                     f"{tail} tail events of 5e7 x 300, 4096 bins, CoREAS+ZHS, mixed precision, "
                     f"fixed point"),
        "inputs": (f"device-resident replay of 15 seeded library showers ({size} segments each, "
                   f"nearest zenith/Xmax), added by one producer thread per event"),
        "budget_gb": args.serve_budget_gb, "events": len(specs), "pairs": int(sum(pairs)),
        "offered_pairs_per_s": sum(pairs) / max(float(arrivals[-1]), 1e-9),
        "plain_event_by_event": {
            "pairs_per_s": plain, "shape": plain_shape,
            "pairs_per_s_by_shape": plain_rates,
            "sample": (f"every event of the stream, first 1/{args.plain_fraction} of its segments, "
                       f"FP64, the reference's direct and tiled launch shapes (the faster taken), one "
                       f"accumulator per event (accumulate + download_fixed)")},
        "served_vs_plain": overloaded["pairs_per_s"] / plain,
        "accuracy_vs_oracle": {"max_rel_l2_per_trace": worst, "max_peak_error": worst_peak,
                               "traces": traces, "events": "the 3 smallest events of the stream",
                               "reference": "the oracle (FP64 CPU restatement of the reference's "
                                            "projection) on the same records"},
        "stable": stable,
    })


def serve_stream(pkg, showers, torch, args, local, specs, arrivals, configs, dev, itemsize, size, keep):
    """One served stream on a fresh RadioServer: returns (summary, {event: fixed
    traces} for the events in `keep`)."""
    import threading

    server = pkg.RadioServer(budget_bytes=int(args.serve_budget_gb * 1e9), round_pairs=args.serve_round_pairs,
                             chunk_tracks=args.serve_chunk)

    def feed(event, spec, count, stream):
        base = dev[showers.library_key(spec)].data_ptr()
        for offset, n in showers.replay_slices(count, size):
            server.add_device(event, base + offset * itemsize, n, stream=stream)

    # warm-up: one small event (module loads, occupancy queries)
    warm = server.open(configs[0])
    feed(warm, specs[0], min(specs[0].segments, 100_000), 0)
    server.close_event(warm)
    server.fetch_fixed(warm)

    results = [None] * len(specs)
    kept = {}
    errors = []
    start = time.perf_counter() + 0.1

    def handle(k):
        try:
            torch.cuda.set_device(local)
            stream = torch.cuda.Stream()
            delay = start + arrivals[k] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            event = server.open(configs[k])
            feed(event, specs[k], specs[k].segments, stream.cuda_stream)
            server.close_event(event)
            server.wait(event)
            coreas, zhs, counters, info = server.fetch_fixed(event)
            done = time.perf_counter()
            results[k] = {"latency": done - (start + arrivals[k]), "done": done, "info": info,
                          "overflows": counters["fixed_point_overflows"]}
            if k in keep:
                kept[k] = (coreas, zhs)
        except Exception as exc:  # reported below
            errors.append(f"event {k}: {exc!r}")

    threads = [threading.Thread(target=handle, args=(k,)) for k in range(len(specs))]
    with ClockSampler(local) as clocks:
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    stats = server.stats()
    server.close()
    if errors:
        raise RuntimeError("; ".join(errors))
    pairs = [s.segments * s.antennas for s in specs]
    latency = np.array([r["latency"] for r in results])
    makespan = max(r["done"] for r in results) - start
    tail = [k for k, s in enumerate(specs) if s.segments == max(x.segments for x in specs)]
    others = np.array([latency[k] for k in range(len(specs)) if k not in tail])
    pct = lambda a, q: float(np.percentile(a, q))  # noqa: E731
    return {
        "makespan_s": makespan, "pairs_per_s": sum(pairs) / makespan,
        "offered_pairs_per_s": sum(pairs) / max(float(arrivals[-1]), 1e-9),
        "latency_s": {"p50": pct(latency, 50), "p95": pct(latency, 95), "p99": pct(latency, 99),
                      "max": float(latency.max())},
        "latency_non_tail_s": {"p50": pct(others, 50), "p95": pct(others, 95), "p99": pct(others, 99)},
        "rounds": stats["rounds"], "launches": stats["launches"],
        "arena_peak_gb": stats["arena_peak_bytes"] / 1e9,
        "fixed_point_overflows": int(sum(r["overflows"] for r in results)),
        "clocks": clocks.summary(),
    }, kept


# ------------------------------------------------------------------ batched
def run_batched(args):
    """--batched: the batched workload alone, one JSON line."""
    import torch

    pkg = entry.load_package()
    from corsika8_kokkos_b200 import showers

    library = showers.shower_library(args.library_segments)
    dev = {k: torch.from_numpy(v.view(np.uint8).reshape(-1)).cuda() for k, v in library.items()}
    out = batched_leg(pkg, showers, torch, args, library, dev, steps=args.steps, warmup=args.warmup)
    print(json.dumps(dict(out, metric="track-antenna pairs/s", unit="pairs/s")), flush=True)


def batched_leg(pkg, showers, torch, args, library, dev, steps: int, warmup: int) -> dict:
    """Batched workload: `batch_events` events (segments log-uniform 1e5-2e7,
    16-300 antennas, zenith 0-60 deg, Xmax 550-850 g/cm^2, 4096 bins), each
    staged into its own accumulator (mixed precision) from a device-resident
    library of seeded showers, then projected together by one persistent launch
    per algorithm, replayed from a captured CUDA graph.  The tile (track
    segments per stage = threads per CTA, tracks per work item, bin window; one
    antenna per CTA) comes from the tuning cache when it holds one for this
    device, build and workload, else from the autotuner on the first eighth of
    the events, which is then stored.  Timed: `steps` graph replays, CUDA
    events."""
    specs = showers.batched_event_specs(events=args.batch_events)
    size = args.library_segments
    itemsize = next(iter(library.values())).itemsize
    stream = torch.cuda.Stream()
    events = []
    for spec in specs:
        wl, _ = showers.event_workload(spec)
        acc = pkg.RadioAccumulator(showers.make_config(wl, precision=1, kernel=2),
                                   stream=stream.cuda_stream)
        acc.reserve_track_capacity(spec.segments)
        base = dev[showers.library_key(spec)].data_ptr()
        for offset, n in showers.replay_slices(spec.segments, size):
            acc.stage_lepton_tracks(base + offset * itemsize, n)
        events.append(acc)
    stream.synchronize()
    pairs = sum(s.segments * s.antennas for s in specs)
    batch = pkg.RadioBatch(stream=stream.cuda_stream)
    label = (f"batched_c3 events={len(specs)} bins=4096 precision=mixed library={size} "
             f"segments={sum(s.segments for s in specs)}")
    cache = Path(args.tuning_cache)
    best = pkg.tuning_cache_load(cache, label)
    source, tune_ms, tuned_events = "tuning cache", None, 0
    if best is None:
        tune = events[: max(1, len(events) // 8)]
        best, tune_ms = batch.autotune(tune, repetitions=1)
        pkg.tuning_cache_store(cache, label, best)
        reloaded = pkg.tuning_cache_load(cache, label, require=True)
        assert (reloaded.team_size, reloaded.track_tile_size, reloaded.observer_tile_size) == \
            (best.team_size, best.track_tile_size, best.observer_tile_size)
        source, tuned_events = "autotuner (stored in the tuning cache)", len(tune)
    for acc in events:
        acc.set_tuning(best)
    for _ in range(max(1, warmup)):
        batch.project(events, graph=True, keep_staged=True)
    stream.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clocks:
        start.record(stream)
        for _ in range(steps):
            batch.project(events, graph=True, keep_staged=True)
        end.record(stream)
        stream.synchronize()
    ms = start.elapsed_time(end) / steps
    captures = batch.graph_captures()
    batch.close()
    for acc in events:
        acc.close()
    torch.cuda.empty_cache()
    return {
        "value": pairs / (ms * 1e-3),
        "workload": f"batched_c3: {len(specs)} events, segments log-uniform 1e5-2e7, 16-300 antennas, "
                    f"zenith 0-60, Xmax 550-850, 4096 bins, CoREAS+ZHS, mixed precision, fixed point",
        "inputs": f"device-resident replay of 15 seeded library showers ({size} segments each), staged",
        "events": len(specs), "segments": int(sum(s.segments for s in specs)), "pairs_per_step": int(pairs),
        "steps": steps, "ms_per_step": ms, "launches_per_step": 2, "graph_captures": int(captures),
        "tile": {"segments_per_stage": best.team_size or 640, "antennas_per_cta": 1,
                 "bin_window": best.observer_tile_size or 4096,
                 "tracks_per_item": best.track_tile_size or "auto (about 16 items per CTA)"},
        "tuning": {"source": source, "autotune_ms_per_projection": tune_ms, "autotune_events": tuned_events,
                   "workload_label": label},
        "clocks": clocks.summary(),
    }


# ------------------------------------------------------------------ precision study
STUDY_MODES = (("fp64", 0, 2), ("mixed", 1, 2), ("study_fp64", 4, 0), ("double_fp32", 2, 0),
               ("fp32", 3, 0))


def run_precision_study(args):
    """The ice workload (uniform n = 1.78, antennas on and +-0.5 deg around the
    Cherenkov cone) with its arrival times, distances, directions and Cherenkov
    denominators in FP64 (the reference's arithmetic), the mixed production
    path, and the generic study kernel in FP64, compensated double-FP32 and
    FP32.  Per mode: samples whose bin differs from FP64 (from sample-count
    traces), per-trace relative L2 and peak-amplitude error of the decoded
    traces against FP64, and pairs/s."""
    import torch

    pkg, showers, wl, records = build_workload("ice_c2", args.segments, seed=2000)
    raw = torch.from_numpy(records.view(np.uint8).reshape(-1)).cuda()
    observers = wl["observers"]
    bins = int(observers["number_of_bins"][0])
    pairs = records.size * len(observers)

    def project(precision, kernel, count_samples, timed=False):
        config = showers.make_config(wl, precision=precision, kernel=kernel, count_samples=count_samples)
        acc = pkg.RadioAccumulator(config)
        if timed:
            acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
            acc.reset()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
        torch.cuda.synchronize()
        seconds = time.perf_counter() - t0
        out = acc.download_fixed() if count_samples else acc.download()
        acc.close()
        return out, seconds

    reference_counts = None
    reference = None
    rows = {}
    for name, precision, kernel in STUDY_MODES:
        (counts_c, counts_z, counters), _ = project(precision, kernel, True)
        waveforms, seconds = project(precision, kernel, False, timed=True)
        if reference_counts is None:
            reference_counts = (counts_c, counts_z, counters)
            reference = waveforms
        row = {"pairs_per_s": pairs / seconds, "kernel": "windowed" if kernel == 2 else "study"}
        for label, got, want, key in (("coreas", counts_c, reference_counts[0], "coreas_contributions"),
                                      ("zhs", counts_z, reference_counts[1], "zhs_contributions")):
            moved = int(np.abs(got[0] - want[0]).sum()) // 2 + abs(int(got[0].sum()) - int(want[0].sum())) // 2
            row[f"{label}_samples"] = int(counters[key])
            row[f"{label}_samples_in_other_bins"] = moved
            row[f"{label}_bin_agreement"] = 1.0 - moved / max(int(want[0].sum()), 1)
        for label, got, want in (("coreas", waveforms.coreas, reference.coreas),
                                 ("zhs", waveforms.zhs, reference.zhs)):
            g = got.reshape(3, -1, bins)
            w = want.reshape(3, -1, bins)
            norm = np.sqrt((w ** 2).sum(axis=(0, 2)))
            ok = norm > 0
            rel = np.sqrt(((g - w) ** 2).sum(axis=(0, 2)))[ok] / norm[ok]
            gp = np.abs(g).max(axis=(0, 2))[ok]
            wp = np.abs(w).max(axis=(0, 2))[ok]
            row[f"{label}_max_rel_l2"] = float(rel.max()) if rel.size else 0.0
            row[f"{label}_median_rel_l2"] = float(np.median(rel)) if rel.size else 0.0
            row[f"{label}_max_peak_error"] = float((np.abs(gp - wp) / wp).max()) if rel.size else 0.0
        rows[name] = row
        print(f"# {name}: {json.dumps(row)}", file=sys.stderr, flush=True)
    print(json.dumps({"study": "arrival-time precision", "workload": "ice_c2",
                      "segments": int(records.size), "antennas": int(len(observers)), "bins": bins,
                      "pairs": pairs, "reference_mode": "fp64 (windowed, the reference's arithmetic)",
                      "modes": rows}), flush=True)


def run_e2e(pkg, showers, wl, records, precision, kernel, stream, args, torch, barrier,
            max_over_ranks, world):
    """reset + enqueueHostLeptonTracks(pinned host records) + download(pinned traces).
    The library uploads the span of each record the ingest reads (208 of 752
    bytes) with a pitched copy.

    Host batches of up to 2^22 records (--e2e-batch): each copy hides behind
    the previous batch's projection; the library starts at 1/32 of that and
    doubles each batch, so the first projection waits for a short copy only."""
    config = showers.make_config(wl, precision=precision, kernel=kernel)
    tuning = pkg.TuningParameters(batch_size=args.e2e_batch)
    acc = pkg.RadioAccumulator(config, tuning, stream=stream.cuda_stream)
    cudart = torch.cuda.cudart()
    registered = cudart.cudaHostRegister(records.ctypes.data, records.nbytes, 0) == 0
    out_c = torch.empty(3 * acc.coreas_bins, dtype=torch.float64, pin_memory=True).numpy()
    out_z = torch.empty(3 * acc.zhs_bins, dtype=torch.float64, pin_memory=True).numpy()
    for _ in range(max(1, args.warmup)):
        acc.reset()
        acc.enqueue_host_lepton_tracks(records)
        acc.download_into(out_c, out_z)
    barrier()
    steps = max(1, args.steps)
    t0 = time.perf_counter()
    for _ in range(steps):
        acc.reset()
        acc.enqueue_host_lepton_tracks(records)
        acc.download_into(out_c, out_z)
    seconds = (time.perf_counter() - t0) / steps
    seconds = max_over_ranks(seconds)
    # the last step's uploaded bytes (reset clears the statistics): the used
    # 208-byte span of each 752-byte record
    h2d = int(acc.statistics().host_to_device_bytes)
    acc.close()
    if registered:
        cudart.cudaHostUnregister(records.ctypes.data)
    pairs = records.size * len(wl["observers"])
    return {"value": world * pairs / seconds, "unit": "pairs/s",
            "h2d_bytes_per_step": h2d, "host_record_bytes_per_step": int(records.nbytes),
            "d2h_bytes_per_step": int(out_c.nbytes + out_z.nbytes),
            "ms_per_step": seconds * 1e3, "steps": steps, "pinned_input": bool(registered)}


def main():
    args = parse_args()
    if args.precision_study:
        run_precision_study(args)
    elif args.batched:
        run_batched(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
