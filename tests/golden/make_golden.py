"""Writes tests/golden/reference_digests.json from the reference's own projection
code (oracle/_ref/libc8ref.so, built from the reference sources by oracle/Makefile).

For every case: the SHA-256 of the int64 fixed-point traces (CoREAS then ZHS,
little-endian, SoA order) and the integer counters.  The cases are the
reference's test inputs (tests/cases.py) and small seeded synthetic showers.
Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

import __graft_entry__ as entry  # noqa: E402

COUNTERS = ("coreas_contributions", "zhs_contributions", "zhs_subtracks", "valid_tracks",
            "fixed_point_overflows")


def digest(coreas, zhs) -> str:
    h = hashlib.sha256()
    h.update(coreas.astype("<i8").tobytes())
    h.update(zhs.astype("<i8").tobytes())
    return h.hexdigest()


def golden_cases():
    """Yields (label, config, records) in a fixed order."""
    import cases

    pkg = entry.load_package()
    from corsika8_kokkos_b200 import showers

    for name, config, record in cases.scalar_cases():
        for mode in (1, 2, 3):
            config.deterministic = True
            config.coreas_enabled = bool(mode & 1)
            config.zhs_enabled = bool(mode & 2)
            yield f"scalar/{name}/mode{mode}", config, record
    name, config, record = cases.scalar_cases()[0]
    for index in (1.0, 1.0003, 1.78):
        config.propagation.homogeneous_refractive_index = index
        config.zhs_subtrack_refinement = 3
        yield f"homogeneous/{index}/refine3", config, record
    for label, config, count in cases.accumulator_grid():
        if config.deterministic:
            yield f"accumulator/{label}", config, cases.accumulator_tracks(count)
    for workload, count in (("plain_c0", 3000), ("tiled_c1", 400), ("ice_c2", 2000)):
        wl, gen, _ = showers.workload_config(workload)
        if gen.get("ice"):
            records = showers.ice_records(count, seed=17, **gen)
        else:
            records = showers.shower_records(count, seed=17, **gen)
        yield f"shower/{workload}/{count}", showers.make_config(wl), records


def main():
    oracle = entry.load_oracle()
    if not oracle.reference_available():
        raise SystemExit("oracle/_ref/libc8ref.so is not built; run make -C oracle ref")
    out = {}
    for label, config, records in golden_cases():
        coreas, zhs, counters = oracle.reference().project(config, records, threads=1)
        out[label] = {"sha256": digest(coreas, zhs), **{k: int(counters[k]) for k in COUNTERS}}
    path = HERE / "reference_digests.json"
    path.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(out)} digests to {path}")


if __name__ == "__main__":
    main()
