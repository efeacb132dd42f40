"""The windowed launches' plan arithmetic on the host (no GPU): work lists
from append_work cover every track once in items no longer than the deferred
entries' offset field, and the deferred-list storage of one- and two-pass
launches (deferred_words / attach_deferred) keeps the first pass's lists, the
second pass's lists, the item states and the counter disjoint and inside the
allocation, with two passes only for fixed-point ZHS launches within the
storage cap.  tests/plan_check.cu, compiled for the host with nvcc."""
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "corsika8-kokkos_b200" / "csrc"


def test_launch_plans_stay_inside_their_storage(tmp_path):
    out = tmp_path / "plan_check"
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(CSRC), "-x", "cu", str(HERE / "plan_check.cu"), "-o", str(out)]
    built = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert built.returncode == 0, built.stderr
    run = subprocess.run([str(out)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stdout + run.stderr
