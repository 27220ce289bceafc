"""bench.py's multi-rank launch on the CPU: `--gpus 2` outside a torchrun environment
re-launches the script as two local ranks, which meet on the gloo backend
(`--dist-check` does no GPU work), and rank 0 prints one JSON line with n_gpus 2."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                       timeout=240, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def test_bench_gpus_2_spawns_two_ranks():
    out = _run(["--gpus", "2", "--dist-check"])
    assert out["n_gpus"] == 2 and out["ranks_seen"] == 2 and out["backend"] == "gloo"


def test_bench_single_rank_needs_no_spawn():
    out = _run(["--dist-check"])
    assert out["n_gpus"] == 1 and out["ranks_seen"] == 1
