"""Multi-rank plumbing of bench.py on the CPU (gloo, world size 2): replicas
only, so the only cross-rank step is the max over ranks of each timing, and
the job rate counts every rank's units over the slowest rank's time.  The
reference arm runs on rank 0 alone; other ranks exit 0 without output."""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        t = bench.max_over_ranks(10.0 + 5.0 * rank, world, torch.device("cpu"))
        out[rank] = (t, bench.replica_rate(3, world, t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate_gloo():
    port = 29500 + (os.getpid() % 2000)
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    # both ranks see the slowest rank's time; 2 replicas x 3 units over 15 s
    assert res[0] == res[1] == (15.0, 0.4)


def test_single_rank_helpers():
    assert bench.max_over_ranks(7.5, 1, None) == 7.5
    assert bench.replica_rate(4, 1, 2.0) == 2.0


@pytest.mark.timeout(120)
def test_reference_arm_other_ranks_exit_silently():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


@pytest.mark.timeout(300)
def test_reference_arm_json_line():
    """Rank 0 of the reference arm prints one JSON line with the bench keys;
    the value is the host oracle's, timed on this machine's cores."""
    import json

    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                        "square512", "--steps", "1", "--warmup", "0", "--cpu-budget", "0.5"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "steps", "warmup", "higher_is_better", "config", "cpu_baseline",
                "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "SVD/s" and d["n_gpus"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # a step is the bounded sample actually timed: its time fits the run
    assert 0 < d["ms_per_step"] <= 1e3 * (0.5 * 4 + 5) and "step" in d


def test_nominal_rate_model():
    """F_nom = S_plain * n(n-1)/2 * (12m + 6n) per SVD; the batch's nominal
    flops use the same per-matrix model."""
    import numpy as np

    r = bench.nominal_rate(512, 512, 14, 50.0)
    f = 14 * 512 * 511 / 2 * (12 * 512 + 6 * 512)
    assert r["gflop_per_svd"] == pytest.approx(f / 1e9)
    assert r["gflops"] == pytest.approx(50.0 * f / 1e9)
    assert r["plain_sweeps"] == 14
    assert bench.nominal_rate(512, 512, None, 50.0) is None
    assert bench.nominal_rate(512, 512, 14, None) is None
    one = bench.batch_flops(np.array([512]), np.array([512]), np.array([14]))
    assert one == pytest.approx(f)


def test_cpu_baseline_contract_fields():
    """The cpu_baseline object of the bench line: the oracle on a bounded
    sample of rounds, extrapolated; kind "port", the threads used as cores."""
    import numpy as np

    rng = np.random.default_rng(1)
    wl = {"name": "t", "a": rng.standard_normal((300, 101)), "eps": 1e-14}
    cb = bench.cpu_baseline(wl, sweeps=10, budget_s=0.2, threads=2)
    assert cb["unit"] == "SVD/s" and cb["kind"] == "port" and cb["cores"] == 2
    assert cb["value"] > 0 and "rounds of one sweep of the same 300x101 input" in cb["sample"]
    assert "x 10 sweeps" in cb["sample"]


def test_rounds_per_sweep_used_for_extrapolation():
    """cpu_baseline extrapolates over n - 1 rounds (even n) or n rounds (odd
    n): the schedule's round count."""
    import oracle as O

    for n in (2, 3, 10, 11, 64, 65):
        assert len(O.schedule(n)) == (n - 1 if n % 2 == 0 else n)


def test_batch_cpu_baseline_contract_fields():
    import numpy as np

    rng = np.random.default_rng(2)
    mats = [rng.standard_normal((20 + k, 8 + k % 5)).astype(np.float32) for k in range(40)]
    cb = bench.batch_cpu_baseline(mats, budget_s=0.05, threads=2)
    assert cb["unit"] == "SVD/s" and cb["kind"] == "port" and cb["cores"] == 2 and cb["value"] > 0
    assert cb["sample"].startswith("first ") and "of 40 matrices" in cb["sample"]


@pytest.mark.parametrize("workload", ["serve", "large"])
def test_reference_arm_unavailable_lines(workload):
    import json

    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                        workload], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr[-1000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["unavailable"]


def test_profile_commands_use_committed_files_and_current_flags():
    """Every ncu summary under profiles/ gives the command that made it: the
    script it runs exists, each bench flag it passes is one bench.py still
    accepts, and every ncu command keeps --clock-control none."""
    import glob
    import re

    help_text = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True,
                               text=True, check=True).stdout
    files = [p for p in glob.glob(os.path.join(ROOT, "profiles", "*.md")) if not p.endswith("README.md")]
    assert files
    for path in files:
        text = open(path).read()
        if "-Xptxas -v" in text:  # a compiler resource summary: its nvcc command on committed sources
            assert re.search(r"^nvcc .*-gencode arch=compute_100a,code=sm_100a", text, flags=re.M), path
            assert os.path.isdir(os.path.join(ROOT, "jacobi-svd-cuda_b200", "csrc")), path
            continue
        cmds = re.findall(r'"(python \S+[^"]*)"', text)
        assert cmds, path
        for cmd in cmds:
            script = cmd.split()[1]
            assert os.path.exists(os.path.join(ROOT, script)), (path, script)
            for flag in re.findall(r"(--[a-z][a-z0-9-]*)", cmd):
                assert flag in help_text, (path, flag)
        for line in re.findall(r"^\s*ncu .*$", text, flags=re.M):
            assert "--clock-control none" in line, (path, line)
