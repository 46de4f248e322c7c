"""Benchmark of the one-sided Jacobi SVD on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload tall|square512|batch|serve|large]
                    [--path auto|plain|precond|mixed|blocked|blockpair]

One step = one pass of the hot path over one batch of synthetic input (for the
single-matrix workloads: one full SVD).  `value` is whole-job SVDs/s with the
input resident in HBM; `e2e` repeats the measurement through the host-buffer
C-ABI call (H2D of A and D2H of U, sigma, V inside the timed region).  Under
torchrun every rank solves its own replica (no collective on the data path):
`scaling` is "weak" and the time is the max over ranks.

`--impl reference` times the reference's CPU arithmetic - the FP64 host
oracle, a restatement of the reference's kernels (the reference has no CPU
path of its own) - on the host cores, on a bounded sample of the same
workload, extrapolated to SVDs/s.  Its line carries the launched N as n_gpus;
the arm itself uses no GPU.

Single-matrix lines also carry `nominal`: the rate in the nominal FP64 count
S_plain * n(n-1)/2 * (12m + 6n) per SVD, S_plain being the plain path's sweep
count on the same input, so that paths with fewer sweeps are compared on the
plain path's work.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "jacobi-svd-cuda_b200"))

FLUSH_BYTES = 256 << 20  # > 126 MB L2

# Sweep counts of the plain path on the seeded inputs (identical in the oracle,
# which reproduces the GPU arithmetic bit for bit); used to extrapolate the
# bounded CPU samples to whole SVDs.
PLAIN_SWEEPS = {"tall": 30, "square512": 14}


def max_over_ranks(x: float, world: int, device) -> float:
    """Maximum of a per-rank scalar over all ranks (times: the job is as slow
    as its slowest replica); identity on one rank.  `device` is where the
    process group's backend reduces (a CUDA device for NCCL, cpu for gloo)."""
    if world <= 1:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Whole-job throughput of `world` independent replicas: all units that
    all ranks processed, over the slowest rank's time."""
    return world * units_per_rank / max_seconds


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi's start-up (NVML initialisation) stalls CUDA calls of this
        # process for a few hundred ms: let it finish before the timed region.
        t0 = time.time()
        while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# workloads


# DRAM bytes (read + write) per launch measured by one ncu capture of the
# named kernel at the named swept shape (rows, columns); caches are flushed
# between ncu passes, so these are cold-cache figures.  Other shapes: null.
L2_BYTES = 126e6  # B200 L2

PROFILED_TRAFFIC = {("plain_round_kernel", 1024, 1024): 8408576.0}


def make_workload(name: str):
    import workloads as W

    if name == "tall":
        a, s = W.tall_case(seed=2)
        return {"name": name, "a": a, "sigma_true": s, "eps": 1e-14,
                "desc": "4096x1024 FP64, A = U diag(sigma) V^T, Haar U,V (seed 2), sigma geometric 1..1e-6"}
    if name == "square512":
        a = W.gaussian_splitmix(512, 512, 1)
        return {"name": name, "a": a, "sigma_true": None, "eps": 1e-14,
                "desc": "512x512 FP64 N(0,1) (SplitMix64 seed 1)"}
    raise SystemExit(f"unknown workload {name}")


def algorithmic_round_bytes(m: int, n: int) -> float:
    """Per launch of the fused round kernel: every pair reads its two A columns
    and writes them back (2 reads + 2 writes of m doubles)."""
    return (n // 2) * 4.0 * m * 8.0


def time_single(args, wl, path, device, stream, steps, warmup, flush, world):
    """Device-timed SVDs of one workload matrix through one path; returns
    (total_ms, sweeps list, per-path stats, last sigma)."""
    import torch
    import jsvd

    a = wl["a"]
    m, n = a.shape
    cfg = jsvd.default_config(epsilon=wl["eps"], **({"threads_per_block": args.threads} if args.threads else {}))
    da = torch.from_numpy(a).to(device)
    du = torch.empty((m, n), dtype=torch.float64, device=device)
    ds = torch.empty(n, dtype=torch.float64, device=device)
    dv = torch.empty((n, n), dtype=torch.float64, device=device)
    fn = {"precond": jsvd.precond_svd_device, "blocked": jsvd.blocked_svd_device,
          "blockpair": jsvd.blockpair_svd_device, "mixed": jsvd.mixed_svd_device}.get(path, jsvd.plain_svd_device)

    def step():
        return fn(da.data_ptr(), m, n, du.data_ptr(), ds.data_ptr(), dv.data_ptr(), cfg, stream.cuda_stream)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(device)
    jsvd.plain_stats_reset()
    jsvd.precond_stats_reset()
    jsvd.blocked_stats_reset()
    jsvd.blockpair_stats_reset()
    jsvd.mixed_stats_reset()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(device)
    total_ms, sweeps = 0.0, []
    for _ in range(steps):
        flush.zero_()  # evict A, V and the working copies from L2 between steps
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sweeps.append(step())
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize(device)
    total_ms = max_over_ranks(total_ms, world, device)
    return total_ms, sweeps, (jsvd.plain_stats(), jsvd.precond_stats(), jsvd.blocked_stats(),
                              jsvd.blockpair_stats(), jsvd.mixed_stats()), ds.cpu().numpy(), (du, dv)


def nominal_rate(m: int, n: int, plain_sweeps: int | None, svd_per_s: float | None) -> dict | None:
    """Nominal FP64 rate of a path: F_nom = S_plain * P * (12 m + 6 n) flops
    per SVD, P = n(n-1)/2 and S_plain the plain path's sweep count on the same
    input, times the path's SVDs/s, so that paths with fewer or cheaper sweeps
    are compared on the plain path's work."""
    if not plain_sweeps or svd_per_s is None:
        return None
    f_nom = float(plain_sweeps) * n * (n - 1) / 2.0 * (12.0 * m + 6.0 * n)
    return {"gflop_per_svd": f_nom / 1e9, "gflops": f_nom * svd_per_s / 1e9, "plain_sweeps": int(plain_sweeps),
            "model": "S_plain * n(n-1)/2 * (12m + 6n) per SVD"}


def blocked_sweep_flops(rows: int, n: int, b: int = 32) -> float:
    """FP64 flops of one blocked sweep: for every block pair, the panel Gram
    (2 rows w^2) and the panel update of X and V (2 (rows + n) w^2), w = 2b."""
    nb = -(-n // b)
    w = 2 * b
    return nb * (nb - 1) / 2 * (2.0 * rows * w * w + 2.0 * (rows + n) * w * w)


ORACLE_FIXTURES = {"tall": os.path.join(ROOT, "tests", "golden", "tall_4096x1024_oracle.npz")}


def oracle_sigma_check(wl, sigma) -> dict | None:
    """Error of `sigma` against the FP64 oracle's sigma on the same input (the
    reference's arithmetic; tests/golden/tall_4096x1024_oracle.npz, made by
    tests/golden/make_tall_sigma.py), when the fixture belongs to this input."""
    import hashlib

    p = ORACLE_FIXTURES.get(wl["name"])
    if not p or not os.path.exists(p):
        return None
    d = np.load(p)
    if hashlib.sha256(np.ascontiguousarray(wl["a"]).tobytes()).hexdigest() != str(d["a_sha256"]):
        return {"oracle": "fixture does not match this input (not compared)"}
    ref = np.sort(d["sigma"])[::-1]
    got = np.sort(np.asarray(sigma))[::-1]
    err = np.abs(got - ref)
    return {"sigma_max_rel_vs_oracle": float(np.max(err / ref)),
            "sigma_normwise_vs_oracle": float(err.max() / ref[0]),
            "oracle_vs_analytic_max_rel": float(np.max(np.abs(ref - np.sort(d["sigma_analytic"])[::-1])
                                                       / np.sort(d["sigma_analytic"])[::-1])),
            "oracle_sweeps": int(d["sweeps"])}


def mixed_roofline(mst, hbm_peak: float, peak_kind: str, step_ms: float) -> dict:
    """Roofline of the mixed path's dominant kernel from the block rounds
    sampled inside the timed solves (events around each launch; rounds 0 and
    rounds/2 of every sweep).  Algorithmic work per launch:
      * Gram: reads the whole swept factor once (rows_pad x cols_pad
        elements, 8 bytes each: FP64, or the TF32 head and tail) - HBM bound;
      * rotation: reads and writes the 64 columns of X and of V of every
        block pair that rotated ((rows_pad + cols_pad) x 64 x 16 bytes per
        pair) - HBM bound;
      * eigen-solve: FP64 flops of the 64 x 64 two-sided Jacobi rounds of
        every block pair (per inner round: 496 off-diagonal 2 x 2 blocks of
        G at 24 flops, 32 diagonal blocks at 4, 64 x 32 rotations of W rows
        at 6; 63 rounds per inner sweep) against the measured FP64 FMA
        throughput - it is latency-bound, far below that peak.
    The kernel with the largest sampled time share is reported."""
    import jsvd

    k = {}
    for ph, g, e, r, n, pairs in (("tc", mst.tc_gram_ms, mst.tc_evd_ms, mst.tc_rot_ms, mst.tc_sampled_rounds,
                                   mst.tc_sampled_pairs),
                                  ("f64", mst.f64_gram_ms, mst.f64_evd_ms, mst.f64_rot_ms, mst.f64_sampled_rounds,
                                   mst.f64_sampled_pairs)):
        if n:
            k[ph] = {"gram_us": 1e3 * g / n, "evd_us": 1e3 * e / n, "rot_us": 1e3 * r / n,
                     "rot_pairs_per_launch": pairs / n, "rounds": int(n)}
    rp, cp = mst.rows_pad, mst.cols_pad
    total = {name: sum(v[name + "_us"] * v["rounds"] for v in k.values()) for name in ("gram", "evd", "rot")}
    if not k:
        return {"bound": "hbm", "kernel": None, "achieved": 0.0, "peak": hbm_peak, "unit": "GB/s", "frac": 0.0,
                "traffic": None}
    inner = int(jsvd.mixed_resolved_options(mst.cols_pad).inner_sweeps)
    evd_flops = mst.block_pairs * inner * 63 * (496 * 24 + 32 * 4 + 64 * 32 * 6)
    kernels = {}
    for ph, v in k.items():
        tcp = ph == "tc"
        kernels["mx_gram_tc" if tcp else "mx_gram_f64"] = {
            "bound": "hbm", "us": v["gram_us"], "work": rp * cp * 8.0, "share": v["gram_us"] * v["rounds"]}
        kernels["mx_rot_tc" if tcp else "mx_rot_f64"] = {
            "bound": "hbm", "us": v["rot_us"], "work": v["rot_pairs_per_launch"] * (rp + cp) * 64 * 16.0,
            "share": v["rot_us"] * v["rounds"]}
        e = kernels.setdefault("mx_evd", {"bound": "fp64", "us": 0.0, "work": float(evd_flops), "share": 0.0,
                                          "rounds": 0})
        e["share"] += v["evd_us"] * v["rounds"]
        e["rounds"] += v["rounds"]
    kernels["mx_evd"]["us"] = kernels["mx_evd"]["share"] / max(1, kernels["mx_evd"]["rounds"])
    tsum = max(1e-9, sum(total.values()))
    name, top = max(kernels.items(), key=lambda kv: kv[1]["share"])
    common = {"kernel": name, "avg_launch_us": top["us"], "sampled_kernel_share": {kk: vv / tsum for kk, vv in
                                                                                    total.items()},
              "per_phase": k}
    if top["bound"] == "fp64":
        fp64_peak = jsvd.probe_fp64_tflops()
        achieved = top["work"] / (top["us"] * 1e-6) / 1e12
        return {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "peak_kind": "measured FP64 FMA probe (jsvd_probe_fp64_tflops)", "frac": achieved / fp64_peak,
                "traffic": None, "algorithmic_flops_per_launch": top["work"], **common,
                "note": "the block eigen-solve is latency-bound: one CTA per block pair runs 63 dependent "
                        "rounds per inner sweep (one barrier and one angle chain each); its DRAM traffic is "
                        "the 64 x 64 Gram partials in and W out"}
    achieved = top["work"] / (top["us"] * 1e-6) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "peak_kind": peak_kind,
            "frac": achieved / hbm_peak, "traffic": PROFILED_TRAFFIC.get((name, rp, cp)),
            "algorithmic_bytes_per_launch": top["work"], **common}


def run_ours(args, rank: int, world: int, device):
    import ctypes

    import torch
    import jsvd

    wl = make_workload(args.workload)
    a = wl["a"]
    m, n = a.shape
    path = args.path if args.path != "auto" else "mixed"
    cfg = jsvd.default_config(epsilon=wl["eps"], **({"threads_per_block": args.threads} if args.threads else {}))
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    torch.cuda.synchronize(device)
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)

    sampler = ClockSampler(device.index if device.index is not None else 0)
    sampler.start()
    total_ms, sweeps, (pst, cst, bst, kst, mst), sig, (du, dv) = time_single(args, wl, path, device, stream,
                                                                            args.steps, args.warmup, flush, world)
    clocks = sampler.stop()
    ms_per_step = total_ms / args.steps
    value = replica_rate(args.steps, world, total_ms / 1e3)
    launches = int(pst.round_launches + pst.vpass_launches + pst.other_launches)
    if kst.solves:
        # outer rounds + per solve: layout in, identity, sigma, U and V layout out
        launches += int(kst.round_launches) + 5 * int(kst.solves)
    if path in ("precond", "mixed"):
        # per solve, the QR stage: 2 factorisations x 3 passes x (Gram, shift?, ceil(n/64) x (diagonal block,
        # panel, trailing update) + ceil(n/64) x (solve, update) + R copy) + 2 R products, and the U, V products
        blocks = (n + 63) // 64
        launches += args.steps * (2 * 3 * (2 + 5 * blocks + 1) + 4 + 4)
    if path == "mixed":
        # block rounds (Gram, eigen-solve, rotation) + layout, split, identity, polar steps, X V', sigma, U, V
        launches += int(mst.tc_gram_launches + mst.tc_rot_launches + mst.f64_gram_launches + mst.f64_rot_launches
                        + mst.evd_launches) + args.steps * 16

    # accuracy guard on the timed configuration (sigma vs the analytic spectrum,
    # and the reference's residual metrics on the returned factors)
    sig_cols = sig.copy()
    sig = np.sort(sig)[::-1]
    guard = None
    if wl["sigma_true"] is not None:
        t = np.sort(wl["sigma_true"])[::-1]
        guard = {"sigma_max_rel_vs_analytic": float(np.max(np.abs(sig - t) / t)),
                 "sigma_normwise_vs_analytic": float(np.max(np.abs(sig - t)) / t[0])}
    if m * n <= (1 << 22):  # the library's validation metrics (jsvd_residuals, host threads)
        guard = dict(guard or {}, **jsvd.residuals(a, du.cpu().numpy(), sig_cols, dv.cpu().numpy()))
    oc = oracle_sigma_check(wl, sig_cols)
    if oc:
        guard = dict(guard or {}, **oc)
    oracle_ref = None  # sigma of the FP64 oracle's arithmetic on this very input

    # e2e through the host-buffer C-ABI call, pinned host memory
    ha = torch.from_numpy(a).pin_memory().numpy()
    hu = torch.empty((m, n), dtype=torch.float64).pin_memory().numpy()
    hs = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    hv = torch.empty((n, n), dtype=torch.float64).pin_memory().numpy()
    lib = jsvd.lib()
    entry = {"precond": lib.jsvd_precond_svd, "blocked": lib.jsvd_blocked_svd,
             "blockpair": lib.jsvd_blockpair_svd, "mixed": lib.jsvd_mixed_svd}.get(path, lib.jsvd_plain_svd)
    sw = ctypes.c_int(0)
    e2e_steps = 0 if args.no_e2e else args.steps
    for _ in range(max(1, args.warmup) if e2e_steps else 0):
        jsvd.check(entry(ha.ctypes.data, m, n, ctypes.byref(cfg), hu.ctypes.data, hs.ctypes.data, hv.ctypes.data,
                         ctypes.byref(sw)))
    e2e_s = 0.0
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        jsvd.check(entry(ha.ctypes.data, m, n, ctypes.byref(cfg), hu.ctypes.data, hs.ctypes.data, hv.ctypes.data,
                         ctypes.byref(sw)))
        e2e_s += time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world, device)
    e2e_value = replica_rate(e2e_steps, world, e2e_s) if e2e_steps else None

    # the plain drop-in on the same input, for the speed-up of the fast path
    plain = None
    if path != "plain" and not args.no_plain_compare:
        p_ms, p_sw, _, p_sig, _ = time_single(args, wl, "plain", device, stream, 2, 1, flush, world)
        plain = {"value": world * 2 / (p_ms / 1e3), "ms_per_step": p_ms / 2, "sweeps_per_svd": p_sw[0]}
        oc = oracle_sigma_check(wl, p_sig)
        if oc:
            plain["check"] = oc
        oracle_ref = p_sig
    if oracle_ref is not None and guard is not None and "sigma_max_rel_vs_oracle" not in guard:
        # The plain path reproduces the oracle bit for bit (tests/test_plain_gpu.py pins it against the oracle,
        # and the oracle against the reference's own outputs), so its sigma in this run is the oracle's sigma on
        # this input even where the committed fixture's input (made on another CPU) differs in the last bits.
        r = np.sort(oracle_ref)[::-1]
        e = np.abs(sig - r)
        guard.update({"sigma_max_rel_vs_oracle": float(np.max(e / r)), "sigma_normwise_vs_oracle": float(e.max() / r[0]),
                      "oracle_source": "plain path in this run (bit-identical to the FP64 oracle)"})

    hbm_peak, _, peak_kind = peaks()
    mx = n if path in ("precond", "mixed") else m  # rows of the swept matrix
    if path == "mixed":
        roof = mixed_roofline(mst, hbm_peak, peak_kind, total_ms / world)
    elif kst.round_launches:
        # block-pair outer round: every column of X (mx rows) and of V (n rows)
        # is read and written once per launch
        avg_ms = kst.round_ms / kst.round_launches
        bytes_per = 16.0 * n * (mx + n)
        roof = {"bound": "hbm", "kernel": "bp_round_kernel", "achieved": bytes_per / (avg_ms * 1e-3) / 1e9,
                "peak": hbm_peak, "unit": "GB/s", "peak_kind": peak_kind, "traffic": None,
                "avg_launch_us": avg_ms * 1e3, "algorithmic_bytes_per_launch": bytes_per,
                "round_share_of_step": kst.round_ms / max(total_ms / world, 1e-9),
                "outer_sweeps": kst.sweeps / max(1, kst.solves)}
    elif pst.round_launches:
        avg_round_ms = pst.round_ms / pst.round_launches
        roof = {"bound": "hbm", "kernel": "plain_round_kernel",
                "achieved": algorithmic_round_bytes(mx, n) / (avg_round_ms * 1e-3) / 1e9, "peak": hbm_peak,
                "unit": "GB/s", "peak_kind": peak_kind,
                "traffic": PROFILED_TRAFFIC.get(("plain_round_kernel", mx, n)), "avg_launch_us": avg_round_ms * 1e3,
                "algorithmic_bytes_per_launch": algorithmic_round_bytes(mx, n),
                "round_share_of_step": pst.round_ms / max(total_ms / world, 1e-9),
                "vpass_ms_per_sweep": pst.vpass_ms / max(1, pst.vpass_launches)}
    else:
        # blocked sweep: FP64 work of the Gram and apply kernels against the
        # measured FP64 FMA peak
        fp64_peak = jsvd.probe_fp64_tflops()
        flops = blocked_sweep_flops(mx, n) * bst.sweeps
        roof = {"bound": "fp64", "kernel": "blk_gram + blk_solve + blk_apply",
                "achieved": flops / (bst.sweep_ms * 1e-3) / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                "peak_kind": "measured FP64 FMA probe (jsvd_probe_fp64_tflops)", "traffic": None,
                "flops_per_sweep": blocked_sweep_flops(mx, n),
                "sweep_share_of_step": bst.sweep_ms / max(total_ms / world, 1e-9)}
    roof["frac"] = roof["achieved"] / roof["peak"]
    # The swept matrix (and V) of these workloads fit in the 126 MB L2: the
    # algorithmic bytes are served from L2, so `achieved` can pass the HBM
    # copy rate and `frac` above 1 is expected there.
    roof["l2_resident"] = bool(8.0 * (mx + n) * n <= L2_BYTES)
    phases = None
    if path == "precond" and cst.solves:
        phases = {"qr_ms": cst.qr_ms / cst.solves, "jacobi_ms": cst.jacobi_ms / cst.solves,
                  "u_ms": cst.u_ms / cst.solves, "fallbacks": int(cst.fallbacks),
                  "gram_checks": pst.gram_checks / cst.solves}
    if path == "mixed" and mst.solves:
        phases = {"qr_ms": mst.qr_ms / mst.solves, "tensor_core_phase_ms": mst.tc_ms / mst.solves,
                  "orthogonalise_ms": mst.orth_ms / mst.solves, "fp64_refine_ms": mst.refine_ms / mst.solves,
                  "output_ms": mst.out_ms / mst.solves, "tc_sweeps": mst.tc_sweeps / mst.solves,
                  "fp64_sweeps": mst.f64_sweeps / mst.solves, "fallbacks": int(mst.fallbacks),
                  "tc_discarded": int(mst.tc_discarded),
                  "sweep_history": [[p, o, r] for p, o, r in jsvd.mixed_sweep_history()]}
    if bst.solves:
        phases = dict(phases or {}, blocked_sweeps=bst.sweeps / bst.solves,
                      blocked_sweep_ms=bst.sweep_ms / max(1, bst.sweeps),
                      block_rounds_per_sweep=bst.block_rounds / max(1, bst.sweeps))
    line = {
        "metric": "SVDs/s",
        "value": value,
        "unit": "SVD/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["desc"],
                   "path": {"precond": "QR-preconditioned: two shifted CholeskyQR3 factorisations (A = QR, "
                                       "R^T = Q1 P) + FP64 Jacobi on P^T (" +
                                       ("block-pair" if kst.solves else "plain round-robin") + " sweep)",
                            "blocked": "blocked FP64 one-sided Jacobi on A (32-column blocks)",
                            "mixed": "blocked mixed precision: the QR stage, then block-pair sweeps with tcgen05 "
                                     "3xTF32 Gram and rotation GEMMs (TMA-fed, TMEM accumulators) and FP64 block "
                                     "eigen-solves, FP64 re-orthogonalisation of V, FP64 blocked refinement "
                                     "sweeps (DMMA)",
                            "blockpair": "block-pair FP64 one-sided Jacobi on A"}.get(
                       path, "plain FP64 drop-in (reference arithmetic, round-robin)"),
                   "epsilon": wl["eps"], "sweeps_per_svd": sweeps[0] if sweeps else None,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
                   "phases_ms": phases},
        "plain_path": plain,
        "nominal": nominal_rate(m, n, plain["sweeps_per_svd"] if plain else (
            sweeps[0] if path == "plain" and sweeps else PLAIN_SWEEPS.get(wl["name"])), value),
        "e2e": {"value": e2e_value, "unit": "SVD/s", "h2d_bytes_per_step": a.nbytes,
                "d2h_bytes_per_step": (m * n + n + n * n) * 8, "timer": "host wall clock around the synchronous call"},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clocks,
        "check": guard,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl, PLAIN_SWEEPS.get(wl["name"], 12), budget_s=args.cpu_budget)
    if wl["name"] == "tall" and world == 1 and not args.no_extras:
        line["other_configs"] = run_extras(args, path, device, stream, flush)
        line["reference_gpu"] = reference_gpu_timing()
    return line


REF_GPU_LIB = os.path.join(ROOT, "oracle", "_ref", "libjsvd_ref.so")


def reference_gpu_timing() -> dict:
    """The reference's own GPU solver (jacobi::svd::one_sided_jacobi_svd,
    compiled unmodified from its sources into oracle/_ref/libjsvd_ref.so by
    oracle/Makefile) timed through its full host path (its own cudaMalloc,
    host<->device copies and per-round synchronisations) on the config-2
    input (one solve) and on config 1 (best of two): the GPU comparator of the
    plain drop-in.  Wall clock around the call, host buffers in and out."""
    import ctypes

    if not os.path.exists(REF_GPU_LIB):
        return {"unavailable": "oracle/_ref/libjsvd_ref.so not built (build() compiles it where the "
                               "reference sources are present)"}
    L = ctypes.CDLL(REF_GPU_LIB)
    P, S, I, D = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_double
    L.ref_plain_svd.argtypes = [P, S, S, D, I, I, I, P, P, P, P]
    L.ref_plain_svd.restype = I
    out = {"kind": "reference GPU binary (unmodified sources, oracle/_ref)", "unit": "SVD/s"}
    for name, reps in (("tall", 1), ("square512", 2)):
        wl = make_workload(name)
        a = np.ascontiguousarray(wl["a"])
        m, n = a.shape
        u, sg, v = np.empty((m, n)), np.empty(n), np.empty((n, n))
        sw = ctypes.c_int(0)
        best = None
        for _ in range(reps):
            t0 = time.perf_counter()
            rc = L.ref_plain_svd(a.ctypes.data, m, n, wl["eps"], 128, 256, 0, u.ctypes.data, sg.ctypes.data,
                                 v.ctypes.data, ctypes.byref(sw))
            dt = time.perf_counter() - t0
            if rc != 0:
                out[name] = {"error": f"ref_plain_svd returned {rc}"}
                break
            best = dt if best is None else min(best, dt)
        else:
            out[name] = {"value": 1.0 / best, "seconds": best, "sweeps": int(sw.value), "epsilon": wl["eps"]}
    return out


def run_extras(args, path: str, device, stream, flush) -> dict:
    """Short measurements of the other configurations beside the headline
    line (device-resident inputs, L2 flushed between steps, CUDA events):
    the other fast path on the same 4096 x 1024 input, config 1 (512 x 512
    N(0,1), plain drop-in, checked bit for bit against the reference's own
    output), config 3 (the 20,000-matrix batch), the 16384 x 8192 graded
    and clustered matrix through the mixed path, the plain drop-in on the
    4096 x 1024 input, and config 4 at one arrival rate (serve_1000; the
    serving core's throughput is host wall clock)."""
    import jsvd

    out = {}
    other = "precond" if path == "mixed" else "mixed"
    wl = make_workload("tall")
    o_ms, o_sw, _, o_sig, _ = time_single(args, wl, other, device, stream, 3, 1, flush, 1)
    out[f"tall_{other}"] = {"value": 3 / (o_ms / 1e3), "unit": "SVD/s", "ms_per_step": o_ms / 3,
                            "sweeps_per_svd": o_sw[0], "check": oracle_sigma_check(wl, o_sig)}
    if path != "plain":
        # the plain FP64 drop-in on the same input (the ratio config 2 is quoted against)
        p_ms, p_sw, _, p_sig, _ = time_single(args, wl, "plain", device, stream, 1, 1, flush, 1)
        out["tall_plain"] = {"value": 1 / (p_ms / 1e3), "unit": "SVD/s", "ms_per_step": p_ms,
                             "sweeps_per_svd": p_sw[0], "check": oracle_sigma_check(wl, p_sig)}
    wl1 = make_workload("square512")
    s_ms, s_sw, _, s_sig, _ = time_single(args, wl1, "plain", device, stream, 3, 1, flush, 1)
    g = np.load(os.path.join(ROOT, "tests", "golden", "cfg1_512x512.npz"))
    out["square512_plain"] = {"value": 3 / (s_ms / 1e3), "unit": "SVD/s", "ms_per_step": s_ms / 3,
                              "sweeps_per_svd": s_sw[0], "epsilon": wl1["eps"],
                              "sigma_bitwise_equal_to_reference": bool(np.array_equal(s_sig, g["sigma"])) if float(
                                  g["eps"]) == wl1["eps"] else None}
    # config 4, briefly: one arrival rate, 500 requests, large ones on the mixed path
    sargs = argparse.Namespace(**vars(args))
    sargs.rates, sargs.serve_count, sargs.serve_plain_sample, sargs.serve_large_path = "1000", 500, 20, 2
    sl = run_serve(sargs, 0, 1, device)
    r = sl["config"]["per_rate"][0]
    out["serve_1000"] = {"value": sl["value"], "unit": "SVD/s", "rate_req_s": r["rate_req_s"],
                         "requests": r["requests"], "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"],
                         "sweep_steps": r["batches"], "small_requests": r["batched_requests"],
                         "large_solves": r["large_solves"],
                         "plain_one_at_a_time_svd_s": sl["config"]["plain_one_at_a_time_svd_s"],
                         "note": "the serve workload's trace, first 500 requests; bench.py --workload serve runs "
                                 "five rates x 2000"}
    bargs = argparse.Namespace(**vars(args))
    bargs.steps, bargs.warmup, bargs.no_cpu_baseline = 2, 1, True
    b = run_batch(bargs, 0, 1, device)
    out["batch"] = {"value": b["value"], "unit": "SVD/s", "ms_per_step": b["ms_per_step"],
                    "matrices": BATCH_COUNT if bargs.batch_count == BATCH_COUNT else bargs.batch_count,
                    "class_ms_per_step": b["config"]["classes"]["ms_per_step"], "roofline": b["roofline"],
                    "plain_one_at_a_time_svd_s": batch_plain_rate(device, 40), "plain_sample": 40}
    # config 1 through the blocked mixed-precision path (accuracy against the
    # reference's own sigma for this input)
    m_ms, m_sw, _, m_sig, _ = time_single(args, wl1, "mixed", device, stream, 3, 1, flush, 1)
    ref1 = np.sort(np.asarray(g["sigma"]))[::-1]
    got1 = np.sort(np.asarray(m_sig))[::-1]
    out["square512_mixed"] = {"value": 3 / (m_ms / 1e3), "unit": "SVD/s", "ms_per_step": m_ms / 3,
                              "sweeps_per_svd": m_sw[0],
                              "sigma_normwise_vs_reference": float(np.max(np.abs(got1 - ref1)) / ref1[0]),
                              "sigma_max_rel_vs_reference": float(np.max(np.abs(got1 - ref1) / ref1))}
    out["large_mixed"] = run_large_device(args, device, "mixed")
    return out


def batch_plain_rate(device, k: int) -> float:
    """The plain drop-in one matrix at a time (host buffers, as a caller of
    one_sided_jacobi_svd would) on k matrices drawn from the config-3
    distribution (seed 3), promoted to FP64: SVD/s."""
    import jsvd
    import workloads as W

    mats = W.batch_workload_torch(k, seed=3, device=device)
    cfg = jsvd.default_config(epsilon=1e-14)
    a64 = [np.asarray(a, dtype=np.float64) for a in mats]
    jsvd.plain_svd(a64[0], cfg)  # warm-up
    t0 = time.perf_counter()
    for a in a64:
        jsvd.plain_svd(a, cfg)
    return k / (time.perf_counter() - t0)


def run_large_device(args, device, path: str, steps: int = 1, warmup: int = 1) -> dict:
    """The 16384 x 8192 graded and clustered matrix (sigma_i = 10^(-10 i/n),
    8 clusters of 16 with gaps 1e-10, Haar U and V, seed 5), generated on the
    GPU and solved from device memory by one path (CUDA events)."""
    import torch
    import jsvd
    import workloads as W

    m, n = args.large_m, args.large_n
    sig = np.ascontiguousarray(W.graded_clustered_sigma(n))
    t0 = time.time()
    da = large_matrix_device(m, n, sig, device)
    gen_s = time.time() - t0
    du = torch.empty((m, n), dtype=torch.float64, device=device)
    ds = torch.empty(n, dtype=torch.float64, device=device)
    dv = torch.empty((n, n), dtype=torch.float64, device=device)
    cfg = jsvd.default_config(epsilon=1e-14)
    fn = {"mixed": jsvd.mixed_svd_device, "precond": jsvd.precond_svd_device}[path]
    st = torch.cuda.current_stream(device)
    for _ in range(warmup):
        fn(da.data_ptr(), m, n, du.data_ptr(), ds.data_ptr(), dv.data_ptr(), cfg, st.cuda_stream)
    jsvd.mixed_stats_reset()
    torch.cuda.synchronize(device)
    total, sw = 0.0, 0
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        sw = fn(da.data_ptr(), m, n, du.data_ptr(), ds.data_ptr(), dv.data_ptr(), cfg, st.cuda_stream)
        e1.record(st)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    ref = np.sort(sig)[::-1]
    got = np.sort(ds.cpu().numpy())[::-1]
    err = np.abs(got - ref)
    mst = jsvd.mixed_stats()
    res = {"value": steps / (total / 1e3), "unit": "SVD/s", "s_per_svd": total / 1e3 / steps, "sweeps_per_svd": sw,
           "path": path, "generation_s": gen_s,
           "check": {"sigma_normwise_vs_analytic": float(err.max() / ref[0]),
                     "sigma_max_rel_top_half": float(np.max((err / ref)[: n // 2]))}}
    if path == "mixed" and mst.solves:
        res["phases_ms"] = {"qr": mst.qr_ms / mst.solves, "tensor_core_phase": mst.tc_ms / mst.solves,
                            "orthogonalise": mst.orth_ms / mst.solves, "fp64_refine": mst.refine_ms / mst.solves,
                            "tc_sweeps": mst.tc_sweeps / mst.solves, "fp64_sweeps": mst.f64_sweeps / mst.solves}
        res["roofline"] = mixed_roofline(mst, peaks()[0], peaks()[2], total / steps)
    del da, du, dv
    torch.cuda.empty_cache()
    return res


def large_matrix_device(m: int, n: int, sig: np.ndarray, device):
    """A = U diag(sig) V^T on the GPU, U (m x n) and V (n x n) Haar from QR of
    seeded Gaussians (torch, FP64), row-major."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(5)
    qu, ru = torch.linalg.qr(torch.randn((m, n), generator=g, dtype=torch.float64, device=device))
    qu *= torch.sign(torch.diagonal(ru))[None, :]
    del ru
    qv, rv = torch.linalg.qr(torch.randn((n, n), generator=g, dtype=torch.float64, device=device))
    qv *= torch.sign(torch.diagonal(rv))[None, :]
    del rv
    qu *= torch.from_numpy(sig).to(device)[None, :]
    a = (qu @ qv.T).contiguous()
    del qu, qv
    torch.cuda.empty_cache()
    return a


def cpu_baseline(wl, sweeps: int, budget_s: float = 12.0, threads: int | None = None) -> dict:
    """Oracle (reference arithmetic) on the host cores: a bounded number of
    rounds of one sweep, extrapolated to a whole SVD with `sweeps` sweeps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    a = wl["a"]
    m, n = a.shape
    threads = threads or os.cpu_count() or 1
    rounds_total = n - 1 if n % 2 == 0 else n
    probe = min(4, rounds_total)
    t0 = time.perf_counter()
    O.partial_sweep(a, wl["eps"], rounds=probe, threads=threads)
    per_round = (time.perf_counter() - t0) / probe
    r = int(max(probe, min(rounds_total, budget_s / max(per_round, 1e-9))))
    t0 = time.perf_counter()
    O.partial_sweep(a, wl["eps"], rounds=r, threads=threads)
    dt = time.perf_counter() - t0
    per_svd = dt / r * rounds_total * sweeps
    return {"value": 1.0 / per_svd, "unit": "SVD/s", "cores": threads, "kind": "port", "sample_s": dt,
            "sample": f"{r} of {rounds_total} rounds of one sweep of the same {m}x{n} input "
                      f"({dt:.1f} s), extrapolated x{rounds_total / r:.2f} rounds x {sweeps} sweeps"}


BATCH_COUNT = 20000


def batch_flops(rows, cols, sweeps) -> float:
    """Nominal FP64 flops: sweeps * P * (12 m + 6 n) per matrix, P = n(n-1)/2
    (every pair counted as rotating)."""
    m = rows.astype(np.float64)
    n = cols.astype(np.float64)
    return float(np.sum(sweeps.astype(np.float64) * n * (n - 1) / 2 * (12 * m + 6 * n)))


def run_batch(args, rank: int, world: int, device):
    import torch
    import jsvd
    import workloads as W

    t0 = time.time()
    mats = W.batch_workload_torch(args.batch_count, seed=3, device=device)
    gen_s = time.time() - t0
    cfg = jsvd.default_config(epsilon=1e-14)
    b = jsvd.DeviceBatch(mats, device, f32=True, want_u=False, want_v=True)
    fp64_peak = jsvd.probe_fp64_tflops()
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    torch.cuda.synchronize(device)
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)
    for _ in range(args.warmup):
        b.solve(cfg, stream=stream.cuda_stream)
    jsvd.batch_stats_reset()
    sampler = ClockSampler(device.index if device.index is not None else 0)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(device)
    sampler.start()
    total_ms = 0.0
    step_ms = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.solve(cfg, stream=stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        total_ms += step_ms[-1]
    clocks = sampler.stop()
    st = jsvd.batch_stats()
    total_ms = max_over_ranks(total_ms, world, device)
    value = replica_rate(args.steps * b.count, world, total_ms / 1e3)
    flops = batch_flops(b.rows, b.cols, b.sweeps)
    kernel_ms = st.kernel_ms / max(1, st.calls)
    achieved = flops / (kernel_ms * 1e-3) / 1e12

    # e2e: pinned FP32 input H2D + solve + D2H of sigma and V, every step
    host_in = b.host_a.pin_memory()
    host_s = torch.empty(b.sigma.shape, dtype=torch.float64).pin_memory()
    host_v = torch.empty(b.v.shape, dtype=torch.float64).pin_memory()
    e2e_s = 0.0
    for i in range(args.steps + 1):
        flush.zero_()
        torch.cuda.synchronize(device)
        t1 = time.perf_counter()
        b.a.copy_(host_in, non_blocking=True)
        b.solve(cfg, stream=stream.cuda_stream)
        host_s.copy_(b.sigma, non_blocking=True)
        host_v.copy_(b.v, non_blocking=True)
        torch.cuda.synchronize(device)
        if i > 0:
            e2e_s += time.perf_counter() - t1
    e2e_s = max_over_ranks(e2e_s, world, device)
    line = {
        "metric": "SVDs/s",
        "value": value,
        "unit": "SVD/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": f"{b.count} FP32-stored matrices, m~U{{16..256}}, n~U{{8..m}}, Haar U,V, sigma "
                               f"log-uniform [1/kappa,1], kappa log-uniform [1e1,1e6] (seed 3); sigma and V",
                   "path": "batched persistent kernels, plain arithmetic: one CTA per matrix for the size classes "
                           "that fit one CTA's shared memory, one thread-block cluster per matrix (A and V in "
                           "distributed shared memory) for the two largest",
                   "epsilon": 1e-14, "mean_sweeps": float(np.mean(b.sweeps)),
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
                   "generation_s": gen_s, "step_ms": step_ms,
                   "launch_shapes": jsvd.batch_builtin_tuning(),
                   "classes": {"count": [int(x) for x in st.class_count],
                               "ms_per_step": [x / max(1, st.calls) for x in st.class_ms]}},
        "e2e": {"value": replica_rate(args.steps * b.count, world, e2e_s), "unit": "SVD/s",
                "h2d_bytes_per_step": b.h2d_bytes,
                "d2h_bytes_per_step": int((b.sigma.numel() + b.v.numel()) * 8),
                "timer": "host wall clock around H2D + solve + D2H"},
        "gpu_launches": int(st.launches),
        "roofline": {"bound": "fp64", "kernel": "batch_kernel + batch_cluster_kernel", "achieved": achieved,
                     "peak": fp64_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                     "peak_kind": "measured FP64 FMA probe (jsvd_probe_fp64_tflops)",
                     "traffic": None, "flops_per_launch_set": flops,
                     "flop_model": "sweeps * n(n-1)/2 * (12m + 6n) per matrix"},
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = batch_cpu_baseline(mats, budget_s=args.cpu_budget)
    return line


def batch_cpu_baseline(mats, budget_s: float = 10.0, threads: int | None = None) -> dict:
    """Oracle on the host cores, threads across matrices, on the first
    matrices of the same batch until the time budget is used."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    threads = threads or os.cpu_count() or 1
    done, t_used, k = 0, 0.0, 0
    chunk = max(threads, 16)
    while t_used < budget_s and k < len(mats):
        part = [a.astype(np.float64) for a in mats[k: k + chunk]]
        t0 = time.perf_counter()
        O.batch_svd(part, eps=1e-14, threads=threads)
        t_used += time.perf_counter() - t0
        done += len(part)
        k += chunk
    return {"value": done / t_used, "unit": "SVD/s", "cores": threads, "kind": "port", "sample_s": t_used,
            "sample": f"first {done} of {len(mats)} matrices of the same batch ({t_used:.1f} s), oracle, "
                      f"one matrix per thread"}


def serve_requests(count: int, seed: int, device):
    """Matrices of the serving workload (shapes and kappas from
    workloads.serving_requests, Haar factors from FP64 QR on the GPU)."""
    import torch
    import workloads as W

    t, ms, ns, kappas, rng = W.serving_requests(count, 1.0, seed=seed)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    mats = []
    for m, n, kappa in zip(ms, ns, kappas):
        m, n = int(m), int(n)
        s = np.sort(10.0 ** rng.uniform(-np.log10(kappa), 0.0, size=n))[::-1].copy()
        s[0] = 1.0
        qu, ru = torch.linalg.qr(torch.randn((m, n), generator=g, dtype=torch.float64, device=device))
        qv, rv = torch.linalg.qr(torch.randn((n, n), generator=g, dtype=torch.float64, device=device))
        qu = qu * torch.sign(torch.diagonal(ru))[None, :]
        qv = qv * torch.sign(torch.diagonal(rv))[None, :]
        a = (qu * torch.from_numpy(s).to(device)[None, :]) @ qv.T
        mats.append(np.ascontiguousarray(a.cpu().numpy()))
    return t, mats


def run_serve(args, rank: int, world: int, device):
    """Poisson arrivals at several rates through the serving core; one step =
    one arrival trace.  value = completed SVDs/s at the highest rate."""
    import torch
    import jsvd

    rates = [float(r) for r in args.rates.split(",")]
    t_unit, mats = serve_requests(args.serve_count, seed=4, device=device)
    cfg = jsvd.default_config(epsilon=1e-14)
    budget = 40 << 30
    per_rate = []
    sampler = ClockSampler(device.index if device.index is not None else 0)
    sampler.start()
    for rate in rates:
        arrivals = t_unit / rate
        with jsvd.Server(cfg, budget_bytes=budget, large_path=args.serve_large_path,
                         large_workers=args.serve_large_workers) as srv:
            # warm the worker plans and kernels
            srv.wait(srv.submit(mats[0]))
            tickets = [None] * len(mats)
            lat = [0.0] * len(mats)
            sweeps = [0] * len(mats)

            def collect():
                for i in range(len(mats)):
                    while tickets[i] is None:
                        time.sleep(0.0002)
                    _, _, _, sweeps[i], lat[i] = srv.wait(tickets[i])

            th = threading.Thread(target=collect)
            th.start()
            t0 = time.perf_counter()
            for i, a in enumerate(mats):
                dt = arrivals[i] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                tickets[i] = srv.submit(a)
            th.join()
            wall = time.perf_counter() - t0
            st = srv.stats()
        lat_sorted = np.sort(np.array(lat))
        per_rate.append({"rate_req_s": rate, "requests": len(mats), "svd_s": len(mats) / wall,
                         "p50_ms": float(np.percentile(lat_sorted, 50)), "p99_ms": float(np.percentile(lat_sorted, 99)),
                         "batches": int(st.batches), "batched_requests": int(st.batched_requests),
                         "large_solves": int(st.large_solves), "peak_device_gb": st.peak_device_bytes / 2**30})
    clocks = sampler.stop()
    # the plain drop-in, one request at a time, on a sample of the same trace
    k = min(len(mats), args.serve_plain_sample)
    t0 = time.perf_counter()
    for a in mats[:k]:
        jsvd.plain_svd(a, cfg)
    plain_rate = k / (time.perf_counter() - t0)
    top = per_rate[-1]
    in_bytes = sum(a.nbytes for a in mats)
    out_bytes = sum((a.shape[1] + a.shape[1] ** 2) * 8 for a in mats)
    return {
        "metric": "SVDs/s",
        "value": top["svd_s"],
        "unit": "SVD/s",
        "n_gpus": world,
        "steps": len(rates),
        "warmup": 1,
        "ms_per_step": 1e3 * top["requests"] / top["svd_s"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": f"serving: Poisson arrivals, {args.serve_count} requests per rate, m log-uniform "
                               f"32..2048, n = m*U(0.25,1), FP64, kappa log-uniform [1e2,1e8], 40 GB budget (seed 4)",
                   "path": "serving core: small requests batched by sweep, large requests on worker streams (" + {0: "plain", 1: "QR-preconditioned", 2: "blocked mixed precision"}[args.serve_large_path] + " path)",
                   "epsilon": 1e-14, "per_rate": per_rate,
                   "plain_one_at_a_time_svd_s": plain_rate, "plain_sample": k},
        "e2e": {"value": top["svd_s"], "unit": "SVD/s", "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": out_bytes, "timer": "host wall clock, submit of the first request to "
                                                          "completion of the last (host buffers in and out)"},
        "gpu_launches": None,
        "clocks": clocks,
    }


def run_large(args, rank: int, world: int, device):
    """Large streamed case: an m x n FP64 matrix with sigma_i = 10^(-10 i / n)
    and 8 clusters of 16 values with relative gaps 1e-10, Haar U and V, written
    to disk in the *.mat format and solved by the CLI pipeline (mmap reader,
    serving core, the chosen solver - mixed by default, or precond or plain -
    mmap writer).  One step = one run of the CLI on the file; timed on the
    host wall clock (file in, file out).  The line also carries the same
    matrix solved from device memory (`device_resident`, CUDA events)."""
    import workloads as W

    m, n = args.large_m, args.large_n
    solver = args.path if args.path in ("mixed", "precond", "plain") else "mixed"
    sig = np.ascontiguousarray(W.graded_clustered_sigma(n))
    t0 = time.time()
    a = large_matrix_device(m, n, sig, device).cpu().numpy()
    gen_s = time.time() - t0
    work = args.large_dir or "/tmp/jsvd_large"
    os.makedirs(work, exist_ok=True)
    src, dst = os.path.join(work, "large_in.mat"), os.path.join(work, "large_out.mat")
    with open(src, "wb") as f:
        f.write(np.array([m, n], dtype=">u8").tobytes())
        a.astype(">f8").tofile(f)
    del a
    cli = os.path.join(ROOT, "jacobi-svd-cuda_b200", "jacobi-svd-b200")
    cmd = [cli, src, dst, "-e", "1e-14", "--solver", solver, "--force", "-q", "--json-report"]
    times = []
    for i in range(args.warmup + args.steps):
        t1 = time.perf_counter()
        out = subprocess.run(cmd, capture_output=True, text=True)
        dt = time.perf_counter() - t1
        if out.returncode != 0:
            raise SystemExit(f"CLI failed: {out.stderr}")
        if i >= args.warmup:
            times.append(dt)
    report = json.loads(out.stdout[out.stdout.index("{"):])
    # sigma is the second record of the output stream: U (m x n), Sigma (1 x n), V
    with open(dst, "rb") as f:
        f.seek(16 + 8 * m * n)
        hdr = np.frombuffer(f.read(16), dtype=">u8")
        got = np.frombuffer(f.read(8 * n), dtype=">f8").astype(np.float64)
    got = np.sort(got)[::-1]
    ref = np.sort(sig)[::-1]
    err = np.abs(got - ref)
    elapsed = float(np.mean(times))
    return {
        "metric": "SVDs/s",
        "value": 1.0 / elapsed,
        "unit": "SVD/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": f"{m}x{n} FP64, sigma_i = 10^(-10 i/n) with 8 clusters of 16 (gaps 1e-10), Haar U,V "
                               f"(seed 5), streamed from a *.mat file through the CLI pipeline",
                   "path": f"CLI pipeline -> serving core -> {solver} solver", "epsilon": 1e-14,
                   "pipeline_report": report, "generation_s": gen_s, "sigma_header": hdr.tolist()},
        "e2e": {"value": 1.0 / elapsed, "unit": "SVD/s", "h2d_bytes_per_step": 8 * m * n,
                "d2h_bytes_per_step": 8 * (m * n + n + n * n), "timer": "host wall clock around the CLI process"},
        "check": {"sigma_normwise_vs_analytic": float(err.max() / ref[0]),
                  "sigma_max_rel_vs_analytic": float(np.max(err / ref)),
                  "sigma_max_rel_top_half": float(np.max((err / ref)[: n // 2]))},
        "gpu_launches": None,
        "device_resident": run_large_device(args, device, solver if solver != "plain" else "precond"),
    }


def run_reference(args):
    if args.workload in ("serve", "large"):
        why = {"serve": "the reference has no serving path (its pipeline solves one matrix per host thread); its "
                        "CPU arithmetic is timed on the tall, square512 and batch workloads",
               "large": "the CPU sample extrapolates sampled rounds by the plain path's sweep count, and no "
                        "plain-path sweep count has been measured on the 16384x8192 input; the reference's CPU "
                        "arithmetic is timed on the tall, square512 and batch workloads"}
        return {"impl": "reference", "unavailable": why[args.workload]}
    if args.workload == "batch":
        import workloads as W
        mats = W.batch_workload(min(args.batch_count, 400), seed=3)
        vals, secs = [], []
        for i in range(args.warmup + args.steps):
            cb = batch_cpu_baseline(mats, budget_s=args.cpu_budget)
            if i >= args.warmup:
                vals.append(cb["value"])
                secs.append(cb["sample_s"])
        value = statistics.mean(vals)
        cb["value"] = value
        return {"impl": "reference", "metric": "SVDs/s", "value": value, "unit": "SVD/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(secs),
                "step": "one bounded sample of the batch (cpu_baseline.sample); value = matrices solved / "
                        "sample time", "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": {"workload": "batch (FP32-stored, m~U{16..256}, n~U{8..m}), sample of the same "
                                       "distribution", "path": "FP64 host oracle",
                           "devices": "host cores only (rank 0); no GPU is used by this arm"},
                "cpu_baseline": cb,
                "e2e": {"value": value, "unit": "SVD/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    wl = make_workload(args.workload)
    m, n = wl["a"].shape
    sweeps = PLAIN_SWEEPS.get(wl["name"], 12)
    vals, secs = [], []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(wl, sweeps, budget_s=args.cpu_budget)
        if i >= args.warmup:
            vals.append(cb["value"])
            secs.append(cb["sample_s"])
    value = statistics.mean(vals)
    cb["value"] = value
    return {
        "impl": "reference",
        "metric": "SVDs/s",
        "value": value,
        "unit": "SVD/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        # a step is one bounded sample (rounds of one sweep), timed on the host
        # cores; value extrapolates it to whole SVDs (cpu_baseline.sample)
        "ms_per_step": 1e3 * statistics.mean(secs),
        "step": "one bounded sample of the solve (cpu_baseline.sample); value = 1 / (sample time x the "
                "extrapolation factor)",
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["desc"], "path": "FP64 host oracle (reference arithmetic; the reference has "
                                                   "no CPU path)", "epsilon": wl["eps"],
                   "devices": "host cores only (rank 0); no GPU is used by this arm"},
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": "SVD/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="tall")
    ap.add_argument("--path", default="auto")
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-count", type=int, default=BATCH_COUNT)
    ap.add_argument("--no-plain-compare", action="store_true")
    ap.add_argument("--rates", default="50,200,500,1000,2000",
                    help="Poisson arrival rates (req/s) of the serve workload")
    ap.add_argument("--serve-count", type=int, default=2000, help="requests per rate of the serve workload")
    ap.add_argument("--serve-plain-sample", type=int, default=40)
    ap.add_argument("--serve-large-workers", type=int, default=0, help="0 = the serving core's default")
    ap.add_argument("--serve-large-path", type=int, default=2, choices=[0, 1, 2],
                    help="serve workload: path of the large requests (0 plain, 1 QR-preconditioned, 2 mixed)")
    ap.add_argument("--large-m", type=int, default=16384)
    ap.add_argument("--large-n", type=int, default=8192)
    ap.add_argument("--large-dir", default="")
    ap.add_argument("--sweep-mode", type=int, default=0, choices=[0, 1, 2, 3],
                    help="0: per-round kernels replayed from a graph, angle derived once per CTA; "
                         "1: persistent sweep kernel; 2: as 0 with programmatic dependent launch; "
                         "3: as 0 with every warp deriving the angle")
    ap.add_argument("--threads", type=int, default=0,
                    help="threads_per_block (reduction width T) of the config; 0 = the reference default 256")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the host-buffer leg (profiling runs: only the warm-up and timed solves launch)")
    ap.add_argument("--no-extras", action="store_true",
                    help="tall workload: skip the other-configuration sub-objects (other_configs)")
    ap.add_argument("--precond-inner", type=int, default=1, choices=[0, 1],
                    help="Jacobi stage of the QR-preconditioned path: 0 block-pair where it applies, 1 plain")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return 0

    import torch

    device = torch.device(f"cuda:{local}")
    torch.cuda.set_device(device)
    import jsvd
    jsvd.set_sweep_mode(args.sweep_mode)
    jsvd.precond_set_inner(args.precond_inner)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    # A rank that fails raises at once, without a further collective (the
    # others end in theirs: the launcher stops them, or the process group's
    # timeout does); ranks that succeed meet at the barrier.
    if args.workload == "batch":
        line = run_batch(args, rank, world, device)
    elif args.workload == "serve":
        line = run_serve(args, rank, world, device)
    elif args.workload == "large":
        line = run_large(args, rank, world, device)
    elif args.workload == "large_device":
        # the large graded/clustered matrix solved from device memory only
        # (no file pipeline): the form the kernel profiles are captured on
        path = args.path if args.path in ("mixed", "precond") else "mixed"
        res = run_large_device(args, device, path, steps=args.steps, warmup=args.warmup)
        line = {"metric": "SVDs/s", "value": res["value"], "unit": "SVD/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * res["s_per_svd"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, on device)",
                "config": {"workload": f"{args.large_m}x{args.large_n} FP64 graded + clustered sigma, device-resident",
                           "path": path}, **{k: v for k, v in res.items() if k not in ("value", "unit")}}
    else:
        line = run_ours(args, rank, world, device)
    if world > 1:
        torch.distributed.barrier()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
