"""Regenerates csrc/mixed_tuning_table.h, the blocked mixed-precision path's
built-in choices by matrix width, from timings on this machine's GPU.

    python jacobi-svd-cuda_b200/mixed_autotune.py --out jacobi-svd-cuda_b200/csrc/mixed_tuning_table.h

For each width n of --shapes (m x n, default 4n rows) it times solves of a
seeded A = U diag(sigma) V^T (Haar U and V, sigma geometric from 1 to 1e-6,
as in the config-2 input; generated on the GPU), epsilon 1e-14, through
jsvd_mixed_svd_device, over a grid of the tunable options:
  * tensor-core sweep cap x inner sweeps of the block eigen-solve, then
  * the Gram row splits for the best pair.
A candidate counts only if its sigma is within 1e-12 normwise of the
analytic sigma.  Each candidate runs --reps times after one warm-up solve;
the minimum is kept.  A candidate replaces the library's current choice for
that width only when it is more than 2% faster.  Entry i of the table covers
widths up to shape i's width (the last covers all).  Rebuild the library
(make) after writing.
"""
from __future__ import annotations

import argparse
import datetime
import os
import re
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

TC_CAPS = (0, 3, 4, 6, 10)
INNER = (1, 2)
SPLITS = (0, 2, 4, 8, 16, 32)
GATE = 1e-12


def render_table(entries: list[tuple[int, int, int, int]], notes: list[str], meta: dict) -> str:
    """Text of mixed_tuning_table.h: entries (max_cols, tc_max_sweeps,
    inner_sweeps, gram_splits) in lookup order, the last with max_cols 0."""
    lines = [
        "/* Built-in choices of the blocked mixed-precision path by matrix width:",
        " * {largest column count the entry covers (0 = any), tensor-core sweep cap,",
        " * inner sweeps of the block eigen-solve, Gram row splits (0 = automatic)}.",
        " * The first entry whose column bound covers the input applies.",
        " *",
        f" * Generated by jacobi-svd-cuda_b200/mixed_autotune.py on {meta['device']},",
        f" * {meta['date']}: {meta['workload']}; {meta['reps']} timed solves per",
        " * candidate after a warm-up, minimum kept; candidates with sigma off by",
        " * more than 1e-12 normwise rejected; a candidate replaces the previous",
        " * choice only when it is more than 2% faster.",
        " *",
    ]
    lines += [" * " + n for n in notes]
    lines += [" */", "#pragma once", "", "#define JSVD_MIXED_TUNING_TABLE \\"]
    lines.append("    { " + ", ".join("{%d, %d, %d, %d}" % e for e in entries) + " }")
    return "\n".join(lines) + "\n"


def parse_table(text: str) -> list[tuple[int, int, int, int]]:
    """Entries of a mixed_tuning_table.h text."""
    m = re.search(r"#define JSVD_MIXED_TUNING_TABLE \\\s*\{(.*)\}", text, flags=re.S)
    if not m:
        raise ValueError("no JSVD_MIXED_TUNING_TABLE")
    ents = [tuple(int(x) for x in e.split(",")) for e in re.findall(r"\{([^{}]*)\}", m.group(1))]
    if not ents or any(len(e) != 4 for e in ents):
        raise ValueError("entries must have four integers")
    if ents[-1][0] != 0:
        raise ValueError("the last entry must cover every width (max_cols 0)")
    return ents


def test_matrix(m: int, n: int, device):
    """The seeded test input on the GPU (row-major FP64) and its sigma."""
    import numpy as np
    import torch

    sig = np.geomspace(1.0, 1e-6, n)
    g = torch.Generator(device=device)
    g.manual_seed(1000 + n)
    qu, ru = torch.linalg.qr(torch.randn((m, n), generator=g, dtype=torch.float64, device=device))
    qu *= torch.sign(torch.diagonal(ru))[None, :]
    qv, rv = torch.linalg.qr(torch.randn((n, n), generator=g, dtype=torch.float64, device=device))
    qv *= torch.sign(torch.diagonal(rv))[None, :]
    qu *= torch.from_numpy(sig).to(device)[None, :]
    return (qu @ qv.T).contiguous(), sig


def time_candidate(da, m: int, n: int, sig, outs, opts: dict, reps: int) -> tuple[float, float]:
    """(best ms, normwise sigma error) of the mixed solve with `opts`."""
    import numpy as np
    import torch

    import jsvd

    du, ds, dv = outs
    cfg = jsvd.default_config(epsilon=1e-14)
    jsvd.mixed_set_options(**opts)
    try:
        best = float("inf")
        for i in range(reps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            jsvd.mixed_svd_device(da.data_ptr(), m, n, du.data_ptr(), ds.data_ptr(), dv.data_ptr(), cfg)
            torch.cuda.synchronize()
            if i > 0:
                best = min(best, (time.perf_counter() - t0) * 1e3)
        got = np.sort(ds.cpu().numpy())[::-1]
        err = float(np.max(np.abs(got - np.sort(sig)[::-1])) / sig.max())
    finally:
        jsvd.mixed_set_options(None)
    return best, err


def tune_shape(m: int, n: int, reps: int = 2, tc_caps=TC_CAPS, inner=INNER, splits=SPLITS, device=None):
    """Best (tc_max_sweeps, inner_sweeps, gram_splits) for an m x n input and
    the timings behind it: a dict with 'best', 'best_ms', 'default_ms',
    'tried', 'rejected'."""
    import torch

    import jsvd

    device = device or torch.device("cuda", torch.cuda.current_device())
    da, sig = test_matrix(m, n, device)
    outs = (torch.empty((m, n), dtype=torch.float64, device=device), torch.empty(n, dtype=torch.float64, device=device),
            torch.empty((n, n), dtype=torch.float64, device=device))
    tried, rejected, results = 0, 0, {}
    for cap in tc_caps:
        for inn in inner:
            ms, err = time_candidate(da, m, n, sig, outs, dict(tc_max_sweeps=cap, inner_sweeps=inn, gram_splits=0),
                                     reps)
            tried += 1
            if err > GATE:
                rejected += 1
                continue
            results[(cap, inn, 0)] = ms
    if not results:
        raise RuntimeError(f"no candidate met the accuracy gate for {m} x {n}")
    cap, inn, _ = min(results, key=results.get)
    for sp in splits:
        if sp == 0:
            continue
        ms, err = time_candidate(da, m, n, sig, outs, dict(tc_max_sweeps=cap, inner_sweeps=inn, gram_splits=sp), reps)
        tried += 1
        if err > GATE:
            rejected += 1
            continue
        results[(cap, inn, sp)] = ms
    best = min(results, key=results.get)
    default_ms, _ = time_candidate(da, m, n, sig, outs, {}, reps)
    r = jsvd.mixed_resolved_options(n)
    current = (int(r.tc_max_sweeps), int(r.inner_sweeps), int(r.gram_splits))
    if results[best] > default_ms / 1.02:  # not clearly faster: keep the current choice
        best, best_ms = current, default_ms
    else:
        best_ms = results[best]
    return {"best": best, "best_ms": best_ms, "default_ms": default_ms, "tried": tried, "rejected": rejected}


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--shapes", default="1024x256,2048x512,4096x1024,8192x2048,8192x4096",
                    help="m x n list, narrowest first; entry i covers widths up to shape i's")
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args()
    import torch

    shapes = [tuple(int(v) for v in s.split("x")) for s in args.shapes.split(",")]
    if any(m < n or n < 128 for m, n in shapes) or [n for _, n in shapes] != sorted(n for _, n in shapes):
        raise SystemExit("shapes must be m x n with m >= n >= 128, in increasing n")
    entries, notes = [], ["width: shape, candidates tried (rejected), ms with the previous table -> chosen"]
    for i, (m, n) in enumerate(shapes):
        r = tune_shape(m, n, args.reps)
        cap, inn, sp = r["best"]
        entries.append((n if i + 1 < len(shapes) else 0, cap, inn, sp))
        notes.append(f"  {n}: {m} x {n}, {r['tried']} ({r['rejected']}), {r['default_ms']:.1f} -> {r['best_ms']:.1f}")
        print(notes[-1], flush=True)
    meta = {"device": torch.cuda.get_device_name(0), "date": datetime.date.today().isoformat(),
            "workload": "A = U diag(sigma) V^T, Haar U and V, sigma geometric 1 .. 1e-6, epsilon 1e-14",
            "reps": args.reps}
    text = render_table(entries, notes, meta)
    parse_table(text)
    with open(args.out, "w") as f:
        f.write(text)
    print(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())
