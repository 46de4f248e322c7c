"""Regenerates csrc/batch_tuning_table.h, the batched solver's built-in launch
shapes, from jsvd_batch_autotune run on this machine's GPU.

    python jacobi-svd-cuda_b200/batch_autotune.py --out jacobi-svd-cuda_b200/csrc/batch_tuning_table.h

It also times every size class that thread-block clusters can take, once
with one CTA per matrix and once with a cluster per matrix, and records the
choice (JSVD_BATCH_CLUSTER_CLASSES).  The timed workload is the mixed-size
batch (m ~ U{16..256}, n ~ U{8..m}, A = U diag(sigma) V^T with Haar factors,
sigma log-uniform in [1/kappa, 1], kappa log-uniform in [1e1, 1e6], stored as
FP32; sigma and V computed, epsilon 1e-14).  Rebuild the library (make) after
writing the table.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

CLASS_NAMES = [
    "A and V in <= 48 KiB of shared memory",
    "A and V in <= 100 KiB of shared memory",
    "A and V in <= ~226 KiB of shared memory",
    "A in shared memory, V in global memory",
    "A and V in global memory",
]


# Size classes whose members a thread-block cluster can take (bit c = class c).
CLUSTER_CAPABLE = (1 << 2) | (1 << 3) | (1 << 4)


def choose_cluster_mask(single_ms: list, cluster_ms: list, members: list, previous: int) -> int:
    """Per cluster-capable class, clusters or one CTA per matrix: the previous
    choice stays unless the other is more than 2% faster (a class without
    members keeps it)."""
    mask = previous & CLUSTER_CAPABLE
    for c in range(5):
        if not (CLUSTER_CAPABLE >> c) & 1 or members[c] == 0:
            continue
        on = bool((previous >> c) & 1)
        t_prev, t_other = (cluster_ms[c], single_ms[c]) if on else (single_ms[c], cluster_ms[c])
        if t_other < 0.98 * t_prev:
            mask ^= 1 << c
    return mask


def render_table(report: dict, meta: dict, cluster: dict) -> str:
    """Text of batch_tuning_table.h for an autotune report given as a dict of
    per-class lists (best, builtin, best_ms, builtin_ms, members, sampled,
    candidates; best/builtin entries are (threads, ctas_per_sm, max_ctas)) and
    the cluster choice (mask, single_ms, cluster_ms per class, and a line
    saying how they were measured)."""
    lines = [
        "/* Built-in launch shapes of the batched solver, one entry per size class:",
        " * {threads per CTA, persistent CTAs per SM, grid cap (0 = none)}.",
        " *",
        f" * Generated by jacobi-svd-cuda_b200/batch_autotune.py on {meta['device']}",
        f" * ({meta['sms']} SMs), {meta['date']}, from jsvd_batch_autotune over {meta['workload']};",
        f" * {meta['reps']} runs per shape, L2 flushed before each, minimum kept.  A shape",
        " * replaces the previous built-in one only when it is more than 2% faster.",
        " *",
        " * class: members timed / in batch, shapes tried, ms previous -> chosen",
    ]
    for c, name in enumerate(CLASS_NAMES):
        if report["members"][c] == 0:
            lines.append(f" *   {c} ({name}): no members, shape kept")
        else:
            lines.append(
                f" *   {c} ({name}): {report['sampled'][c]} / {report['members'][c]}, "
                f"{report['candidates'][c]} shapes, {report['builtin_ms'][c]:.2f} -> {report['best_ms'][c]:.2f}")
    lines += [
        " *",
        " * CTAs per matrix: the classes whose bit is set in JSVD_BATCH_CLUSTER_CLASSES",
        " * are solved by a thread-block cluster per matrix (2, 4 or 8 CTAs, the",
        " * smallest that holds it), the others by one CTA per matrix; a class goes",
        " * over only when that is more than 2% faster.",
        f" * {cluster['note']}",
        " * class: ms one CTA per matrix, ms clusters -> chosen",
    ]
    for c in range(5):
        if (CLUSTER_CAPABLE >> c) & 1:
            choice = "clusters" if (cluster["mask"] >> c) & 1 else "one CTA"
            lines.append(f" *   {c}: {cluster['single_ms'][c]:.1f}, {cluster['cluster_ms'][c]:.1f} -> {choice}")
    lines += [" */", "#pragma once", "", "#define JSVD_BATCH_TUNING_TABLE \\"]
    ents = []
    for c in range(5):
        t = report["best"][c] if report["members"][c] > 0 else report["builtin"][c]
        ents.append("{%d, %d, %d}" % tuple(t))
    lines.append("    { " + ", ".join(ents) + " }")
    lines += ["", "#define JSVD_BATCH_CLUSTER_CLASSES 0x%x" % cluster["mask"]]
    return "\n".join(lines) + "\n"


def parse_cluster_mask(text: str) -> int:
    """The JSVD_BATCH_CLUSTER_CLASSES mask of a table header."""
    m = re.search(r"#define\s+JSVD_BATCH_CLUSTER_CLASSES\s+(0x[0-9a-fA-F]+|\d+)", text)
    if m is None:
        raise ValueError("no JSVD_BATCH_CLUSTER_CLASSES in the table")
    return int(m.group(1), 0)


def time_cluster_choice(b, cfg, reps: int, device) -> tuple[list, list]:
    """Per-class device ms (mean of reps, L2 flushed before each) of the whole
    batch with every cluster-capable class on clusters, and with none."""
    import torch

    import jsvd

    flush = torch.empty(256 << 18, dtype=torch.float32, device=device)
    out = []
    old = jsvd.batch_set_cluster_classes(0)
    try:
        for mask in (0, CLUSTER_CAPABLE):
            jsvd.batch_set_cluster_classes(mask)
            b.solve(cfg)
            jsvd.batch_stats_reset()
            for _ in range(reps):
                flush.zero_()
                b.solve(cfg)
            st = jsvd.batch_stats()
            out.append([x / max(1, st.calls) for x in st.class_ms])
    finally:
        jsvd.batch_set_cluster_classes(old)
    return out[0], out[1]


def parse_table(text: str) -> list[tuple[int, int, int]]:
    """The five (threads, ctas_per_sm, max_ctas) entries of a table header."""
    body = text.split("#define JSVD_BATCH_TUNING_TABLE", 1)[1]
    ents = re.findall(r"\{\s*(\d+)\s*,\s*(\d+)\s*,\s*(\d+)\s*\}", body)
    if len(ents) != 5:
        raise ValueError(f"expected 5 entries, found {len(ents)}")
    return [tuple(int(x) for x in e) for e in ents]


def report_dict(rep) -> dict:
    def tun(arr):
        return [(t.threads, t.ctas_per_sm, t.max_ctas) for t in arr]

    return {
        "best": tun(rep.best), "builtin": tun(rep.builtin),
        "best_ms": list(rep.best_ms), "builtin_ms": list(rep.builtin_ms),
        "members": list(rep.members), "sampled": list(rep.sampled), "candidates": list(rep.candidates),
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=" ".join(__doc__.split("\n\n")[0].split()))
    ap.add_argument("--out", required=True, help="path of the table header to write")
    ap.add_argument("--json", help="also write the report as JSON here")
    ap.add_argument("--count", type=int, default=20000, help="matrices in the timed batch")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--sample", type=int, default=0, help="matrices timed per class (0 = all)")
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args(argv)

    import torch

    import jsvd
    import workloads as W

    if not torch.cuda.is_available():
        raise SystemExit("batch_autotune needs a CUDA device")
    device = torch.device("cuda:0")
    torch.cuda.set_device(device)
    mats = W.batch_workload_torch(args.count, seed=args.seed, device=device)
    b = jsvd.DeviceBatch(mats, device, f32=True, want_u=False, want_v=True)
    torch.cuda.synchronize(device)
    cfg = jsvd.default_config(epsilon=1e-14)
    rep = report_dict(b.autotune(cfg, sample=args.sample, reps=args.reps))
    previous = (1 << 3) | (1 << 4)  # the library's default when a table names no choice
    if os.path.exists(args.out):
        try:
            previous = parse_cluster_mask(open(args.out).read())
        except ValueError:
            pass
    single_ms, cluster_ms = time_cluster_choice(b, cfg, max(args.reps, 3), device)
    props = torch.cuda.get_device_properties(device)
    meta = {
        "device": props.name, "sms": props.multi_processor_count,
        "date": datetime.date.today().isoformat(), "reps": args.reps,
        "workload": f"{args.count} FP32-stored matrices m ~ U{{16..256}}, n ~ U{{8..m}} (seed {args.seed})",
    }
    cluster = {"mask": choose_cluster_mask(single_ms, cluster_ms, rep["members"], previous),
               "single_ms": single_ms, "cluster_ms": cluster_ms,
               "note": f"Timed on the same batch, all classes, mean of {max(args.reps, 3)} runs, L2 flushed."}
    text = render_table(rep, meta, cluster)
    with open(args.out, "w") as f:
        f.write(text)
    if args.json:
        with open(args.json, "w") as f:
            json.dump({"meta": meta, "report": rep, "cluster": cluster}, f, indent=1)
    sys.stdout.write(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())
