"""The C structs of include/jsvd.h and their ctypes mirrors in jsvd.py agree
field by field (offsets and total size), so an FFI caller using the ctypes
binding reads and writes the same bytes as C.  A C program generated from the
ctypes field names is compiled with gcc against the header (a renamed field
fails to compile) and prints sizeof and every offsetof.  No GPU."""
import ctypes
import os
import subprocess

import pytest

import jsvd
from conftest import ROOT

PAIRS = {
    "jsvd_config": jsvd.Config,
    "jsvd_autotune_report": jsvd.AutoTuneReport,
    "jsvd_plain_stats": jsvd.PlainStats,
    "jsvd_residual_report": jsvd.ResidualReport,
    "jsvd_batch_tuning": jsvd.BatchTuning,
    "jsvd_batch_autotune_report": jsvd.BatchAutotuneReport,
    "jsvd_blockpair_stats": jsvd.BlockPairStats,
    "jsvd_batch_stats": jsvd.BatchStats,
    "jsvd_blocked_stats": jsvd.BlockedStats,
    "jsvd_precond_stats": jsvd.PrecondStats,
    "jsvd_server_options": jsvd.ServerOptions,
    "jsvd_server_stats": jsvd.ServerStats,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    d = tmp_path_factory.mktemp("layout")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "jsvd.h"', "int main(void) {"]
    for cname, cls in PAIRS.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{cname}.{field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                           "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.splitlines())}


@pytest.mark.parametrize("cname", sorted(PAIRS))
def test_struct_layout_matches_ctypes(c_layout, cname):
    cls = PAIRS[cname]
    assert c_layout[cname] == ctypes.sizeof(cls), f"sizeof({cname})"
    for field, _ in cls._fields_:
        assert c_layout[f"{cname}.{field}"] == getattr(cls, field).offset, f"{cname}.{field}"
