"""Pipeline extensions on the host (no GPU): the per-testcase residual record
(include/pipeline_ext.hpp) and the CLI's --residual-report flag.

The record carries what the reference's design asks a test report to hold
((m, n), epsilon, max_sweeps, sweeps, rho_A, rho_U, rho_V;
tex/sections/03-gpu-parallel-reduction.tex:53-58), one JSON object per line.
"""
import json
import os
import subprocess

import pytest

import matfile
from conftest import PKG, ROOT

DRIVER = os.path.join(ROOT, "tests", "cpp", "pipeline_driver.cpp")
CLI = os.path.join(PKG, "jacobi-svd-b200")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = tmp_path_factory.mktemp("pipe") / "pipeline_driver"
    subprocess.check_call(["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), DRIVER, "-o", str(out),
                           "-L", PKG, "-ljsvd", f"-Wl,-rpath,{PKG}"])
    return str(out)


def test_record_json_round_trips(driver):
    lines = subprocess.run([driver, "record-json"], capture_output=True, text=True, check=True).stdout.splitlines()
    assert len(lines) == 2
    r = json.loads(lines[0])
    assert r == {"index": 7, "rows": 300, "columns": 260, "epsilon": 1e-14, "max_sweeps": 128, "sweeps": 13,
                 "rho_A": 3.0000000000000001e-15, "rho_U": 1.25e-13, "rho_V": 0.1}
    r = json.loads(lines[1])
    assert r["rho_A"] is None and r["rho_U"] == -1.0


def test_report_path_setting(driver, tmp_path):
    p = str(tmp_path / "r.jsonl")
    out = subprocess.run([driver, "report-path", p], capture_output=True, text=True, check=True).stdout
    assert out.splitlines() == [p, "[]"]


def _cli(*args):
    return subprocess.run([CLI, *map(str, args)], capture_output=True, text=True)


def test_cli_residual_report_flag(tmp_path):
    src = tmp_path / "case.mat"
    matfile.write(src, [[[1.0, 2.0], [3.0, 4.0]]])
    r = _cli(src, "--dry-run")
    assert r.returncode == 0 and "residual-report : off" in r.stdout
    rep = tmp_path / "res.jsonl"
    r = _cli(src, "--dry-run", "--residual-report", rep)
    assert r.returncode == 0 and f"residual-report : {rep}" in r.stdout
    for clash in (src, tmp_path / "case.svd.mat"):
        r = _cli(src, "--dry-run", "--residual-report", clash)
        assert r.returncode == 2 and "--residual-report must name a file other than" in r.stderr
    r = _cli("-h")
    assert "--residual-report PATH" in r.stdout


def test_last_run_stats_are_zero_before_a_run(driver):
    out = subprocess.run([driver, "last-run"], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["0"] * 7
