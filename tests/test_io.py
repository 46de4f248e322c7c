"""The *.mat / *.txt stream formats (include/io.hpp) and the CLI's argument
handling, on CPU.

*.mat records are u64 rows | u64 columns | f64 values, big-endian, row-major
(reference include/io.hpp:40-51); the C++ codec must round-trip byte for byte
with the independent Python codec, reject truncated records with the
reference's messages, and print text with max_digits10 (exact round trip).
"""
import os
import subprocess

import numpy as np
import pytest

import matfile
from conftest import PKG, ROOT

DRIVER = os.path.join(ROOT, "tests", "cpp", "io_driver.cpp")
CLI = os.path.join(PKG, "jacobi-svd-b200")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = tmp_path_factory.mktemp("io") / "io_driver"
    subprocess.check_call(["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"),
                           "-I/usr/local/cuda/include", DRIVER, "-o", str(out), "-L", PKG, "-ljsvd",
                           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{PKG}"])
    return str(out)


def _mats(seed=0):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((3, 2)), np.arange(12.0).reshape(4, 3) - 5.5, np.array([[1e-300, -0.0]]),
            rng.standard_normal((1, 7)) * 1e200, np.array([[np.pi]])]


def run(driver, *args):
    return subprocess.run([driver, *map(str, args)], capture_output=True, text=True)


def test_mat_roundtrip_bytes(driver, tmp_path):
    src, dst = tmp_path / "a.mat", tmp_path / "b.mat"
    matfile.write(src, _mats())
    r = run(driver, "mat-copy", src, dst)
    assert r.returncode == 0, r.stdout
    assert dst.read_bytes() == src.read_bytes()
    r = run(driver, "stream-copy", src, tmp_path / "c.mat")
    assert r.returncode == 0 and "records 5" in r.stdout
    assert (tmp_path / "c.mat").read_bytes() == src.read_bytes()


def test_mat_to_txt_is_exact(driver, tmp_path):
    src, txt, back = tmp_path / "a.mat", tmp_path / "a.txt", tmp_path / "b.txt"
    mats = _mats(1)
    matfile.write(src, mats)
    assert run(driver, "mat-to-txt", src, txt).returncode == 0
    text = txt.read_text()
    blocks = [b for b in text.split("\n\n") if b.strip()]
    assert len(blocks) == len(mats)
    for blk, a in zip(blocks, mats):
        got = np.array([[float(x) for x in line.split()] for line in blk.strip().splitlines()])
        assert got.shape == a.shape and np.array_equal(got, a)
    assert run(driver, "txt-copy", txt, back).returncode == 0
    assert back.read_text() == text


@pytest.mark.parametrize("cut,msg", [(10, "Truncated *.mat header."), (16 + 8 * 5, "Truncated *.mat payload.")])
def test_truncated_mat(driver, tmp_path, cut, msg):
    src = tmp_path / "t.mat"
    data = matfile.encode(_mats()[:2])
    src.write_bytes(data[:cut])
    r = run(driver, "mat-copy", src, tmp_path / "o.mat")
    assert r.returncode == 1 and msg in r.stdout


def test_dispatch_refuses_oversized_claim_before_reserving(driver, tmp_path):
    """A record header that claims more payload than the file holds (here 1e12
    x 8 doubles) is refused as truncated before pinned memory is reserved."""
    import struct

    bad = tmp_path / "bad.mat"
    bad.write_bytes(struct.pack(">QQ", 10**12, 8) + b"\0" * 64)
    r = run(driver, "dispatch-count", bad, tmp_path / "unused")
    assert r.returncode == 1 and r.stdout.strip() == "error: Truncated *.mat payload while dispatch reading."


def test_txt_errors(driver, tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("1 2\n3\n")
    r = run(driver, "txt-copy", bad, tmp_path / "o.txt")
    assert r.returncode == 1 and "Inconsistent column count in text matrix block." in r.stdout
    bad.write_text("1 x\n")
    r = run(driver, "txt-copy", bad, tmp_path / "o.txt")
    assert r.returncode == 1 and "Invalid numeric token in text matrix row." in r.stdout


def test_empty_mat_file(driver, tmp_path):
    src = tmp_path / "e.mat"
    src.write_bytes(b"")
    assert run(driver, "mat-copy", src, tmp_path / "o.mat").returncode == 0
    assert (tmp_path / "o.mat").read_bytes() == b""


# ---- CLI (argument handling needs no GPU) -----------------------------------------

def cli(*args, cwd=None):
    return subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, cwd=cwd)


def test_cli_version_and_help():
    r = cli("--version")
    assert r.returncode == 0 and "sm_100a" in r.stdout
    r = cli("-h")
    assert r.returncode == 0 and "--layout-transpose-mode" in r.stdout and "--queue-capacity" in r.stdout


def test_cli_argument_errors(tmp_path):
    assert cli().returncode == 2
    r = cli(tmp_path / "missing.mat")
    assert r.returncode == 2 and "Input file does not exist" in r.stderr
    src = tmp_path / "a.mat"
    matfile.write(src, _mats())
    r = cli(src, "--epsilon", "-1")
    assert r.returncode == 2 and "must be a positive finite number" in r.stderr
    r = cli(src, "--max-sweeps", "x")
    assert r.returncode == 2 and "Invalid integer value for --max-sweeps." in r.stderr
    r = cli(src, "--bogus")
    assert r.returncode == 2 and "Unknown option: --bogus" in r.stderr
    r = cli(src, src)
    assert r.returncode == 2 and "must be different files" in r.stderr
    (tmp_path / "a.svd.mat").write_bytes(b"")
    r = cli(src)
    assert r.returncode == 2 and "Use --force to overwrite" in r.stderr
    r = cli(tmp_path / "noext", "--dry-run")
    assert r.returncode == 2


def test_cli_dry_run_defaults(tmp_path):
    src = tmp_path / "case.txt"
    src.write_text("1 2\n3 4\n")
    r = cli(src, "--dry-run", "-e", "1e-12", "-t", "128", "--layout-transpose-mode", "off")
    assert r.returncode == 0
    assert f"output          : {tmp_path / 'case.svd.txt'}" in r.stdout
    assert "epsilon         : 1e-12" in r.stdout
    assert "threads-per-blk : 128" in r.stdout and "layout-mode     : off" in r.stdout
    r = cli(src, tmp_path / "out", "--dry-run")
    assert f"output          : {tmp_path / 'out.txt'}" in r.stdout


@pytest.mark.gpu
def test_dispatch_reader_roundtrip(cuda_device, driver, tmp_path):
    """MatDispatchReader (pinned task buffers, needs a CUDA device) reads every
    record in order with the requested workspace; decoding them all and
    writing them back reproduces the input bytes."""
    src = tmp_path / "in.mat"
    matfile.write(src, _mats())
    out = tmp_path / "out.mat"
    r = subprocess.run([driver, "dispatch", str(src), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert out.read_bytes() == src.read_bytes()


# Property test of the *.mat codec: random record lists (empty ones and
# records with a zero dimension included) with NaN, infinities, subnormals,
# signed zeros and extreme values go through the C++ reader and writer
# unchanged, byte for byte and bit for bit.
from hypothesis import HealthCheck, given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402

_SPECIAL = st.sampled_from([0.0, -0.0, float("inf"), float("-inf"), float("nan"), 5e-324, -5e-324,
                            1.7976931348623157e308, -2.2250738585072014e-308])
_VALUE = st.one_of(st.floats(allow_nan=True, allow_infinity=True, width=64), _SPECIAL)


@st.composite
def _records(draw):
    out = []
    for _ in range(draw(st.integers(0, 5))):
        r, c = draw(st.integers(0, 6)), draw(st.integers(0, 6))
        vals = draw(st.lists(_VALUE, min_size=r * c, max_size=r * c))
        out.append(np.array(vals, dtype=np.float64).reshape(r, c))
    return out


@settings(derandomize=True, max_examples=40, deadline=None,
          suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(mats=_records())
def test_mat_codec_round_trip_property(driver, tmp_path_factory, mats):
    d = tmp_path_factory.mktemp("prop")
    src, dst = d / "in.mat", d / "out.mat"
    matfile.write(src, mats)
    for cmd in ("mat-copy", "stream-copy"):
        r = run(driver, cmd, src, dst)
        assert r.returncode == 0, r.stdout
        assert dst.read_bytes() == src.read_bytes(), cmd
    back = matfile.read(dst)
    assert len(back) == len(mats)
    for x, y in zip(back, mats):
        assert x.shape == y.shape and np.array_equal(x.view(np.uint64), y.view(np.uint64))


@st.composite
def _finite_records(draw):
    out = []
    for _ in range(draw(st.integers(1, 4))):
        r, c = draw(st.integers(1, 5)), draw(st.integers(1, 5))
        vals = draw(st.lists(st.one_of(st.floats(allow_nan=False, allow_infinity=False, width=64),
                                       st.sampled_from([0.0, -0.0, 5e-324, -1e-310, 1.7976931348623157e308])),
                             min_size=r * c, max_size=r * c))
        out.append(np.array(vals, dtype=np.float64).reshape(r, c))
    return out


@settings(derandomize=True, max_examples=30, deadline=None,
          suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(mats=_finite_records())
def test_txt_codec_round_trip_property(driver, tmp_path_factory, mats):
    """*.txt with finite values (subnormals and -0.0 included): the C++ reader
    and writer keep every bit (max_digits10 output), and a second pass writes
    the same bytes."""
    d = tmp_path_factory.mktemp("txtprop")
    src, mid, end = d / "in.txt", d / "mid.txt", d / "end.txt"
    src.write_text("\n".join("\n".join(" ".join(repr(float(x)) for x in row) for row in a) + "\n" for a in mats))
    assert run(driver, "txt-copy", src, mid).returncode == 0
    assert run(driver, "txt-copy", mid, end).returncode == 0
    assert end.read_bytes() == mid.read_bytes()
    blocks = [b for b in mid.read_text().split("\n\n") if b.strip()]
    assert len(blocks) == len(mats)
    for blk, a in zip(blocks, mats):
        got = np.array([[float(t) for t in ln.split()] for ln in blk.strip().splitlines()])
        assert got.shape == a.shape and np.array_equal(got.view(np.uint64), a.view(np.uint64))


def test_cli_reports_solver_failure_with_exit_1(tmp_path):
    """A solve that fails (here: no CUDA device) reaches the CLI through the
    serving core, the writer thread and the pipeline's exception path: exit
    code 1 and the reference's "Execution failed:" message
    (src/main.cpp:1289-1298)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("checks the failure path of a machine without a GPU")
    src = tmp_path / "in.mat"
    matfile.write(src, _mats())
    r = subprocess.run([CLI, str(src), str(tmp_path / "out.mat"), "-q"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1, (r.returncode, r.stderr)
    assert r.stderr.startswith("Execution failed: ") and "CUDA" in r.stderr


def test_policy_concepts_accept_user_policies(tmp_path):
    """io.hpp's MatrixInputPolicy / MatrixOutputPolicy concepts (reference
    include/io.hpp:630-661): the file policies satisfy them, a policy without
    flush does not (static_asserts), and a user-defined in-memory policy runs
    through the stream templates."""
    exe = tmp_path / "policy_driver"
    subprocess.check_call(["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"),
                           "-I/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "policy_driver.cpp"),
                           "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["3", "3", "1", "3", "5", "7"]


@pytest.fixture(scope="module")
def asan_driver(tmp_path_factory):
    """The io driver with the codec (csrc/io.cpp) compiled in under
    AddressSanitizer and UndefinedBehaviorSanitizer."""
    out = tmp_path_factory.mktemp("asan") / "io_asan"
    subprocess.check_call(["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined",
                           "-fno-sanitize-recover=all", "-fno-omit-frame-pointer",
                           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "csrc"),
                           "-I/usr/local/cuda/include", DRIVER, os.path.join(PKG, "csrc", "io.cpp"), "-o", str(out),
                           "-L/usr/local/cuda/lib64", "-lcudart"])
    return str(out)


def test_codec_clean_under_sanitizers(asan_driver, tmp_path):
    """Valid, special-valued, truncated and corrupt inputs through every codec
    command: results as in the plain build, no sanitizer report."""
    import struct

    matfile.write(tmp_path / "a.mat", _mats() + [np.zeros((0, 4)), np.array([[np.nan, np.inf, -0.0, 5e-324]])])
    (tmp_path / "t.txt").write_text("1 2 3\n4 5 6\n\n7.5\n")
    (tmp_path / "trunc.mat").write_bytes((tmp_path / "a.mat").read_bytes()[:-5])
    (tmp_path / "claim.mat").write_bytes(struct.pack(">QQ", 10**12, 8) + b"\0" * 64)
    (tmp_path / "huge.mat").write_bytes(struct.pack(">QQ", 2**62, 2**62))
    (tmp_path / "ragged.txt").write_text("1 2\n3\n")
    cases = [("mat-copy", "a.mat", 0), ("stream-copy", "a.mat", 0), ("mat-to-txt", "a.mat", 0),
             ("txt-copy", "t.txt", 0), ("mat-copy", "trunc.mat", 1), ("dispatch-count", "claim.mat", 1),
             ("mat-copy", "huge.mat", 1), ("txt-copy", "ragged.txt", 1)]
    for cmd, name, rc in cases:
        r = run(asan_driver, cmd, tmp_path / name, tmp_path / "out.bin")
        assert r.returncode == rc, (cmd, name, r.stdout, r.stderr[-800:])
        assert "Sanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-800:]
    assert (tmp_path / "out.bin").exists()


@settings(derandomize=True, max_examples=25, deadline=None,
          suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(mats=_records())
def test_mat_round_trip_under_sanitizers(asan_driver, tmp_path_factory, mats):
    d = tmp_path_factory.mktemp("asanprop")
    matfile.write(d / "in.mat", mats)
    r = run(asan_driver, "stream-copy", d / "in.mat", d / "out.mat")
    assert r.returncode == 0 and "Sanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-800:]
    assert (d / "out.mat").read_bytes() == (d / "in.mat").read_bytes()


def test_cli_option_syntax_like_the_reference(tmp_path):
    """Option forms the reference's parser accepts (src/main.cpp:925-1100):
    --name=value, --name value, -xVALUE, -x VALUE, clustered flags (-yq), and
    `--` ending the options; with the same argument errors (exit code 2)."""
    src = tmp_path / "c.txt"
    src.write_text("1 2\n3 4\n")
    for form in (["--epsilon=1e-12"], ["--epsilon", "1e-12"], ["-e1e-12"], ["-e", "1e-12"]):
        r = cli(src, *form, "--dry-run")
        assert r.returncode == 0 and "epsilon         : 1e-12" in r.stdout, (form, r.stderr)
    r = cli(src, "--max-sweeps=7", "-t64", "-yq", "--dry-run")
    assert r.returncode == 0 and "max-sweeps      : 7" in r.stdout and "threads-per-blk : 64" in r.stdout
    assert "force-overwrite : true" in r.stdout
    for args, msg in ((["--force=1"], "Option --force does not take a value."),
                      (["-z"], "Unknown short option: -z"),
                      (["--dry-run", "-e"], "Missing value for --epsilon.")):
        r = cli(src, *args, "--dry-run") if args[-1] != "-e" else cli(src, *args)
        assert r.returncode == 2 and msg in r.stderr, (args, r.stderr)
    # after `--` everything is positional: here the output path
    r = cli(src, "--dry-run", "--", str(tmp_path / "--out.txt"))
    assert r.returncode == 0 and f"output          : {tmp_path / '--out.txt'}" in r.stdout


def test_cli_verify_checks_a_result_file(tmp_path):
    """--verify IN RESULT prints each testcase's rho_A, rho_U, rho_V (the
    reference design's validation metrics) for a result file made by any
    implementation - here the reference CLI's own output - without solving."""
    import json

    import oracle as O

    inp = os.path.join(ROOT, "tests", "golden", "pipeline_in.mat")
    ref_out = os.path.join(ROOT, "tests", "golden", "pipeline_ref_out.mat")
    r = subprocess.run([CLI, inp, "--verify", ref_out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    recs = [json.loads(line) for line in r.stdout.splitlines()]
    mats, res = matfile.read(inp), matfile.read(ref_out)
    assert [d["index"] for d in recs] == list(range(len(mats)))
    for d, a in zip(recs, mats):
        k = d["index"]
        exp = O.residuals(a, res[3 * k], res[3 * k + 1].ravel(), res[3 * k + 2])
        assert (d["rows"], d["columns"]) == a.shape and d["rho_A"] < 1e-13
        for key in ("rho_A", "rho_U", "rho_V"):
            assert abs(d[key] - exp[key]) <= 1e-14 + 1e-10 * exp[key]
    # a tampered U value shows in that testcase's rho_A
    bad = [x.copy() for x in res]
    bad[3 * 6][2, 1] += 1e-3
    matfile.write(tmp_path / "bad.mat", bad)
    recs = [json.loads(line) for line in subprocess.run([CLI, inp, "--verify", tmp_path / "bad.mat"],
                                                          capture_output=True, text=True, check=True).stdout.splitlines()]
    assert recs[6]["rho_A"] > 1e-5 and all(d["rho_A"] < 1e-13 for d in recs if d["index"] != 6)
    # a record missing, and records in the wrong order
    matfile.write(tmp_path / "short.mat", res[:-1])
    r = subprocess.run([CLI, inp, "--verify", tmp_path / "short.mat"], capture_output=True, text=True)
    assert r.returncode == 1 and "expected 3 (U, Sigma, V) for each of the 12 testcases" in r.stderr
    matfile.write(tmp_path / "swapped.mat", [res[1], res[0]] + res[2:])
    r = subprocess.run([CLI, inp, "--verify", tmp_path / "swapped.mat"], capture_output=True, text=True)
    assert r.returncode == 1 and "Testcase[0] result shapes do not match the input." in r.stderr
    r = subprocess.run([CLI, inp, "--verify", tmp_path / "missing.mat"], capture_output=True, text=True)
    assert r.returncode == 2 and "Input file does not exist" in r.stderr
