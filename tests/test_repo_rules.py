"""Where the oracle may be used, and what committed files may refer to (host,
no GPU).

The oracle is test infrastructure: the product (the package) never imports
it, and bench.py calls it only in the functions that time the CPU baseline.
Committed sources do not refer to the scratch folder `_work/`.
"""
import ast
import os
import re
import subprocess

from conftest import PKG, ROOT

BENCH_ORACLE_FUNCTIONS = {"cpu_baseline", "batch_cpu_baseline"}


def _tracked_files():
    out = subprocess.run(["git", "ls-files"], cwd=ROOT, capture_output=True, text=True)
    if out.returncode != 0:
        return []
    return [os.path.join(ROOT, f) for f in out.stdout.splitlines()]


def _imports_oracle(node) -> bool:
    if isinstance(node, ast.Import):
        return any(a.name.split(".")[0] == "oracle" for a in node.names)
    if isinstance(node, ast.ImportFrom):
        return (node.module or "").split(".")[0] == "oracle"
    return False


def test_package_never_imports_the_oracle():
    for name in os.listdir(PKG):
        if name.endswith(".py"):
            tree = ast.parse(open(os.path.join(PKG, name)).read())
            assert not any(_imports_oracle(n) for n in ast.walk(tree)), name


def test_bench_imports_the_oracle_only_for_the_cpu_baseline():
    tree = ast.parse(open(os.path.join(ROOT, "bench.py")).read())
    assert not any(_imports_oracle(n) for n in tree.body), "module-level import of the oracle"
    users = set()
    for fn in ast.walk(tree):
        if isinstance(fn, ast.FunctionDef):
            for stmt in fn.body:  # direct statements: nested helpers would show up as their own function
                if any(_imports_oracle(n) for n in ast.walk(stmt)):
                    users.add(fn.name)
    assert users and users <= BENCH_ORACLE_FUNCTIONS, users


def test_no_committed_file_refers_to_the_scratch_folder():
    pattern = re.compile(r"(?<![A-Za-z0-9])_work\b")
    offenders = []
    for path in _tracked_files():
        # .gitignore lists the folder; this file names it to look for it; the
        # review files are written by the reviewers, not by this repository
        if os.path.basename(path) in (".gitignore", "VERDICT.md", "ADVICE.md") or os.path.abspath(
            path
        ) == os.path.abspath(__file__):
            continue
        if not os.path.isfile(path):
            continue
        try:
            text = open(path, encoding="utf-8").read()
        except UnicodeDecodeError:
            continue
        if pattern.search(text):
            offenders.append(os.path.relpath(path, ROOT))
    assert offenders == [], offenders


def test_sources_name_no_build_notes_or_machine_paths():
    """Code and comments stand on their own: no source names the build's
    notes, its benchmark descriptor, the remote-run tool or this machine's
    paths.  The oracle's Makefile is the one recipe that reads the reference
    where it lies."""
    pattern = re.compile(r"SURVEY|DESIGN\.md|BASELINE|VERDICT|ADVICE|north_star|gpurun|/root/|configs\[")
    skip_suffixes = (".md", ".json", ".gitignore", ".gpurunignore")
    allowed = {("oracle/Makefile", "/root/")}
    offenders = []
    for path in _tracked_files():
        rel = os.path.relpath(path, ROOT)
        if rel.endswith(skip_suffixes) or os.path.abspath(path) == os.path.abspath(__file__):
            continue
        if not os.path.isfile(path):
            continue
        try:
            text = open(path, encoding="utf-8").read()
        except UnicodeDecodeError:
            continue
        for m in pattern.finditer(text):
            if (rel, m.group(0)) not in allowed:
                offenders.append((rel, m.group(0)))
    assert offenders == [], offenders
