"""The reference's C++ program API on the B200 library.

* tests/transitive_closure.cpp of the reference, compiled unchanged against
  parallel-ra_b200/cxx/src (build.py), must print the reference's relation sizes.
* tests/cxx/api_driver.cpp runs the TC and SG builders of oracle/programs.h
  through the C++ classes and must reproduce the golden history and rows.
"""
import os
import runpy
import subprocess

import numpy as np
import pytest

import parallel_ra_b200 as P
from conftest import GOLDEN, ROOT, golden_input, load_golden, rows_digest

PKG = os.path.join(ROOT, "parallel-ra_b200")
TC_BIN = os.path.join(PKG, "cxx", "bin", "TC")
DRIVER_SRC = os.path.join(ROOT, "tests", "cxx", "api_driver.cpp")


def build_driver(tmp):
    out = os.path.join(tmp, "api_driver")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(PKG, "cxx", "src"), "-I", os.path.join(ROOT, "include"),
                    DRIVER_SRC, "-o", out, "-L", PKG, "-lparallel_ra", "-lra_b200", f"-Wl,-rpath,{PKG}"], check=True)
    return out


def test_api_driver_compiles(tmp_path):
    assert os.path.exists(build_driver(str(tmp_path)))


def test_reference_tc_program_was_built_unchanged():
    if not os.path.exists(TC_BIN):
        pytest.skip("reference program binary not built here (needs the reference tree at build time)")
    out = subprocess.run(["nm", "-D", "--undefined-only", TC_BIN], capture_output=True, text=True).stdout
    assert "LIE7execute" in out and "relation" in out


def tc_layout(tmp):
    """cwd with ../data/g5955/path_2_1_2 (the empty T relation TC loads by relative path)."""
    run = os.path.join(tmp, "run")
    os.makedirs(run)
    P.datagen.write_empty_relation(os.path.join(tmp, "data", "g5955", "path_2_1_2"))
    return run


@pytest.mark.gpu
@pytest.mark.parametrize("fixture,count", [("g5955", 10), ("g13236", 573)])
def test_unchanged_transitive_closure_program(tmp_path, fixture, count):
    if not os.path.exists(TC_BIN):
        pytest.skip("reference program binary not built")
    run = tc_layout(str(tmp_path))
    edge = os.path.join(GOLDEN, f"{fixture}_edge_2_1_2")
    r = subprocess.run([TC_BIN, edge], cwd=run, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    g = load_golden(f"{fixture}_tc")["relations"]["G"]["count"]
    assert f"T: {{2}}. ({count} total facts)" in r.stdout
    assert f"G: {{2}}. ({g} total facts)" in r.stdout
    assert f"Total facts across all relations {count + g}" in r.stdout


@pytest.mark.gpu
def test_unchanged_transitive_closure_bad_args():
    if not os.path.exists(TC_BIN):
        pytest.skip("reference program binary not built")
    r = subprocess.run([TC_BIN], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Usage" in r.stdout


@pytest.mark.gpu
def test_unchanged_transitive_closure_missing_file(tmp_path):
    if not os.path.exists(TC_BIN):
        pytest.skip("reference program binary not built")
    run = tc_layout(str(tmp_path))
    r = subprocess.run([TC_BIN, os.path.join(str(tmp_path), "nope")], cwd=run, capture_output=True, text=True,
                       timeout=60)
    assert r.returncode != 0 and "I/O error" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("id_order", ["emission", "reference"])
@pytest.mark.parametrize("name", ["g13236_tc", "er200_tc", "er2000_tc", "tree256_sg", "tree1024_sg"])
def test_cxx_api_matches_goldens(tmp_path, name, id_order):
    tmp = str(tmp_path)
    drv = build_driver(tmp)
    case = load_golden(name)
    rows = golden_input(case)
    edge = os.path.join(tmp, "edge")
    P.datagen.write_relation(edge, rows)
    empty = os.path.join(tmp, "empty")
    P.datagen.write_empty_relation(empty)
    out = os.path.join(tmp, "out")
    env = dict(os.environ, RA_ID_ORDER=id_order)
    r = subprocess.run([drv, case["program"], edge, empty, out], capture_output=True, text=True, timeout=600,
                       env=env)
    assert r.returncode == 0, r.stderr
    hist = []
    for line in open(os.path.join(out, "history.txt")):
        a = line.split()
        if a[0] == "scc":
            hist.append([int(a[1]), []])
        else:
            hist[-1][1].append([int(a[0]), int(a[1])])
    assert hist == case["history"]
    for rname, exp in case["relations"].items():
        got = np.fromfile(os.path.join(out, rname + ".bin"), dtype="<u8").reshape(-1, exp["arity"] + 1)
        assert got.shape[0] == exp["count"]
        if id_order == "reference":
            assert rows_digest(got) == exp["sha256"], rname
        else:
            assert rows_digest(np.ascontiguousarray(got[:, :-1])) == exp["data_sha256"], rname


def _python_blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return [b.split("```", 1)[0].lstrip("\n") for b in text.split("```python")[1:]]


def test_integration_md_quotes_the_example_files():
    """INTEGRATION.md's Python examples are these test files, verbatim."""
    blocks = _python_blocks()
    for name in ("integration_ctypes_example.py", "integration_batch_example.py"):
        with open(os.path.join(ROOT, "tests", name)) as f:
            assert f.read() in blocks, name


@pytest.mark.gpu
def test_integration_ctypes_example_runs():
    """The ctypes example (quoted in INTEGRATION.md) computes TC of a 2-edge chain (3 pairs)."""
    cwd = os.getcwd()
    os.chdir(ROOT)
    try:
        env = runpy.run_path(os.path.join(ROOT, "tests", "integration_ctypes_example.py"))
    finally:
        os.chdir(cwd)
    assert env["f"].value == 3


@pytest.mark.gpu
def test_integration_batch_example_runs():
    """The batching example (quoted in INTEGRATION.md) runs and its assertion holds."""
    env = runpy.run_path(os.path.join(ROOT, "tests", "integration_batch_example.py"))
    assert len(env["results"]) == 3
