"""C++ drop-in tests: programs written against the reference's C++
interfaces, linked against libhytgraph.so."""
from __future__ import annotations

import subprocess

import pytest

from conftest import BUILD, ROOT, compile_cpp, run_cpp


def test_dropin_host_classes():
    exe = compile_cpp("drop_in_tests", ["drop_in_tests.cpp"])
    r = run_cpp(exe, "cpu")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "checks passed (cpu)" in r.stdout


def test_transfer_and_scheduling_parity_with_reference():
    ref = ROOT / "oracle" / "_ref" / "libhytref.so"
    if not ref.exists():
        pytest.skip("oracle/_ref (the reference's compiled classes) is not built here")
    exe = compile_cpp("transfer_parity", ["transfer_parity.cpp"])
    r = run_cpp(exe, str(ref), "300")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "parity checks passed over 300 random cases" in r.stdout


def test_host_checks_without_gpu():
    """NULL creation options select the current device; the no-alloc
    entry point's pointer test refuses host memory and other GPUs' memory
    (hytgraph_b200/csrc/host_checks.hpp, exercised with made-up pointer
    attributes, so no second GPU is needed)."""
    BUILD.mkdir(parents=True, exist_ok=True)
    exe = BUILD / "host_checks_tests"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(ROOT / "include"), "-I",
                    str(ROOT / "hytgraph_b200" / "csrc"), "-I", "/usr/local/cuda/include",
                    str(ROOT / "tests" / "cpp" / "host_checks_tests.cpp"), "-o", str(exe)], check=True)
    r = run_cpp(exe)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host checks passed" in r.stdout


@pytest.mark.gpu
def test_dropin_gpu_entry_points(gpu):
    exe = compile_cpp("drop_in_tests", ["drop_in_tests.cpp"])
    r = run_cpp(exe, "gpu")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "checks passed (gpu)" in r.stdout
