"""C++ drop-in tests: programs written against the reference's C++
interfaces, linked against libhytgraph.so."""
from __future__ import annotations

import pytest

from conftest import ROOT, compile_cpp, run_cpp


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


@pytest.mark.gpu
def test_dropin_gpu_entry_points(gpu):
    exe = compile_cpp("drop_in_tests", ["drop_in_tests.cpp"])
    r = run_cpp(exe, "gpu")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "checks passed (gpu)" in r.stdout
