"""The reference's own test programs -- tests/algorithm_tests.cpp,
tests/unit_tests.cpp and tests/cuda_algorithm_tests.cu of the reference --
compiled unchanged against this project's headers and linked against the
drop-in libraries (oracle/Makefile, target `ref`, with the reference
checkout named by REF or HYT_REFERENCE).  They exercise the C++ interfaces
exactly as the reference's callers do: CSRGraph, GraphLoader, the transfer
engines and cost model, TaskCombiner, HubSorter, reorder_vertices,
ContributionScheduler, the runtime config / result JSON, pagerank_gpu and
sssp_gpu.  The binaries are built where the reference sources are present
and travel with the build; without them these tests are skipped.
"""
from __future__ import annotations

import pytest

from conftest import ROOT, run_cpp

BIN = ROOT / "oracle" / "_ref" / "tests"


def _binary(name):
    exe = BIN / name
    if not exe.exists():
        pytest.skip(f"{exe.relative_to(ROOT)} is not built (no reference checkout when building)")
    return exe


def test_reference_algorithm_tests_pass_on_the_drop_in():
    r = run_cpp(_binary("algorithm_tests"))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "CPU tests passed" in r.stdout


def test_reference_cuda_tests_build_and_skip_without_a_gpu(hyt):
    if hyt.device_count() > 0:
        pytest.skip("a GPU is present: the -m gpu test runs the suite")
    r = run_cpp(_binary("cuda_algorithm_tests"))
    assert r.returncode == 77, r.stdout + r.stderr  # the reference's own skip code


@pytest.mark.gpu
def test_reference_cuda_algorithm_tests_pass_on_the_drop_in(gpu):
    """pagerank_gpu / sssp_gpu of the drop-in against the reference's
    pagerank_cpu / sssp_cpu, as the reference's CUDA test checks them."""
    r = run_cpp(_binary("cuda_algorithm_tests"))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "CUDA algorithm tests passed" in r.stdout


@pytest.mark.gpu
def test_reference_unit_tests_pass_on_the_drop_in(gpu):
    """The reference's unit tests (the drop-in's loader, hub sort, reorder
    and contribution paths run on the GPU)."""
    r = run_cpp(_binary("unit_tests"), timeout=900)
    assert r.returncode == 0, (r.stdout + r.stderr)[-4000:]
    assert "unit tests passed" in r.stdout
