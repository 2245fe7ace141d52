"""Shared fixtures.  `-m gpu` tests need a CUDA device; everything else runs
on CPU.  The C-ABI library and the oracle are built on demand."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
BUILD = ROOT / "_build" / "tests"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on a B200 with -m gpu)")


def _ensure_built():
    core = ROOT / "hytgraph_b200" / "lib" / "libhyt_core.so"
    host = ROOT / "hytgraph_b200" / "lib" / "libhytgraph.so"
    if not core.exists() or not host.exists():
        subprocess.run(["make", "-C", str(ROOT / "hytgraph_b200"), "-j8"], check=True, stdout=subprocess.DEVNULL)
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, stdout=subprocess.DEVNULL)


_ensure_built()


@pytest.fixture(scope="session")
def hyt():
    import hytgraph_b200

    return hytgraph_b200


@pytest.fixture(scope="session")
def oracle():
    from oracle.bindings import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.bindings import Reference

    if not Reference.available():
        pytest.skip("oracle/_ref (the reference's compiled CPU code) is not built here")
    return Reference()


@pytest.fixture(scope="session")
def gpu(hyt):
    if hyt.device_count() == 0:
        pytest.fail("test marked gpu but no CUDA device is visible")
    return True


@pytest.fixture(scope="session")
def golden():
    import json

    d = ROOT / "tests" / "golden"
    return {"npz": np.load(d / "rmat_reference.npz"), "meta": json.load(open(d / "known_answers.json"))}


def compile_cpp(name: str, sources, extra=()) -> Path:
    """Compiles a C++ test program against the product's headers and
    libhytgraph.so into _build/tests/<name>."""
    BUILD.mkdir(parents=True, exist_ok=True)
    out = BUILD / name
    srcs = [str(ROOT / "tests" / "cpp" / s) for s in sources]
    newest = max(Path(s).stat().st_mtime for s in srcs)
    lib = ROOT / "hytgraph_b200" / "lib" / "libhytgraph.so"
    if not out.exists() or out.stat().st_mtime < max(newest, lib.stat().st_mtime):
        cmd = ["g++", "-O1", "-std=c++17", "-I", str(ROOT / "include"), *srcs, "-o", str(out),
               "-L", str(lib.parent), "-lhytgraph", "-lhyt_core", f"-Wl,-rpath,{lib.parent}", "-ldl", *extra]
        subprocess.run(cmd, check=True)
    return out


def run_cpp(binary: Path, *args, env=None, timeout=600):
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.run([str(binary), *args], capture_output=True, text=True, env=e, timeout=timeout)
