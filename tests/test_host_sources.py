"""The TypeScript host (host/ts/cuda-solver.ts) and its N-API addon
(host/napi/addon.cc) against each other and against the C ABI, on the CPU.

No Node toolchain exists here, so these checks stand in for a build: every
addon function the TS class calls is exported by the addon, every cs_* call
the addon makes is declared in include/closim_cuda.h and exported by
libclosim_cuda.so, and the addon compiles (syntax and types) against the
public N-API declarations.
"""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TS = os.path.join(ROOT, "host", "ts", "cuda-solver.ts")
ADDON = os.path.join(ROOT, "host", "napi", "addon.cc")
HEADER = os.path.join(ROOT, "include", "closim_cuda.h")


def addon_exports():
    src = open(ADDON).read()
    return set(re.findall(r'\{"(\w+)", nullptr, \w+, nullptr', src))


def test_ts_calls_only_addon_exports():
    ts = open(TS).read()
    called = set(re.findall(r"\bcs\.(\w+)\(", ts))
    assert called, "no addon calls found"
    missing = called - addon_exports()
    assert not missing, f"the TS class calls addon functions that are not exported: {sorted(missing)}"
    # the ClothSolver interface (src/backend/solver.ts:5-13) is implemented
    for method in ["initialize", "step", "setMaterial", "pinVertex", "unpinVertex", "getPositions",
                   "getVelocities"]:
        assert re.search(rf"^\s+{method}\(", ts, re.M), method
    assert "implements ClothSolver" in ts and "lastStats" in ts


def test_addon_calls_declared_and_exported_c_abi():
    src = open(ADDON).read()
    calls = set(re.findall(r"\b(cs_[a-z_0-9]+)\(", src)) - {"cs_ok"}
    header = open(HEADER).read()
    from closim_b200 import _lib
    lib = _lib.load()
    for fn in sorted(calls):
        assert re.search(rf"\b{fn}\(", header), f"{fn} is not declared in closim_cuda.h"
        assert hasattr(lib, fn), f"{fn} is not exported by libclosim_cuda.so"


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_addon_compiles_against_napi_declarations():
    stub = os.path.join(ROOT, "tests", "napi_stub")
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I", stub, "-I",
                        os.path.join(ROOT, "include"), ADDON], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
