"""CPU-only checks of the product library: it loads, exports every symbol the
C header declares, and its host-side mesh preprocessing matches the oracle bit
for bit. No GPU compute is called here."""
import ctypes
import os
import re

import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import _lib
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = []
    for name in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if name.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", name)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            out += re.findall(r"\b(cs_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(out))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) >= set(_lib.EXPORTS)


@pytest.mark.parametrize("args", [(40, 8, 1.0, 0.2), (63, 63, 0.8, 0.8), (7, 3, 0.3, 0.1), (1, 1, 1.0, 1.0)])
def test_grid_and_preprocess_match_oracle(args):
    pos, uv, idx = cb.buildGrid(*args)
    p2, uv2, idx2 = O.build_grid(*args)
    assert np.array_equal(pos, p2) and np.array_equal(uv, uv2) and np.array_equal(idx, idx2)
    me = cb.preprocess(pos, uv, idx, 0.2)
    om = O.Mesh(pos, uv, idx, 0.2)
    assert me.hinges.shape[0] == om.hg
    for a, b in [(me.invDm, om.invDm), (me.areas, om.areas), (me.masses, om.masses),
                 (me.hinges.ravel(), om.hinges), (me.hingeMeta.ravel(), om.hinge_meta)]:
        assert np.array_equal(a, b)


def test_preprocess_rejects_degenerate_and_bad_indices():
    pos = np.zeros(9, np.float32)
    uv = np.zeros(6, np.float32)
    with pytest.raises(ValueError):
        cb.preprocess(pos, uv, np.array([0, 1, 2], np.uint32), 0.2)
    with pytest.raises(ValueError):
        cb.preprocess(pos, uv, np.array([0, 1, 7], np.uint32), 0.2)


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(cb.ClothSolverError):
        cb.CudaSolver()


def test_null_handle_is_an_argument_error():
    lib = _lib.load()
    assert lib.cs_step(None, 0.01) == _lib.CS_E_ARG
    assert lib.cs_get_positions(None, None) == _lib.CS_E_ARG
