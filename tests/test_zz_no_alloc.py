"""The allocation-free membrane HVP (cs_membrane_hvp_static) against the handle
entry point (cs_membrane_hvp), through the C ABI, on two calls in a row.

cs_membrane_hvp_static serves callers that may not allocate device memory while
they step (graph capture, real-time loops, memory owned by another runtime): the
test allocates the device buffers itself, as such a caller would, and the entry
point only uses the fixed scratch array compiled into the library. This file is
named to run last, so a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import _lib, configs

pytestmark = pytest.mark.gpu


def incidence(indices, n):
    """Membrane incidence records (triangle * 4 + corner), ascending triangle order."""
    idx = np.asarray(indices, np.int64).reshape(-1, 3)
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum(np.bincount(idx.ravel(), minlength=n))
    rec = np.zeros(idx.size, np.uint32)
    cur = off[:-1].astype(np.int64).copy()
    for t in range(len(idx)):
        for c in range(3):
            v = idx[t, c]
            rec[cur[v]] = t * 4 + c
            cur[v] += 1
    return off, rec


def test_membrane_hvp_static_matches_handle_entry_point():
    import torch
    lib = _lib.load()
    f = lib.cs_membrane_hvp_static
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_int32] + [C.c_void_p] * 5 + [C.POINTER(_lib.cs_material)] + [C.c_void_p] * 4
    cfg = configs.floor_drape(nx=40, ny=30, w=0.5, hgt=0.4)
    sc = configs.make_scene(cfg)
    solver = cb.CudaSolver("fp64")
    solver.initialize(sc)
    me = sc.mesh
    n, m = me.count, me.triCount
    off, rec = incidence(me.indices, n)
    dev = torch.device("cuda:0")
    as_dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    d_idx = as_dev(me.indices.view(np.int32))
    d_inv = as_dev(me.invDm)
    d_area = as_dev(me.areas)
    d_off = as_dev(off.view(np.int32))
    d_rec = as_dev(rec.view(np.int32))
    mat = sc.material._c()
    stream = torch.cuda.current_stream(dev).cuda_stream
    rng = np.random.default_rng(17)
    for call in range(2):
        x = cfg["x"] + rng.uniform(-1e-3, 1e-3, 3 * n)
        p = rng.normal(0.0, 1.0, 3 * n)
        d_x, d_p = as_dev(x), as_dev(p)
        d_out = torch.empty(3 * n, dtype=torch.float64, device=dev)
        rc = f(n, m, d_idx.data_ptr(), d_inv.data_ptr(), d_area.data_ptr(), d_off.data_ptr(), d_rec.data_ptr(),
               C.byref(mat), d_x.data_ptr(), d_p.data_ptr(), d_out.data_ptr(), stream)
        assert rc == _lib.CS_OK, (call, rc)
        torch.cuda.synchronize(dev)
        got = d_out.cpu().numpy()
        want = solver.membraneHvp(x, p)
        # both entry points run the same kernels in the same order: bit equality
        assert np.array_equal(got, want), (call, float(np.max(np.abs(got - want))))
    # beyond the stated limits: a clear capacity error, nothing launched
    rc = f(70000, m, d_idx.data_ptr(), d_inv.data_ptr(), d_area.data_ptr(), d_off.data_ptr(), d_rec.data_ptr(),
           C.byref(mat), d_x.data_ptr(), d_p.data_ptr(), d_out.data_ptr(), stream)
    assert rc == _lib.CS_E_CAPACITY
