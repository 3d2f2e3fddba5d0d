"""Mixed-precision path (FP32 linear solve, FP64 gradients / energies / contact)
against the FP64 path, through the C ABI.

Target (FP32 vs FP64 trajectories): relative position error <= 1e-5 over the
run, no admitted intersection (every accepted trial passed the FP64 CCD gate,
so no vertex ends at or below the floor's hard core).
"""
import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5


def trajectory(cfg, precision, steps):
    sc = configs.make_scene(cfg)
    s = cb.CudaSolver(precision, **cfg["options"])
    s.initialize(sc)
    out = []
    for k in range(steps):
        sc.pinned.clear()
        sc.pinned.update(configs.pins_at(cfg, k))
        s.step(cfg["h"])
        out.append(sc.positions.copy())
    return out, s


def rel_err(a, b):
    return max(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-30) for x, y in zip(a, b))


def test_strip_pull_mixed_vs_fp64():
    cfg = configs.strip_pull()
    a, _ = trajectory(cfg, "fp64", cfg["steps"])
    b, s = trajectory(cfg, "mixed", cfg["steps"])
    err = rel_err(b, a)
    print(f"strip_pull mixed vs fp64 over {cfg['steps']} steps: max rel pos err {err:.3e}")
    assert np.all(np.isfinite(b[-1]))
    assert err <= POS_TOL


def test_floor_drape_mixed_vs_fp64_no_intersection():
    cfg = configs.floor_drape(nx=31, ny=31, w=0.4, hgt=0.4, steps=60)
    cfg["x"][1::3] -= 0.28  # start 2 cm above the floor so contact engages early
    a, _ = trajectory(cfg, "fp64", cfg["steps"])
    b, s = trajectory(cfg, "mixed", cfg["steps"])
    err = rel_err(b, a)
    miny = min(float(x[1::3].min()) for x in b)
    print(f"floor drape 32x32 mixed vs fp64 over {cfg['steps']} steps: max rel pos err {err:.3e}, min y {miny:.3e}")
    assert miny > cfg["contact"]["dMinM"] - 1e-12
    assert s.lastStats.contact["activePairs"] > 0
    assert err <= POS_TOL
