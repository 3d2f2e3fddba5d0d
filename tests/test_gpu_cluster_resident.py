"""Resident phase A of the one-cluster mixed PCG against the gathering one.

With the per-CTA element lists, the (Ap, p, x, r) dof records and the packed
Schwarz inverses in shared memory (the default where they fit, Schwarz
preconditioners only) the HVP adds the same per-corner shares as the
vertex-major gathers, only in a different order, and the preconditioner is
the symmetrized FP32 inverse, so both kernels solve the same systems to the
same tolerance. Checked where Newton converges (32 x 32 drape through landing in
exact-Newton mode, 30 steps): positions agree to 1e-8 relative, every step
converges on both. At the reference budgets (strip pull, 20 steps) the
truncated solves amplify the FP32 ordering differences; the bound there is
the one the mixed path meets against FP64 (1e-4).
"""
import os

import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs

pytestmark = pytest.mark.gpu


def run(cfg, steps, resident, exact=None):
    old = os.environ.get("CLOSIM_MX_RESIDENT")
    os.environ["CLOSIM_MX_RESIDENT"] = "1" if resident else "0"
    try:
        sc = configs.make_scene(cfg)
        s = cb.CudaSolver("mixed", **cfg["options"])
        s.initialize(sc)
    finally:
        if old is None:
            del os.environ["CLOSIM_MX_RESIDENT"]
        else:
            os.environ["CLOSIM_MX_RESIDENT"] = old
    if exact:
        s.setNewtonMode("exact", exact)
    xs, conv = [], 0
    for k in range(steps):
        sc.pinned.clear()
        sc.pinned.update(configs.pins_at(cfg, k))
        s.step(cfg["h"])
        xs.append(sc.positions.copy())
        conv += bool(s.lastStats.converged)
    return xs, conv, s.launchInfo()


def rel(a, b):
    return max(float(np.max(np.abs(x - y)) / np.max(np.abs(y))) for x, y in zip(a, b))


def test_resident_matches_gather_converged_drape():
    cfg = configs.floor_drape(nx=31, ny=31, w=0.4, hgt=0.4, steps=30)
    cfg["x"][1::3] -= 0.28
    cfg["options"] = dict(cfg["options"], newtonIters=40, pcgMaxIters=3000, gradTol=1e-8)
    a, ca, ia = run(cfg, cfg["steps"], True, exact=1e-6)
    b, cb_, ib = run(cfg, cfg["steps"], False, exact=1e-6)
    assert ia["pcgClusterCtas"] > 0 and ia["residentSmemExact"] > 0, ia
    assert ib["residentSmem"] == 0 and ib["residentSmemExact"] == 0, ib
    err = rel(a, b)
    print(f"resident vs gather, converged 32x32 drape: {err:.3e}; converged {ca}/{cb_}")
    assert ca == cfg["steps"] and cb_ == cfg["steps"]
    assert err <= 1e-8, err


def test_resident_matches_gather_reference_budget_strip():
    cfg = configs.strip_pull(steps=20)
    cfg["options"] = dict(cfg["options"], precond="schwarz")  # the resident kernel serves the Schwarz PCG
    a, _, ia = run(cfg, cfg["steps"], True)
    b, _, _ = run(cfg, cfg["steps"], False)
    assert ia["residentSmem"] > 0, ia
    err = rel(a, b)
    print(f"resident vs gather, strip at the reference budgets: {err:.3e}")
    assert err <= 1e-4, err
