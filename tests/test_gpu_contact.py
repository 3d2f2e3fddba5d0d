"""GPU parity of the contact path (FP64) against the oracle, through the C ABI.

Scenes are the reference's own contact tests (tests/floor-contact.test.ts,
determinism.test.ts, self-contact.test.ts, static-collider.test.ts) plus a
small floor drape. Tolerance: 1e-9 relative per step on positions and total
energy; contact diagnostics (candidate / active counts) must match exactly.
"""
import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs
from oracle import oracle as O
from tests.helpers import merge_parts, offset_mesh, oracle_scene, oracle_step_kwargs

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9
DEFAULT_MAT = dict(arealDensityKgM2=0.15, thickness=0.001, stretchWarp=20000.0, stretchWeft=20000.0,
                   stretchCoupling=0.0, shear=5000.0, bendWarp=1e-5, bendWeft=1e-5, damping=0.001)


def scene_cfg(parts, steps, h=1 / 60, gravity=(0.0, -9.81, 0.0), mu=0.3, floor=None, static=None, v=None,
              density=0.15):
    pos, uv, idx = merge_parts(parts)
    n = len(pos) // 3
    contact = dict(dHatM=0.002, kappaJ=50.0, dMinM=1e-4, frictionMu=mu, frictionEpsM=1e-4, floorY=floor)
    if static is not None:
        contact["staticPos"], contact["staticIdx"] = static
    return dict(name="scene", pos=pos, uv=uv, idx=idx, density=density, material=dict(DEFAULT_MAT),
                x=pos.astype(np.float64), v=np.zeros(n * 3) if v is None else v, gravity=gravity, h=h, steps=steps,
                options=dict(newtonIters=10, pcgMaxIters=60, gradTol=1e-5, lineSearchIters=10, precond="jacobi"),
                fixed_pins=[], moving_pins=[], pin_velocity=(0.0, 0.0, 0.0), contact=contact, seed=0)


def run_pair(cfg, steps=None):
    steps = cfg["steps"] if steps is None else steps
    osc = oracle_scene(cfg)
    sc = configs.make_scene(cfg)
    solver = cb.CudaSolver("fp64", **cfg["options"])
    solver.initialize(sc)
    kw = oracle_step_kwargs(cfg)
    worst = 0.0
    for s in range(steps):
        ost = osc.step(cfg["h"], **kw)
        solver.step(cfg["h"])
        xo = osc.positions
        err = np.max(np.abs(sc.positions - xo)) / max(np.max(np.abs(xo)), 1e-30)
        verr = np.max(np.abs(sc.velocities - osc.velocities)) / max(np.max(np.abs(osc.velocities)), 1e-30)
        st = solver.lastStats
        e_err = abs(st.energy - ost["energy"]) / max(abs(ost["energy"]), 1e-30)
        worst = max(worst, err, e_err)
        assert err <= REL_TOL and e_err <= REL_TOL and verr <= REL_TOL, (s, err, e_err, verr)
        c = st.contact
        for k in ["candidatePairs", "activePairs", "vtPairs", "eePairs", "floorPairs", "rejectedLineSearchSteps",
                  "ccdFailures"]:
            assert c[k] == ost[k], (s, k, c[k], ost[k])
        assert st.pcgIters == ost["pcgIters"], (s, st.pcgIters, ost["pcgIters"])
    return worst, solver, osc


def test_floor_patch_parity():
    """tests/floor-contact.test.ts scene: 6x6 patch 5 cm over a y = 0 floor."""
    g = offset_mesh(6, 6, 0.1, 0.1, 0, 0.05, 0)
    cfg = scene_cfg([g], 90, floor=0.0)
    worst, solver, _ = run_pair(cfg)
    print(f"floor patch: worst rel err {worst:.3e}")
    assert solver.lastStats.contact["activePairs"] > 0


def test_determinism_scene_parity():
    """tests/determinism.test.ts scene (5x5 patch, floor, 30 steps)."""
    g = offset_mesh(5, 5, 0.1, 0.1, 0, 0.04, 0.01)
    run_pair(scene_cfg([g], 30, floor=0.0))


def test_self_contact_head_on_parity():
    """tests/self-contact.test.ts:11-36: two patches fly at each other (VT/EE actives)."""
    A = offset_mesh(4, 4, 0.08, 0.08, -0.07, 0.02, 0)
    B = offset_mesh(4, 4, 0.08, 0.08, 0.07, 0.02, 0)
    nA = len(A[0]) // 3
    n = nA + len(B[0]) // 3
    v = np.zeros(n * 3)
    v[0::3] = np.where(np.arange(n) < nA, 0.3, -0.3)
    cfg = scene_cfg([A, B], 60, gravity=(0.0, 0.0, 0.0), mu=0.0, v=v)
    worst, solver, osc = run_pair(cfg)
    print(f"head-on: worst rel err {worst:.3e}")


def test_static_plate_parity():
    """tests/static-collider.test.ts:34-70: patch drapes over a static two-triangle plate."""
    g = offset_mesh(4, 4, 0.08, 0.08, 0.01, 0.08, 0.01)
    spos = np.array([-0.05, 0.03, -0.05, 0.15, 0.03, -0.05, 0.15, 0.03, 0.15, -0.05, 0.03, 0.15], np.float32)
    sidx = np.array([0, 1, 2, 0, 2, 3], np.uint32)
    cfg = scene_cfg([g], 60, static=(spos, sidx))
    worst, solver, _ = run_pair(cfg)
    assert solver.lastStats.contact["vtPairs"] >= 0


def test_small_floor_drape_parity():
    """The floor-drape workload at 16 x 16 vertices (Schwarz PCG)."""
    cfg = configs.floor_drape(nx=15, ny=15, w=0.2, hgt=0.2, steps=12)
    run_pair(cfg)
