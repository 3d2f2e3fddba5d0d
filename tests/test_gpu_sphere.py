"""Sheet dropped onto a static sphere collider (the self-contact-heavy workload
scaled down): FP64 path bit-for-bit against the oracle, mixed path free of
intersections, through the C ABI.

The static sphere exercises the cloth-vs-static candidates (3 VT + 9 EE per
static pair, static ids -(i+2)), the static CCD with zero static motion and
the static traversal of the LBVH (contact-assembly.ts:96-140, 556-580).
"""
import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs
from tests.helpers import audit_min_distance, oracle_scene, oracle_step_kwargs

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9


def small_sphere_drape(steps):
    """32 x 32 sheet (0.3 m), sphere r = 0.08 m (12 x 6) whose top is 1 cm below it."""
    return configs.sphere_drape(nx=31, ny=31, w=0.3, hgt=0.3, steps=steps, radius=0.08, drop=0.09, segments=12,
                                rings=6)


def test_sphere_drape_fp64_parity():
    cfg = small_sphere_drape(45)
    osc = oracle_scene(cfg)
    sc = configs.make_scene(cfg)
    solver = cb.CudaSolver("fp64", **cfg["options"])
    solver.initialize(sc)
    kw = oracle_step_kwargs(cfg)
    static_active = 0
    for s in range(cfg["steps"]):
        ost = osc.step(cfg["h"], **kw)
        solver.step(cfg["h"])
        err = np.max(np.abs(sc.positions - osc.positions)) / np.max(np.abs(osc.positions))
        e_err = abs(solver.lastStats.energy - ost["energy"]) / max(abs(ost["energy"]), 1e-30)
        assert err <= REL_TOL and e_err <= REL_TOL, (s, err, e_err)
        c = solver.lastStats.contact
        for k in ["candidatePairs", "activePairs", "vtPairs", "eePairs", "rejectedLineSearchSteps", "ccdFailures"]:
            assert c[k] == ost[k], (s, k, c[k], ost[k])
        assert solver.lastStats.pcgIters == ost["pcgIters"]
        static_active = max(static_active, c["activePairs"])
    print(f"sphere drape 32x32: {cfg['steps']} steps bit-identical, max active contacts {static_active}")
    assert static_active > 0


def test_sphere_drape_mixed_no_intersection():
    cfg = small_sphere_drape(80)
    sc = configs.make_scene(cfg)
    solver = cb.CudaSolver("mixed", **cfg["options"])
    solver.initialize(sc)
    sph = cfg["sphere"]
    centre = np.asarray(sph["centre"])
    for s in range(cfg["steps"]):
        solver.step(cfg["h"])
    x = sc.positions.reshape(-1, 3)
    assert np.all(np.isfinite(x))
    # every vertex outside the faceted sphere's inscribed radius (r cos(pi / rings))
    r_in = sph["radius"] * np.cos(np.pi / sph["rings"]) * np.cos(np.pi / sph["segments"])
    assert np.min(np.linalg.norm(x - centre, axis=1)) > r_in
    mesh = configs.make_scene(cfg).mesh
    assert audit_min_distance(sc.positions, mesh) > 0
    assert solver.lastStats.contact["activePairs"] > 0
