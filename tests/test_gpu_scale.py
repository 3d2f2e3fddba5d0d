"""Parity at the workloads' own scale (the other GPU tests use small meshes).

- Floor drape, 64 x 64 (7,938 triangles), FP64 path against the oracle over
  steps 0..41: free fall, self-contacts of the wrinkling sheet, and the first
  floor contacts (from step 36 at the reference's stepper budget). Positions and energies within 1e-9 relative per step;
  PCG iterations and the candidate / active / floor counts equal; the active
  set after the last step equal record for record.
- Sphere drape, 256 x 256 (130,050 triangles) on the 960-triangle sphere, FP64,
  two steps from a state 0.3 mm above the sphere (inside dHat = 0.5 mm, so the
  static VT/EE candidates are live): the same checks, the active set compared
  record for record (kind, ids, weights, normals).
- Material fit, 96 x 96 (18,050 triangles): the adjoint of a 5-step rollout
  (one checkpoint segment) against central differences with Richardson
  extrapolation, 1e-4 relative, for dL/d(C00, C11, G, k_bend) and a direction
  of dL/dv0. Each of the 22 forward rollouts converges every step to
  gradTol 1e-10, which the FD quotients need; 5 steps keep the test within a
  few minutes.
"""
import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs
from tests.helpers import oracle_scene, oracle_step_kwargs

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9


def lockstep(cfg, steps):
    osc = oracle_scene(cfg)
    sc = configs.make_scene(cfg)
    solver = cb.CudaSolver("fp64", **cfg["options"])
    solver.initialize(sc)
    kw = oracle_step_kwargs(cfg)
    seen_floor = 0
    for s in range(steps):
        ost = osc.step(cfg["h"], **kw)
        solver.step(cfg["h"])
        xo = osc.positions
        err = np.max(np.abs(sc.positions - xo)) / np.max(np.abs(xo))
        e_err = abs(solver.lastStats.energy - ost["energy"]) / max(abs(ost["energy"]), 1e-30)
        assert err <= REL_TOL and e_err <= REL_TOL, (s, err, e_err)
        st = solver.lastStats
        assert st.pcgIters == ost["pcgIters"], (s, st.pcgIters, ost["pcgIters"])
        for k in ("candidatePairs", "activePairs", "vtPairs", "eePairs", "floorPairs"):
            assert st.contact[k] == ost[k], (s, k, st.contact[k], ost[k])
        seen_floor = max(seen_floor, ost["floorPairs"])
    return solver, osc, seen_floor


def check_active_equal(solver, osc):
    ids_g, w_g = solver.activeContacts()
    ids_o, w_o = osc._cs.active()
    assert ids_g.shape == ids_o.shape
    assert np.array_equal(ids_g, ids_o)
    if len(w_o):
        scale = np.maximum(np.abs(w_o), 1e-300)
        assert np.max(np.abs(w_g - w_o) / scale) <= REL_TOL
    return len(ids_o)


def test_floor_drape_64x64_fp64_through_landing():
    cfg = configs.floor_drape()
    solver, osc, seen_floor = lockstep(cfg, 42)
    assert seen_floor > 0, "the sheet did not reach the floor within the window"
    assert check_active_equal(solver, osc) > 0


def test_sphere_drape_256x256_fp64_contact_steps():
    cfg = configs.sphere_drape(drop=0.2 + 3e-4)
    solver, osc, _ = lockstep(cfg, 2)
    st = solver.lastStats.contact
    assert st["activePairs"] > 0 and st["candidatePairs"] > 0, st
    assert check_active_equal(solver, osc) == st["activePairs"]


def test_material_fit_96x96_adjoint_matches_central_differences():
    cfg = configs.material_fit(steps=5, checkpoint_every=5, newton_iters=30, pcg_max_iters=3000, grad_tol=1e-10)

    def rollout(theta, v0=None):
        c = configs.with_theta(cfg, theta)
        sc = configs.make_scene(c)
        s = cb.CudaSolver("fp64", **c["options"])
        s.initialize(sc)
        s.setNewtonMode("exact", 1e-10)
        s.setAdjointOptions(4000, 1e-12)
        if v0 is not None:
            sc.velocities[:] = v0
            s.push_state()
        return s.forward(cfg["h"], cfg["steps"], cfg["checkpoint_every"]).copy(), s

    xs, s_gt = rollout(cfg["theta_gt"])
    assert s_gt.adjointStats()["forwardConverged"] == cfg["steps"]
    th0 = cfg["theta0"].copy()
    x0, s = rollout(th0)
    assert s.adjointStats()["forwardConverged"] == cfg["steps"]
    n = len(x0) // 3

    def loss(x):
        return float(np.sum((x - xs) ** 2) / n)

    dth, dv0 = s.backward(2 * (x0 - xs) / n)
    assert s.adjointStats()["maxRelResidual"] < 1e-9
    adj = [dth["C00"], dth["C11"], dth["G"], dth["kBend"]]

    def central(f, h):
        return (f(h) - f(-h)) / (2 * h)

    def richardson(f, h):
        return (4 * central(f, h / 2) - central(f, h)) / 3

    for j, name in enumerate(["C00", "C11", "G", "kBend"]):
        def f(dh, j=j):
            t = th0.copy()
            t[j] *= 1 + dh
            return loss(rollout(t)[0])
        fd = richardson(f, 1e-2) / th0[j]
        rel = abs(adj[j] - fd) / max(abs(fd), 1e-300)
        print(f"96x96 dL/d{name}: adjoint {adj[j]:.8e}  FD {fd:.8e}  rel {rel:.2e}")
        assert rel <= 1e-4, (name, adj[j], fd)
    u = np.random.default_rng(11).standard_normal(3 * n) * 1e-3
    for pid in cfg["fixed_pins"]:
        u[pid * 3:pid * 3 + 3] = 0
    fd = richardson(lambda e: loss(rollout(th0, cfg["v"] + e * u)[0]), 1.0)
    ad = float(dv0 @ u)
    rel = abs(ad - fd) / max(abs(fd), 1e-300)
    print(f"96x96 dL/dv0 . u: adjoint {ad:.8e}  FD {fd:.8e}  rel {rel:.2e}")
    assert rel <= 1e-4
