"""Exact-Newton mode: its first iterate, and the oracle's restatement of it.

Exact-Newton mode starts Newton from x0 + h v instead of the reference's
inertial target yHat = x0 + h v + h^2 g (CLOSIM_DRIFT_GUESS=0 restores it).
The energy still has yHat as its inertial target, so every converged step is
the same: on a small drape through landing and rest, both starts converge on
every step, to positions within 1e-7 of each other, and the drift start needs
fewer Newton iterations once the sheet rests on the floor.

The oracle restates the mode on the CPU (implicit_step_exact). On the same
drape, with and without friction, both GPU paths converge on every step to
the oracle's positions within 1e-7. At the benchmark's scale and budget (the
64x64 drape, 120 steps, PCG tolerance 3e-4) the oracle's trajectory is a
committed fixture (tests/golden/make_exact_drape.py), and both GPU paths match
it within 1e-7 after the landing and at step 120. With friction on one-sided
static contacts (the reference's static-plate drape) both GPU paths converge
on every step, as the oracle does, to its positions within 1e-7; so they do
on frictionless cloth-cloth self-contact (two sliding patches).
"""
import os

import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs
from tests.helpers import oracle_scene, oracle_step_kwargs

pytestmark = pytest.mark.gpu


def drape(steps, mu=0.3):
    cfg = configs.floor_drape(nx=15, ny=15, w=0.2, hgt=0.2, steps=steps, height=0.004)
    cfg["contact"] = dict(cfg["contact"], frictionMu=mu)
    cfg["options"] = dict(cfg["options"], newtonIters=40, pcgMaxIters=3000, gradTol=1e-8)
    return cfg


def run(drift, precision, steps=40, mu=0.3):
    old = os.environ.get("CLOSIM_DRIFT_GUESS")
    os.environ["CLOSIM_DRIFT_GUESS"] = "1" if drift else "0"
    try:
        cfg = drape(steps, mu)
        sc = configs.make_scene(cfg)
        s = cb.CudaSolver(precision, **cfg["options"])
        s.initialize(sc)
    finally:
        if old is None:
            del os.environ["CLOSIM_DRIFT_GUESS"]
        else:
            os.environ["CLOSIM_DRIFT_GUESS"] = old
    s.setNewtonMode("exact", 1e-6)
    xs, newton, conv = [], [], 0
    for _ in range(steps):
        s.step(cfg["h"])
        xs.append(sc.positions.copy())
        newton.append(s.lastStats.newtonItersUsed)
        conv += bool(s.lastStats.converged)
    return xs, np.array(newton), conv


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_first_iterate_does_not_change_the_converged_steps(precision):
    a, na, ca = run(True, precision)
    b, nb, cb_ = run(False, precision)
    assert ca == len(a) and cb_ == len(b), (ca, cb_)
    err = max(float(np.max(np.abs(x - y)) / np.max(np.abs(y))) for x, y in zip(a, b))
    print(f"{precision}: drift vs yHat start {err:.3e}; Newton iterations {na.sum()} vs {nb.sum()} "
          f"(last 10 steps {na[-10:].sum()} vs {nb[-10:].sum()})")
    assert err <= 1e-7, err
    assert na[-10:].sum() < nb[-10:].sum()


_ORACLE = {}


def oracle_run(mu, steps=40):
    if mu not in _ORACLE:
        cfg = drape(steps, mu)
        osc = oracle_scene(cfg)
        kw = oracle_step_kwargs(cfg)
        xs, conv = [], 0
        for _ in range(steps):
            st = osc.step(cfg["h"], exact=True, pcg_tol=1e-6, drift=True, **kw)
            xs.append(osc.positions)
            conv += st["converged"] > 0
        _ORACLE[mu] = (xs, conv)
    return _ORACLE[mu]


@pytest.mark.parametrize("precision,mu", [("fp64", 0.3), ("mixed", 0.3), ("fp64", 0.0), ("mixed", 0.0)])
def test_exact_mode_matches_the_oracle_exact_mode(precision, mu):
    xo, co = oracle_run(mu)
    xg, _, cg = run(True, precision, mu=mu)
    assert co == len(xo) and cg == len(xg), (co, cg)
    err = max(float(np.max(np.abs(a - b)) / np.max(np.abs(b))) for a, b in zip(xg, xo))
    print(f"{precision}, mu {mu}: GPU exact mode vs oracle exact mode {err:.3e}")
    assert err <= 1e-7, err


GOLD_DRAPE = os.path.join(os.path.dirname(__file__), "golden", "exact_drape_64.npz")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_exact_mode_matches_the_oracle_on_the_64x64_drape(precision):
    g = np.load(GOLD_DRAPE)
    keep = [int(k) for k in g["keep"]]
    steps = len(g["converged"])
    assert int(g["converged"].sum()) == steps
    cfg = configs.floor_drape()
    cfg["options"] = dict(cfg["options"], newtonIters=40, pcgMaxIters=3000, gradTol=float(g["grad_tol"]))
    sc = configs.make_scene(cfg)
    s = cb.CudaSolver(precision, **cfg["options"])
    s.initialize(sc)
    s.setNewtonMode("exact", float(g["pcg_tol"]))
    conv, newton, errs = 0, 0, {}
    for k in range(steps):
        s.step(cfg["h"])
        conv += bool(s.lastStats.converged)
        newton += s.lastStats.newtonItersUsed
        if k in keep:
            xo = g[f"x{k}"]
            errs[k] = float(np.max(np.abs(sc.positions - xo)) / np.max(np.abs(xo)))
    print(f"{precision}: 64x64 drape vs oracle exact mode {errs}; converged {conv}/{steps}; "
          f"Newton {newton} (oracle {int(g['newton'].sum())})")
    assert conv == steps, conv
    assert max(errs.values()) <= 1e-7, errs


def static_plate(steps):
    """tests/static-collider.test.ts:34-70's plate drape (mu 0.3): a 5x5 patch
    falls onto a static two-triangle plate; VT and EE contacts against the
    static mesh, with friction."""
    from tests.helpers import merge_parts, offset_mesh
    pos, uv, idx = merge_parts([offset_mesh(4, 4, 0.08, 0.08, 0.01, 0.08, 0.01)])
    n = len(pos) // 3
    spos = np.array([-0.05, 0.03, -0.05, 0.15, 0.03, -0.05, 0.15, 0.03, 0.15, -0.05, 0.03, 0.15], np.float32)
    sidx = np.array([0, 1, 2, 0, 2, 3], np.uint32)
    mat = dict(arealDensityKgM2=0.15, thickness=0.001, stretchWarp=20000.0, stretchWeft=20000.0, stretchCoupling=0.0,
               shear=5000.0, bendWarp=1e-5, bendWeft=1e-5, damping=0.001)
    return dict(name="static_plate", pos=pos, uv=uv, idx=idx, density=0.15, material=mat, x=pos.astype(np.float64),
                v=np.zeros(n * 3), gravity=(0.0, -9.81, 0.0), h=1 / 60, steps=steps,
                options=dict(newtonIters=40, pcgMaxIters=2000, gradTol=1e-8, lineSearchIters=10, precond="jacobi"),
                fixed_pins=[], moving_pins=[], pin_velocity=(0.0, 0.0, 0.0),
                contact=dict(dHatM=0.002, kappaJ=50.0, dMinM=1e-4, frictionMu=0.3, frictionEpsM=1e-4, floorY=None,
                             staticPos=spos, staticIdx=sidx), seed=0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_exact_mode_static_collider_friction_matches_the_oracle(precision):
    """Friction on one-sided static contacts is a potential gradient, so every
    exact step converges, on the GPU as in the oracle's exact mode, to the
    same positions."""
    steps = 30
    cfg = static_plate(steps)
    osc = oracle_scene(cfg)
    kw = oracle_step_kwargs(cfg)
    sc = configs.make_scene(cfg)
    s = cb.CudaSolver(precision, **cfg["options"])
    s.initialize(sc)
    s.setNewtonMode("exact", 1e-6)
    worst, co, cg, vt, ee = 0.0, 0, 0, 0, 0
    for _ in range(steps):
        st = osc.step(cfg["h"], exact=True, pcg_tol=1e-6, drift=True, **kw)
        s.step(cfg["h"])
        co += st["converged"] > 0
        cg += bool(s.lastStats.converged)
        vt, ee = max(vt, st["vtPairs"]), max(ee, st["eePairs"])
        xo = osc.positions
        worst = max(worst, float(np.max(np.abs(sc.positions - xo)) / np.max(np.abs(xo))))
    print(f"{precision}: static plate, exact mode vs oracle {worst:.3e}; converged GPU {cg}/{steps}, "
          f"oracle {co}/{steps}; VT {vt}, EE {ee}")
    assert vt > 0 and ee > 0
    assert co == steps and cg == steps, (co, cg)
    assert worst <= 1e-7, worst


def sliding_patches(steps):
    """Patch B lands on patch A, which rests on a floor, and slides across it:
    cloth-cloth VT and EE contacts plus floor contacts, without friction (the
    reference's cloth-cloth friction term is no potential gradient)."""
    from tests.helpers import merge_parts, offset_mesh
    A = offset_mesh(4, 4, 0.08, 0.08, 0.0, 0.02, 0)
    B = offset_mesh(4, 4, 0.08, 0.08, 0.03, 0.0215, 0.011)
    pos, uv, idx = merge_parts([A, B])
    n, nA = len(pos) // 3, len(A[0]) // 3
    v = np.zeros(n * 3)
    v[0::3] = np.where(np.arange(n) < nA, 0.1, -0.1)
    cfg = static_plate(steps)
    cfg.update(name="sliding_patches", pos=pos, uv=uv, idx=idx, x=pos.astype(np.float64), v=v)
    cfg["contact"] = dict(dHatM=0.002, kappaJ=50.0, dMinM=1e-4, frictionMu=0.0, frictionEpsM=1e-4, floorY=0.0185)
    return cfg


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_exact_mode_frictionless_self_contact_matches_the_oracle(precision):
    steps = 12
    cfg = sliding_patches(steps)
    osc = oracle_scene(cfg)
    kw = oracle_step_kwargs(cfg)
    sc = configs.make_scene(cfg)
    s = cb.CudaSolver(precision, **cfg["options"])
    s.initialize(sc)
    s.setNewtonMode("exact", 1e-6)
    worst, co, cg, vt, ee = 0.0, 0, 0, 0, 0
    for _ in range(steps):
        st = osc.step(cfg["h"], exact=True, pcg_tol=1e-6, drift=True, **kw)
        s.step(cfg["h"])
        co += st["converged"] > 0
        cg += bool(s.lastStats.converged)
        vt, ee = max(vt, st["vtPairs"]), max(ee, st["eePairs"])
        xo = osc.positions
        worst = max(worst, float(np.max(np.abs(sc.positions - xo)) / np.max(np.abs(xo))))
    print(f"{precision}: sliding patches, exact mode vs oracle {worst:.3e}; converged GPU {cg}/{steps}, "
          f"oracle {co}/{steps}; VT {vt}, EE {ee}")
    assert vt > 0 and ee > 0
    assert co == steps and cg == steps, (co, cg)
    assert worst <= 1e-7, worst
