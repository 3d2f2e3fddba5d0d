"""GPU parity of the CUDA solver (FP64 path) against the oracle, through the C ABI.

Tolerance: positions and total energy within 1e-9 relative per step (the FP64
target). Per-element arithmetic is op-for-op identical to the oracle; the only
differences come from reduction order (tree sums on the device, sequential sums
in the reference) and libm ulps, so observed errors are far below the bound.
"""
import math

import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs
from tests.helpers import oracle_scene, oracle_step_kwargs

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9


def run_pair(cfg, steps, precision="fp64", check=True):
    osc = oracle_scene(cfg)
    sc = configs.make_scene(cfg)
    solver = cb.CudaSolver(precision, **cfg["options"])
    solver.initialize(sc)
    kw = oracle_step_kwargs(cfg)
    worst = 0.0
    worst_e = 0.0
    for s in range(steps):
        pins = configs.pins_at(cfg, s)
        osc.set_pins(pins)
        sc.pinned.clear()
        sc.pinned.update(pins)
        ost = osc.step(cfg["h"], **kw)
        solver.step(cfg["h"])
        xo = osc.positions
        xg = solver.getPositions()
        err = np.max(np.abs(xg - xo)) / max(np.max(np.abs(xo)), 1e-30)
        e_err = abs(solver.lastStats.energy - ost["energy"]) / max(abs(ost["energy"]), 1e-30)
        worst = max(worst, err)
        worst_e = max(worst_e, e_err)
        if check:
            assert err <= REL_TOL, (s, err)
            assert e_err <= REL_TOL, (s, e_err, solver.lastStats.energy, ost["energy"])
            assert solver.lastStats.pcgIters == ost["pcgIters"], (s, solver.lastStats, ost)
    return worst, worst_e, solver, osc


def test_strip_pull_fp64_parity_jacobi():
    cfg = configs.strip_pull()
    worst, worst_e, solver, _ = run_pair(cfg, cfg["steps"])
    print(f"strip_pull fp64 jacobi: max rel pos err {worst:.3e}, energy {worst_e:.3e}")
    assert solver.kernelLaunches() > 0


def test_strip_pull_fp64_parity_schwarz():
    cfg = configs.strip_pull(steps=40)
    cfg["options"] = dict(cfg["options"], precond="schwarz")
    worst, worst_e, _, _ = run_pair(cfg, cfg["steps"])
    print(f"strip_pull fp64 schwarz: max rel pos err {worst:.3e}, energy {worst_e:.3e}")


def test_gpu_runs_are_bit_identical():
    cfg = configs.strip_pull(steps=20)
    outs = []
    for _ in range(2):
        sc = configs.make_scene(cfg)
        s = cb.CudaSolver("fp64", **cfg["options"])
        s.initialize(sc)
        for k in range(cfg["steps"]):
            sc.pinned.clear()
            sc.pinned.update(configs.pins_at(cfg, k))
            s.step(cfg["h"])
        outs.append(sc.positions.copy())
    assert np.array_equal(outs[0], outs[1])


def test_solver_interface_semantics():
    cfg = configs.strip_pull(steps=3)
    s = cb.CudaSolver("fp64")
    with pytest.raises(cb.ClothSolverError, match="not initialized"):
        s.step(0.01)
    sc = configs.make_scene(cfg)
    s.initialize(sc)
    s.step(0.01)
    # results land in the scene's own arrays (cpu-solver.ts:40-48)
    assert s.getPositions() is sc.positions
    assert np.all(np.isfinite(sc.positions))
    # pinVertex without a position pins at the current position; unpin frees it
    x = sc.positions.copy()
    s.pinVertex(5)
    assert sc.pinned[5] == tuple(float(q) for q in x[15:18])
    s.step(0.01)
    assert np.array_equal(sc.positions[15:18], x[15:18])
    s.unpinVertex(5)
    assert 5 not in sc.pinned
    s.pinVertex(7, (0.5, 0.25, 0.1))
    assert np.array_equal(sc.positions[21:24], [0.5, 0.25, 0.1])
    m = cb.ClothMaterial(**dict(cfg["material"], stretchWarp=9e3))
    s.setMaterial(m)
    assert sc.material.stretchWarp == 9e3
    s.step(0.01)
    assert s.lastStats.newtonIters == 10


def test_nonfinite_gradient_raises():
    cfg = configs.strip_pull(steps=1)
    sc = configs.make_scene(cfg)
    sc.positions[10] = math.nan
    s = cb.CudaSolver("fp64")
    s.initialize(sc)
    with pytest.raises(FloatingPointError, match="non-finite gradient"):
        s.step(0.01)


def test_membrane_hvp_bit_exact():
    """membraneHvp (fem.ts:108-130) on the GPU equals the oracle bit for bit."""
    from oracle import oracle as O
    cfg = configs.floor_drape(nx=20, ny=13, w=0.3, hgt=0.2)
    sc = configs.make_scene(cfg)
    s = cb.CudaSolver("fp64")
    s.initialize(sc)
    mesh = O.Mesh(cfg["pos"], cfg["uv"], cfg["idx"], cfg["density"])
    m = cfg["material"]
    mat = dict(arealDensity=m["arealDensityKgM2"], thickness=m["thickness"], C00=m["stretchWarp"],
               C11=m["stretchWeft"], C01=m["stretchCoupling"], G=m["shear"], bendWarp=m["bendWarp"],
               bendWeft=m["bendWeft"], damping=m["damping"])
    rng = np.random.default_rng(4)
    for _ in range(3):
        x = cfg["x"] + rng.uniform(-2e-3, 2e-3, len(cfg["x"]))
        p = rng.normal(0, 1, len(cfg["x"]))
        assert np.array_equal(s.membraneHvp(x, p), O.membrane_hvp(mesh, mat, x, p))
