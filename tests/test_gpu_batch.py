"""Batched solver (include/closim_batch.h) through the C ABI.

- Converged regime: soft strips of different sizes pinned at both ends (both
  solvers converge on at least 80% of the steps, the rest end within a few
  gradient tolerances); each sheet of the batch against the single-sheet FP64
  solver: relative position error <= 1e-5.
- A sheet's trajectory does not depend on the rest of the batch (one block per
  sheet, fixed-order block reductions): bit-identical alone and in a batch.
- A graph-replayed multi-step call equals the same steps issued one by one.
- Floor contact: sheets dropped onto the floor stay above dMin.
- The autotuner returns a candidate block size and leaves the state unchanged.
- At a converging budget each sheet matches the oracle's exact-Newton mode.
"""
import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs
from closim_b200.batch import BatchSolver

pytestmark = pytest.mark.gpu


def soft_strip(nx, ny, seed):
    cfg = configs.strip_pull(seed=seed, nx=nx, ny=ny, w=nx * 0.025, hgt=ny * 0.025, steps=30)
    for k in ["stretchWarp", "stretchWeft"]:
        cfg["material"][k] = 500.0
    cfg["material"]["shear"] = 100.0
    cfg["fixed_pins"] = cfg["fixed_pins"] + cfg["moving_pins"]
    cfg["moving_pins"] = []
    cfg["options"] = dict(cfg["options"], newtonIters=20, pcgMaxIters=200, gradTol=1e-5)
    return cfg


def single_fp64(cfg, steps):
    sc = configs.make_scene(cfg)
    s = cb.CudaSolver("fp64", **cfg["options"])
    s.initialize(sc)
    conv = 0
    for _ in range(steps):
        s.step(cfg["h"])
        conv += bool(s.lastStats.converged)
    return sc.positions.copy(), conv


def test_batch_matches_single_sheet_fp64_converged():
    sheets = [soft_strip(nx, ny, seed) for nx, ny, seed in [(40, 8, 1), (24, 12, 2), (16, 16, 3), (31, 5, 4)]]
    steps = 30
    bs = BatchSolver(sheets)
    conv = np.zeros(len(sheets))
    for _ in range(steps):
        bs.step(sheets[0]["h"])
        conv += [st["converged"] == 1 for st in bs.stats()]
    for i, cfg in enumerate(sheets):
        ref, rconv = single_fp64(cfg, steps)
        xb = bs.positions(i)
        err = np.max(np.abs(xb - ref)) / np.max(np.abs(ref))
        print(f"sheet {i} ({len(ref) // 3} verts): batch converged {int(conv[i])}/{steps}, fp64 {rconv}/{steps}, "
              f"max rel pos err {err:.3e}")
        assert conv[i] >= 0.8 * steps and rconv >= 0.8 * steps
        assert err <= 1e-5


def test_sheet_independent_of_batch_and_graph_replay():
    sheets = configs.batch_sheets(count=12, side_min=8, side_max=40, seed=9)
    h = sheets[0]["h"]
    full = BatchSolver(sheets)
    full.step(h, 6)  # graph-captured
    alone = BatchSolver([sheets[5]])
    for _ in range(6):
        alone.step(h)  # one launch per step
    assert np.array_equal(full.positions(5), alone.positions(0))
    again = BatchSolver(sheets)
    for _ in range(6):
        again.step(h)
    assert np.array_equal(full.allPositions(), again.allPositions())


def test_batch_floor_contact_no_penetration():
    sheets = configs.batch_sheets(count=16, side_min=8, side_max=32, seed=11, floor_y=-0.02)
    bs = BatchSolver(sheets)
    miny = np.inf
    for _ in range(40):
        bs.step(sheets[0]["h"])
        x = bs.allPositions()
        miny = min(miny, float(x[1::3].min()))
    st = bs.stats()
    assert np.all(np.isfinite(bs.allPositions()))
    assert miny > -0.02 + sheets[0]["contact"]["dMinM"] - 1e-12
    assert sum(s["floorContacts"] for s in st) > 0


def test_autotune_keeps_state():
    sheets = configs.batch_sheets(count=20, side_min=16, side_max=48, seed=13)
    bs = BatchSolver(sheets)
    bs.step(0.01, 2)
    x0 = bs.allPositions()
    t = bs.autotune(0.01)
    assert t in (128, 256, 512)
    assert np.array_equal(bs.allPositions(), x0)
    bs.step(0.01)
    assert np.all(np.isfinite(bs.allPositions()))


def test_batch_matches_the_oracle_exact_mode_when_converged():
    """Each sheet of the batch at a converging budget (gradTol 1e-8) against the
    oracle's exact-Newton mode, an independent CPU implementation of the same
    equations (both take the exact hinge gradient): the oracle converges every
    step and the batch all but at most one per sheet (its Armijo search, the
    reference's, has no near-convergence rule, so a step can stop just short of
    the tolerance), and the positions agree."""
    from tests.helpers import oracle_scene, oracle_step_kwargs
    sheets = [soft_strip(nx, ny, seed) for nx, ny, seed in [(24, 12, 2), (31, 5, 4)]]
    budget = dict(newtonIters=40, pcgMaxIters=400, gradTol=1e-8)
    steps = 20
    h = sheets[0]["h"]
    bs = BatchSolver(sheets, options=budget)
    conv = np.zeros(len(sheets))
    for _ in range(steps):
        bs.step(h)
        conv += [st["converged"] == 1 for st in bs.stats()]
    for i, cfg in enumerate(sheets):
        osc = oracle_scene(cfg)
        kw = dict(oracle_step_kwargs(cfg), newton_iters=40, pcg_max_iters=3000, grad_tol=1e-8)
        co = 0
        for k in range(steps):
            osc.set_pins(configs.pins_at(cfg, k))
            co += osc.step(h, exact=True, pcg_tol=1e-6, drift=True, **kw)["converged"] > 0
        xo = osc.positions
        err = float(np.max(np.abs(bs.positions(i) - xo)) / np.max(np.abs(xo)))
        print(f"sheet {i}: batch vs oracle exact mode {err:.3e}; converged batch {int(conv[i])}/{steps}, "
              f"oracle {co}/{steps}")
        assert co == steps and conv[i] >= steps - 1, (conv[i], co)
        assert err <= 1e-7, err
