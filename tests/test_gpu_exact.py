"""Exact-Newton mode's first iterate.

Exact-Newton mode starts Newton from x0 + h v instead of the reference's
inertial target yHat = x0 + h v + h^2 g (CLOSIM_DRIFT_GUESS=0 restores it).
The energy still has yHat as its inertial target, so every converged step is
the same: on a small drape through landing and rest, both starts converge on
every step, to positions within 1e-7 of each other, and the drift start needs
fewer Newton iterations once the sheet rests on the floor.
"""
import os

import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs

pytestmark = pytest.mark.gpu


def run(drift, precision, steps=40):
    old = os.environ.get("CLOSIM_DRIFT_GUESS")
    os.environ["CLOSIM_DRIFT_GUESS"] = "1" if drift else "0"
    try:
        cfg = configs.floor_drape(nx=15, ny=15, w=0.2, hgt=0.2, steps=steps, height=0.004)
        cfg["options"] = dict(cfg["options"], newtonIters=40, pcgMaxIters=3000, gradTol=1e-8)
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
