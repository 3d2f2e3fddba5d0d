"""SimulationSession.doStep hand-off (src/view/sim-session.ts:120-150) on the
device: NaN scan and stable snapshot without a host scan, restoreStable."""
import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs
from closim_b200.session import SimulationSession

pytestmark = pytest.mark.gpu


def test_session_steps_publish_and_restore():
    cfg = configs.floor_drape(nx=15, ny=15, w=0.2, hgt=0.2, steps=10)
    sc = configs.make_scene(cfg)
    published = []
    sess = SimulationSession(cb.CudaSolver("mixed", **cfg["options"]), lambda x: published.append(x.copy()))
    sess.attach(sc, cfg["h"])
    assert sess.status == "ready" and len(published) == 1
    sess.stepOnce(5)
    assert sess.stepCount == 5 and sess.lastStepNaNFree and sess.stableStep == 5
    assert np.array_equal(published[-1], sc.positions)
    assert sess.lastStats is not None and sess.lastStats.newtonIters == 10
    x5 = sc.positions.copy()
    sess.stepOnce(2)
    x7 = sc.positions.copy()
    assert sess.stableStep == 7
    assert sess.restoreStable()
    assert np.array_equal(sc.positions, x7)
    assert np.all(sc.velocities == 0)
    sess.play()
    sess.tick(3 * cfg["h"] + 1e-9)
    assert sess.stepCount == 10
    assert not np.array_equal(sc.positions, x5)


def test_session_flags_nonfinite_positions_and_keeps_snapshot():
    """A non-finite state (planted on the host through the scene) is reported
    and the last finite snapshot survives."""
    cfg = configs.strip_pull(steps=5)
    sc = configs.make_scene(cfg)
    sess = SimulationSession(cb.CudaSolver("fp64", **cfg["options"]), lambda x: None)
    sess.attach(sc, cfg["h"])
    sess.stepOnce(2)
    good = sc.positions.copy()
    solver = sess.solver
    sc.positions[5] = np.nan
    solver.push_state()
    with pytest.raises(FloatingPointError):
        sess.stepOnce(1)
    assert sess.restoreStable()
    assert np.array_equal(sc.positions, good)


def test_session_published_positions_match_oracle_through_contact():
    """Every position the session publishes (cs_session_step's device hand-off)
    equals the oracle's state after the same step, through the landing of a
    sheet on the floor (barrier, friction and restitution active)."""
    from tests.helpers import oracle_scene, oracle_step_kwargs
    cfg = configs.floor_drape(nx=11, ny=11, w=0.15, hgt=0.15, steps=14, height=0.012)
    sc = configs.make_scene(cfg)
    published = []
    sess = SimulationSession(cb.CudaSolver("fp64", **cfg["options"]), lambda x: published.append(x.copy()))
    sess.attach(sc, cfg["h"])
    osc = oracle_scene(cfg)
    kw = oracle_step_kwargs(cfg)
    floor_contacts = 0
    for s in range(cfg["steps"]):
        sess.stepOnce(1)
        ost = osc.step(cfg["h"], **kw)
        xo = osc.positions
        err = np.max(np.abs(published[-1] - xo)) / np.max(np.abs(xo))
        assert err <= 1e-9, (s, err)
        assert sess.lastStats.contact["floorPairs"] == ost["floorPairs"], s
        floor_contacts = max(floor_contacts, ost["floorPairs"])
    assert floor_contacts > 0, "the sheet never reached the floor"
    assert sess.stableStep == cfg["steps"] and len(published) == cfg["steps"] + 1
