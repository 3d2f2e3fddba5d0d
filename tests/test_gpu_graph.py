"""Graph-captured steps (cs_set_graph_mode) against the host-driven step.

A captured step replays the same kernels with the Newton / Armijo /
trust-region decisions taken on the device, so its results must equal the
host-driven step's bit for bit: positions, velocities and every counter of
StepStats and ContactDiagnostics, on every step. Scenes: the strip pull
(moving pins, no contact), a small floor drape through its landing (barrier,
friction, restitution, superset rebuilds), the same drape in exact-Newton mode
(friction potential, Gauss-Newton bending), the 64 x 64 floor drape, and a
garment under a moving collider (the static mesh moves between steps).
Captured steps keep the contact CSR and the broadphase pair superset across
steps when nothing they depend on changed; these comparisons cover both.
"""
import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs

pytestmark = pytest.mark.gpu

KEYS = ["pcgIters", "newtonItersUsed", "armijoTrials", "converged", "gradNorm", "energy", "maxStrain"]
CKEYS = ["candidatePairs", "activePairs", "vtPairs", "eePairs", "floorPairs", "minDistance", "minTOI",
         "barrierEnergy", "frictionWork", "rejectedLineSearchSteps", "ccdFailures"]


def run(cfg, graph, steps, exact=None):
    sc = configs.make_scene(cfg)
    s = cb.CudaSolver("mixed", **cfg["options"])
    s.initialize(sc)
    s.setGraphMode(graph)
    if exact:
        s.setNewtonMode("exact", exact)
    out = []
    for k in range(steps):
        sc.pinned.clear()
        sc.pinned.update(configs.pins_at(cfg, k))
        s.step(cfg["h"])
        st = s.lastStats
        out.append((sc.positions.copy(), sc.velocities.copy(), {k2: getattr(st, k2) for k2 in KEYS},
                    dict(st.contact) if st.contact else None))
    return out, s.graphInfo()


def compare(cfg, steps, exact=None):
    host, gi_h = run(cfg, False, steps, exact)
    graph, gi_g = run(cfg, True, steps, exact)
    assert gi_h["graphSteps"] == 0
    assert gi_g["graphSteps"] + gi_g["hostRepeats"] >= steps and gi_g["graphSteps"] > 0, gi_g
    for k, (a, b) in enumerate(zip(host, graph)):
        assert np.array_equal(a[0], b[0]), (k, float(np.max(np.abs(a[0] - b[0]))))
        assert np.array_equal(a[1], b[1]), k
        assert a[2] == b[2], (k, a[2], b[2])
        if a[3] is not None:
            for key in CKEYS:
                assert a[3][key] == b[3][key], (k, key, a[3][key], b[3][key])
    return graph, gi_g


def test_graph_equals_host_strip_pull():
    cfg = configs.strip_pull(steps=20)
    compare(cfg, cfg["steps"])


def test_graph_equals_host_small_drape_landing():
    cfg = configs.floor_drape(nx=15, ny=15, w=0.2, hgt=0.2, steps=16, height=0.012)
    graph, _ = compare(cfg, cfg["steps"])
    assert max(g[3]["floorPairs"] for g in graph) > 0, "the sheet never reached the floor"


def test_graph_equals_host_small_drape_exact_newton():
    cfg = configs.floor_drape(nx=15, ny=15, w=0.2, hgt=0.2, steps=12, height=0.006)
    cfg["options"] = dict(cfg["options"], newtonIters=40, pcgMaxIters=3000, gradTol=1e-8)
    compare(cfg, cfg["steps"], exact=1e-6)


def test_graph_equals_host_floor_drape_64x64():
    cfg = configs.floor_drape()
    compare(cfg, 45)


def test_graph_equals_host_moving_collider_schwarz():
    """Irregular garment (annulus) under a rising sphere collider, mixed path
    with the Schwarz PCG: the collider's static mesh moves before every step,
    which must invalidate the pair superset the captured steps keep across
    steps."""
    from closim_b200.avatar import AvatarCollider, LinearMotion, SphereGeometry, Transform, toCollisionObject
    from closim_b200.garment import AssembledGarment, AvatarDriver, createFittingScene
    from tests.test_gpu_garment import annulus
    h, steps = 0.01, 16

    def run(graph):
        sphere = AvatarCollider("torso", "torso", SphereGeometry(0.08, 12, 6), 0.004,
                                motion=LinearMotion(Transform((0.0, -0.1, 0.0)), Transform((0.0, 0.06, 0.0)), 0.0,
                                                    steps * h))
        pos, uv, idx = annulus()
        material = cb.ClothMaterial(arealDensityKgM2=0.2, thickness=1.0, stretchWarp=5e3, stretchWeft=5e3,
                                    stretchCoupling=0.0, shear=1e3, bendWarp=1e-4, bendWeft=1e-4, damping=0.0)
        params = cb.ContactParams(dHatM=1e-3, kappaJ=50.0, dMinM=1e-4, frictionMu=0.3, frictionEpsM=1e-4)
        fs = createFittingScene(AssembledGarment(pos, uv, idx), avatar=toCollisionObject(sphere, 0.0),
                                material=material, contact=params, arealDensityKgM2=0.2)
        s = cb.CudaSolver("mixed", newtonIters=10, pcgMaxIters=60, gradTol=1e-5, lineSearchIters=10,
                          precond="schwarz")
        s.initialize(fs.scene)
        s.setGraphMode(graph)
        driver = AvatarDriver([sphere], s)
        out, active = [], 0
        for k in range(steps):
            driver.advance_to((k + 1) * h)
            s.step(h)
            st = s.lastStats
            out.append((fs.scene.positions.copy(), {k2: getattr(st, k2) for k2 in KEYS}, dict(st.contact)))
            active = max(active, st.contact["activePairs"])
        return out, s.graphInfo(), active

    host, _, active = run(False)
    graph, gi, _ = run(True)
    assert active > 0, "the collider never reached the garment"
    assert gi["graphSteps"] > 0, gi
    for k, (a, b) in enumerate(zip(host, graph)):
        assert np.array_equal(a[0], b[0]), (k, float(np.max(np.abs(a[0] - b[0]))))
        assert a[1] == b[1], (k, a[1], b[1])
        for key in CKEYS:
            assert a[2][key] == b[2][key], (k, key, a[2][key], b[2][key])
