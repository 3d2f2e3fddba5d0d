"""A garment scene with a moving avatar collider, FP64 path against the oracle.

The garment is a triangulated annulus (a skirt-like ring, not a grid: 120
vertices, 192 triangles) built by createFittingScene with a sphere collider
below it; the sphere moves up through the ring's plane with a LinearMotion.
Before every step the collider is sampled at the step's end time and the
static mesh moved there (CudaSolver.setStaticPositions on the GPU,
ContactSystem.setStaticMesh on the oracle, as the reference's session does).
Positions and energies within 1e-9 relative on every step; the contact counts
equal; the sphere does reach the garment (static contacts appear).
"""
import math

import numpy as np
import pytest

import closim_b200 as cb
from closim_b200.avatar import AvatarCollider, LinearMotion, SphereGeometry, Transform, toCollisionObject
from closim_b200.garment import AssembledGarment, AvatarDriver, createFittingScene
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def annulus(r0=0.05, r1=0.2, segments=24, rings=4, y=0.0):
    pos, uv = [], []
    for j in range(rings + 1):
        r = r0 + (r1 - r0) * j / rings
        for i in range(segments):
            a = 2 * math.pi * (i + 0.5 * (j % 2)) / segments
            pos += [r * math.cos(a), y, r * math.sin(a)]
            uv += [r * math.cos(a), r * math.sin(a)]
    idx = []
    for j in range(rings):
        for i in range(segments):
            a, b = j * segments + i, j * segments + (i + 1) % segments
            c, d = a + segments, b + segments
            idx += [a, c, b, b, c, d] if j % 2 == 0 else [a, c, d, a, d, b]
    return np.asarray(pos, np.float32), np.asarray(uv, np.float32), np.asarray(idx, np.uint32)


def test_moving_collider_fp64_parity_with_oracle():
    h, steps = 0.01, 16
    sphere = AvatarCollider("torso", "torso", SphereGeometry(0.08, 12, 6), 0.004,
                            motion=LinearMotion(Transform((0.0, -0.1, 0.0)), Transform((0.0, 0.06, 0.0)), 0.0,
                                                steps * h))
    pos, uv, idx = annulus()
    material = cb.ClothMaterial(arealDensityKgM2=0.2, thickness=1.0, stretchWarp=5e3, stretchWeft=5e3,
                                stretchCoupling=0.0, shear=1e3, bendWarp=1e-4, bendWeft=1e-4, damping=0.0)
    params = cb.ContactParams(dHatM=1e-3, kappaJ=50.0, dMinM=1e-4, frictionMu=0.3, frictionEpsM=1e-4)
    fs = createFittingScene(AssembledGarment(pos, uv, idx), avatar=toCollisionObject(sphere, 0.0), material=material,
                            contact=params, arealDensityKgM2=0.2)
    opts = dict(newtonIters=10, pcgMaxIters=60, gradTol=1e-5, lineSearchIters=10, precond="jacobi")
    solver = cb.CudaSolver("fp64", **opts)
    solver.initialize(fs.scene)
    driver = AvatarDriver([sphere], solver)

    omesh = O.Mesh(pos, uv, idx, 0.2)
    mat = dict(arealDensity=0.2, thickness=1.0, C00=5e3, C11=5e3, C01=0.0, G=1e3, bendWarp=1e-4, bendWeft=1e-4,
               damping=0.0)
    osc = O.Scene(omesh, mat, x=pos.astype(np.float64))
    ocs = O.ContactSystem(dict(dHat=1e-3, kappa=50.0, dMin=1e-4, mu=0.3, eps=1e-4), omesh.indices)
    sidx = fs.contact.staticIdx
    ocs.set_static_mesh(fs.contact.staticPos, sidx)
    osc.set_contact(ocs)
    static_contacts = 0
    for k in range(steps):
        sp = driver.advance_to((k + 1) * h)
        ocs.set_static_mesh(sp, sidx)
        ost = osc.step(h, newton_iters=10, pcg_max_iters=60, grad_tol=1e-5, ls_iters=10, precond="jacobi")
        solver.step(h)
        xo = osc.positions
        err = np.max(np.abs(fs.scene.positions - xo)) / np.max(np.abs(xo))
        e_err = abs(solver.lastStats.energy - ost["energy"]) / max(abs(ost["energy"]), 1e-30)
        assert err <= 1e-9 and e_err <= 1e-9, (k, err, e_err)
        st = solver.lastStats.contact
        for key in ("candidatePairs", "activePairs", "vtPairs", "eePairs"):
            assert st[key] == ost[key], (k, key, st[key], ost[key])
        assert solver.lastStats.pcgIters == ost["pcgIters"], k
        static_contacts = max(static_contacts, st["activePairs"])
    assert static_contacts > 0, "the collider never reached the garment"
