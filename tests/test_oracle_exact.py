"""The oracle's restatement of the CUDA solver's exact-Newton mode.

The reference has no exact-Newton mode; these tests pin each of its pieces to
the reference quantity it differentiates or replaces:
- the exact hinge gradient against central differences of the reference
  hinge energy (bending.ts:7-16), away from flat, and against central
  differences of the smooth signed-angle form near flat; its exact Hessian
  against differences of the gradient;
- the positive part of the membrane stress against an eigendecomposition;
- the internal Newton matrix against differences of the exact gradient, and
  its positive semi-definiteness under compression;
- the friction potential against the reference's Coulomb friction force
  (friction.ts:14-23 through contact-assembly.ts:318-341) on floor contacts;
- the exact step against the reference step where both equations coincide
  (no bending, no friction): both converge to the same positions;
- the exact step on frictionless self-contact (VT and EE), where it converges
  and the reference step does not, and the reason it cannot on cloth-cloth
  friction: there the reference's friction term is not a potential gradient;
- the exact step under friction on one-sided static contacts, where every
  step converges.
"""
import math

import numpy as np

from oracle import oracle as O

MAT = O.DEFAULT_MATERIAL


def _hinge(rng, fold):
    """A hinge (v0, v1 shared; v2, v3 the wings) folded by `fold` radians from flat."""
    e = rng.uniform(0.01, 0.02)
    a = rng.uniform(0.006, 0.012)
    b = rng.uniform(0.006, 0.012)
    q = np.zeros(12)
    q[3:6] = [e, 0, 0]
    q[6:9] = [rng.uniform(0.2, 0.8) * e, a, 0]
    q[9:12] = [rng.uniform(0.2, 0.8) * e, -b * math.cos(fold), b * math.sin(fold)]
    R, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    q = (q.reshape(4, 3) @ R.T + rng.uniform(-0.1, 0.1, 3)).ravel()
    meta = np.array([rng.uniform(2.5, 3.1), e, 0.5 * e * (a + b)])
    return q, meta


def _theta_smooth(q):
    """Bend angle pi - |phi|, phi = atan2((n1 x m2).e0/|e0|, n1.m2): the same
    angle as the reference's acos of the normals' cosine, smooth near flat."""
    x0, x1, x2, x3 = q.reshape(4, 3)
    e0 = x1 - x0
    n1 = np.cross(e0, x2 - x0)
    m2 = np.cross(x3 - x0, e0)
    phi = math.atan2(np.dot(np.cross(n1, m2), e0) / np.linalg.norm(e0), np.dot(n1, m2))
    return math.pi - abs(phi)


def test_hinge_grad_exact_vs_fd_of_reference_energy():
    rng = np.random.default_rng(3)
    k = 1e-5
    for _ in range(40):
        q, meta = _hinge(rng, rng.choice([-1, 1]) * rng.uniform(0.2, 2.5))
        g = O.hinge_grad_exact(q, meta, k)
        fd = np.zeros(12)
        h = 1e-7
        for j in range(12):
            qp, qm = q.copy(), q.copy()
            qp[j] += h
            qm[j] -= h
            fd[j] = (O.hinge_energy(qp, meta, k) - O.hinge_energy(qm, meta, k)) / (2 * h)
        assert np.max(np.abs(g - fd)) <= 1e-6 * np.max(np.abs(g)), (g, fd)
        # the angle is rigid-motion invariant: the gradient carries no net force or torque
        assert np.max(np.abs(g.reshape(4, 3).sum(0))) <= 1e-12 * np.max(np.abs(g))


def test_hinge_grad_exact_near_flat():
    """Near flat the reference's acos form loses its derivative to rounding;
    the exact gradient follows the smooth signed-angle form there."""
    rng = np.random.default_rng(5)
    k = 1e-5
    for fold in [1e-3, -1e-4, 1e-6]:
        q, meta = _hinge(rng, fold)
        w = meta[1] ** 2 / meta[2]
        g = O.hinge_grad_exact(q, meta, k)
        th = _theta_smooth(q)
        fd = np.zeros(12)
        h = 1e-9
        for j in range(12):
            qp, qm = q.copy(), q.copy()
            qp[j] += h
            qm[j] -= h
            fd[j] = k * w * (th - meta[0]) * (_theta_smooth(qp) - _theta_smooth(qm)) / (2 * h)
        assert np.max(np.abs(g - fd)) <= 1e-5 * np.max(np.abs(g)), (fold, g, fd)
    # exactly flat at a flat rest angle: zero
    q, meta = _hinge(rng, 0.0)
    q = q.reshape(4, 3)
    q[:, :] = q - q[0]
    q[:, 2] = 0  # the four points in one plane
    meta[0] = math.pi
    assert np.max(np.abs(O.hinge_grad_exact(q.ravel(), meta, k))) == 0


def test_hinge_hess_exact_vs_differences_of_exact_gradient():
    rng = np.random.default_rng(4)
    k = 1e-5
    for fold in [0.7, -1.9, 2.8, 1e-3, -1e-5]:
        q, meta = _hinge(rng, fold)
        H = O.hinge_hess_exact(q, meta, k)
        assert np.array_equal(H, H.T)
        h = 1e-8
        fd = np.zeros((12, 12))
        for j in range(12):
            qp, qm = q.copy(), q.copy()
            qp[j] += h
            qm[j] -= h
            fd[:, j] = (O.hinge_grad_exact(qp, meta, k) - O.hinge_grad_exact(qm, meta, k)) / (2 * h)
        assert np.max(np.abs(H - fd)) <= 1e-5 * np.max(np.abs(H)), (fold, np.max(np.abs(H - fd)))
        # rigid translations are in its null space
        for a in range(3):
            t = np.zeros(12)
            t[a::3] = 1
            assert np.max(np.abs(H @ t)) <= 1e-9 * np.max(np.abs(H))


def test_stress_positive_part():
    rng = np.random.default_rng(7)
    for _ in range(200):
        s00, s11, s01 = rng.normal(size=3) * rng.uniform(1, 1e4)
        S = np.array([[s00, s01], [s01, s11]])
        lam, V = np.linalg.eigh(S)
        ref = V @ np.diag(np.maximum(lam, 0)) @ V.T
        p00, p11, p01 = O.stress_positive_part(s00, s11, s01)
        got = np.array([[p00, p01], [p01, p11]])
        assert np.max(np.abs(got - ref)) <= 1e-12 * max(np.max(np.abs(S)), 1e-300)
    # diagonal and isotropic corner cases
    assert O.stress_positive_part(3.0, -2.0, 0.0) == (3.0, 0.0, 0.0)
    assert O.stress_positive_part(-3.0, 2.0, 0.0) == (0.0, 2.0, 0.0)
    assert O.stress_positive_part(-1.0, -1.0, 0.0) == (0.0, 0.0, 0.0)
    assert O.stress_positive_part(2.0, 2.0, 0.0) == (2.0, 2.0, 0.0)


def _grid(nx, sx, sz, fold=0.0):
    pos, uv, idx = O.build_grid(nx, nx, 0.1, 0.1)
    mesh = O.Mesh(pos, uv, idx, 0.15)
    x = mesh.positions.astype(np.float64).copy()
    x[0::3] *= sx
    x[2::3] *= sz
    x[1::3] += fold * np.sin(40 * x[0::3])
    return mesh, x


def test_internal_hvp_exact_matches_differences_of_exact_gradient():
    """In tension (no stress to clamp) the exact-mode Newton matrix is the
    Hessian of the energy whose gradient is eval_internal_exact."""
    rng = np.random.default_rng(9)
    mesh, x = _grid(6, 1.02, 1.03, fold=0.004)
    for _ in range(3):
        v = rng.normal(size=x.size)
        hv = O.internal_hvp_exact(mesh, MAT, x, v)
        h = 1e-7
        fd = (O.eval_internal_exact(mesh, MAT, x + h * v)[1] - O.eval_internal_exact(mesh, MAT, x - h * v)[1]) / (2 * h)
        assert np.max(np.abs(hv - fd)) <= 1e-5 * np.max(np.abs(hv)), np.max(np.abs(hv - fd))
    # its membrane part equals the reference's analytic HVP there
    mat0 = dict(MAT, bendWarp=0.0, bendWeft=0.0)
    v = rng.normal(size=x.size)
    assert np.allclose(O.internal_hvp_exact(mesh, mat0, x, v), O.eval_membrane_hvp(mesh, mat0, x, v),
                       rtol=1e-10, atol=1e-10 * np.max(np.abs(O.eval_membrane_hvp(mesh, mat0, x, v))))


def test_internal_hvp_exact_is_psd_under_compression():
    rng = np.random.default_rng(13)
    mat0 = dict(MAT, bendWarp=0.0, bendWeft=0.0)
    mesh, x = _grid(6, 0.95, 0.97, fold=0.002)
    neg_ref = 0
    for i in range(30):
        v = rng.normal(size=x.size)
        if i % 2:
            v[0::3] = 0  # out-of-plane only: the geometric term dominates
            v[2::3] = 0
        q = float(v @ O.internal_hvp_exact(mesh, mat0, x, v))
        assert q >= -1e-12 * float(v @ v) * np.max(np.abs(O.internal_hvp_exact(mesh, mat0, x, np.ones(x.size)))), q
        neg_ref += float(v @ O.eval_membrane_hvp(mesh, mat0, x, v)) < 0
    # the unclamped compressive stress makes the reference's matrix indefinite here
    assert neg_ref > 0


def _floor_sheet(y):
    pos, uv, idx = O.build_grid(4, 4, 0.03, 0.03)
    mesh = O.Mesh(pos, uv, idx, 0.15)
    x = mesh.positions.astype(np.float64).copy()
    x[1::3] = y
    return mesh, x


def test_friction_potential_gradient_is_the_reference_friction_force():
    """On floor contacts the gradient of the frozen potential at its freeze
    point is the reference's lagged friction term of energyGrad."""
    rng = np.random.default_rng(17)
    mesh, x0 = _floor_sheet(0.0009)
    params = dict(O.DEFAULT_CONTACT)
    with_f = O.ContactSystem(params, mesh.indices)
    no_f = O.ContactSystem(dict(params, mu=0.0), mesh.indices)
    for cs in (with_f, no_f):
        cs.set_floor(0.0)
        cs.begin_step(x0)
    xf = x0.copy()
    xf[0::3] += rng.uniform(-3e-4, 3e-4, mesh.n)
    xf[2::3] += rng.uniform(-3e-4, 3e-4, mesh.n)
    xf[1::3] += rng.uniform(-1e-4, 1e-4, mesh.n)
    for cs in (with_f, no_f):
        cs.update_active_set(xf)
    assert len(with_f.active()[0]) == mesh.n
    g_fric = with_f.energy_grad(xf)[1] - no_f.energy_grad(xf)[1]
    fd = np.zeros(xf.size)
    h = 1e-9
    for j in range(xf.size):
        xp, xm = xf.copy(), xf.copy()
        xp[j] += h
        xm[j] -= h
        fd[j] = (with_f.friction_potential(xf, xp) - with_f.friction_potential(xf, xm)) / (2 * h)
    assert np.max(np.abs(fd - g_fric)) <= 1e-6 * np.max(np.abs(g_fric)), np.max(np.abs(fd - g_fric))
    # the Hessian along v against second differences of the potential
    for _ in range(3):
        v = rng.normal(size=xf.size) * 1e-4
        _, hv = with_f.friction_potential(xf, xf, v)
        e = 1e-3
        d2 = (with_f.friction_potential(xf, xf + e * v) - 2 * with_f.friction_potential(xf, xf)
              + with_f.friction_potential(xf, xf - e * v)) / (e * e)
        assert abs(d2 - float(v @ hv)) <= 1e-5 * abs(float(v @ hv)) + 1e-18, (d2, float(v @ hv))
        assert float(v @ hv) >= 0


def _drape(nx, mu, bend=True, drift=True, exact=True, steps=30):
    pos, uv, idx = O.build_grid(nx, nx, 0.08, 0.08)
    pos = pos.copy()
    pos[1::3] = (pos[1::3].astype(np.float64) + 0.004).astype(np.float32)
    mesh = O.Mesh(pos, uv, idx, 0.15)
    mat = MAT if bend else dict(MAT, bendWarp=0.0, bendWeft=0.0)
    sc = O.Scene(mesh, mat)
    cs = O.ContactSystem(dict(O.DEFAULT_CONTACT, mu=mu), mesh.indices)
    cs.set_floor(0.0)
    sc.set_contact(cs)
    xs, newton, conv = [], [], 0
    for _ in range(steps):
        st = sc.step(1 / 60, newton_iters=40, pcg_max_iters=2000, grad_tol=1e-8, exact=exact, pcg_tol=1e-6,
                     drift=drift)
        xs.append(sc.positions)
        newton.append(st["newtonItersUsed"])
        conv += st["converged"] > 0
    return xs, np.array(newton), conv


def test_exact_step_drift_start_converges_to_the_same_steps():
    a, na, ca = _drape(8, 0.3, drift=True)
    b, nb, cb = _drape(8, 0.3, drift=False)
    assert ca == len(a) and cb == len(b), (ca, cb)
    err = max(float(np.max(np.abs(x - y)) / np.max(np.abs(y))) for x, y in zip(a, b))
    assert err <= 1e-7, err
    assert na[-10:].sum() < nb[-10:].sum(), (na, nb)


def test_exact_step_reaches_the_reference_steps_stationary_point():
    """Without bending and friction both modes solve the same equations; run
    to a tight gradient tolerance they land on the same positions."""
    a, _, ca = _drape(7, 0.0, bend=False, exact=True)
    b, _, cb = _drape(7, 0.0, bend=False, exact=False)
    assert ca == len(a), ca
    assert cb >= len(b) - 2, cb
    err = max(float(np.max(np.abs(x - y)) / np.max(np.abs(y))) for x, y in zip(a, b))
    assert err <= 1e-7, err


def _sliding_patches(mu):
    """Patch B lands on patch A (which rests on a floor) and slides across it:
    cloth-cloth VT and EE contacts plus floor contacts."""
    from tests.helpers import offset_mesh, preprocess_merged
    A = offset_mesh(4, 4, 0.08, 0.08, 0.0, 0.02, 0)
    B = offset_mesh(4, 4, 0.08, 0.08, 0.03, 0.0215, 0.011)
    mesh = preprocess_merged([A, B], 0.15)
    nA = len(A[0]) // 3
    v = np.zeros(mesh.n * 3)
    v[0::3] = np.where(np.arange(mesh.n) < nA, 0.1, -0.1)
    sc = O.Scene(mesh, MAT, v=v)
    cs = O.ContactSystem(dict(O.DEFAULT_CONTACT, mu=mu), mesh.indices)
    cs.set_floor(0.0185)
    sc.set_contact(cs)
    return sc, cs, mesh


def test_exact_step_converges_on_frictionless_self_contact():
    """VT and EE contacts between two patches: every exact step converges; the
    reference step at the same budget does not."""
    conv = {}
    for exact in (True, False):
        sc, _, _ = _sliding_patches(0.0)
        conv[exact] = 0
        for _ in range(12):
            st = sc.step(1 / 60, newton_iters=40, pcg_max_iters=2000, grad_tol=1e-8, exact=exact, pcg_tol=1e-6)
            assert st["vtPairs"] > 0 and st["eePairs"] > 0
            conv[exact] += st["converged"] > 0
    assert conv[True] == 12 and conv[False] < 12, conv


def test_cloth_cloth_friction_term_is_not_the_potential_gradient():
    """The reference's lagged friction term (contact-assembly.ts:318-341) on
    cloth-cloth contacts is not the gradient of the slip potential: it applies
    an EE contact's force to the second edge with the weights' sign flipped
    (both edges are pushed the same way), and a VT contact's force reaches the
    triangle's third vertex, which relativeSlip (contact-assembly.ts:344-367)
    leaves out. No merit is then consistent with the reference's equations, so
    exact-Newton mode converges there only without friction (the previous
    test); floor and one-sided static contacts match (the floor test above)."""
    rng = np.random.default_rng(23)
    sc, cs, mesh = _sliding_patches(0.3)
    x0 = sc.positions
    cs.begin_step(x0)
    no_f = O.ContactSystem(dict(O.DEFAULT_CONTACT, mu=0.0), mesh.indices)
    no_f.set_floor(0.0185)
    no_f.begin_step(x0)
    x = x0.copy()
    x[1::3] -= 0.0003 * (np.arange(mesh.n) >= mesh.n // 2)  # bring B within reach of A
    x[0::3] += rng.uniform(-2e-4, 2e-4, mesh.n)
    x[2::3] += rng.uniform(-2e-4, 2e-4, mesh.n)
    for c in (cs, no_f):
        c.update_active_set(x)
    ids, _ = cs.active()
    kinds = set(ids[:, 0].tolist())
    assert {0, 1, 2} <= kinds, kinds
    g_fric = cs.energy_grad(x)[1] - no_f.energy_grad(x)[1]
    fd = np.zeros(x.size)
    h = 1e-9
    for j in range(x.size):
        xp, xm = x.copy(), x.copy()
        xp[j] += h
        xm[j] -= h
        fd[j] = (cs.friction_potential(x, xp) - cs.friction_potential(x, xm)) / (2 * h)
    # the floor-only vertices (patch A's vertices in no cloth-cloth contact) agree ...
    cloth = set()
    for k, p, a, b, c, d in ids.tolist():
        if k in (0, 1):
            cloth.update(q for q in (p, a, b, c, d) if q >= 0)
    rest = [v for v in range(mesh.n) if v not in cloth]
    sel = np.array([3 * v + i for v in rest for i in range(3)])
    assert np.max(np.abs(fd[sel] - g_fric[sel])) <= 1e-6 * np.max(np.abs(g_fric)) + 1e-15
    # ... the cloth-cloth ones do not
    csel = np.array([3 * v + i for v in sorted(cloth) for i in range(3)])
    assert np.max(np.abs(fd[csel] - g_fric[csel])) > 0.1 * np.max(np.abs(g_fric[csel]))


def test_exact_step_converges_on_static_collider_friction():
    """tests/static-collider.test.ts:34-70's plate drape (mu 0.3): on one-sided
    static contacts (cloth vertex against static triangle, cloth edge against
    static edge) the friction potential's gradient is the reference's friction
    term, and every exact step converges; the reference step at the same
    budget mostly does not."""
    from tests.helpers import offset_mesh, preprocess_merged
    conv = {}
    for exact in (True, False):
        g = offset_mesh(4, 4, 0.08, 0.08, 0.01, 0.08, 0.01)
        mesh = preprocess_merged([g], 0.15)
        sc = O.Scene(mesh, MAT)
        spos = np.array([-0.05, 0.03, -0.05, 0.15, 0.03, -0.05, 0.15, 0.03, 0.15, -0.05, 0.03, 0.15], np.float32)
        cs = O.ContactSystem({"mu": 0.3}, mesh.indices)
        cs.set_static_mesh(spos, np.array([0, 1, 2, 0, 2, 3], np.uint32))
        sc.set_contact(cs)
        conv[exact], vt, ee = 0, 0, 0
        for _ in range(30):
            st = sc.step(1 / 60, newton_iters=40, pcg_max_iters=2000, grad_tol=1e-8, exact=exact, pcg_tol=1e-6)
            conv[exact] += st["converged"] > 0
            vt, ee = max(vt, st["vtPairs"]), max(ee, st["eePairs"])
        assert vt > 0 and ee > 0
    assert conv[True] == 30 and conv[False] < 15, conv
