"""The device contact primitives (closim_b200/csrc/contact_math.cuh and
jsmath.cuh), compiled for the host, agree bit for bit with the oracle on
random and edge-case inputs. Catches porting slips without a GPU. The device
math of exact-Newton mode (adjoint_math.cuh: hinge gradient and HVP, clamped
stress, clamped membrane block) agrees with the oracle's exact-mode pieces to
rounding."""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "hostcheck", "libhostcheck.so")


@pytest.fixture(scope="module")
def hc():
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "hostcheck")], check=True)
    L = C.CDLL(LIB)
    d = C.c_double
    p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    for name, res, args in [("hc_js_acos", d, [d]), ("hc_js_log", d, [d]), ("hc_js_cbrt", d, [d]),
                            ("hc_hypot3", d, [d, d, d]), ("hc_closest_vt", None, [p, p]),
                            ("hc_closest_ee", None, [p, p]), ("hc_vt_ccd", d, [p, p, d]), ("hc_ee_ccd", d, [p, p, d]),
                            ("hc_trial_ccd", d, [p, p, d, C.c_int]),
                            ("hc_solve_cubic01", C.c_int, [d, d, d, d, p]), ("hc_barrier_value", d, [d, d]),
                            ("hc_barrier_grad", d, [d, d, d]), ("hc_barrier_curv", d, [d, d, d])]:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


def same(a, b):
    return (a == b) or (math.isnan(a) and math.isnan(b))


def test_js_math_matches_oracle(hc):
    ol = O.lib()
    for f in ["orc_js_acos", "orc_js_log", "orc_js_cbrt"]:
        getattr(ol, f).restype = C.c_double
        getattr(ol, f).argtypes = [C.c_double]
    rng = np.random.default_rng(5)
    xs = list(rng.uniform(-1, 1, 3000)) + list(np.exp(rng.uniform(-700, 700, 3000))) + \
        [0.0, -0.0, 1.0, -1.0, 5e-324, 1e-310, math.inf, -math.inf, math.nan, 1 - 1e-16, -1 + 1e-16]
    for x in xs:
        assert same(hc.hc_js_acos(x), ol.orc_js_acos(x)), x
        assert same(hc.hc_js_log(x), ol.orc_js_log(x)), x
        assert same(hc.hc_js_cbrt(x), ol.orc_js_cbrt(x)), x
        assert same(hc.hc_js_cbrt(-x), ol.orc_js_cbrt(-x)), x


def _random_stencils(rng, k, scale):
    base = rng.uniform(-scale, scale, (k, 4, 3))
    move = base + rng.normal(0, scale * 0.3, (k, 4, 3)) * rng.integers(0, 2, (k, 1, 1))
    return base, move


def test_closest_points_match_oracle(hc):
    rng = np.random.default_rng(1)
    for _ in range(3000):
        q = rng.uniform(-1, 1, 12) * rng.choice([1e-3, 1.0])
        o1 = np.zeros(6)
        hc.hc_closest_vt(q, o1)
        assert np.array_equal(o1, O.closest_vt(q[0:3], q[3:6], q[6:9], q[9:12]))
        hc.hc_closest_ee(q, o1)
        assert np.array_equal(o1, O.closest_ee(q[0:3], q[3:6], q[6:9], q[9:12]))


def test_ccd_matches_oracle(hc):
    rng = np.random.default_rng(2)
    hits = 0
    for _ in range(3000):
        P0, P1 = _random_stencils(rng, 1, 0.01)
        P0 = np.ascontiguousarray(P0.ravel())
        P1 = np.ascontiguousarray(P1.ravel())
        for th in (1e-4, 2e-3):
            a = hc.hc_vt_ccd(P0, P1, th)
            b = O.vt_ccd(P0, P1, th)
            assert same(a, b), (a, b)
            c = hc.hc_ee_ccd(P0, P1, th)
            d = O.ee_ccd(P0, P1, th)
            assert same(c, d), (c, d)
            hits += (0 < a < 1) + (0 < c < 1)
    assert hits > 0


def _stencil_dist(P, kind):
    q = P.reshape(4, 3)
    o = O.closest_vt(q[0], q[1], q[2], q[3]) if kind == 0 else O.closest_ee(q[0], q[1], q[2], q[3])
    return float(o[2])


def test_trial_ccd_gate_matches_oracle(hc):
    """The trial kernel's CCD skips the root search when the sweep bound
    (d0 + dT) / 2 - E, or its lower bound dT - 2E, clears the thickness. It must
    return exactly the reference's CCD: random stencils, cloth-like near-parallel
    layers closing in, and thicknesses placed on and around each gate's
    threshold (relative offsets down to 1e-9)."""
    rng = np.random.default_rng(11)
    checked = gated = 0

    def check(P0, P1, th):
        nonlocal checked
        for kind, ref in ((0, O.vt_ccd), (1, O.ee_ccd)):
            a = hc.hc_trial_ccd(P0, P1, th, kind)
            b = ref(P0, P1, th)
            assert same(a, b), (kind, th, a, b, P0.tolist(), P1.tolist())
            checked += 1

    for it in range(1500):
        if it % 2 == 0:
            P0, P1 = _random_stencils(rng, 1, 0.01)
            P0 = np.ascontiguousarray(P0.ravel())
            P1 = np.ascontiguousarray(P1.ravel())
        else:
            # two cloth layers: a triangle and a vertex (or edges) a few dHat apart, closing in
            h = 4e-3
            tri = np.array([[0, 0, 0], [h, 0, 0], [0, 0, h]]) + rng.normal(0, 2e-4, (3, 3))
            top = np.array([h / 3, 0, h / 3]) + rng.normal(0, 2e-4, 3)
            top[1] = rng.uniform(1e-4, 2e-3)
            P0 = np.concatenate([top, tri.ravel()]) + rng.uniform(-1, 1)
            P1 = P0 + rng.normal(0, 1, 12) * 10 ** rng.uniform(-6, -3)
            P1 += np.tile(rng.normal(0, 1e-2, 3), 4)  # common translation
        for kind in (0, 1):
            dT = _stencil_dist(P1, kind)
            d0 = _stencil_dist(P0, kind)
            m0 = P1.reshape(4, 3) - P0.reshape(4, 3)
            E = float(np.max(np.linalg.norm(m0 - m0.mean(axis=0), axis=1)))
            dev = float(np.max(np.abs(m0 - m0.mean(axis=0))))
            for crit in (dT - 2 * E, (d0 + dT) / 2 - E, d0 - 4 * dev, d0):
                if not (crit > 0):
                    continue
                for rel in (-1e-5, -1e-7, -1e-9, 0.0, 1e-9, 1e-7, 1e-5):
                    th = crit * (1 + rel)
                    gated += dT - 2 * E > th
                    check(P0, P1, th)
        for th in (1e-4, 2e-3):
            check(P0, P1, th)
    assert checked > 40000 and gated > 1000, (checked, gated)


def test_cubic_and_barrier_match_oracle(hc):
    rng = np.random.default_rng(3)
    o = np.zeros(3)
    for _ in range(5000):
        a = rng.normal(0, 1, 4) * rng.choice([1e-14, 1e-6, 1.0], 4)
        k = hc.hc_solve_cubic01(*a, o)
        assert list(o[:k]) == O.solve_cubic01(*a)
    for d in np.concatenate([rng.uniform(0, 2e-3, 2000), [1e-12, 1e-13, 2e-3, 5e-3, 0.0]]):
        assert same(hc.hc_barrier_value(d, 2e-3), O.barrier_value(d, 2e-3))
        assert same(hc.hc_barrier_grad(d, 2e-3, 50.0), O.lib().orc_barrier_grad_scalar(d, 2e-3, 50.0, 1.0))


def test_bending_gradient_and_hvp(hc):
    """The adjoint's analytic hinge gradient against central differences of the
    reference's hinge energy (acos form, bending.ts:7-16), and its dual-number
    HVP against central differences of that gradient. Near-flat hinges with
    flat (pi) and curved (2.5 rad) rest angles."""
    p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    hc.hc_bend_grad.restype = C.c_double
    hc.hc_bend_grad.argtypes = [p, p, C.c_double, p]
    hc.hc_bend_hvp.restype = None
    hc.hc_bend_hvp.argtypes = [p, p, p, C.c_double, p]
    rng = np.random.default_rng(11)
    base = np.array([0, 0, 0, 1, 0, 0, 0.4, 0, 1, 0.6, 0, -1], np.float64)
    worst_e = worst_g = worst_h = 0.0
    for trial in range(60):
        q = base + rng.uniform(-1, 1, 12) * (0.01 if trial < 30 else 0.1)
        meta = np.array([np.pi if trial % 2 else 2.5, 0.7, 0.9])
        k = 2e-4
        g = np.zeros(12)
        e = hc.hc_bend_grad(q, meta, k, g)
        e_ref = O.hinge_energy(q, meta, k)
        worst_e = max(worst_e, abs(e - e_ref) / max(abs(e_ref), 1e-30))
        fd = np.zeros(12)
        for a in range(12):
            qp, qm = q.copy(), q.copy()
            qp[a] += 1e-6
            qm[a] -= 1e-6
            fd[a] = (O.hinge_energy(qp, meta, k) - O.hinge_energy(qm, meta, k)) / 2e-6
        worst_g = max(worst_g, np.max(np.abs(fd - g)) / max(np.max(np.abs(g)), 1e-30))
        v = rng.uniform(-1, 1, 12)
        hv = np.zeros(12)
        hc.hc_bend_hvp(q, v, meta, k, hv)
        gp, gm = np.zeros(12), np.zeros(12)
        hc.hc_bend_grad(q + 1e-6 * v, meta, k, gp)
        hc.hc_bend_grad(q - 1e-6 * v, meta, k, gm)
        worst_h = max(worst_h, np.max(np.abs((gp - gm) / 2e-6 - hv)) / max(np.max(np.abs(hv)), 1e-30))
    assert worst_e < 1e-7, worst_e
    assert worst_g < 1e-4, worst_g
    assert worst_h < 1e-6, worst_h


def test_bending_gradient_large_angles(hc):
    """The mixed path takes the analytic hinge gradient in place of the
    reference's central differences (bending.ts:19-44), so it must hold away
    from flat too: hinges folded by 0.3 to 3.1 rad about the shared edge, flat
    rest angle, against central differences of the reference's hinge energy."""
    p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    hc.hc_bend_grad.restype = C.c_double
    hc.hc_bend_grad.argtypes = [p, p, C.c_double, p]
    rng = np.random.default_rng(3)
    meta = np.array([np.pi, 0.7, 0.9])
    k = 2e-4
    for ang in (0.3, 1.0, 1.5, 2.0, 2.5, 2.9, 3.1):
        worst = 0.0
        for _ in range(10):
            # edge along x; wing 2 in +z, wing 3 turned by `ang` about x from -z
            q = np.array([0, 0, 0, 1, 0, 0, 0.4, 0, 1, 0.6, np.sin(ang), -np.cos(ang)], np.float64)
            q = q + rng.uniform(-0.02, 0.02, 12)
            g = np.zeros(12)
            hc.hc_bend_grad(q, meta, k, g)
            fd = np.zeros(12)
            for a in range(12):
                qp, qm = q.copy(), q.copy()
                qp[a] += 1e-6
                qm[a] -= 1e-6
                fd[a] = (O.hinge_energy(qp, meta, k) - O.hinge_energy(qm, meta, k)) / 2e-6
            worst = max(worst, np.max(np.abs(fd - g)) / max(np.max(np.abs(fd)), 1e-30))
        assert worst < 1e-6, (ang, worst)


def test_membrane_block9_matches_oracle(hc):
    """The mixed path's closed-form 9x9 membrane block against the oracle's
    restatement of membrane-blocks.ts:21-98 (same Hessian, different algebra)."""
    p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    hc.hc_membrane_block9.restype = None
    hc.hc_membrane_block9.argtypes = [p, p, C.c_double, p, p]
    rng = np.random.default_rng(21)
    worst = 0.0
    for trial in range(40):
        x9 = np.array([0, 0, 0, 0.02, 0, 0, 0, 0, 0.02]) + rng.uniform(-4e-3, 4e-3, 9)
        inv = np.array([50.0, 0.0, 0.0, 50.0]) + rng.uniform(-5, 5, 4)
        area = 2e-4 * (1 + 0.1 * rng.uniform())
        mat = dict(arealDensity=0.2, thickness=1.0, C00=rng.uniform(2e3, 1e4), C11=rng.uniform(2e3, 1e4),
                   C01=rng.uniform(0, 500), G=rng.uniform(5e2, 2e3), bendWarp=1e-4, bendWeft=1e-4, damping=0)
        ref = O.tri_hessian9(x9, inv, np.float32(area), mat)
        h = np.zeros(81)
        hc.hc_membrane_block9(x9, inv, mat["thickness"] * float(np.float32(area)),
                              np.array([mat["C00"], mat["C11"], mat["C01"], mat["G"]]), h)
        worst = max(worst, np.max(np.abs(h.reshape(9, 9) - ref)) / np.max(np.abs(ref)))
    assert worst < 1e-12, worst


def test_exact_mode_bending_matches_the_oracle(hc):
    """Exact-Newton mode's hinge gradient and full bending HVP (the FP64
    path's) against the oracle's exact hinge gradient and Hessian, written
    independently (hyper-dual numbers): agreement to rounding, near flat and
    folded up to 2.8 rad, flat and curved rest angles."""
    p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    hc.hc_bend_grad.restype = C.c_double
    hc.hc_bend_grad.argtypes = [p, p, C.c_double, p]
    hc.hc_bend_hvp.restype = None
    hc.hc_bend_hvp.argtypes = [p, p, p, C.c_double, p]
    rng = np.random.default_rng(19)
    k = 2e-4
    worst_g = worst_h = 0.0
    for trial, ang in enumerate([1e-6, 1e-3, 0.05, 0.3, 1.0, 2.0, 2.8] * 6):
        q = np.array([0, 0, 0, 1, 0, 0, 0.4, 0, 1, 0.6, np.sin(ang), -np.cos(ang)], np.float64)
        q = q * 0.02 + rng.uniform(-1e-4, 1e-4, 12) * (trial % 2)
        meta = np.array([np.pi if trial % 3 else 2.6, 0.02, 3e-4])
        g = np.zeros(12)
        hc.hc_bend_grad(q, meta, k, g)
        go = O.hinge_grad_exact(q, meta, k)
        worst_g = max(worst_g, np.max(np.abs(g - go)) / max(np.max(np.abs(go)), 1e-300))
        v = rng.uniform(-1, 1, 12)
        hv = np.zeros(12)
        hc.hc_bend_hvp(q, v, meta, k, hv)
        ho = O.hinge_hess_exact(q, meta, k) @ v
        worst_h = max(worst_h, np.max(np.abs(hv - ho)) / max(np.max(np.abs(ho)), 1e-300))
    assert worst_g < 1e-9, worst_g
    assert worst_h < 1e-8, worst_h


def test_exact_mode_psd_stress_matches_the_oracle(hc):
    p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    hc.hc_psd_stress.restype = None
    hc.hc_psd_stress.argtypes = [p]
    rng = np.random.default_rng(29)
    cases = [rng.normal(size=3) * rng.uniform(1, 1e4) for _ in range(500)]
    cases += [np.array(c, float) for c in ([3, -2, 0], [-3, 2, 0], [-1, -1, 0], [2, 2, 0], [0, 0, 0], [1, -1, 1e-20])]
    for c in cases:
        s = c.copy()
        hc.hc_psd_stress(s)
        ref = np.array(O.stress_positive_part(*c))
        assert np.max(np.abs(s - ref)) <= 1e-13 * max(np.max(np.abs(c)), 1e-300), (c, s, ref)


def test_exact_mode_membrane_block_matches_the_oracle(hc):
    """The Schwarz / FP64 exact-mode membrane block with the clamped stress
    (membrane_block9, psd) against the oracle's exact-mode membrane HVP on
    single compressed, sheared and stretched triangles."""
    p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    hc.hc_membrane_block9_psd.restype = None
    hc.hc_membrane_block9_psd.argtypes = [p, p, C.c_double, p, p]
    rng = np.random.default_rng(31)
    mat = dict(O.DEFAULT_MATERIAL, C00=5e3, C11=3e3, C01=400.0, G=1e3, bendWarp=0.0, bendWeft=0.0)
    pos = np.array([0, 0, 0, 0.01, 0, 0, 0.002, 0, 0.012], np.float32)
    mesh = O.Mesh(pos, np.array([0, 0, 1, 0, 0, 1], np.float32), np.array([0, 1, 2], np.uint32), 0.2)
    inv = mesh.invDm.astype(np.float64)
    s = mat["thickness"] * float(mesh.areas[0])
    C4 = np.array([mat["C00"], mat["C11"], mat["C01"], mat["G"]])
    worst = 0.0
    for trial in range(60):
        A = np.eye(3) + rng.uniform(-0.08, 0.08, (3, 3))
        A[0, 0] *= (0.9, 1.0, 1.05)[trial % 3]
        x = (pos.astype(np.float64).reshape(3, 3) @ A.T + rng.uniform(-1, 1, 3)).ravel()
        H = np.zeros(81)
        hc.hc_membrane_block9_psd(x, inv, s, C4, H)
        v = rng.uniform(-1, 1, 9)
        ho = O.internal_hvp_exact(mesh, mat, x, v)
        hv = H.reshape(9, 9) @ v
        worst = max(worst, np.max(np.abs(hv - ho)) / np.max(np.abs(ho)))
        assert np.min(np.linalg.eigvalsh(H.reshape(9, 9))) >= -1e-9 * np.max(np.abs(H))
    assert worst < 1e-10, worst
