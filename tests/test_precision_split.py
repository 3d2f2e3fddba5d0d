"""Why the mixed path assembles the Newton gradient in FP64 (CPU check).

The mixed path runs the linear solve (HVP, Schwarz, PCG vectors) in FP32 and
keeps the gradient assembly, dot products, energies and CCD in FP64. An FP32
gradient would set a floor under the Newton residual: on the 64 x 64 floor
drape sheet, evaluating the same membrane gradient in FP32 differs from the
FP64 one by about 1e-2 in the 2-norm, set by the rounding of positions
(0.3-0.8 m) in FP32, whatever the strain. Newton cannot converge below that
floor, while the 1e-5 relative position gate needs gradient norms near 1e-8
(the converged steps reach 1e-9..1e-11). This test measures the floor with a
restatement of the membrane gradient (membrane.ts:17-80) in numpy, checked
against the oracle in FP64.
"""
import numpy as np

from closim_b200 import configs
from oracle import oracle as O


def membrane_gradient(x, idx, inv, area, mat, dt):
    X = x.reshape(-1, 3).astype(dt)
    a, b, c, d = [inv[:, k].astype(dt) for k in range(4)]
    e1 = X[idx[:, 1]] - X[idx[:, 0]]
    e2 = X[idx[:, 2]] - X[idx[:, 0]]
    F0 = a[:, None] * e1 + c[:, None] * e2
    F1 = b[:, None] * e1 + d[:, None] * e2
    E00 = dt(0.5) * ((F0 * F0).sum(1) - 1)
    E11 = dt(0.5) * ((F1 * F1).sum(1) - 1)
    E01 = dt(0.5) * (F0 * F1).sum(1)
    S00 = dt(mat["C00"]) * E00 + dt(mat["C01"]) * E11
    S11 = dt(mat["C11"]) * E11 + dt(mat["C01"]) * E00
    S01 = dt(2 * mat["G"]) * E01
    P0 = F0 * S00[:, None] + F1 * S01[:, None]
    P1 = F0 * S01[:, None] + F1 * S11[:, None]
    s = (dt(mat["thickness"]) * area.astype(dt))[:, None]
    g1 = s * (P0 * a[:, None] + P1 * b[:, None])
    g2 = s * (P0 * c[:, None] + P1 * d[:, None])
    G = np.zeros_like(X)
    np.add.at(G, idx[:, 0], -(g1 + g2))
    np.add.at(G, idx[:, 1], g1)
    np.add.at(G, idx[:, 2], g2)
    return G.ravel().astype(np.float64)


def test_fp32_gradient_floor_exceeds_the_converged_tolerance():
    cfg = configs.floor_drape()
    mesh = O.Mesh(cfg["pos"], cfg["uv"], cfg["idx"], cfg["density"])
    m = cfg["material"]
    mat = dict(arealDensity=m["arealDensityKgM2"], thickness=m["thickness"], C00=m["stretchWarp"],
               C11=m["stretchWeft"], C01=m["stretchCoupling"], G=m["shear"], bendWarp=0.0, bendWeft=0.0, damping=0.0)
    idx = cfg["idx"].reshape(-1, 3).astype(np.int64)
    inv = mesh.invDm.reshape(-1, 4).astype(np.float64)
    area = mesh.areas.astype(np.float64)
    rng = np.random.default_rng(0)
    for amp in (1e-4, 1e-3):
        x = cfg["x"] + rng.uniform(-amp, amp, cfg["x"].size)
        g64 = membrane_gradient(x, idx, inv, area, mat, np.float64)
        _, gref, _ = O.eval_internal(mesh, mat, x)
        assert np.linalg.norm(g64 - gref) <= 1e-12 * np.linalg.norm(gref)  # the restatement is the oracle's
        floor = np.linalg.norm(membrane_gradient(x, idx, inv, area, mat, np.float32) - g64)
        print(f"jitter {amp:g} m: FP32 gradient floor {floor:.3e}")
        assert floor > 1e-4 > 1e-8  # four orders above any tolerance the 1e-5 gate can use
