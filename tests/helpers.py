"""Scene builders shared by the tests (mirrors tests/helpers.ts of the reference)."""
import math

import numpy as np

from oracle import oracle as O


def offset_mesh(nx, ny, w, h, ox, oy, oz):
    """tests/helpers.ts:5-17 offsetMesh: buildGrid + Float32Array offsets."""
    pos, uv, idx = O.build_grid(nx, ny, w, h)
    p = pos.astype(np.float64)
    p[0::3] += ox
    p[1::3] += oy
    p[2::3] += oz
    return p.astype(np.float32), uv, idx


def merge_parts(parts):
    """tests/helpers.ts:19-37 mergeParts."""
    pos, uv, idx = [], [], []
    vo = 0
    for p, u, i in parts:
        pos.append(p)
        uv.append(u)
        idx.append(i.astype(np.int64) + vo)
        vo += len(p) // 3
    return (np.concatenate(pos).astype(np.float32), np.concatenate(uv).astype(np.float32),
            np.concatenate(idx).astype(np.uint32))


def preprocess_merged(parts, density):
    pos, uv, idx = merge_parts(parts)
    return O.Mesh(pos, uv, idx, density)


def audit_min_distance(x, mesh, exclude_adjacent=True):
    """tests/helpers.ts:45-80 auditMinDistance (brute force, small meshes only)."""
    idx = mesh.indices.reshape(-1, 3)
    m = len(idx)
    v2t = {}
    for t in range(m):
        for v in idx[t]:
            v2t.setdefault(int(v), []).append(t)
    adj = set()
    if exclude_adjacent:
        for lst in v2t.values():
            for i in range(len(lst)):
                for j in range(i + 1, len(lst)):
                    adj.add((min(lst[i], lst[j]), max(lst[i], lst[j])))
    P = lambda v: x[v * 3:v * 3 + 3]
    best = math.inf
    edges = [(0, 1), (1, 2), (2, 0)]
    for tA in range(m):
        for tB in range(tA + 1, m):
            if exclude_adjacent and (tA, tB) in adj:
                continue
            A, B = idx[tA], idx[tB]
            for p in A:
                best = min(best, O.closest_vt(P(p), P(B[0]), P(B[1]), P(B[2]))[2])
            for p in B:
                best = min(best, O.closest_vt(P(p), P(A[0]), P(A[1]), P(A[2]))[2])
            for ea in edges:
                for eb in edges:
                    a, b, c, d = A[ea[0]], A[ea[1]], B[eb[0]], B[eb[1]]
                    if a == c or a == d or b == c or b == d:
                        continue
                    best = min(best, O.closest_ee(P(a), P(b), P(c), P(d))[2])
    return best


def pin_column(x, pred):
    pins = {}
    n = len(x) // 3
    for i in range(n):
        if pred(x[i * 3], x[i * 3 + 1], x[i * 3 + 2], i):
            pins[i] = (x[i * 3], x[i * 3 + 1], x[i * 3 + 2])
    return pins


def oracle_scene(cfg):
    """Oracle scene (CpuSolver equivalent) from a closim_b200.configs workload dict."""
    mesh = O.Mesh(cfg["pos"], cfg["uv"], cfg["idx"], cfg["density"])
    m = cfg["material"]
    mat = dict(arealDensity=m["arealDensityKgM2"], thickness=m["thickness"], C00=m["stretchWarp"],
               C11=m["stretchWeft"], C01=m["stretchCoupling"], G=m["shear"], bendWarp=m["bendWarp"],
               bendWeft=m["bendWeft"], damping=m["damping"])
    sc = O.Scene(mesh, mat, gravity=cfg["gravity"], x=cfg["x"], v=cfg["v"])
    c = cfg["contact"]
    if c is not None:
        cs = O.ContactSystem(dict(dHat=c["dHatM"], kappa=c["kappaJ"], dMin=c["dMinM"], mu=c["frictionMu"],
                                  eps=c["frictionEpsM"]), mesh.indices)
        if c.get("floorY") is not None:
            cs.set_floor(c["floorY"])
        if c.get("staticPos") is not None:
            cs.set_static_mesh(c["staticPos"], c["staticIdx"])
        sc.set_contact(cs)
        sc._cs = cs
    return sc


def oracle_step_kwargs(cfg):
    o = cfg["options"]
    return dict(newton_iters=o["newtonIters"], pcg_max_iters=o["pcgMaxIters"], grad_tol=o["gradTol"],
                ls_iters=o["lineSearchIters"], precond=o["precond"])
