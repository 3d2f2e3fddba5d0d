"""Synthetic workloads of the cloth step (seeded), in the reference's y-up frame.

A workload is a plain dict (arrays + parameters) so the same inputs can be fed
to the CUDA solver and to any checker. Config text uses z-up; here config "z"
is the reference's y (vertical), config "z = c" floors are y = c.

  strip_pull    41 x 9 strip, left column pinned, right column pulled +x at 0.1 m/s
  floor_drape   64 x 64 sheet released 0.3 m above a y = 0 floor (barrier + friction)
  sphere_drape  256 x 256 sheet dropped onto a static sphere, folding onto itself
  material_fit  96 x 96 sheet hung from two corners, loss on the final positions (adjoint)
  batch_sheets  512 independent sheets of uneven size, stepped together (batched solver)
"""
from __future__ import annotations

import numpy as np

from .solver import (ClothMaterial, ClothScene, ContactParams, ContactSystem, buildGrid, createScene,
                     preprocess)

# Grid builder of the workloads: buildGrid (src/mesh/mesh.ts:17-48) through the
# CUDA library's cs_build_grid by default. A caller that must not load the
# library (a CPU-only timing of the same workload) installs another
# implementation of the same function with set_grid_builder.
_GRID_BUILDER = None


def set_grid_builder(fn) -> None:
    """fn(nx, ny, w, h) -> (pos f32[3n], uv f32[2n], idx u32[6 nx ny]); None restores buildGrid."""
    global _GRID_BUILDER
    _GRID_BUILDER = fn


def _grid(nx, ny, w, h):
    return (_GRID_BUILDER or buildGrid)(nx, ny, w, h)


def _material(**kw):
    m = dict(arealDensityKgM2=0.2, thickness=1.0, stretchWarp=5e3, stretchWeft=5e3, stretchCoupling=0.0,
             shear=1e3, bendWarp=1e-4, bendWeft=1e-4, damping=0.0)
    m.update(kw)
    return m


def strip_pull(seed: int = 1, nx: int = 40, ny: int = 8, w: float = 1.0, hgt: float = 0.2, steps: int = 100):
    """1.0 x 0.2 m strip, 41 x 9 vertices (640 triangles); C00 = C11 = 5e3 N/m,
    G = 1e3, k_bend = 1e-4, 0.2 kg/m^2; h = 0.01 s; Newton tol 1e-6; Jacobi PCG.
    Seeded U(+-1e-4) jitter on the vertical coordinate of the initial state."""
    pos, uv, idx = _grid(nx, ny, w, hgt)
    n = len(pos) // 3
    rng = np.random.default_rng(seed)
    x = pos.astype(np.float64)
    x[1::3] += rng.uniform(-1e-4, 1e-4, n)
    left = [i for i in range(n) if i % (nx + 1) == 0]
    right = [i for i in range(n) if i % (nx + 1) == nx]
    return dict(name="strip_pull", pos=pos, uv=uv, idx=idx, density=0.2, material=_material(), x=x,
                v=np.zeros(n * 3), gravity=(0.0, -9.81, 0.0), h=0.01, steps=steps,
                options=dict(newtonIters=10, pcgMaxIters=60, gradTol=1e-6, lineSearchIters=10, precond="jacobi"),
                fixed_pins=left, moving_pins=right, pin_velocity=(0.1, 0.0, 0.0), contact=None, seed=seed)


def floor_drape(seed: int = 2, nx: int = 63, ny: int = 63, w: float = 0.8, hgt: float = 0.8, steps: int = 240,
                precond: str = "schwarz", height: float = 0.3):
    """0.8 x 0.8 m sheet, 64 x 64 vertices (7938 triangles), 0.3 m (`height`)
    above a y = 0 floor; dHat = 1e-3 m, mu = 0.3; C00 = 5e3, C11 = 3e3, G = 1e3;
    h = 1/120 s; Schwarz-block PCG. Seeded U(+-1e-3) vertical noise."""
    pos, uv, idx = _grid(nx, ny, w, hgt)
    pos = pos.copy()
    pos[1::3] = (pos[1::3].astype(np.float64) + height).astype(np.float32)
    n = len(pos) // 3
    rng = np.random.default_rng(seed)
    x = pos.astype(np.float64)
    x[1::3] += rng.uniform(-1e-3, 1e-3, n)
    return dict(name="floor_drape", pos=pos, uv=uv, idx=idx, density=0.2, material=_material(stretchWeft=3e3),
                x=x, v=np.zeros(n * 3), gravity=(0.0, -9.81, 0.0), h=1.0 / 120, steps=steps,
                options=dict(newtonIters=10, pcgMaxIters=60, gradTol=1e-5, lineSearchIters=10, precond=precond),
                fixed_pins=[], moving_pins=[], pin_velocity=(0.0, 0.0, 0.0),
                contact=dict(dHatM=1e-3, kappaJ=50.0, dMinM=1e-4, frictionMu=0.3, frictionEpsM=1e-4, floorY=0.0),
                seed=seed)


def sphere_mesh(radius: float, segments: int = 12, rings: int = 6, center=(0.0, 0.0, 0.0)):
    """Static UV-sphere collider (src/collision/avatar-collider.ts:273-300):
    a top pole, rings - 1 rings of `segments` vertices, a bottom pole;
    2 * segments * (rings - 1) triangles. The vertices are the reference's
    positions moved by `center` (added in double precision) and stored as f32,
    as ContactSystem.setStaticMesh stores them."""
    if not (6 <= segments <= 64 and 3 <= rings <= 32 and radius > 0):
        raise ValueError("sphere needs radius > 0, 6 <= segments <= 64, 3 <= rings <= 32")
    pts = [(0.0, radius, 0.0)]
    for j in range(1, rings):
        theta = np.pi * j / rings
        for i in range(segments):
            phi = 2 * np.pi * i / segments
            pts.append((radius * np.sin(theta) * np.cos(phi), radius * np.cos(theta), radius * np.sin(theta) * np.sin(phi)))
    bottom = len(pts)
    pts.append((0.0, -radius, 0.0))
    idx = []
    for i in range(segments):
        nxt = (i + 1) % segments
        idx += [0, 1 + i, 1 + nxt]
        for ring in range(rings - 2):
            a, b = 1 + ring * segments + i, 1 + ring * segments + nxt
            c, d = a + segments, b + segments
            idx += [a, c, b, b, c, d]
        last = 1 + (rings - 2) * segments
        idx += [last + i, bottom, last + nxt]
    pos = (np.asarray(pts, np.float64) + np.asarray(center, np.float64)).astype(np.float32).ravel()
    return pos, np.asarray(idx, np.uint32)


def sphere_drape(seed: int = 3, nx: int = 255, ny: int = 255, w: float = 1.0, hgt: float = 1.0, steps: int = 300,
                 radius: float = 0.2, drop: float = 0.4, segments: int = 32, rings: int = 16,
                 precond: str = "schwarz"):
    """1.0 x 1.0 m sheet, 256 x 256 vertices (130,050 triangles), dropped onto a
    static sphere (r = 0.2 m, centre 0.4 m below the sheet under its middle,
    32 segments x 16 rings = 960 triangles) and folding onto itself: LBVH
    broadphase, VT + EE CCD, IPC barrier dHat = 5e-4 m, mu = 0.2, h = 1/200 s.
    Seeded U(+-5e-4) in-plane (x, z) jitter of the initial state."""
    pos, uv, idx = _grid(nx, ny, w, hgt)
    n = len(pos) // 3
    rng = np.random.default_rng(seed)
    x = pos.astype(np.float64)
    x[0::3] += rng.uniform(-5e-4, 5e-4, n)
    x[2::3] += rng.uniform(-5e-4, 5e-4, n)
    centre = (0.5 * w, float(pos[1]) - drop, 0.5 * hgt)
    spos, sidx = sphere_mesh(radius, segments, rings, centre)
    return dict(name="sphere_drape", pos=pos, uv=uv, idx=idx, density=0.2, material=_material(), x=x,
                v=np.zeros(n * 3), gravity=(0.0, -9.81, 0.0), h=1.0 / 200, steps=steps,
                options=dict(newtonIters=10, pcgMaxIters=60, gradTol=1e-5, lineSearchIters=10, precond=precond),
                fixed_pins=[], moving_pins=[], pin_velocity=(0.0, 0.0, 0.0),
                contact=dict(dHatM=5e-4, kappaJ=50.0, dMinM=1e-4, frictionMu=0.2, frictionEpsM=1e-4, floorY=None,
                             staticPos=spos, staticIdx=sidx),
                sphere=dict(radius=radius, segments=segments, rings=rings, centre=centre), seed=seed)


def material_fit(seed: int = 4, nx: int = 95, ny: int = 95, w: float = 0.6, hgt: float = 0.6, steps: int = 200,
                 checkpoint_every: int = 20, perturb: float = 0.2, floor_y: float = -0.7,
                 newton_iters: int = 40, pcg_max_iters: int = 600, grad_tol: float = 1e-9):
    """Material fit through the adjoint: a 0.6 x 0.6 m sheet of 96 x 96
    vertices (18,050 triangles) hung from the two corners of its z = 0 edge,
    200 steps of h = 0.01 s, floor contact at y = -0.7. The target final
    positions come from ground-truth parameters (C00 = 6e3, C11 = 3e3,
    G = 8e2, k_bend = 2e-4 N/m); the fit starts from each parameter scaled by a
    seeded U(1 - perturb, 1 + perturb). Loss = mean over vertices of
    |x_N - x_N*|^2. The stepper budget lets every step converge (gradTol 1e-9),
    which the implicit-function-theorem gradient assumes."""
    pos, uv, idx = _grid(nx, ny, w, hgt)
    n = len(pos) // 3
    rng = np.random.default_rng(seed)
    theta_gt = np.array([6e3, 3e3, 8e2, 2e-4])
    theta0 = theta_gt * rng.uniform(1 - perturb, 1 + perturb, 4)
    mat = _material(stretchWarp=theta0[0], stretchWeft=theta0[1], shear=theta0[2], bendWarp=theta0[3],
                    bendWeft=theta0[3])
    return dict(name="material_fit", pos=pos, uv=uv, idx=idx, density=0.2, material=mat, x=pos.astype(np.float64),
                v=np.zeros(n * 3), gravity=(0.0, -9.81, 0.0), h=0.01, steps=steps, checkpoint_every=checkpoint_every,
                options=dict(newtonIters=newton_iters, pcgMaxIters=pcg_max_iters, gradTol=grad_tol,
                             lineSearchIters=10, precond="schwarz"),
                fixed_pins=[0, nx], moving_pins=[], pin_velocity=(0.0, 0.0, 0.0),
                contact=dict(dHatM=1e-3, kappaJ=50.0, dMinM=1e-4, frictionMu=0.3, frictionEpsM=1e-4, floorY=floor_y),
                theta_gt=theta_gt, theta0=theta0, seed=seed)


def batch_sheets(seed: int = 5, count: int = 512, side_min: int = 16, side_max: int = 128, steps: int = 100,
                 sheet_size: float = 0.5, floor_y: float = -0.5, spacing: float = 0.0):
    """Batched uneven instances: `count` independent sheets, vertex-grid side
    s ~ U{side_min..side_max} (seeded), each buildGrid(s-1, s-1, L, L) with
    L = sheet_size; C00, C11 ~ U[2e3, 1e4], G ~ U[5e2, 2e3], k_bend ~ logU[1e-5,
    1e-3]; pinned at two seeded boundary vertices; floor contact at y = -0.5;
    h = 0.01 s. Sheets do not interact (each is its own scene); `spacing`
    only offsets them in x for viewing. Returns a list of single-sheet
    workload dicts sharing h, gravity, contact parameters and options."""
    rng = np.random.default_rng(seed)
    sheets = []
    for i in range(count):
        sd = int(rng.integers(side_min, side_max + 1))
        pos, uv, idx = _grid(sd - 1, sd - 1, sheet_size, sheet_size)
        n = len(pos) // 3
        x = pos.astype(np.float64)
        x[0::3] += i * spacing
        c00, c11 = rng.uniform(2e3, 1e4, 2)
        g = rng.uniform(5e2, 2e3)
        kb = float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-3))))
        boundary = [j for j in range(n) if j % sd in (0, sd - 1) or j // sd in (0, sd - 1)]
        pins = sorted(int(v) for v in rng.choice(boundary, 2, replace=False))
        sheets.append(dict(name=f"batch_sheet_{i}", pos=pos, uv=uv, idx=idx, density=0.2,
                           material=_material(stretchWarp=float(c00), stretchWeft=float(c11), shear=float(g),
                                              bendWarp=kb, bendWeft=kb),
                           x=x, v=np.zeros(n * 3), gravity=(0.0, -9.81, 0.0), h=0.01, steps=steps,
                           options=dict(newtonIters=10, pcgMaxIters=60, gradTol=1e-5, lineSearchIters=10,
                                        precond="jacobi"),
                           fixed_pins=pins, moving_pins=[], pin_velocity=(0.0, 0.0, 0.0),
                           contact=dict(dHatM=1e-3, kappaJ=50.0, dMinM=1e-4, frictionMu=0.3, frictionEpsM=1e-4,
                                        floorY=floor_y),
                           side=sd, seed=seed))
    return sheets


def with_theta(cfg: dict, theta) -> dict:
    """Copy of a workload with material (C00, C11, G, k_bend) = theta."""
    out = dict(cfg)
    out["material"] = dict(cfg["material"], stretchWarp=float(theta[0]), stretchWeft=float(theta[1]),
                           shear=float(theta[2]), bendWarp=float(theta[3]), bendWeft=float(theta[3]))
    return out


def pins_at(cfg: dict, step: int) -> dict:
    """Pin map before `step` (0-based): fixed pins at their initial position,
    moving pins displaced by velocity * h * (step + 1)."""
    x = cfg["x"]
    pins = {}
    for i in cfg["fixed_pins"]:
        pins[i] = (float(x[i * 3]), float(x[i * 3 + 1]), float(x[i * 3 + 2]))
    t = cfg["h"] * (step + 1)
    vx, vy, vz = cfg["pin_velocity"]
    for i in cfg["moving_pins"]:
        pins[i] = (float(x[i * 3] + vx * t), float(x[i * 3 + 1] + vy * t), float(x[i * 3 + 2] + vz * t))
    return pins


def make_scene(cfg: dict) -> ClothScene:
    """ClothScene for CudaSolver from a workload dict."""
    mesh = preprocess(cfg["pos"], cfg["uv"], cfg["idx"], cfg["density"])
    sc = createScene(mesh, ClothMaterial(**cfg["material"]), cfg["gravity"])
    sc.positions = cfg["x"].copy()
    sc.velocities = cfg["v"].copy()
    sc.pinned = pins_at(cfg, 0)
    c = cfg["contact"]
    if c is not None:
        cs = ContactSystem(ContactParams(c["dHatM"], c["kappaJ"], c["dMinM"], c["frictionMu"], c["frictionEpsM"]),
                           mesh.indices)
        cs.setFloor(c.get("floorY"))
        if c.get("staticPos") is not None:
            cs.setStaticMesh(c["staticPos"], c["staticIdx"])
        sc.contact = cs
    return sc
