"""Synthetic workloads of the cloth step (seeded), in the reference's y-up frame.

A workload is a plain dict (arrays + parameters) so the same inputs can be fed
to the CUDA solver and to any checker. Config text uses z-up; here config "z"
is the reference's y (vertical), config "z = c" floors are y = c.

  strip_pull   41 x 9 strip, left column pinned, right column pulled +x at 0.1 m/s
  floor_drape  64 x 64 sheet released 0.3 m above a y = 0 floor (barrier + friction)
"""
from __future__ import annotations

import numpy as np

from .solver import (ClothMaterial, ClothScene, ContactParams, ContactSystem, buildGrid, createScene,
                     preprocess)


def _material(**kw):
    m = dict(arealDensityKgM2=0.2, thickness=1.0, stretchWarp=5e3, stretchWeft=5e3, stretchCoupling=0.0,
             shear=1e3, bendWarp=1e-4, bendWeft=1e-4, damping=0.0)
    m.update(kw)
    return m


def strip_pull(seed: int = 1, nx: int = 40, ny: int = 8, w: float = 1.0, hgt: float = 0.2, steps: int = 100):
    """1.0 x 0.2 m strip, 41 x 9 vertices (640 triangles); C00 = C11 = 5e3 N/m,
    G = 1e3, k_bend = 1e-4, 0.2 kg/m^2; h = 0.01 s; Newton tol 1e-6; Jacobi PCG.
    Seeded U(+-1e-4) jitter on the vertical coordinate of the initial state."""
    pos, uv, idx = buildGrid(nx, ny, w, hgt)
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
                precond: str = "schwarz"):
    """0.8 x 0.8 m sheet, 64 x 64 vertices (7938 triangles), 0.3 m above a y = 0
    floor; dHat = 1e-3 m, mu = 0.3; C00 = 5e3, C11 = 3e3, G = 1e3; h = 1/120 s;
    Schwarz-block PCG. Seeded U(+-1e-3) vertical noise."""
    pos, uv, idx = buildGrid(nx, ny, w, hgt)
    pos = pos.copy()
    pos[1::3] = (pos[1::3].astype(np.float64) + 0.3).astype(np.float32)
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
