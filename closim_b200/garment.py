"""Garment fitting scenes: a garment mesh draped on avatar colliders.

Mirrors (mohdabraralikhan/closim):
  createFittingScene     src/garment/assembly.ts:469-505
  FittingScene           the {scene, mesh, contact} it returns

createFittingScene builds the simulation scene of an assembled garment (any
triangle mesh, not only grids): the preprocessed mesh, the material, gravity,
a ContactSystem with the avatar's collision meshes merged into one static
mesh, and an optional floor. AvatarDriver then moves those colliders between
steps: it re-samples every collider's pose at the step's end time and hands
the merged positions to CudaSolver.setStaticPositions, which is what the
reference's session does with ContactSystem.setStaticMesh and
toCollisionObject (src/collision/avatar-collider.ts:205-237).
"""
from __future__ import annotations

from dataclasses import dataclass, replace
from typing import List, Optional, Sequence

import numpy as np

from .avatar import AvatarCollider, CollisionObject, toCollisionObject
from .solver import (DEFAULT_CONTACT_PARAMS, DEFAULT_MATERIAL, ClothMaterial, ClothMeshData, ClothScene,
                     ContactParams, ContactSystem, createScene, preprocess)


@dataclass
class AssembledGarment:
    """The garment's welded mesh (assembly.ts's AssembledGarment): positions
    3n, uv 2n, triangle indices 3m."""
    positions: np.ndarray
    uv: np.ndarray
    indices: np.ndarray


@dataclass
class FittingScene:
    scene: ClothScene
    mesh: ClothMeshData
    contact: ContactSystem


def merge_collision_objects(objs: Sequence[CollisionObject]):
    """One static mesh from several collision objects: positions concatenated,
    each object's indices offset by the vertices before it."""
    if not objs:
        raise ValueError("no collision objects")
    pos = np.concatenate([np.asarray(o.positions, np.float32) for o in objs])
    idx, base = [], 0
    for o in objs:
        idx.append(np.asarray(o.indices, np.int64) + base)
        base += len(o.positions) // 3
    return pos, np.concatenate(idx).astype(np.uint32)


def createFittingScene(garment: AssembledGarment, avatar=None, floorY: Optional[float] = None,
                       material: Optional[ClothMaterial] = None, contact: Optional[ContactParams] = None,
                       gravity=(0.0, -9.81, 0.0), arealDensityKgM2: float = 0.15) -> FittingScene:
    """createFittingScene (assembly.ts:469-505). `avatar`: a CollisionObject or
    a list of them (merged into one static mesh)."""
    idx = np.asarray(garment.indices, np.uint32)
    if idx.size == 0:
        raise ValueError("assembly: cannot create a scene from an empty garment")
    pos = np.asarray(garment.positions, np.float64)
    if not np.all(np.isfinite(pos)):
        raise ValueError("assembly: garment state contains NaN/Inf")
    mesh = preprocess(pos.astype(np.float32), np.asarray(garment.uv, np.float32), idx, arealDensityKgM2)
    scene = createScene(mesh, replace(material) if material else replace(DEFAULT_MATERIAL), gravity)
    cs = ContactSystem(replace(contact) if contact else replace(DEFAULT_CONTACT_PARAMS), mesh.indices)
    if avatar is not None:
        objs = list(avatar) if isinstance(avatar, (list, tuple)) else [avatar]
        sp, si = merge_collision_objects(objs)
        cs.setStaticMesh(sp, si)
    if floorY is not None:
        cs.setFloor(floorY)
    scene.contact = cs
    return FittingScene(scene, mesh, cs)


class AvatarDriver:
    """Moves a fitting scene's avatar colliders with their motion providers:
    before the step that ends at time t, `advance_to(t)` samples every
    collider at t and moves the solver's static mesh there."""

    def __init__(self, colliders: List[AvatarCollider], solver, t0: float = 0.0):
        self.colliders = list(colliders)
        self.solver = solver
        self.t = float(t0)
        self._tris = merge_collision_objects([toCollisionObject(c, t0) for c in self.colliders])[1]

    def objects_at(self, t: float) -> List[CollisionObject]:
        return [toCollisionObject(c, t) for c in self.colliders]

    def positions_at(self, t: float) -> np.ndarray:
        pos, tris = merge_collision_objects(self.objects_at(t))
        if not np.array_equal(tris, self._tris):
            raise ValueError("a collider's tessellation changed with its pose (welded vertices differ)")
        return pos

    def advance_to(self, t: float) -> np.ndarray:
        pos = self.positions_at(t)
        self.solver.setStaticPositions(pos)
        self.t = float(t)
        return pos
