"""Avatar colliders for the cloth step: rigid collision shapes, their motion,
and the hand-off to the contact system's static mesh.

Mirrors (mohdabraralikhan/closim):
  Transform / MotionProvider / StaticMotionProvider   src/collision/avatar-collider.ts:9-95
  sampleMotion, interpolateTransform                 avatar-collider.ts:97-143
  preprocessCollisionMesh                            avatar-collider.ts:151-187
  toCollisionObject, toCollisionObjectMotion,
  attachCollisionObject, horizontalPlaneHeight        avatar-collider.ts:205-250
  sphere / capsule / box / compound tessellation      avatar-collider.ts:252-354

A collider is a sphere, capsule, box, triangle mesh or compound of these in
local metres, placed by a rigid transform and moved by a motion provider. Its
pose is sampled at a time and tessellated into the f32 positions and u32
triangles the contact system takes as its static mesh; a moving collider is
re-sampled every step and handed to CudaSolver.setStaticPositions (the same
triangles, new positions), which is what the reference does by calling
ContactSystem.setStaticMesh with each new pose. The tessellations keep the
reference's vertex and triangle order, so the static meshes are the same.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

Vec3 = Tuple[float, float, float]
Quat = Tuple[float, float, float, float]  # x, y, z, w


@dataclass(frozen=True)
class Transform:
    translation: Vec3 = (0.0, 0.0, 0.0)
    rotation: Quat = (0.0, 0.0, 0.0, 1.0)


IDENTITY_TRANSFORM = Transform()


def _finite(v, name):
    if not isinstance(v, (int, float)) or isinstance(v, bool) or not math.isfinite(v):
        raise ValueError(f"{name} must be finite")
    return float(v)


def _positive(v, name):
    v = _finite(v, name)
    if not v > 0:
        raise ValueError(f"{name} must be positive")
    return v


def _nonnegative(v, name):
    v = _finite(v, name)
    if v < 0:
        raise ValueError(f"{name} must be nonnegative")
    return v


def _resolution(v, name, lo, hi):
    if not isinstance(v, int) or isinstance(v, bool) or v < lo or v > hi:
        raise ValueError(f"{name} must be an integer in [{lo}, {hi}]")
    return v


def _check_transform(t: Transform) -> None:
    if len(t.translation) != 3 or len(t.rotation) != 4:
        raise ValueError("invalid rigid transform dimensions")
    for i, v in enumerate(t.translation):
        _finite(v, f"translation[{i}]")
    for i, v in enumerate(t.rotation):
        _finite(v, f"rotation[{i}]")
    if not math.hypot(*t.rotation) > 1e-12:
        raise ValueError("rotation quaternion must be nonzero")


def _unit(q) -> Tuple[float, float, float, float]:
    n = math.hypot(*q)
    if not (n > 1e-12) or not math.isfinite(n):
        raise ValueError("rotation quaternion must be finite and nonzero")
    return (q[0] / n, q[1] / n, q[2] / n, q[3] / n)


def _canonical(q):
    """Unit quaternion with its first clearly nonzero component positive (a
    representative of q and -q)."""
    u = _unit(q)
    for c in u:
        if abs(c) <= 1e-15:
            continue
        return tuple(-x for x in u) if c < 0 else u
    return u


def _rotate(q, p) -> Tuple[float, float, float]:
    """p rotated by the unit quaternion q: p + w t + (q.xyz x t), t = 2 q.xyz x p."""
    x, y, z, w = q
    tx = 2 * (y * p[2] - z * p[1])
    ty = 2 * (z * p[0] - x * p[2])
    tz = 2 * (x * p[1] - y * p[0])
    return (p[0] + w * tx + y * tz - z * ty, p[1] + w * ty + z * tx - x * tz, p[2] + w * tz + x * ty - y * tx)


def _compose(a: Transform, b: Transform) -> Transform:
    """a after b: rotations multiplied (Hamilton product a.q b.q), b's
    translation rotated into a's frame."""
    qa, qb = _unit(a.rotation), _unit(b.rotation)
    p = _rotate(qa, b.translation)
    ax, ay, az, aw = qa
    bx, by, bz, bw = qb
    return Transform(
        (a.translation[0] + p[0], a.translation[1] + p[1], a.translation[2] + p[2]),
        (aw * bx + ax * bw + ay * bz - az * by,
         aw * by - ax * bz + ay * bw + az * bx,
         aw * bz + ax * by - ay * bx + az * bw,
         aw * bw - ax * bx - ay * by - az * bz))


class MotionProvider:
    """The body's rigid world transform as a function of time (seconds)."""

    def sample(self, timeSeconds: float) -> Transform:  # pragma: no cover - interface
        raise NotImplementedError


class StaticMotionProvider(MotionProvider):
    def __init__(self, transform: Transform = IDENTITY_TRANSFORM):
        _check_transform(transform)
        self._t = transform

    def sample(self, timeSeconds: float) -> Transform:
        _finite(timeSeconds, "timeSeconds")
        return self._t


class LinearMotion(MotionProvider):
    """Interpolation between two poses over [t0, t1] (held outside it):
    translation lerp, rotation slerp (interpolateTransform)."""

    def __init__(self, start: Transform, end: Transform, t0: float, t1: float):
        _check_transform(start)
        _check_transform(end)
        if not t1 > t0:
            raise ValueError("motion interval must satisfy t1 > t0")
        self.start, self.end, self.t0, self.t1 = start, end, float(t0), float(t1)

    def sample(self, timeSeconds: float) -> Transform:
        a = min(1.0, max(0.0, (_finite(timeSeconds, "timeSeconds") - self.t0) / (self.t1 - self.t0)))
        return interpolateTransform(self.start, self.end, a)


@dataclass(frozen=True)
class MotionInterval:
    t0: float
    t1: float
    start: Transform
    end: Transform


def sampleMotion(provider: MotionProvider, t0: float, t1: float) -> MotionInterval:
    _finite(t0, "t0")
    _finite(t1, "t1")
    if t1 < t0:
        raise ValueError("motion interval must satisfy t1 >= t0")
    a, b = provider.sample(t0), provider.sample(t1)
    _check_transform(a)
    _check_transform(b)
    return MotionInterval(float(t0), float(t1), a, b)


def interpolateTransform(a: Transform, b: Transform, alpha: float) -> Transform:
    """Translation lerp plus shortest-arc slerp of the rotation (a normalized
    lerp when the two rotations are within about 1.8 degrees)."""
    _check_transform(a)
    _check_transform(b)
    alpha = _finite(alpha, "alpha")
    if alpha < 0 or alpha > 1:
        raise ValueError("interpolation alpha must be in [0, 1]")
    qa, qb = _canonical(a.rotation), list(_canonical(b.rotation))
    dot = sum(qa[k] * qb[k] for k in range(4))
    if dot < 0:
        qb = [-c for c in qb]
        dot = -dot
    dot = max(-1.0, min(1.0, dot))
    if dot > 0.9995:
        q = [qa[k] + alpha * (qb[k] - qa[k]) for k in range(4)]
    else:
        th = math.acos(dot)
        s = math.sin(th)
        wa, wb = math.sin((1 - alpha) * th) / s, math.sin(alpha * th) / s
        q = [qa[k] * wa + qb[k] * wb for k in range(4)]
    t = tuple(a.translation[k] + alpha * (b.translation[k] - a.translation[k]) for k in range(3))
    return Transform(t, _unit(q))


# ---- geometry ------------------------------------------------------------------------


@dataclass
class TriangleMeshGeometry:
    positions: Sequence[float]
    indices: Sequence[int]
    triangleBodyParts: Optional[List[str]] = None
    kind: str = "triangle-mesh"


@dataclass
class SphereGeometry:
    radiusM: float
    segments: int = 12
    rings: int = 6
    kind: str = "sphere"


@dataclass
class CapsuleGeometry:
    radiusM: float
    cylinderLengthM: float
    segments: int = 12
    hemisphereRings: int = 3
    kind: str = "capsule"


@dataclass
class BoxGeometry:
    halfExtentsM: Vec3
    kind: str = "box"


@dataclass
class CompoundChild:
    geometry: object
    transform: Optional[Transform] = None
    bodyPart: Optional[str] = None


@dataclass
class CompoundGeometry:
    children: List[CompoundChild] = field(default_factory=list)
    kind: str = "compound"


@dataclass
class AvatarCollider:
    id: str
    bodyPart: str
    geometry: object
    thicknessM: float
    transform: Optional[Transform] = None
    motion: Optional[MotionProvider] = None


@dataclass
class CollisionObject:
    positions: np.ndarray          # f32 [3 ns]
    indices: np.ndarray            # u32 [3 ms]
    thicknessM: float
    triangleBodyParts: List[str]


@dataclass
class CollisionObjectMotion:
    interval: MotionInterval
    start: CollisionObject
    end: CollisionObject


def _check_geometry(g) -> None:
    if g.kind == "triangle-mesh":
        npos, nidx = len(g.positions), len(g.indices)
        if npos < 9 or npos % 3 or nidx < 3 or nidx % 3:
            raise ValueError("triangle mesh requires xyz vertices and triangle indices")
        for i, v in enumerate(g.positions):
            _finite(float(v), f"positions[{i}]")
        for v in g.indices:
            if int(v) != v or v < 0 or v >= npos // 3:
                raise ValueError(f"invalid triangle index {v}")
        if g.triangleBodyParts is not None and len(g.triangleBodyParts) != nidx // 3:
            raise ValueError("triangleBodyParts length mismatch")
    elif g.kind == "sphere":
        _positive(g.radiusM, "sphere radiusM")
        _resolution(g.segments, "sphere segments", 6, 64)
        _resolution(g.rings, "sphere rings", 3, 32)
    elif g.kind == "capsule":
        _positive(g.radiusM, "capsule radiusM")
        _nonnegative(g.cylinderLengthM, "capsule cylinderLengthM")
        _resolution(g.segments, "capsule segments", 6, 64)
        _resolution(g.hemisphereRings, "capsule hemisphereRings", 2, 16)
    elif g.kind == "box":
        for i, v in enumerate(g.halfExtentsM):
            _positive(v, f"box halfExtentsM[{i}]")
    elif g.kind == "compound":
        if not g.children:
            raise ValueError("compound collider must contain children")
        for c in g.children:
            if c.transform is not None:
                _check_transform(c.transform)
            _check_geometry(c.geometry)
    else:
        raise ValueError(f"unknown collider geometry {g.kind!r}")


def _uv_sphere(g: SphereGeometry) -> TriangleMeshGeometry:
    """Top pole, rings - 1 rings of `segments` vertices, bottom pole; a fan at
    each pole and two triangles per quad between rings."""
    r = g.radiusM
    seg, rings = g.segments, g.rings
    pos = [0.0, r, 0.0]
    for j in range(1, rings):
        th = math.pi * j / rings
        for i in range(seg):
            ph = 2 * math.pi * i / seg
            pos += [r * math.sin(th) * math.cos(ph), r * math.cos(th), r * math.sin(th) * math.sin(ph)]
    bottom = len(pos) // 3
    pos += [0.0, -r, 0.0]
    idx = []
    for i in range(seg):
        nxt = (i + 1) % seg
        idx += [0, 1 + i, 1 + nxt]
        for ring in range(rings - 2):
            a, b = 1 + ring * seg + i, 1 + ring * seg + nxt
            idx += [a, a + seg, b, b, a + seg, b + seg]
        last = 1 + (rings - 2) * seg
        idx += [last + i, bottom, last + nxt]
    return TriangleMeshGeometry(pos, idx)


def _capsule(g: CapsuleGeometry) -> TriangleMeshGeometry:
    """Rings of `segments` vertices from the top pole region down: the upper
    hemisphere (hemisphereRings + 1 rings), then the lower one; quads between
    consecutive rings."""
    r, seg, hemi = g.radiusM, g.segments, g.hemisphereRings
    half = 0.5 * g.cylinderLengthM
    ys = [half + r * math.cos((math.pi / 2) * j / hemi) for j in range(hemi + 1)]
    ys += [-half - r * math.sin((math.pi / 2) * j / hemi) for j in range(1, hemi + 1)]
    pos = []
    for y in ys:
        cap = half if y > half else -half if y < -half else y
        rad = math.sqrt(max(0.0, r * r - (y - cap) ** 2))
        for i in range(seg):
            ph = 2 * math.pi * i / seg
            pos += [rad * math.cos(ph), y, rad * math.sin(ph)]
    idx = []
    for ring in range(len(ys) - 1):
        for i in range(seg):
            nxt = (i + 1) % seg
            a, b = ring * seg + i, ring * seg + nxt
            idx += [a, b, a + seg, b, b + seg, a + seg]
    return TriangleMeshGeometry(pos, idx)


# corner order and faces of the unit box (two triangles per face, outward)
_BOX_CORNERS = [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)]
_BOX_TRIS = [0, 2, 1, 0, 3, 2, 4, 5, 6, 4, 6, 7, 0, 1, 5, 0, 5, 4, 1, 2, 6, 1, 6, 5, 2, 3, 7, 2, 7, 6, 3, 0, 4, 3, 4, 7]


def _box(g: BoxGeometry) -> TriangleMeshGeometry:
    hx, hy, hz = (float(v) for v in g.halfExtentsM)
    pos = [c for sx, sy, sz in _BOX_CORNERS for c in (sx * hx, sy * hy, sz * hz)]
    return TriangleMeshGeometry(pos, list(_BOX_TRIS))


def _transformed(mesh: TriangleMeshGeometry, t: Transform) -> TriangleMeshGeometry:
    _check_transform(t)
    q = _unit(t.rotation)
    p = np.asarray(mesh.positions, np.float64).reshape(-1, 3)
    out = np.empty_like(p)
    for i, v in enumerate(p):
        r = _rotate(q, v)
        out[i] = (r[0] + t.translation[0], r[1] + t.translation[1], r[2] + t.translation[2])
    return TriangleMeshGeometry(out.ravel().tolist(), list(mesh.indices), mesh.triangleBodyParts)


def _mesh_of(g, bodyPart: str) -> TriangleMeshGeometry:
    if g.kind == "triangle-mesh":
        return g
    if g.kind == "sphere":
        return _uv_sphere(g)
    if g.kind == "capsule":
        return _capsule(g)
    if g.kind == "box":
        return _box(g)
    pos, idx, labels = [], [], []
    for c in g.children:
        part = c.bodyPart or bodyPart
        m = _transformed(_mesh_of(c.geometry, part), c.transform or IDENTITY_TRANSFORM)
        off = len(pos) // 3
        pos += list(m.positions)
        idx += [int(i) + off for i in m.indices]
        labels += list(m.triangleBodyParts) if m.triangleBodyParts else [part] * (len(m.indices) // 3)
    if not idx:
        raise ValueError("compound collider must contain geometry")
    return TriangleMeshGeometry(pos, idx, labels)


def preprocessCollisionMesh(mesh: TriangleMeshGeometry, defaultBodyPart: str):
    """Validates the mesh, welds vertices with identical coordinates (-0 taken
    as 0, first occurrence kept) and drops degenerate or repeated triangles
    (the same vertex set in any order). Returns (f32 positions, u32 indices,
    per-triangle body parts)."""
    _check_geometry(mesh)
    p = np.asarray(mesh.positions, np.float64).reshape(-1, 3) + 0.0  # -0 -> 0
    if not np.all(np.isfinite(p.astype(np.float32))):
        raise ValueError("a vertex cannot be represented in the f32 collision buffers")
    ids = {}
    weld = np.empty(len(p), np.int64)
    kept = []
    for i, v in enumerate(p):
        k = (float(v[0]), float(v[1]), float(v[2]))
        j = ids.get(k)
        if j is None:
            j = len(kept)
            ids[k] = j
            kept.append(v)
        weld[i] = j
    kept = np.asarray(kept)
    idx, labels, seen = [], [], set()
    tris = np.asarray(mesh.indices, np.int64).reshape(-1, 3)
    for t, (a0, b0, c0) in enumerate(tris):
        a, b, c = int(weld[a0]), int(weld[b0]), int(weld[c0])
        if a == b or b == c or c == a:
            continue
        u, w = kept[b] - kept[a], kept[c] - kept[a]
        cr = np.cross(u, w)
        if float(cr @ cr) <= 1e-24:
            continue
        key = tuple(sorted((a, b, c)))
        if key in seen:
            continue
        seen.add(key)
        idx += [a, b, c]
        labels.append(mesh.triangleBodyParts[t] if mesh.triangleBodyParts else defaultBodyPart)
    if not idx:
        raise ValueError("collision mesh has no nondegenerate triangles")
    return kept.astype(np.float32).ravel(), np.asarray(idx, np.uint32), labels


def _check_collider(c: AvatarCollider) -> None:
    if not c.id or not c.bodyPart:
        raise ValueError("collider id and bodyPart are required")
    _nonnegative(c.thicknessM, "thicknessM")
    if c.transform is not None:
        _check_transform(c.transform)
    _check_geometry(c.geometry)


def toCollisionObject(collider: AvatarCollider, timeSeconds: float) -> CollisionObject:
    """The collider's mesh at time t: motion pose composed with the collider's
    own transform, tessellated, welded, in f32."""
    _check_collider(collider)
    _finite(timeSeconds, "timeSeconds")
    world = collider.motion.sample(timeSeconds) if collider.motion else IDENTITY_TRANSFORM
    _check_transform(world)
    root = _compose(world, collider.transform or IDENTITY_TRANSFORM)
    mesh = _transformed(_mesh_of(collider.geometry, collider.bodyPart), root)
    pos, idx, labels = preprocessCollisionMesh(mesh, collider.bodyPart)
    return CollisionObject(pos, idx, collider.thicknessM, labels)


def toCollisionObjectMotion(collider: AvatarCollider, t0: float, t1: float) -> CollisionObjectMotion:
    interval = sampleMotion(collider.motion or StaticMotionProvider(), t0, t1)
    a = AvatarCollider(collider.id, collider.bodyPart, collider.geometry, collider.thicknessM, collider.transform,
                       StaticMotionProvider(interval.start))
    b = AvatarCollider(collider.id, collider.bodyPart, collider.geometry, collider.thicknessM, collider.transform,
                       StaticMotionProvider(interval.end))
    return CollisionObjectMotion(interval, toCollisionObject(a, t0), toCollisionObject(b, t1))


def attachCollisionObject(target, obj: CollisionObject) -> None:
    """Hands the sampled mesh to anything with setStaticMesh(positions, indices)
    (a ContactSystem)."""
    target.setStaticMesh(obj.positions, obj.indices)


def horizontalPlaneHeight(obj: CollisionObject, toleranceM: float = 1e-6) -> float:
    """The y of a collider whose vertices all lie on one horizontal plane
    (then the floor representation can stand in for it)."""
    p = np.asarray(obj.positions)
    if p.size < 9 or p.size % 3:
        raise ValueError("invalid collision positions")
    _nonnegative(toleranceM, "toleranceM")
    y = float(p[1])
    if np.any(np.abs(p[1::3].astype(np.float64) - y) > toleranceM):
        raise ValueError("collider is not a horizontal plane")
    return y
