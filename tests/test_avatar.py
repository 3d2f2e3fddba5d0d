"""Avatar colliders (closim_b200.avatar) and fitting scenes (closim_b200.garment)
on the CPU, after the reference's tests/avatar-collider.test.ts: static and
moving poses, rigid rotation, compound primitives with body-part labels,
thickness metadata and the setStaticMesh hand-off, deterministic shortest-arc
interpolation, input rejection, and a horizontal collider plane against the
floor representation (through the oracle's ContactSystem)."""
import math

import numpy as np
import pytest

from closim_b200.avatar import (AvatarCollider, BoxGeometry, CapsuleGeometry, CompoundChild, CompoundGeometry,
                                LinearMotion, SphereGeometry, Transform, TriangleMeshGeometry, attachCollisionObject,
                                horizontalPlaneHeight, interpolateTransform, preprocessCollisionMesh, sampleMotion,
                                toCollisionObject, toCollisionObjectMotion)
from closim_b200.garment import AssembledGarment, createFittingScene, merge_collision_objects
from oracle import oracle as O

TRI = TriangleMeshGeometry([0, 0, 0, 1, 0, 0, 0, 1, 0], [0, 1, 2])


def collider(**kw):
    base = dict(id="body-collider", bodyPart="torso", geometry=TRI, thicknessM=0.004)
    base.update(kw)
    return AvatarCollider(**base)


def test_static_triangle_mesh_adapts_to_static_buffers():
    m = toCollisionObject(collider(), 0)
    assert np.array_equal(m.positions, np.asarray(TRI.positions, np.float32))
    assert np.array_equal(m.indices, np.asarray(TRI.indices, np.uint32))
    assert m.triangleBodyParts == ["torso"]


def test_motion_sampled_at_both_ends():
    motion = LinearMotion(Transform((0, 0, 0)), Transform((2, -1, 3)), 0, 2)
    s = sampleMotion(motion, 0, 2)
    assert s.start.translation == (0, 0, 0) and s.end.translation == (2, -1, 3)
    objs = toCollisionObjectMotion(collider(motion=motion), 0, 2)
    assert objs.start.positions[0] == 0 and objs.end.positions[0] == 2 and objs.end.positions[1] == -1


def test_rigid_rotation():
    quarter = Transform((0, 0, 0), (0, 0, math.sqrt(0.5), math.sqrt(0.5)))
    m = toCollisionObject(collider(transform=quarter), 0)
    assert m.positions[0] == pytest.approx(0, abs=1e-6) and m.positions[1] == pytest.approx(0, abs=1e-6)
    assert m.positions[3] == pytest.approx(0, abs=1e-6) and m.positions[4] == pytest.approx(1)


def test_compound_primitives_with_labels():
    comp = collider(geometry=CompoundGeometry([
        CompoundChild(SphereGeometry(0.1, 8, 4), bodyPart="head"),
        CompoundChild(BoxGeometry((0.2, 0.1, 0.1)), Transform((0, -0.3, 0)), "chest"),
        CompoundChild(CapsuleGeometry(0.05, 0.3, 8, 2), bodyPart="arm")]))
    m = toCollisionObject(comp, 0)
    assert len(m.indices) > 0 and set(m.triangleBodyParts) == {"head", "chest", "arm"}
    assert len(m.positions) // 3 > 8
    # the sphere's tessellation is the static sphere of the sphere-drape workload
    from closim_b200.configs import sphere_mesh
    sp, si = sphere_mesh(0.1, 8, 4)
    sph = toCollisionObject(collider(geometry=SphereGeometry(0.1, 8, 4)), 0)
    assert np.array_equal(sph.positions, sp) and np.array_equal(sph.indices, si)


def test_thickness_metadata_and_attach():
    m = toCollisionObject(collider(thicknessM=0.0125), 0)
    assert m.thicknessM == 0.0125
    got = []

    class Target:
        def setStaticMesh(self, p, i):
            got.append((p, i))
    attachCollisionObject(Target(), m)
    assert got[0][0] is m.positions and got[0][1] is m.indices


def test_shortest_arc_interpolation_is_deterministic():
    a = Transform((0, 2, 0), (0, 0, 0, 1))
    b = Transform((4, 0, 2), (0, 0, 1, 0))
    first, second = interpolateTransform(a, b, 0.25), interpolateTransform(a, b, 0.25)
    assert first == second and first.translation == (1, 1.5, 0.5)
    assert math.hypot(*first.rotation) == pytest.approx(1)
    assert interpolateTransform(a, Transform(b.translation, (0, 0, -1, 0)), 0.25) == first


def test_rejects_invalid_inputs():
    with pytest.raises(ValueError, match="positive"):
        toCollisionObject(collider(geometry=SphereGeometry(-1)), 0)
    with pytest.raises(ValueError, match="index"):
        toCollisionObject(collider(geometry=TriangleMeshGeometry(TRI.positions, [0, 1, 7])), 0)
    with pytest.raises(ValueError, match="nonzero"):
        toCollisionObject(collider(transform=Transform((0, 0, 0), (0, 0, 0, 0))), 0)
    with pytest.raises(ValueError, match="nonnegative"):
        toCollisionObject(collider(thicknessM=-0.1), 0)
    with pytest.raises(ValueError, match="children"):
        toCollisionObject(collider(geometry=CompoundGeometry([])), 0)
    with pytest.raises(ValueError, match="index"):
        preprocessCollisionMesh(TriangleMeshGeometry(TRI.positions, [0, 1, 8]), "part")


def test_horizontal_plane_matches_floor_distance():
    plane = toCollisionObject(collider(geometry=TriangleMeshGeometry(
        [-1, 0.25, -1, 1, 0.25, -1, 1, 0.25, 1, -1, 0.25, 1], [0, 1, 2, 0, 2, 3])), 0)
    y = horizontalPlaneHeight(plane)
    cloth = np.array([0, 0.251, 0, 0.1, 0.251, 0, 0, 0.251, 0.1])
    params = dict(dHat=0.002, kappa=50.0, dMin=1e-4, mu=0.3, eps=1e-4)
    floor = O.ContactSystem(params, np.array([0, 1, 2], np.uint32))
    floor.set_floor(y)
    floor.begin_step(cloth)
    floor.update_active_set(cloth)
    mesh = O.ContactSystem(params, np.array([0, 1, 2], np.uint32))
    mesh.set_static_mesh(plane.positions, plane.indices)
    mesh.begin_step(cloth)
    mesh.update_active_set(cloth)
    assert floor.diag()["minDistance"] == pytest.approx(0.001, abs=1e-6)
    assert mesh.diag()["minDistance"] == pytest.approx(floor.diag()["minDistance"], abs=1e-6)
    with pytest.raises(ValueError, match="horizontal plane"):
        horizontalPlaneHeight(toCollisionObject(collider(), 0))


def test_fitting_scene_merges_avatar_meshes():
    a = toCollisionObject(collider(geometry=SphereGeometry(0.1)), 0)
    b = toCollisionObject(collider(geometry=BoxGeometry((0.1, 0.1, 0.1)), transform=Transform((0, -0.5, 0))), 0)
    pos, uv, idx = O.build_grid(4, 4, 0.2, 0.2)
    fs = createFittingScene(AssembledGarment(pos, uv, idx), avatar=[a, b], floorY=-1.0)
    sp, si = merge_collision_objects([a, b])
    assert np.array_equal(fs.contact.staticPos, sp) and np.array_equal(fs.contact.staticIdx, si)
    assert si.max() == len(sp) // 3 - 1 and fs.contact.floorY == -1.0 and fs.scene.contact is fs.contact
    with pytest.raises(ValueError, match="empty garment"):
        createFittingScene(AssembledGarment(pos, uv, np.zeros(0, np.uint32)))
