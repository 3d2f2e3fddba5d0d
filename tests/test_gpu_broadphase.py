"""Device LBVH broadphase against the oracle's FP32 mirror of GpuBroadPhase
(src/backend/webgpu/gpu-broadphase.ts) and the CPU TriBvh pair set
(src/collision/bvh.ts), through the C ABI in include/closim_broadphase.h.

Bit-exact: swept boxes, centroids, sorted Morton keys and payload, node boxes,
node topology, root, depth and the pair set (the reference's
tests/webgpu/broadphase-parity.test.ts compares the mirror with the CPU set;
here the device build is compared with both).
"""
import numpy as np
import pytest

from closim_b200.broadphase import GpuBroadPhase
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def grid_scene(nx, ny, w, h, seed, jitter, fold=0.0, drop=0.0):
    """buildGrid sheet lifted into 3D (y-up), seeded in-plane jitter; x1 folds the
    sheet about its middle row by `fold` (rad) and drops it by `drop` (m)."""
    pos, _, idx = O.build_grid(nx, ny, w, h)
    x0 = pos.astype(np.float64).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    x0[:, 0] += rng.uniform(-jitter, jitter, len(x0))
    x0[:, 2] += rng.uniform(-jitter, jitter, len(x0))
    x1 = x0.copy()
    if fold:
        zc = 0.5 * (x0[:, 2].min() + x0[:, 2].max())
        far = x0[:, 2] > zc
        r = x0[far, 2] - zc
        x1[far, 2] = zc + r * np.cos(np.pi - fold)
        x1[far, 1] = x0[far, 1] + r * np.sin(np.pi - fold) + 0.004
    x1[:, 1] -= drop
    return x0.ravel(), x1.ravel(), idx


def device(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


def mirror_equal(dev, ref):
    m = len(ref["morton"])
    assert np.array_equal(dev["aabb"].view(np.uint32), ref["aabb"].view(np.uint32))
    assert np.array_equal(dev["centroid"].view(np.uint32), ref["centroid"].view(np.uint32))
    assert np.array_equal(dev["morton"], ref["morton"])
    assert np.array_equal(dev["payload"], ref["payload"])
    assert np.array_equal(dev["nodeLeft"], ref["left"])
    assert np.array_equal(dev["nodeRight"], ref["right"])
    assert np.array_equal(dev["nodeLeafTri"], ref["leafTri"])
    assert np.array_equal(dev["nodeMin"].view(np.uint32), ref["nodeMin"].view(np.uint32))
    assert np.array_equal(dev["nodeMax"].view(np.uint32), ref["nodeMax"].view(np.uint32))
    assert dev["root"] == ref["root"]
    assert dev["depth"] == ref["depth"]
    assert m == len(dev["payload"])


@pytest.mark.parametrize("fold,drop", [(0.0, 0.0), (0.0, 0.003), (2.8, 0.0)])
def test_mirror_bit_exact_small(fold, drop):
    x0, x1, idx = grid_scene(12, 9, 0.3, 0.22, seed=5, jitter=2e-3, fold=fold, drop=drop)
    m = len(idx) // 3
    ref = O.lbvh_mirror(x0, x1, idx, 0.002)
    bp = GpuBroadPhase(idx, m, 0.002, pairCapacity=1 << 22, n=len(x0) // 3)
    res = bp.build(device(x0), device(x1))
    mirror_equal(bp.lastMirror, ref)
    assert np.array_equal(res["pairs"], ref["pairs"])
    assert res["diagnostics"]["scannedCount"] == ref["scanned"]
    assert res["diagnostics"]["candidateOverflow"] == 0
    # The mirror set equals the CPU BVH set (broadphase-parity.test.ts).
    ex = GpuBroadPhase(idx, m, 0.002, pairCapacity=1 << 22, mode="exact", n=len(x0) // 3)
    assert np.array_equal(ex.build(device(x0), device(x1))["pairs"], O.tri_pairs(x0, x1, idx, 0.002))


def test_overflow_keeps_reference_prefix():
    """A capacity below the scanned count keeps the first pairs in traversal
    order, then sorts them (gpu-broadphase.ts:355-372)."""
    x0, x1, idx = grid_scene(10, 10, 0.2, 0.2, seed=7, jitter=1e-3, fold=2.9)
    m = len(idx) // 3
    cap = 97
    ref = O.lbvh_mirror(x0, x1, idx, 0.002, capacity=cap)
    assert ref["overflow"] == 1
    bp = GpuBroadPhase(idx, m, 0.002, pairCapacity=cap, n=len(x0) // 3)
    res = bp.build(device(x0), device(x1))
    d = res["diagnostics"]
    assert d["candidateOverflow"] == 1 and d["scannedCount"] == ref["scanned"] and d["writtenCount"] == cap
    assert np.array_equal(res["pairs"], ref["pairs"])


def test_equal_centroids_tiebreak():
    """Two coincident layers: every Morton key appears twice, so the hierarchy
    rests on the sorted-position tiebreak (gpu-broadphase.ts:140-145)."""
    pos, _, idx = O.build_grid(6, 5, 0.1, 0.1)
    n = len(pos) // 3
    x0 = np.concatenate([pos, pos]).astype(np.float64)
    idx2 = np.concatenate([idx, idx + n]).astype(np.uint32)
    x1 = x0.copy()
    m = len(idx2) // 3
    ref = O.lbvh_mirror(x0, x1, idx2, 1e-3)
    bp = GpuBroadPhase(idx2, m, 1e-3, pairCapacity=1 << 20, n=2 * n)
    res = bp.build(device(x0), device(x1))
    mirror_equal(bp.lastMirror, ref)
    assert np.array_equal(res["pairs"], ref["pairs"])


@pytest.mark.parametrize("nx", [1, 2])
def test_tiny_meshes(nx):
    """One triangle pair (m = 2) and a single-triangle mesh (m = 1)."""
    pos, _, idx = O.build_grid(nx, 1, 0.1, 0.1)
    if nx == 1:
        idx = idx[:3]
    x0 = pos.astype(np.float64)
    x1 = x0 + 0.001
    m = len(idx) // 3
    ref = O.lbvh_mirror(x0, x1, idx, 1e-3)
    bp = GpuBroadPhase(idx, m, 1e-3, n=len(x0) // 3)
    res = bp.build(device(x0), device(x1))
    mirror_equal(bp.lastMirror, ref)
    assert np.array_equal(res["pairs"], ref["pairs"])


def test_self_contact_sheet_256():
    """Self-contact-heavy sheet: 256 x 256 vertices (130,050 triangles), in-plane
    jitter U(+-5e-4), pad 5e-4, swept from flat to folded over a 0.4 m drop:
    Morton keys, sorted payload, topology and pair set bit-exact."""
    x0, x1, idx = grid_scene(255, 255, 1.0, 1.0, seed=3, jitter=5e-4, fold=2.6, drop=0.004)
    m = len(idx) // 3
    assert m == 130050
    ref = O.lbvh_mirror(x0, x1, idx, 5e-4)
    bp = GpuBroadPhase(idx, m, 5e-4, pairCapacity=1 << 26, n=len(x0) // 3)
    res = bp.build(device(x0), device(x1))
    mirror_equal(bp.lastMirror, ref)
    assert res["diagnostics"]["scannedCount"] == ref["scanned"]
    assert np.array_equal(res["pairs"], ref["pairs"])
    ex = GpuBroadPhase(idx, m, 5e-4, pairCapacity=1 << 26, mode="exact", n=len(x0) // 3)
    assert np.array_equal(ex.build(device(x0), device(x1))["pairs"], O.tri_pairs(x0, x1, idx, 5e-4))
