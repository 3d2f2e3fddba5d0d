"""Per-CTA element lists of the one-cluster PCG's resident phase A (host logic).

The builder (closim_b200/csrc/cluster_plan.cpp) is compiled for the host with
a checker of its invariants (tests/plancheck): the owned vertex ranges cover
the mesh; every owned vertex's triangle and hinge incidences appear in the
membrane and hinge CSRs' order and point at list slots whose halo-local ids
map back to the right global vertices; every listed element touches an owned
vertex; shared-memory regions are 16-byte aligned; every vertex's dofs are
pushed to the phase-B slot of the warp that owns its Schwarz domain. Meshes: the floor drape's
64 x 64 grid (which must fit in a CTA's shared memory at 16 CTAs), the strip,
an irregular annulus and a UV sphere.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from closim_b200 import configs
from tests.test_gpu_garment import annulus

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "plancheck", "libplancheck.so")
SMEM_LIMIT = 227 * 1024 - 4096  # the kernel's dynamic shared-memory budget per CTA


@pytest.fixture(scope="module")
def lib():
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "plancheck")], check=True)
    L = ctypes.CDLL(LIB)
    L.pc_check.restype = ctypes.c_int
    return L


def check(L, mesh, nrank):
    idx = np.ascontiguousarray(mesh.indices, dtype=np.uint32)
    hin = np.ascontiguousarray(np.asarray(mesh.hinges, dtype=np.int32).reshape(-1))
    n = len(mesh.restPositions) // 3
    info = np.zeros(7, dtype=np.int64)
    rest = np.ascontiguousarray(mesh.restPositions, dtype=np.float32)
    rc = L.pc_check(n, len(idx) // 3, len(hin) // 4, idx.ctypes.data_as(ctypes.c_void_p),
                    hin.ctypes.data_as(ctypes.c_void_p), rest.ctypes.data_as(ctypes.c_void_p), nrank,
                    info.ctypes.data_as(ctypes.c_void_p))
    return rc, info


def scene_mesh(cfg):
    return configs.make_scene(cfg).mesh


def test_plan_invariants_floor_drape(lib):
    rc, info = check(lib, scene_mesh(configs.floor_drape()), 16)
    assert rc == 0, rc
    print(f"64x64 at 16 CTAs: shared memory {info[0]} B (reference mode), {info[1]} B (exact-Newton mode)")
    assert info[1] <= SMEM_LIMIT, info


@pytest.mark.parametrize("nrank", [8, 1])
def test_plan_refused_when_a_warp_would_own_more_than_three_domains(lib, nrank):
    # 513 Schwarz domains need at least 171 warps (3 domains each): 16 per CTA
    rc, _ = check(lib, scene_mesh(configs.floor_drape()), nrank)
    assert rc == 1, rc


def test_plan_invariants_strip_and_sphere(lib):
    for cfg in (configs.strip_pull(), configs.sphere_drape(nx=31, ny=31)):
        rc, _ = check(lib, scene_mesh(cfg), 16)
        assert rc == 0, (cfg["name"], rc)


def test_plan_invariants_irregular_mesh(lib):
    from closim_b200.garment import AssembledGarment
    from closim_b200.solver import preprocess
    pos, uv, idx = annulus()
    mesh = preprocess(pos.astype(np.float32), uv.astype(np.float32), idx.astype(np.uint32), 0.15)
    for nrank in (16, 4, 3):
        rc, _ = check(lib, mesh, nrank)
        assert rc == 0, (nrank, rc)


def test_plan_more_ctas_than_vertices(lib):
    # a 3 x 3 sheet over 16 CTAs: most CTAs own nothing
    cfg = configs.floor_drape(nx=2, ny=2, w=0.1, hgt=0.1, steps=2)
    rc, info = check(lib, scene_mesh(cfg), 16)
    assert rc == 0, rc
