"""Oracle binding (test infrastructure only).

ctypes wrapper over oracle/build/liborc.so, the CPU FP64 restatement of the
reference CpuSolver hot path. Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg may import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liborc.so")
_lib = None

F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
U32P = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
VP = C.c_void_p


def build() -> str:
    """Compile the oracle library (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    sig = {
        "orc_build_grid": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, F32P, F32P, U32P]),
        "orc_mesh_create": (VP, [C.c_int, C.c_int, F32P, F32P, U32P, C.c_double]),
        "orc_mesh_destroy": (None, [VP]),
        "orc_mesh_counts": (None, [VP, I32P]),
        "orc_mesh_arrays": (None, [VP, F32P, F32P, F32P, I32P, F64P]),
        "orc_hinge_energy": (C.c_double, [F64P, I32P, F64P, C.c_double]),
        "orc_incidence": (None, [VP, C.c_int, U32P, U32P, U32P, C.POINTER(C.c_int)]),
        "orc_js_hypot3": (C.c_double, [C.c_double, C.c_double, C.c_double]),
        "orc_tri_energy_grad": (None, [F64P, F64P, C.c_double, F64P, F64P]),
        "orc_tri_hvp": (None, [F64P, F64P, F64P, C.c_double, F64P, F64P]),
        "orc_tri_hessian9": (None, [F64P, F64P, C.c_double, F64P, F64P]),
        "orc_dihedral": (C.c_double, [F64P, C.c_int, C.c_int, C.c_int, C.c_int]),
        "orc_eval_internal": (None, [VP, F64P, F64P, F64P, F64P]),
        "orc_internal_energy_only": (C.c_double, [VP, F64P, F64P]),
        "orc_eval_membrane": (C.c_double, [VP, F64P, F64P, F64P]),
        "orc_membrane_hvp": (None, [VP, F64P, F64P, F64P, F64P]),
        "orc_eval_membrane_hvp": (None, [VP, F64P, F64P, F64P, F64P]),
        "orc_eval_membrane_blocks": (None, [VP, F64P, F64P, F64P]),
        "orc_closest_vt": (None, [F64P, F64P]),
        "orc_closest_ee": (None, [F64P, F64P]),
        "orc_vt_ccd": (C.c_double, [F64P, F64P, C.c_double]),
        "orc_ee_ccd": (C.c_double, [F64P, F64P, C.c_double]),
        "orc_solve_cubic01": (C.c_int, [C.c_double] * 4 + [F64P]),
        "orc_barrier_value": (C.c_double, [C.c_double, C.c_double]),
        "orc_barrier_grad_scalar": (C.c_double, [C.c_double] * 4),
        "orc_coulomb_force": (None, [F64P, F64P, C.c_double, C.c_double, C.c_double, F64P]),
        "orc_contact_create": (VP, [F64P, U32P, C.c_int]),
        "orc_contact_destroy": (None, [VP]),
        "orc_contact_set_floor": (None, [VP, C.c_int, C.c_double]),
        "orc_contact_set_static": (None, [VP, F32P, C.c_int, U32P, C.c_int]),
        "orc_contact_begin_step": (None, [VP, F64P, C.c_int]),
        "orc_contact_update_active_set": (None, [VP, F64P, C.c_int]),
        "orc_contact_energy_grad": (C.c_double, [VP, F64P, F64P, C.c_int]),
        "orc_contact_apply_hvp": (None, [VP, F64P, F64P, F64P, C.c_int]),
        "orc_contact_merit_energy": (C.c_double, [VP, F64P]),
        "orc_contact_add_diag_estimate": (None, [VP, F64P, F64P]),
        "orc_contact_commit": (None, [VP, F64P]),
        "orc_contact_check_trial": (C.c_int, [VP, F64P, C.c_int, F64P]),
        "orc_contact_active": (C.c_int, [VP, VP, VP]),
        "orc_contact_candidates": (C.c_int, [VP, F64P, C.c_double, VP, C.c_int]),
        "orc_tri_pairs": (C.c_int, [F64P, F64P, U32P, C.c_int, C.c_double, VP, C.c_int]),
        "orc_contact_diag": (None, [VP, F64P]),
        "orc_schwarz_domains": (VP, [VP, F32P, C.c_int, C.c_int, C.c_int]),
        "orc_schwarz_destroy": (None, [VP]),
        "orc_schwarz_info": (C.c_int, [VP, VP, VP, C.c_int]),
        "orc_pcg_solve": (C.c_int, [VP, F64P, F64P, VP, C.c_double, F64P, F64P, C.c_int, C.c_double,
                                    C.c_int, VP, F64P, C.POINTER(C.c_double)]),
        "orc_scene_create": (VP, [VP, F64P, F64P, F64P, F64P]),
        "orc_scene_destroy": (None, [VP]),
        "orc_scene_set_material": (None, [VP, F64P]),
        "orc_scene_set_pins": (None, [VP, C.c_int, I32P, F64P]),
        "orc_scene_set_contact": (None, [VP, VP]),
        "orc_scene_set_state": (None, [VP, VP, VP]),
        "orc_scene_get_state": (None, [VP, VP, VP]),
        "orc_scene_build_schwarz": (None, [VP, C.c_int, C.c_int, C.c_int]),
        "orc_step": (C.c_int, [VP, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, F64P]),
        "orc_step_exact": (C.c_int, [VP, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                     C.c_double, C.c_int, F64P]),
        "orc_hinge_grad_exact": (None, [F64P, F64P, C.c_double, F64P]),
        "orc_hinge_hess_exact": (None, [F64P, F64P, C.c_double, F64P]),
        "orc_stress_positive_part": (None, [F64P]),
        "orc_eval_internal_exact": (None, [VP, F64P, F64P, F64P, F64P]),
        "orc_internal_hvp_exact": (None, [VP, F64P, F64P, F64P, F64P]),
        "orc_contact_friction_potential": (C.c_double, [VP, F64P, F64P, VP, VP, C.c_int]),
        "orc_lbvh_build": (VP, [F64P, F64P, U32P, C.c_int, C.c_double, C.c_long]),
        "orc_lbvh_destroy": (None, [VP]),
        "orc_lbvh_info": (None, [VP, np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")]),
        "orc_lbvh_arrays": (None, [VP] + [VP] * 10),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---- parameter packing -------------------------------------------------------

DEFAULT_MATERIAL = dict(arealDensity=0.15, thickness=0.001, C00=20000.0, C11=20000.0, C01=0.0,
                        G=5000.0, bendWarp=1e-5, bendWeft=1e-5, damping=0.001)
DEFAULT_CONTACT = dict(dHat=0.002, kappa=50.0, dMin=1e-4, mu=0.3, eps=1e-4)
MAT_KEYS = ["arealDensity", "thickness", "C00", "C11", "C01", "G", "bendWarp", "bendWeft", "damping"]
CON_KEYS = ["dHat", "kappa", "dMin", "mu", "eps"]


def mat_array(mat: dict) -> np.ndarray:
    m = dict(DEFAULT_MATERIAL)
    m.update(mat)
    return np.array([m[k] for k in MAT_KEYS], np.float64)


def contact_array(p: dict) -> np.ndarray:
    c = dict(DEFAULT_CONTACT)
    c.update(p)
    return np.array([c[k] for k in CON_KEYS], np.float64)


# ---- mesh ----------------------------------------------------------------------

def build_grid(nx, ny, w, h):
    n = (nx + 1) * (ny + 1)
    pos = np.zeros(n * 3, np.float32)
    uv = np.zeros(n * 2, np.float32)
    idx = np.zeros(nx * ny * 6, np.uint32)
    lib().orc_build_grid(nx, ny, w, h, pos, uv, idx)
    return pos, uv, idx


class Mesh:
    """Preprocessed cloth mesh (src/mesh/mesh.ts:50-97), f32 constants."""

    def __init__(self, pos, uv, idx, density):
        pos = np.ascontiguousarray(pos, np.float32)
        uv = np.ascontiguousarray(uv, np.float32)
        idx = np.ascontiguousarray(idx, np.uint32)
        self.n = len(pos) // 3
        self.m = len(idx) // 3
        self.h = lib().orc_mesh_create(self.n, self.m, pos, uv, idx, density)
        if not self.h:
            raise ValueError("degenerate triangle")
        cnt = np.zeros(3, np.int32)
        lib().orc_mesh_counts(self.h, cnt)
        self.hg = int(cnt[2])
        self.positions = pos.copy()
        self.uv = uv.copy()
        self.indices = idx.copy()
        self.invDm = np.zeros(self.m * 4, np.float32)
        self.areas = np.zeros(self.m, np.float32)
        self.masses = np.zeros(self.n, np.float32)
        self.hinges = np.zeros(self.hg * 4, np.int32)
        self.hinge_meta = np.zeros(self.hg * 3, np.float64)
        lib().orc_mesh_arrays(self.h, self.invDm, self.areas, self.masses, self.hinges, self.hinge_meta)

    def incidence(self, kind: int):
        nrec = C.c_int(0)
        cap = max(3 * self.m, 4 * self.hg, 1)
        off = np.zeros(self.n + 1, np.uint32)
        ids = np.zeros(cap, np.uint32)
        cor = np.zeros(cap, np.uint32)
        lib().orc_incidence(self.h, kind, off, ids, cor, C.byref(nrec))
        return off, ids[: nrec.value], cor[: nrec.value]

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_mesh_destroy(self.h)
            self.h = None


# ---- element functions ---------------------------------------------------------

def hinge_energy(q12, meta3, k):
    """hingeEnergy (src/physics/bending.ts:7-16) of the 4 vertices in q12."""
    return lib().orc_hinge_energy(np.ascontiguousarray(q12, np.float64), np.arange(4, dtype=np.int32),
                                  np.ascontiguousarray(meta3, np.float64), k)


def hinge_grad_exact(q12, meta3, k):
    """Exact gradient of hinge_energy over the 12 coordinates (exact-Newton mode)."""
    g = np.zeros(12)
    lib().orc_hinge_grad_exact(np.ascontiguousarray(q12, np.float64), np.ascontiguousarray(meta3, np.float64),
                               k, g)
    return g


def hinge_hess_exact(q12, meta3, k):
    """Exact 12x12 Hessian of hinge_energy (hyper-dual numbers)."""
    h = np.zeros(144)
    lib().orc_hinge_hess_exact(np.ascontiguousarray(q12, np.float64), np.ascontiguousarray(meta3, np.float64),
                               k, h)
    return h.reshape(12, 12)


def stress_positive_part(s00, s11, s01):
    """Positive part of the symmetric stress [[s00, s01], [s01, s11]]."""
    s = np.array([s00, s11, s01], np.float64)
    lib().orc_stress_positive_part(s)
    return tuple(s.tolist())


def tri_energy_grad(x0, x1, x2, inv, area, mat):
    out = np.zeros(13)
    lib().orc_tri_energy_grad(np.array([*x0, *x1, *x2], np.float64), np.array(inv, np.float64),
                              float(area), mat_array(mat), out)
    return out[0], out[1:10].copy(), out[10:13].copy()


def tri_hvp(x9, v9, inv, area, mat):
    out = np.zeros(9)
    lib().orc_tri_hvp(np.asarray(x9, np.float64), np.asarray(v9, np.float64), np.array(inv, np.float64),
                      float(area), mat_array(mat), out)
    return out


def tri_hessian9(x9, inv, area, mat):
    out = np.zeros(81)
    lib().orc_tri_hessian9(np.asarray(x9, np.float64), np.array(inv, np.float64), float(area),
                           mat_array(mat), out)
    return out.reshape(9, 9)


def eval_internal(mesh: Mesh, mat, x):
    g = np.zeros(mesh.n * 3)
    o = np.zeros(2)
    lib().orc_eval_internal(mesh.h, mat_array(mat), np.ascontiguousarray(x, np.float64), g, o)
    return o[0], g, o[1]


def internal_energy_only(mesh: Mesh, mat, x):
    return lib().orc_internal_energy_only(mesh.h, mat_array(mat), np.ascontiguousarray(x, np.float64))


def eval_membrane(mesh: Mesh, mat, x):
    g = np.zeros(mesh.n * 3)
    e = lib().orc_eval_membrane(mesh.h, mat_array(mat), np.ascontiguousarray(x, np.float64), g)
    return e, g


def eval_internal_exact(mesh: Mesh, mat, x):
    """eval_internal with the exact hinge gradient (exact-Newton mode)."""
    g = np.zeros(mesh.n * 3)
    o = np.zeros(2)
    lib().orc_eval_internal_exact(mesh.h, mat_array(mat), np.ascontiguousarray(x, np.float64), g, o)
    return o[0], g, o[1]


def internal_hvp_exact(mesh: Mesh, mat, x, p):
    """Exact-Newton mode's internal Newton matrix along p: membrane HVP with the
    positive part of the stress in its geometric term, plus the bending HVP."""
    o = np.zeros(mesh.n * 3)
    lib().orc_internal_hvp_exact(mesh.h, mat_array(mat), np.ascontiguousarray(x, np.float64),
                                 np.ascontiguousarray(p, np.float64), o)
    return o


def membrane_hvp(mesh: Mesh, mat, x, p):
    o = np.zeros(mesh.n * 3)
    lib().orc_membrane_hvp(mesh.h, mat_array(mat), np.ascontiguousarray(x, np.float64),
                           np.ascontiguousarray(p, np.float64), o)
    return o


def eval_membrane_hvp(mesh: Mesh, mat, x, p):
    o = np.zeros(mesh.n * 3)
    lib().orc_eval_membrane_hvp(mesh.h, mat_array(mat), np.ascontiguousarray(x, np.float64),
                                np.ascontiguousarray(p, np.float64), o)
    return o


def eval_membrane_blocks(mesh: Mesh, mat, x):
    o = np.zeros(mesh.n * 9)
    lib().orc_eval_membrane_blocks(mesh.h, mat_array(mat), np.ascontiguousarray(x, np.float64), o)
    return o


def closest_vt(p, a, b, c):
    o = np.zeros(6)
    lib().orc_closest_vt(np.array([*p, *a, *b, *c], np.float64), o)
    return o


def closest_ee(a, b, c, d):
    o = np.zeros(6)
    lib().orc_closest_ee(np.array([*a, *b, *c, *d], np.float64), o)
    return o


def vt_ccd(P0, P1, thickness):
    return lib().orc_vt_ccd(np.asarray(P0, np.float64).ravel(), np.asarray(P1, np.float64).ravel(), thickness)


def ee_ccd(P0, P1, thickness):
    return lib().orc_ee_ccd(np.asarray(P0, np.float64).ravel(), np.asarray(P1, np.float64).ravel(), thickness)


def solve_cubic01(a3, a2, a1, a0):
    o = np.zeros(3)
    k = lib().orc_solve_cubic01(a3, a2, a1, a0, o)
    return list(o[:k])


def barrier_value(d, dHat):
    return lib().orc_barrier_value(d, dHat)


def coulomb_force(u, n, lam, mu, eps):
    o = np.zeros(3)
    lib().orc_coulomb_force(np.array(u, np.float64), np.array(n, np.float64), lam, mu, eps, o)
    return o


def tri_pairs(x0, x1, idx, pad):
    x0 = np.ascontiguousarray(x0, np.float64)
    x1 = np.ascontiguousarray(x1, np.float64)
    idx = np.ascontiguousarray(idx, np.uint32)
    k = lib().orc_tri_pairs(x0, x1, idx, len(idx) // 3, pad, None, 0)
    out = np.zeros(max(k, 1) * 2, np.int32)
    lib().orc_tri_pairs(x0, x1, idx, len(idx) // 3, pad, _ptr(out), k)
    return out[: k * 2].reshape(k, 2)


# ---- ContactSystem ---------------------------------------------------------------

class ContactSystem:
    """src/collision/contact-assembly.ts ContactSystem restated."""

    def __init__(self, params: dict, indices):
        self.idx = np.ascontiguousarray(indices, np.uint32)
        self.h = lib().orc_contact_create(contact_array(params), self.idx, len(self.idx) // 3)

    def set_floor(self, y):
        lib().orc_contact_set_floor(self.h, 0 if y is None else 1, 0.0 if y is None else float(y))

    def set_static_mesh(self, pos, idx):
        self.spos = np.ascontiguousarray(pos, np.float32)
        self.sidx = np.ascontiguousarray(idx, np.uint32)
        lib().orc_contact_set_static(self.h, self.spos, len(self.spos) // 3, self.sidx, len(self.sidx) // 3)

    def begin_step(self, x0):
        x0 = np.ascontiguousarray(x0, np.float64)
        lib().orc_contact_begin_step(self.h, x0, len(x0))

    def update_active_set(self, x):
        x = np.ascontiguousarray(x, np.float64)
        lib().orc_contact_update_active_set(self.h, x, len(x))

    def energy_grad(self, x):
        x = np.ascontiguousarray(x, np.float64)
        g = np.zeros(len(x))
        e = lib().orc_contact_energy_grad(self.h, x, g, len(x))
        return e, g

    def apply_hvp(self, x, v):
        x = np.ascontiguousarray(x, np.float64)
        o = np.zeros(len(x))
        lib().orc_contact_apply_hvp(self.h, x, np.ascontiguousarray(v, np.float64), o, len(x))
        return o

    def merit_energy(self, x):
        return lib().orc_contact_merit_energy(self.h, np.ascontiguousarray(x, np.float64))

    def add_diag_estimate(self, diag, x):
        lib().orc_contact_add_diag_estimate(self.h, diag, np.ascontiguousarray(x, np.float64))

    def commit(self, x):
        lib().orc_contact_commit(self.h, np.ascontiguousarray(x, np.float64))

    def friction_potential(self, xf, x, v=None):
        """Exact-Newton mode: the friction potential of the active contacts
        frozen at xf, evaluated at x; with v, also its Hessian along v."""
        xf = np.ascontiguousarray(xf, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        va = None if v is None else np.ascontiguousarray(v, np.float64)
        out = None if v is None else np.zeros(len(x))
        e = lib().orc_contact_friction_potential(self.h, xf, x, _ptr(va), _ptr(out), len(x))
        return e if v is None else (e, out)

    def check_trial(self, x):
        x = np.ascontiguousarray(x, np.float64)
        o = np.zeros(2)
        v = lib().orc_contact_check_trial(self.h, x, len(x), o)
        return bool(v), o[0], o[1]

    def active(self):
        k = lib().orc_contact_active(self.h, None, None)
        ids = np.zeros(max(k, 1) * 6, np.int32)
        w = np.zeros(max(k, 1) * 7)
        lib().orc_contact_active(self.h, _ptr(ids), _ptr(w))
        return ids[: k * 6].reshape(k, 6), w[: k * 7].reshape(k, 7)

    def candidates(self, x, pad):
        x = np.ascontiguousarray(x, np.float64)
        k = lib().orc_contact_candidates(self.h, x, pad, None, 0)
        ids = np.zeros(max(k, 1) * 6, np.int32)
        lib().orc_contact_candidates(self.h, x, pad, _ptr(ids), k)
        return ids[: k * 6].reshape(k, 6)

    def diag(self):
        o = np.zeros(11)
        lib().orc_contact_diag(self.h, o)
        keys = ["candidatePairs", "activePairs", "vtPairs", "eePairs", "floorPairs", "minDistance",
                "minTOI", "barrierEnergy", "frictionWork", "rejectedLineSearchSteps", "ccdFailures"]
        return dict(zip(keys, o.tolist()))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_contact_destroy(self.h)
            self.h = None


class SchwarzDomains:
    def __init__(self, mesh: Mesh, rest, target=16, min_size=8, max_size=32):
        self.mesh = mesh
        self.h = lib().orc_schwarz_domains(mesh.h, np.ascontiguousarray(rest, np.float32), target,
                                            min_size, max_size)
        self.count = lib().orc_schwarz_info(self.h, None, None, mesh.n)
        self.domain_of = np.zeros(mesh.n, np.uint32)
        self.local_of = np.zeros(mesh.n, np.uint32)
        lib().orc_schwarz_info(self.h, _ptr(self.domain_of), _ptr(self.local_of), mesh.n)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_schwarz_destroy(self.h)
            self.h = None


def pcg_solve(mesh: Mesh, mat, x, contact, invH2, diag, b, max_iters, tol, precond=0, domains=None):
    out = np.zeros(mesh.n * 3)
    res = C.c_double(0)
    it = lib().orc_pcg_solve(mesh.h, mat_array(mat), np.ascontiguousarray(x, np.float64),
                             contact.h if contact is not None else None, invH2,
                             np.ascontiguousarray(diag, np.float64), np.ascontiguousarray(b, np.float64),
                             max_iters, tol, precond, domains.h if domains is not None else None, out,
                             C.byref(res))
    return it, res.value, out


# ---- scene + CpuSolver-equivalent stepping ----------------------------------------

STAT_KEYS = ["newtonIters", "pcgIters", "gradNorm", "energy", "maxStrain", "converged", "hasContact",
             "candidatePairs", "activePairs", "vtPairs", "eePairs", "floorPairs", "minDistance", "minTOI",
             "barrierEnergy", "frictionWork", "rejectedLineSearchSteps", "ccdFailures",
             "newtonItersUsed", "armijoTrials"]

PRECOND = {"jacobi": 0, "schwarz": 1, "block": 2, "mas2": 3, "masX": 4}


class Scene:
    """ClothScene + CpuSolver.step (src/backend/cpu-solver.ts:15-18, implicitStep)."""

    def __init__(self, mesh: Mesh, mat: dict, gravity=(0.0, -9.81, 0.0), x=None, v=None):
        self.mesh = mesh
        self.mat = dict(mat)
        n3 = mesh.n * 3
        x = mesh.positions.astype(np.float64) if x is None else np.ascontiguousarray(x, np.float64)
        v = np.zeros(n3) if v is None else np.ascontiguousarray(v, np.float64)
        self.h = lib().orc_scene_create(mesh.h, mat_array(mat), np.array(gravity, np.float64), x, v)
        self.contact = None
        self.pins = {}

    def set_material(self, mat):
        self.mat = dict(mat)
        lib().orc_scene_set_material(self.h, mat_array(mat))

    def set_pins(self, pins: dict):
        self.pins = dict(pins)
        ids = np.array(list(pins.keys()), np.int32)
        pos = np.array([pins[k] for k in pins], np.float64).reshape(-1)
        if len(ids) == 0:
            ids = np.zeros(1, np.int32)
            pos = np.zeros(3)
            lib().orc_scene_set_pins(self.h, 0, ids, pos)
        else:
            lib().orc_scene_set_pins(self.h, len(ids), ids, pos)

    def set_contact(self, cs: ContactSystem):
        self.contact = cs
        lib().orc_scene_set_contact(self.h, cs.h if cs is not None else None)

    @property
    def positions(self):
        x = np.zeros(self.mesh.n * 3)
        lib().orc_scene_get_state(self.h, _ptr(x), None)
        return x

    @property
    def velocities(self):
        v = np.zeros(self.mesh.n * 3)
        lib().orc_scene_get_state(self.h, None, _ptr(v))
        return v

    def set_state(self, x=None, v=None):
        xa = None if x is None else np.ascontiguousarray(x, np.float64)
        va = None if v is None else np.ascontiguousarray(v, np.float64)
        lib().orc_scene_set_state(self.h, _ptr(xa), _ptr(va))

    def build_schwarz(self, target=8, min_size=1, max_size=8):
        lib().orc_scene_build_schwarz(self.h, target, min_size, max_size)

    def step(self, dt, newton_iters=10, pcg_max_iters=60, grad_tol=1e-5, ls_iters=10, precond="jacobi",
             exact=False, pcg_tol=1e-6, drift=True):
        """implicitStep; exact=True runs the CUDA solver's exact-Newton mode
        (implicit_step_exact) with PCG tolerance pcg_tol and the drift start."""
        st = np.zeros(20)
        if exact:
            rc = lib().orc_step_exact(self.h, dt, newton_iters, pcg_max_iters, grad_tol, ls_iters,
                                      PRECOND[precond], pcg_tol, 1 if drift else 0, st)
        else:
            rc = lib().orc_step(self.h, dt, newton_iters, pcg_max_iters, grad_tol, ls_iters, PRECOND[precond], st)
        if rc == 2:
            raise FloatingPointError("non-finite gradient — blow up; reduce dt/stiffness")
        return dict(zip(STAT_KEYS, st.tolist()))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_scene_destroy(self.h)
            self.h = None


# ---- FP32 LBVH mirror ----------------------------------------------------------------

def lbvh_mirror(x0, x1, idx, pad, capacity=1 << 40):
    x0 = np.ascontiguousarray(x0, np.float64)
    x1 = np.ascontiguousarray(x1, np.float64)
    idx = np.ascontiguousarray(idx, np.uint32)
    m = len(idx) // 3
    L = lib()
    h = L.orc_lbvh_build(x0, x1, idx, m, pad, capacity)
    info = np.zeros(5, np.int64)
    L.orc_lbvh_info(h, info)
    nc = max(1, 2 * m - 1)
    out = dict(
        aabb=np.zeros(m * 6, np.float32), centroid=np.zeros(m * 3, np.float32),
        morton=np.zeros(m, np.uint32), payload=np.zeros(m, np.uint32),
        nodeMin=np.zeros(nc * 3, np.float32), nodeMax=np.zeros(nc * 3, np.float32),
        left=np.zeros(nc, np.int32), right=np.zeros(nc, np.int32), leafTri=np.zeros(nc, np.int32),
        pairs=np.zeros(max(int(info[2]), 1) * 2, np.int32))
    L.orc_lbvh_arrays(h, *[_ptr(out[k]) for k in ["aabb", "centroid", "morton", "payload", "nodeMin",
                                                  "nodeMax", "left", "right", "leafTri", "pairs"]])
    L.orc_lbvh_destroy(h)
    out["pairs"] = out["pairs"][: int(info[2]) * 2].reshape(-1, 2)
    out.update(root=int(info[0]), depth=int(info[1]), scanned=int(info[3]), overflow=int(info[4]))
    return out
