"""Host-side mirror of the reference's cloth backend interface, over the CUDA C ABI.

Mirrors (mohdabraralikhan/closim):
  ClothSolver            src/backend/solver.ts:5-13
  CpuSolver semantics    src/backend/cpu-solver.ts:5-49 (scene kept by reference,
                         results written back into scene.positions/velocities)
  ClothScene/createScene src/physics/scene.ts:5-36
  buildGrid/preprocess   src/mesh/mesh.ts:17-97
  ContactSystem config   src/collision/contact-assembly.ts:63-73
  StepStats              src/solver/newton.ts:10-18

CudaSolver is the drop-in for CpuSolver: the same methods, argument meaning and
error behaviour; every step runs on the GPU through libclosim_cuda.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, replace
from typing import Dict, Optional, Tuple

import numpy as np

from . import _lib as L

# ---- data model -------------------------------------------------------------------


@dataclass
class ClothMaterial:
    """ClothMaterial (src/physics/types.ts:1-12)."""
    arealDensityKgM2: float = 0.15
    thickness: float = 0.001
    stretchWarp: float = 20000.0
    stretchWeft: float = 20000.0
    stretchCoupling: float = 0.0
    shear: float = 5000.0
    bendWarp: float = 1e-5
    bendWeft: float = 1e-5
    damping: float = 0.001

    def _c(self):
        return L.cs_material(self.arealDensityKgM2, self.thickness, self.stretchWarp, self.stretchWeft,
                             self.stretchCoupling, self.shear, self.bendWarp, self.bendWeft, self.damping)


DEFAULT_MATERIAL = ClothMaterial()


@dataclass
class ContactParams:
    """ContactParams (src/collision/types.ts:27-47)."""
    dHatM: float = 0.002
    kappaJ: float = 50.0
    dMinM: float = 1e-4
    frictionMu: float = 0.3
    frictionEpsM: float = 1e-4


DEFAULT_CONTACT_PARAMS = ContactParams()


@dataclass
class ClothMeshData:
    """ClothMeshData (src/mesh/mesh.ts:3-14); constants are Float32."""
    count: int
    triCount: int
    positions: np.ndarray
    restPositions: np.ndarray
    uv: np.ndarray
    indices: np.ndarray
    invDm: np.ndarray
    areas: np.ndarray
    masses: np.ndarray
    hinges: np.ndarray        # int32 (hg, 4): v0, v1, v2, v3
    hingeMeta: np.ndarray     # float64 (hg, 3): restAngle, edgeLen, areaSum


class ContactSystem:
    """Contact configuration of a scene (contact-assembly.ts:63-73): params,
    optional floor plane y = floorY and optional static triangle mesh."""

    def __init__(self, params: ContactParams, clothIndices: np.ndarray):
        self.params = replace(params)
        self.clothIdx = np.ascontiguousarray(clothIndices, np.uint32)
        self.floorY: Optional[float] = None
        self.staticPos: Optional[np.ndarray] = None
        self.staticIdx: Optional[np.ndarray] = None

    def setFloor(self, y: Optional[float]) -> None:
        self.floorY = None if y is None else float(y)

    def setStaticMesh(self, pos, idx) -> None:
        self.staticPos = np.ascontiguousarray(pos, np.float32)
        self.staticIdx = np.ascontiguousarray(idx, np.uint32)


@dataclass
class ClothScene:
    """ClothScene (src/physics/scene.ts:5-14)."""
    mesh: ClothMeshData
    material: ClothMaterial
    gravity: Tuple[float, float, float]
    pinned: Dict[int, Tuple[float, float, float]]
    positions: np.ndarray
    velocities: np.ndarray
    contact: Optional[ContactSystem] = None


@dataclass
class StepStats:
    """StepStats (src/solver/newton.ts:10-18) with ContactDiagnostics."""
    newtonIters: int
    pcgIters: int
    gradNorm: float
    energy: float
    maxStrain: float
    converged: bool
    contact: Optional[dict]
    newtonItersUsed: int = 0
    armijoTrials: int = 0


# ---- mesh helpers ------------------------------------------------------------------

def buildGrid(nx: int, ny: int, w: float, h: float):
    """buildGrid (src/mesh/mesh.ts:17-48): XZ grid at y = 0."""
    n = (nx + 1) * (ny + 1)
    pos = np.zeros(n * 3, np.float32)
    uv = np.zeros(n * 2, np.float32)
    idx = np.zeros(nx * ny * 6, np.uint32)
    rc = L.load().cs_build_grid(nx, ny, w, h, L.ptr(pos), L.ptr(uv), L.ptr(idx))
    if rc != L.CS_OK:
        raise ValueError("buildGrid: invalid arguments")
    return pos, uv, idx


def preprocess(positions, uv, indices, arealDensityKgM2: float) -> ClothMeshData:
    """preprocess (src/mesh/mesh.ts:50-97): Dm^-1, areas, lumped masses, hinges."""
    pos = np.ascontiguousarray(positions, np.float32)
    uv = np.ascontiguousarray(uv, np.float32)
    idx = np.ascontiguousarray(indices, np.uint32)
    n, m = len(pos) // 3, len(idx) // 3
    inv = np.zeros(m * 4, np.float32)
    area = np.zeros(m, np.float32)
    mass = np.zeros(n, np.float32)
    hg = C.c_int32(0)
    lib = L.load()
    rc = lib.cs_preprocess(n, m, L.ptr(pos), L.ptr(uv), L.ptr(idx), arealDensityKgM2, None, None, None,
                           C.byref(hg), None, None)
    if rc != L.CS_OK:
        raise ValueError("preprocess: degenerate triangle or bad indices")
    hinge = np.zeros(max(hg.value, 1) * 4, np.int32)
    meta = np.zeros(max(hg.value, 1) * 3, np.float64)
    rc = lib.cs_preprocess(n, m, L.ptr(pos), L.ptr(uv), L.ptr(idx), arealDensityKgM2, L.ptr(inv), L.ptr(area),
                           L.ptr(mass), C.byref(hg), L.ptr(hinge), L.ptr(meta))
    if rc != L.CS_OK:
        raise ValueError("preprocess: degenerate triangle or bad indices")
    k = hg.value
    return ClothMeshData(n, m, pos.copy(), pos.copy(), uv.copy(), idx.copy(), inv, area, mass,
                         hinge[:k * 4].reshape(k, 4).copy(), meta[:k * 3].reshape(k, 3).copy())


def createScene(mesh: ClothMeshData, material: ClothMaterial, gravity=(0.0, -9.81, 0.0)) -> ClothScene:
    """createScene (src/physics/scene.ts:16-26)."""
    return ClothScene(mesh, material, tuple(gravity), {}, mesh.positions.astype(np.float64),
                      np.zeros(mesh.count * 3), None)


def pinColumn(scene: ClothScene, predicate) -> None:
    """pinColumn (src/physics/scene.ts:28-36)."""
    x = scene.positions
    for i in range(scene.mesh.count):
        if predicate(x[i * 3], x[i * 3 + 1], x[i * 3 + 2], i):
            scene.pinned[i] = (float(x[i * 3]), float(x[i * 3 + 1]), float(x[i * 3 + 2]))


def enforcePins(scene: ClothScene, x: np.ndarray) -> None:
    """enforcePins (src/physics/scene.ts:38-44)."""
    for i, p in scene.pinned.items():
        x[i * 3:i * 3 + 3] = p


# ---- the solver --------------------------------------------------------------------


class ClothSolverError(RuntimeError):
    pass


class CudaSolver:
    """Drop-in for CpuSolver (src/backend/cpu-solver.ts) running on one B200.

    precision: "fp64" (plain path, op-for-op with the reference arithmetic) or
    "mixed". options: StepperOptions (newtonIters, pcgMaxIters, gradTol,
    lineSearchIters) plus precond ("jacobi" | "schwarz" | "mas2": two-level
    Schwarz, src/solver/mas.ts).
    """

    def __init__(self, precision: str = "fp64", device: int = 0, **options):
        self._lib = L.load()
        prec = {"fp64": L.CS_PRECISION_FP64, "mixed": L.CS_PRECISION_MIXED}[precision]
        self._h = self._lib.cs_create(prec, device)
        if not self._h:
            raise ClothSolverError("cs_create failed: no CUDA device or unsupported precision")
        self.precision = precision
        self.scene: Optional[ClothScene] = None
        self.lastStats: Optional[StepStats] = None
        self._pins_sent = None
        self.syncFromScene = False
        self._options = dict(newtonIters=10, pcgMaxIters=60, gradTol=1e-5, lineSearchIters=10, precond="jacobi")
        self.setOptions(**options)

    # -- helpers --
    def _check(self, rc: int):
        if rc == L.CS_OK:
            return
        msg = self._lib.cs_last_error(self._h).decode()
        if rc == L.CS_E_NONFINITE:
            raise FloatingPointError(msg)
        if rc == L.CS_E_UNINIT:
            raise ClothSolverError("CudaSolver not initialized")
        raise ClothSolverError(f"cs error {rc}: {msg}")

    def _need(self):
        if self.scene is None:
            raise ClothSolverError("CudaSolver not initialized")

    def setOptions(self, **o):
        self._options.update(o)
        oo = self._options
        pc = {"jacobi": L.CS_PRECOND_JACOBI, "schwarz": L.CS_PRECOND_SCHWARZ, "mas2": L.CS_PRECOND_MAS2}[oo["precond"]]
        opts = L.cs_stepper_options(int(oo["newtonIters"]), int(oo["pcgMaxIters"]), int(oo["lineSearchIters"]),
                                    pc, float(oo["gradTol"]))
        self._check(self._lib.cs_set_stepper_options(self._h, C.byref(opts)))

    def _send_pins(self, force=False):
        pins = self.scene.pinned
        key = tuple((k, tuple(v)) for k, v in pins.items())
        if not force and key == self._pins_sent:
            return
        ids = np.array(list(pins.keys()), np.int32)
        pos = np.array([pins[k] for k in pins], np.float64).reshape(-1)
        self._check(self._lib.cs_set_pins(self._h, len(ids), L.ptr(ids) if len(ids) else None,
                                          L.ptr(pos) if len(ids) else None))
        self._pins_sent = key

    # -- ClothSolver interface (src/backend/solver.ts:5-13) --
    def initialize(self, scene: ClothScene) -> None:
        me = scene.mesh
        self.scene = scene
        self._keep = [np.ascontiguousarray(a) for a in (me.indices, me.restPositions, me.invDm, me.areas, me.masses,
                                                        me.hinges.astype(np.int32).reshape(-1),
                                                        me.hingeMeta.astype(np.float64).reshape(-1))]
        idx, rest, inv, area, mass, hinge, meta = self._keep
        cm = L.cs_mesh(me.count, me.triCount, len(hinge) // 4, L.ptr(idx), L.ptr(rest), L.ptr(inv), L.ptr(area),
                       L.ptr(mass), L.ptr(hinge), L.ptr(meta))
        mat = scene.material._c()
        g = np.array(scene.gravity, np.float64)
        scene.positions = np.ascontiguousarray(scene.positions, np.float64)
        scene.velocities = np.ascontiguousarray(scene.velocities, np.float64)
        self._check(self._lib.cs_initialize(self._h, C.byref(cm), C.byref(mat), L.ptr(g), L.ptr(scene.positions),
                                            L.ptr(scene.velocities)))
        self._send_pins(force=True)
        c = scene.contact
        if c is not None:
            p = c.params
            cp = L.cs_contact_params(p.dHatM, p.kappaJ, p.dMinM, p.frictionMu, p.frictionEpsM)
            sp, si = c.staticPos, c.staticIdx
            self._check(self._lib.cs_set_contact(
                self._h, C.byref(cp), 0 if c.floorY is None else 1, 0.0 if c.floorY is None else c.floorY,
                L.ptr(sp), 0 if sp is None else len(sp) // 3, L.ptr(si), 0 if si is None else len(si) // 3))

    def step(self, dt: float) -> None:
        """One implicit step; positions/velocities are written back to the scene.

        With syncFromScene set, scene.positions / scene.velocities are uploaded
        first, so edits the caller made to the scene arrays take effect."""
        self._need()
        if self.syncFromScene:
            self.push_state()
        self._send_pins()
        self._check(self._lib.cs_step(self._h, float(dt)))
        self._pull()
        self.lastStats = self._stats()

    def setMaterial(self, material: ClothMaterial) -> None:
        self._need()
        self.scene.material = replace(material)
        mat = material._c()
        self._check(self._lib.cs_set_material(self._h, C.byref(mat)))

    def pinVertex(self, vertexId: int, position=None) -> None:
        self._need()
        x = self.scene.positions
        p = tuple(position) if position is not None else (x[vertexId * 3], x[vertexId * 3 + 1], x[vertexId * 3 + 2])
        self.scene.pinned[int(vertexId)] = tuple(float(q) for q in p)
        enforcePins(self.scene, self.scene.positions)
        self._check(self._lib.cs_set_state(self._h, L.ptr(self.scene.positions), None))
        self._send_pins()

    def unpinVertex(self, vertexId: int) -> None:
        if self.scene is None:
            return
        self.scene.pinned.pop(int(vertexId), None)
        self._send_pins()

    def getPositions(self) -> np.ndarray:
        self._need()
        return self.scene.positions

    def getVelocities(self) -> np.ndarray:
        self._need()
        return self.scene.velocities

    # -- device-resident stepping (no host copies between steps) --
    def advance(self, dt: float, steps: int) -> None:
        self._need()
        self._send_pins()
        self._check(self._lib.cs_step_n(self._h, float(dt), int(steps)))
        self.lastStats = self._stats()

    def pull(self) -> None:
        self._pull()

    def _pull(self):
        self._check(self._lib.cs_get_positions(self._h, L.ptr(self.scene.positions)))
        self._check(self._lib.cs_get_velocities(self._h, L.ptr(self.scene.velocities)))

    def push_state(self) -> None:
        self._check(self._lib.cs_set_state(self._h, L.ptr(self.scene.positions), L.ptr(self.scene.velocities)))

    def _stats(self) -> StepStats:
        st = L.cs_step_stats()
        self._check(self._lib.cs_last_stats(self._h, C.byref(st)))
        con = None
        if st.has_contact:
            con = {k: getattr(st, s) for k, s in [
                ("candidatePairs", "candidate_pairs"), ("activePairs", "active_pairs"), ("vtPairs", "vt_pairs"),
                ("eePairs", "ee_pairs"), ("floorPairs", "floor_pairs"), ("minDistance", "min_distance"),
                ("minTOI", "min_toi"), ("barrierEnergy", "barrier_energy"), ("frictionWork", "friction_work"),
                ("rejectedLineSearchSteps", "rejected_line_search_steps"), ("ccdFailures", "ccd_failures")]}
        return StepStats(st.newton_iters, st.pcg_iters, st.grad_norm, st.energy, st.max_strain, bool(st.converged),
                         con, st.newton_iters_used, st.armijo_trials)

    def membraneHvp(self, x, p) -> np.ndarray:
        """membraneHvp (src/physics/fem.ts:108-130) on the GPU: central-difference
        membrane Hessian-vector product at x along p."""
        self._need()
        x = np.ascontiguousarray(x, np.float64)
        p = np.ascontiguousarray(p, np.float64)
        out = np.zeros_like(x)
        self._check(self._lib.cs_membrane_hvp(self._h, L.ptr(x), L.ptr(p), L.ptr(out)))
        return out

    def activeContacts(self):
        """ContactSystem.active after the last step: (ids [k, 6] int32: kind,
        p, a, b, c, d; weights [k, 7]: w0..w3, nx, ny, nz), in list order."""
        self._need()
        k = C.c_int32(0)
        self._check(self._lib.cs_contact_active(self._h, 0, C.byref(k), None, None))
        ids = np.zeros(max(k.value, 1) * 6, np.int32)
        w = np.zeros(max(k.value, 1) * 7)
        self._check(self._lib.cs_contact_active(self._h, max(k.value, 1), C.byref(k), L.ptr(ids), L.ptr(w)))
        return ids[:k.value * 6].reshape(-1, 6), w[:k.value * 7].reshape(-1, 7)

    def setStaticPositions(self, positions) -> None:
        """Moves the scene's static collider mesh (same triangles) before the
        next step: ContactSystem.setStaticMesh with a collider's sampled pose
        (src/collision/avatar-collider.ts:205-237). The scene's ContactSystem
        keeps the new positions."""
        self._need()
        c = self.scene.contact
        if c is None or c.staticPos is None:
            raise ClothSolverError("the scene has no static mesh")
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1)
        if pos.size != c.staticPos.size:
            raise ValueError("static positions must keep the static mesh's vertex count")
        self._check(self._lib.cs_update_static_positions(self._h, L.ptr(pos), pos.size // 3))
        c.staticPos = pos.copy()

    def setGraphMode(self, enable: bool) -> None:
        """Graph-captured steps with device-side Newton/Armijo control (default
        on; applies to the mixed path's one-cluster sheets); off forces the
        host-driven step."""
        self._check(self._lib.cs_set_graph_mode(self._h, 1 if enable else 0))

    def graphInfo(self) -> dict:
        out = np.zeros(2, np.int64)
        self._check(self._lib.cs_graph_info(self._h, L.ptr(out)))
        return dict(graphSteps=int(out[0]), hostRepeats=int(out[1]))

    def kernelLaunches(self) -> int:
        return int(self._lib.cs_kernel_launches(self._h))

    def stream(self) -> int:
        """The solver's cudaStream_t (for events recorded around calls)."""
        return int(self._lib.cs_stream(self._h) or 0)

    PHASES = ["other", "broadphase", "active_set", "gradient", "precond", "pcg", "trial", "energy", "commit"]

    def profile(self, enable, phases: bool = False) -> None:
        """Per-launch timing of the PCG kernel; phases=True also charges wall
        time to the step's phases (synchronizing at each boundary)."""
        self._check(self._lib.cs_profile(self._h, (2 if phases else 1) if enable else 0))

    # ---- differentiable rollout (no reference counterpart) -------------------------
    def forward(self, dt: float, steps: int, checkpointEvery: int = 20) -> np.ndarray:
        """`steps` steps from the current state with the pins held fixed, keeping
        checkpoints every `checkpointEvery` steps; returns the final positions
        (also written into the scene)."""
        self._need()
        self._send_pins()
        self._check(self._lib.cs_forward(self._h, float(dt), int(steps), int(checkpointEvery)))
        self._pull()
        self.lastStats = self._stats()
        return self.scene.positions

    def backward(self, dLdxN) -> tuple:
        """Gradient of a loss on the final positions: returns
        ({C00, C11, G, kBend}: dL/dtheta, dL/dv0 [3n])."""
        self._need()
        g = np.ascontiguousarray(dLdxN, np.float64)
        if g.size != 3 * self.scene.mesh.count:
            raise ValueError("dL/dx_N must hold 3n values")
        th = np.zeros(4)
        dv = np.zeros(g.size)
        self._check(self._lib.cs_backward(self._h, L.ptr(g), L.ptr(th), L.ptr(dv)))
        return dict(C00=th[0], C11=th[1], G=th[2], kBend=th[3]), dv

    def setNewtonMode(self, mode: str = "reference", tol: float = 1e-8) -> None:
        """'reference': the reference's inexact Newton. 'exact': the full
        Hessian (FP64 path; FP32 with Gauss-Newton bending on the mixed path)
        solved to the relative PCG tolerance `tol`, Newton started from
        x0 + h v, lagged friction as a frozen potential in the merit, the Armijo
        base energy re-evaluated at every iterate: with a tight gradTol every
        step converges (except under cloth-cloth friction, whose reference
        force is no potential gradient), to the same solution in far fewer
        Newton iterations. The benchmark and the differentiable rollouts use it."""
        self._check(self._lib.cs_set_newton_mode(self._h, {"reference": 0, "exact": 1}[mode], tol))

    def setAdjointOptions(self, maxIters: int = 2000, tol: float = 1e-10) -> None:
        self._check(self._lib.cs_set_adjoint_options(self._h, maxIters, tol))

    def adjointStats(self) -> dict:
        out = np.zeros(5)
        self._check(self._lib.cs_adjoint_stats(self._h, L.ptr(out)))
        return dict(pcgIters=int(out[0]), solves=int(out[1]), recomputedSteps=int(out[2]), maxRelResidual=out[3],
                    forwardConverged=int(out[4]))

    def launchInfo(self) -> dict:
        out = np.zeros(6, np.int32)
        self._check(self._lib.cs_solver_info(self._h, L.ptr(out), len(out)))
        return dict(pcgClusterCtas=int(out[0]), pcgGridCtas=int(out[1]), fp64PcgCtas=int(out[2]),
                    schwarzDomains=int(out[3]), residentSmem=int(out[4]), residentSmemExact=int(out[5]))

    def profilePhases(self) -> dict:
        out = np.zeros(len(self.PHASES))
        self._check(self._lib.cs_profile_phases(self._h, L.ptr(out), len(out)))
        return dict(zip(self.PHASES, out.tolist()))

    def profileRead(self) -> dict:
        out = np.zeros(5)
        self._check(self._lib.cs_profile_read(self._h, L.ptr(out)))
        return dict(ms=out[0], launches=int(out[1]), bytes=out[2], iters=int(out[3]), ms_per_launch=out[4])

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
