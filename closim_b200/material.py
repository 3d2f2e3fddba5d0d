"""Material model layer (src/physics/material-model.ts) over the CUDA solver.

Mirrors (mohdabraralikhan/closim):
  PhysicalMaterialParams, MaterialCalibration   material-model.ts:26-115
  validatePhysicalParams / validateCalibration  material-model.ts:134-185
  ClothMaterialModel / OrthotropicStVKMaterial  material-model.ts:191-329
  describeParameters, FRICTION_OWNERSHIP_NOTE   material-model.ts:60-78

OrthotropicStVKMaterial is a validated, immutable snapshot of the orthotropic
StVK parameters with a legacy bridge (fromLegacy / toLegacy) and JSON
round-trips. Its energy / gradient / hessianVector run on the GPU through the
same kernels the solver's FP64 path uses (cs_internal_energy,
cs_internal_gradient, cs_membrane_hvp_analytic), so the model's numerics are
the legacy path's by construction, as the reference's delegation is.
"""
from __future__ import annotations

import copy
import ctypes as C
import json
import math
from collections.abc import Mapping
from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np

from . import _lib as L
from .solver import ClothMaterial, ClothMeshData, CudaSolver, createScene

FRICTION_OWNERSHIP_NOTE = ("Coulomb friction mu is owned by the contact system (ContactParams, dimensionless), "
                           "not the material model.")


def describeParameters():
    """Machine-readable SI unit table (material-model.ts:60-72)."""
    return [
        {"path": "inertia.arealDensityKgM2", "unit": "kg/m^2"},
        {"path": "thicknessM", "unit": "m"},
        {"path": "membrane.warpPa", "unit": "Pa"},
        {"path": "membrane.weftPa", "unit": "Pa"},
        {"path": "membrane.couplingPa", "unit": "Pa"},
        {"path": "membrane.shearPa", "unit": "Pa"},
        {"path": "bending.warpNm", "unit": "N*m"},
        {"path": "bending.weftNm", "unit": "N*m"},
        {"path": "dampingRatio", "unit": "dimensionless"},
    ]


class MaterialValidationError(ValueError):
    """MaterialValidationError (material-model.ts:119-126): carries a code."""

    def __init__(self, code: str, message: str):
        super().__init__(f"invalid material ({code}): {message}")
        self.code = code


def _num(v, path: str) -> float:
    if isinstance(v, bool) or not isinstance(v, (int, float)) or not math.isfinite(v):
        raise MaterialValidationError("non-finite", f"{path} must be a finite number, got {v!r}")
    return float(v)


def _get(obj, key):
    if isinstance(obj, Mapping):
        return obj.get(key)
    return None


def validatePhysicalParams(p) -> None:
    """Structural validation (material-model.ts:134-162): SI ranges and the
    positive-semidefinite coupling C00 * C11 - C01^2 >= 0."""
    if not isinstance(p, Mapping):
        raise MaterialValidationError("shape", "params must be an object")
    rho = _num(_get(p.get("inertia") or {}, "arealDensityKgM2"), "inertia.arealDensityKgM2")
    if rho <= 0:
        raise MaterialValidationError("non-positive-density", f"arealDensityKgM2 must be > 0, got {rho}")
    h = _num(p.get("thicknessM"), "thicknessM")
    if h <= 0:
        raise MaterialValidationError("non-positive-thickness", f"thicknessM must be > 0, got {h}")
    mem = p.get("membrane")
    c00 = _num(_get(mem, "warpPa"), "membrane.warpPa")
    c11 = _num(_get(mem, "weftPa"), "membrane.weftPa")
    c01 = _num(_get(mem, "couplingPa"), "membrane.couplingPa")
    g = _num(_get(mem, "shearPa"), "membrane.shearPa")
    if c00 < 0 or c11 < 0 or g < 0:
        raise MaterialValidationError("negative-stiffness", "membrane moduli must be >= 0")
    if c00 * c11 - c01 * c01 < 0:
        raise MaterialValidationError("indefinite-coupling",
                                      f"|couplingPa| must satisfy C00*C11 - C01^2 >= 0, got {c00}*{c11} - {c01}^2 < 0")
    bend = p.get("bending")
    bw = _num(_get(bend, "warpNm"), "bending.warpNm")
    be = _num(_get(bend, "weftNm"), "bending.weftNm")
    if bw < 0 or be < 0:
        raise MaterialValidationError("negative-stiffness", "bending moduli must be >= 0")
    d = _num(p.get("dampingRatio"), "dampingRatio")
    if d < 0 or d > 1:
        raise MaterialValidationError("damping-range", f"dampingRatio must be in [0,1], got {d}")


def validateCalibration(cal) -> None:
    """Metadata only (material-model.ts:165-178): an elastic dataset is
    required and dissipative models other than "none" are rejected."""
    if cal is None:
        return
    if not isinstance(cal, Mapping):
        raise MaterialValidationError("shape", "calibration must be an object")
    el = cal.get("elastic")
    if not isinstance(el, Mapping) or not isinstance(el.get("dataset"), str) or not el["dataset"]:
        raise MaterialValidationError("calibration", "elastic.dataset (string) is required")
    for kind in ("hysteresis", "plasticity"):
        meta = cal.get(kind)
        if meta is not None and (not isinstance(meta, Mapping) or meta.get("model") != "none"):
            model = meta.get("model") if isinstance(meta, Mapping) else meta
            raise MaterialValidationError("not-implemented",
                                          f'{kind} model "{model}" is not implemented (metadata only)')


def _freeze(v):
    """Deep, immutable copy: dicts become read-only mappings."""
    from types import MappingProxyType
    if isinstance(v, dict):
        return MappingProxyType({k: _freeze(x) for k, x in v.items()})
    if isinstance(v, list):
        return tuple(_freeze(x) for x in v)
    return v


def _thaw(v):
    if isinstance(v, Mapping):
        return {k: _thaw(x) for k, x in v.items()}
    if isinstance(v, tuple):
        return [_thaw(x) for x in v]
    return v


@dataclass
class MaterialModelEval:
    """MaterialModelEval (material-model.ts:191-195)."""
    energy: float
    grad: np.ndarray
    maxStrain: float


class _Evaluator:
    """A CudaSolver handle holding one mesh on the GPU, reused across calls."""

    def __init__(self, mesh: ClothMeshData, device: int):
        self.mesh = mesh
        self.solver = CudaSolver("fp64", device=device)
        self.solver.initialize(createScene(mesh, ClothMaterial()))
        self.material = None

    def bind(self, legacy: ClothMaterial):
        if self.material != legacy:
            self.solver.setMaterial(legacy)
            self.material = legacy

    def x(self, x) -> np.ndarray:
        a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
        if a.size != 3 * self.mesh.count:
            raise ValueError("x must hold 3n values")
        return a


_EVALUATORS: Dict[int, _Evaluator] = {}


def _evaluator(mesh: ClothMeshData, device: int = 0) -> _Evaluator:
    key = id(mesh)
    ev = _EVALUATORS.get(key)
    if ev is None or ev.mesh is not mesh:
        ev = _Evaluator(mesh, device)
        _EVALUATORS[key] = ev
    return ev


class OrthotropicStVKMaterial:
    """OrthotropicStVKMaterial (material-model.ts:218-329)."""

    KIND = "orthotropic-stvk"
    VERSION = 1

    def __init__(self, params: dict, calibration: Optional[dict] = None):
        validatePhysicalParams(params)
        validateCalibration(calibration)
        self._params = _freeze(copy.deepcopy(_thaw(params)))
        self._calibration = None if calibration is None else _freeze(copy.deepcopy(_thaw(calibration)))
        p = self._params
        self._legacy = ClothMaterial(
            arealDensityKgM2=float(p["inertia"]["arealDensityKgM2"]), thickness=float(p["thicknessM"]),
            stretchWarp=float(p["membrane"]["warpPa"]), stretchWeft=float(p["membrane"]["weftPa"]),
            stretchCoupling=float(p["membrane"]["couplingPa"]), shear=float(p["membrane"]["shearPa"]),
            bendWarp=float(p["bending"]["warpNm"]), bendWeft=float(p["bending"]["weftNm"]),
            damping=float(p["dampingRatio"]))

    kind = property(lambda self: self.KIND)
    params = property(lambda self: self._params)
    calibration = property(lambda self: self._calibration)

    @staticmethod
    def fromLegacy(mat: ClothMaterial, calibration: Optional[dict] = None) -> "OrthotropicStVKMaterial":
        """Bridge from the legacy struct; unphysical legacy values raise."""
        return OrthotropicStVKMaterial({
            "inertia": {"arealDensityKgM2": mat.arealDensityKgM2},
            "thicknessM": mat.thickness,
            "membrane": {"warpPa": mat.stretchWarp, "weftPa": mat.stretchWeft,
                         "couplingPa": mat.stretchCoupling, "shearPa": mat.shear},
            "bending": {"warpNm": mat.bendWarp, "weftNm": mat.bendWeft},
            "dampingRatio": mat.damping,
        }, calibration)

    def toLegacy(self) -> ClothMaterial:
        l = self._legacy
        return ClothMaterial(l.arealDensityKgM2, l.thickness, l.stretchWarp, l.stretchWeft, l.stretchCoupling,
                             l.shear, l.bendWarp, l.bendWeft, l.damping)

    # -- numerics on the GPU (the legacy kernels, so bitwise the legacy path) --
    def energy(self, x, mesh: ClothMeshData) -> float:
        """Total internal energy (membrane + bending), J: internalEnergyOnly."""
        ev = _evaluator(mesh)
        ev.bind(self._legacy)
        xa = ev.x(x)
        e = C.c_double(0.0)
        ev.solver._check(ev.solver._lib.cs_internal_energy(ev.solver._h, L.ptr(xa), C.byref(e)))
        return e.value

    def gradient(self, x, mesh: ClothMeshData, out: Optional[np.ndarray] = None) -> MaterialModelEval:
        """Internal energy, gradient and max strain: evalInternal."""
        ev = _evaluator(mesh)
        ev.bind(self._legacy)
        xa = ev.x(x)
        g = out if out is not None else np.zeros(3 * mesh.count)
        if g.dtype != np.float64 or not g.flags.c_contiguous or g.size != 3 * mesh.count:
            raise ValueError("out must be a contiguous float64 array of 3n values")
        e, ms = C.c_double(0.0), C.c_double(0.0)
        ev.solver._check(ev.solver._lib.cs_internal_gradient(ev.solver._h, L.ptr(xa), C.byref(e), L.ptr(g),
                                                             C.byref(ms)))
        return MaterialModelEval(e.value, g, ms.value)

    def hessianVector(self, x, p, mesh: ClothMeshData, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Membrane-only analytic HVP (bending kept in the gradient only, as
        the reference's inexact Newton does): evalMembraneHvp."""
        ev = _evaluator(mesh)
        ev.bind(self._legacy)
        xa = ev.x(x)
        pa = ev.x(p)
        o = out if out is not None else np.zeros(3 * mesh.count)
        if o.dtype != np.float64 or not o.flags.c_contiguous or o.size != 3 * mesh.count:
            raise ValueError("out must be a contiguous float64 array of 3n values")
        ev.solver._check(ev.solver._lib.cs_membrane_hvp_analytic(ev.solver._h, L.ptr(xa), L.ptr(pa), L.ptr(o)))
        return o

    def clone(self) -> "OrthotropicStVKMaterial":
        return OrthotropicStVKMaterial(_thaw(self._params), None if self._calibration is None else
                                       _thaw(self._calibration))

    def toJSON(self) -> dict:
        out = {"kind": self.KIND, "version": self.VERSION, "params": _thaw(self._params)}
        if self._calibration is not None:
            out["calibration"] = _thaw(self._calibration)
        return out

    @staticmethod
    def fromJSON(j) -> "OrthotropicStVKMaterial":
        o = json.loads(j) if isinstance(j, str) else j
        if not isinstance(o, dict):
            raise MaterialValidationError("shape", "model JSON must be an object")
        if o.get("kind") != OrthotropicStVKMaterial.KIND:
            raise MaterialValidationError("unknown-kind",
                                          f'expected kind "{OrthotropicStVKMaterial.KIND}", got {o.get("kind")}')
        if o.get("version") != OrthotropicStVKMaterial.VERSION:
            raise MaterialValidationError("version",
                                          f"expected version {OrthotropicStVKMaterial.VERSION}, got {o.get('version')}")
        return OrthotropicStVKMaterial(o.get("params"), o.get("calibration"))
