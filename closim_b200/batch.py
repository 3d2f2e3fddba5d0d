"""Batched solver: many independent sheets stepped together (include/closim_batch.h).

    bs = BatchSolver(sheets)           # list of single-sheet workload dicts (closim_b200.configs)
    bs.autotune(0.01)                  # optional: pick the block size on this batch
    bs.step(0.01, steps=10)            # one persistent launch per step, graph-replayed
    bs.positions(i)                    # 3n_i positions of sheet i
    bs.stats()                         # per-sheet Newton / PCG / convergence record

Every sheet is its own scene: its own material, pins and Newton decisions.
Contact parameters, gravity, h and the stepper options are shared (taken
from the first sheet); the floor contact is the only contact.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .solver import preprocess

STAT_KEYS = ["newtonIters", "pcgIters", "gradNorm", "energy", "converged", "armijoTrials", "floorContacts",
             "rejectedLineSearchSteps"]


class BatchSolver:
    def __init__(self, sheets, device: int = 0, options: dict | None = None):
        if not sheets:
            raise ValueError("empty batch")
        self._lib = L.load()
        self._h = self._lib.cs_batch_create(device)
        if not self._h:
            raise RuntimeError(f"cs_batch_create failed for device {device}")
        self.S = len(sheets)
        meshes = (L.cs_mesh * self.S)()
        mats = (L.cs_material * self.S)()
        self._keep = []
        xs, vs, pin_counts, pin_ids, pin_pos = [], [], [], [], []
        self.offsets = [0]
        for i, cfg in enumerate(sheets):
            me = preprocess(cfg["pos"], cfg["uv"], cfg["idx"], cfg["density"])
            arrs = [np.ascontiguousarray(a) for a in (me.indices, me.restPositions, me.invDm, me.areas, me.masses,
                                                      me.hinges.astype(np.int32).reshape(-1),
                                                      me.hingeMeta.astype(np.float64).reshape(-1))]
            self._keep.append(arrs)
            idx, rest, inv, area, mass, hinge, meta = arrs
            meshes[i] = L.cs_mesh(me.count, me.triCount, len(hinge) // 4, L.ptr(idx), L.ptr(rest), L.ptr(inv),
                                  L.ptr(area), L.ptr(mass), L.ptr(hinge), L.ptr(meta))
            m = cfg["material"]
            mats[i] = L.cs_material(m["arealDensityKgM2"], m["thickness"], m["stretchWarp"], m["stretchWeft"],
                                    m["stretchCoupling"], m["shear"], m["bendWarp"], m["bendWeft"], m["damping"])
            xs.append(np.asarray(cfg["x"], np.float64))
            vs.append(np.asarray(cfg["v"], np.float64))
            pins = list(cfg["fixed_pins"])
            pin_counts.append(len(pins))
            for p in pins:
                pin_ids.append(p)
                pin_pos.extend(cfg["x"][p * 3:p * 3 + 3])
            self.offsets.append(self.offsets[-1] + me.count)
        self.N = self.offsets[-1]
        x = np.ascontiguousarray(np.concatenate(xs))
        v = np.ascontiguousarray(np.concatenate(vs))
        pc = np.asarray(pin_counts, np.int32)
        pi = np.asarray(pin_ids if pin_ids else [0], np.int32)
        pp = np.asarray(pin_pos if pin_pos else [0.0, 0.0, 0.0], np.float64)
        g = np.asarray(sheets[0]["gravity"], np.float64)
        self._check(self._lib.cs_batch_initialize(self._h, self.S, meshes, mats, L.ptr(x), L.ptr(v), L.ptr(pc),
                                                  L.ptr(pi), L.ptr(pp), L.ptr(g)))
        c = sheets[0]["contact"]
        if c is not None:
            cp = L.cs_contact_params(c["dHatM"], c["kappaJ"], c["dMinM"], c["frictionMu"], c["frictionEpsM"])
            fl = c.get("floorY")
            self._check(self._lib.cs_batch_set_contact(self._h, C.byref(cp), 0 if fl is None else 1,
                                                       0.0 if fl is None else float(fl)))
        o = dict(sheets[0]["options"])
        if options:
            o.update(options)
        opts = L.cs_stepper_options(int(o["newtonIters"]), int(o["pcgMaxIters"]), int(o["lineSearchIters"]),
                                    L.CS_PRECOND_JACOBI, float(o["gradTol"]))
        self._check(self._lib.cs_batch_set_stepper_options(self._h, C.byref(opts)))
        self._x = np.zeros(3 * self.N)

    def _check(self, rc):
        if rc != L.CS_OK:
            raise RuntimeError(f"batch error {rc}: {self._lib.cs_batch_last_error(self._h).decode()}")

    def step(self, dt: float, steps: int = 1) -> None:
        self._check(self._lib.cs_batch_step(self._h, float(dt), int(steps)))

    def autotune(self, dt: float) -> int:
        t = C.c_int32(0)
        self._check(self._lib.cs_batch_autotune(self._h, float(dt), C.byref(t)))
        return t.value

    def launchShape(self) -> dict:
        t, b = C.c_int32(0), C.c_int32(0)
        self._check(self._lib.cs_batch_launch_shape(self._h, C.byref(t), C.byref(b)))
        return dict(threads=t.value, blocks=b.value)

    def setThreads(self, threads: int) -> None:
        self._check(self._lib.cs_batch_set_threads(self._h, int(threads)))

    def allPositions(self) -> np.ndarray:
        out = np.zeros(3 * self.N)
        self._check(self._lib.cs_batch_get_positions(self._h, L.ptr(out)))
        return out

    def allVelocities(self) -> np.ndarray:
        out = np.zeros(3 * self.N)
        self._check(self._lib.cs_batch_get_velocities(self._h, L.ptr(out)))
        return out

    def positions(self, i: int) -> np.ndarray:
        x = self.allPositions()
        return x[3 * self.offsets[i]:3 * self.offsets[i + 1]]

    def stats(self) -> list:
        out = np.zeros(self.S * 8)
        self._check(self._lib.cs_batch_stats(self._h, L.ptr(out)))
        return [dict(zip(STAT_KEYS, out[i * 8:(i + 1) * 8].tolist())) for i in range(self.S)]

    def stream(self) -> int:
        return self._lib.cs_batch_stream(self._h)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
