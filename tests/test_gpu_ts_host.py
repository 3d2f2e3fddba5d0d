"""The TypeScript host's call sequence (host/ts/cuda-solver.ts over
host/napi/addon.cc), replayed through ctypes and checked against the oracle.

No JavaScript runtime exists here, so the test re-issues, call for call, the
cs_* functions the addon makes for each CudaSolver method:
  constructor   cs_create, cs_set_stepper_options
  initialize    cs_initialize, cs_set_pins, cs_set_contact
  step          cs_set_pins (every step: scene.pinned may have changed),
                cs_step, cs_get_positions, cs_get_velocities (into the
                scene's own arrays), cs_last_stats
  setMaterial   copy into scene.material, cs_set_material
  pinVertex     scene.pinned + enforcePins on scene.positions, cs_set_state(x, NULL), cs_set_pins
  unpinVertex   scene.pinned only (sent at the next step)
The scenario mutates the pin map between steps (moving pins, as
src/physics/scene.ts pinColumn scenes and tests/self-contact.test.ts:73-75 do),
pins and unpins a vertex mid-run and changes the material mid-run; after every
step the scene arrays must equal the oracle's state within the FP64 tolerance.
"""
import ctypes as C

import numpy as np
import pytest

from closim_b200 import _lib as L
from closim_b200 import configs
from tests.helpers import oracle_scene, oracle_step_kwargs

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9


class TsCudaSolverReplay:
    """CudaSolver of host/ts/cuda-solver.ts, method for method, over the same C calls."""

    def __init__(self, options, precision="fp64"):
        self.lib = L.load()
        self.h = self.lib.cs_create(L.CS_PRECISION_FP64 if precision == "fp64" else L.CS_PRECISION_MIXED, 0)
        assert self.h
        self.scene = None
        self.lastStats = None
        pc = L.CS_PRECOND_SCHWARZ if options["precond"] == "schwarz" else L.CS_PRECOND_JACOBI
        o = L.cs_stepper_options(options["newtonIters"], options["pcgMaxIters"], options["lineSearchIters"], pc,
                                 options["gradTol"])
        self._ok(self.lib.cs_set_stepper_options(self.h, C.byref(o)))

    def _ok(self, rc):
        assert rc == L.CS_OK, self.lib.cs_last_error(self.h).decode()

    def _send_pins(self):
        pins = self.scene["pinned"]
        ids = np.array(list(pins.keys()), np.int32)
        pos = np.array([pins[k] for k in pins], np.float64).reshape(-1)
        self._ok(self.lib.cs_set_pins(self.h, len(ids), L.ptr(ids) if len(ids) else None,
                                      L.ptr(pos) if len(ids) else None))

    def initialize(self, scene):
        self.scene = scene
        me = scene["mesh"]
        self._keep = [np.ascontiguousarray(a) for a in (me.indices, me.restPositions, me.invDm, me.areas, me.masses,
                                                        me.hinges.astype(np.int32).reshape(-1),
                                                        me.hingeMeta.astype(np.float64).reshape(-1))]
        idx, rest, inv, area, mass, hinge, meta = self._keep
        cm = L.cs_mesh(me.count, me.triCount, len(hinge) // 4, L.ptr(idx), L.ptr(rest), L.ptr(inv), L.ptr(area),
                       L.ptr(mass), L.ptr(hinge), L.ptr(meta))
        mat = scene["material"]._c()
        g = np.array(scene["gravity"], np.float64)
        self._ok(self.lib.cs_initialize(self.h, C.byref(cm), C.byref(mat), L.ptr(g), L.ptr(scene["positions"]),
                                        L.ptr(scene["velocities"])))
        self._send_pins()
        self._ok(self.lib.cs_set_contact(self.h, None, 0, 0.0, None, 0, None, 0))

    def step(self, dt):
        self._send_pins()
        self._ok(self.lib.cs_step(self.h, dt))
        self._ok(self.lib.cs_get_positions(self.h, L.ptr(self.scene["positions"])))
        self._ok(self.lib.cs_get_velocities(self.h, L.ptr(self.scene["velocities"])))
        st = L.cs_step_stats()
        self._ok(self.lib.cs_last_stats(self.h, C.byref(st)))
        self.lastStats = st

    def setMaterial(self, material):
        from dataclasses import replace
        self.scene["material"] = replace(material)
        m = self.scene["material"]._c()
        self._ok(self.lib.cs_set_material(self.h, C.byref(m)))

    def pinVertex(self, vid, position=None):
        x = self.scene["positions"]
        p = tuple(position) if position is not None else tuple(float(q) for q in x[vid * 3:vid * 3 + 3])
        self.scene["pinned"][vid] = p
        for i, q in self.scene["pinned"].items():  # enforcePins
            x[i * 3:i * 3 + 3] = q
        self._ok(self.lib.cs_set_state(self.h, L.ptr(x), None))
        self._send_pins()

    def unpinVertex(self, vid):
        self.scene["pinned"].pop(vid, None)

    def close(self):
        self.lib.cs_destroy(self.h)


def test_ts_host_call_sequence_matches_oracle():
    from closim_b200.solver import ClothMaterial
    cfg = configs.strip_pull(steps=24)
    sc = configs.make_scene(cfg)
    scene = dict(mesh=sc.mesh, material=sc.material, gravity=sc.gravity, pinned=dict(sc.pinned),
                 positions=np.ascontiguousarray(sc.positions, np.float64).copy(),
                 velocities=np.ascontiguousarray(sc.velocities, np.float64).copy())
    pos_array, vel_array = scene["positions"], scene["velocities"]
    solver = TsCudaSolverReplay(cfg["options"])
    solver.initialize(scene)
    osc = oracle_scene(cfg)
    kw = oracle_step_kwargs(cfg)
    extra = {}          # pins added by pinVertex, kept across the moving-pin updates
    free_vertex = 4 * (40 + 1) + 20  # middle of the strip
    for s in range(cfg["steps"]):
        if s == 8:
            solver.pinVertex(free_vertex)
            extra[free_vertex] = scene["pinned"][free_vertex]
            xo = osc.positions.copy()
            xo[free_vertex * 3:free_vertex * 3 + 3] = extra[free_vertex]
            osc.set_state(x=xo)
        if s == 12:
            m = ClothMaterial(**dict(cfg["material"], shear=600.0))
            solver.setMaterial(m)
            assert scene["material"] is not m and scene["material"] == m   # the scene keeps a copy
            mo = dict(arealDensity=m.arealDensityKgM2, thickness=m.thickness, C00=m.stretchWarp, C11=m.stretchWeft,
                      C01=m.stretchCoupling, G=m.shear, bendWarp=m.bendWarp, bendWeft=m.bendWeft, damping=m.damping)
            osc.set_material(mo)
        if s == 16:
            solver.unpinVertex(free_vertex)
            extra.pop(free_vertex)
        # the caller mutates scene.pinned in place between steps
        moving = configs.pins_at(cfg, s)
        scene["pinned"].clear()
        scene["pinned"].update(moving)
        scene["pinned"].update(extra)
        osc.set_pins(dict(scene["pinned"]))
        solver.step(cfg["h"])
        ost = osc.step(cfg["h"], **kw)
        # results land in the scene's own arrays (getPositions returns them)
        assert scene["positions"] is pos_array and scene["velocities"] is vel_array
        xo, vo = osc.positions, osc.velocities
        err = np.max(np.abs(pos_array - xo)) / np.max(np.abs(xo))
        verr = np.max(np.abs(vel_array - vo)) / max(np.max(np.abs(vo)), 1e-30)
        assert err <= REL_TOL and verr <= REL_TOL, (s, err, verr)
        assert solver.lastStats.pcg_iters == ost["pcgIters"], s
        if free_vertex in extra:
            assert np.array_equal(pos_array[free_vertex * 3:free_vertex * 3 + 3], np.array(extra[free_vertex]))
    solver.close()
