"""SimulationSession (src/view/sim-session.ts): fixed-dt stepping, publish,
NaN-free tracking and restoreStable, over the device hand-off
(cs_session_step): the NaN scan and the stable snapshot run on the device and
the positions arrive in the scene's arrays with one synchronization per step.

Differences from the reference: attach() takes a ClothScene and dt instead of
a FittingScene and SimulationConfig (garment assembly is not part of this
package); everything else keeps the reference's names and behaviour.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

MAX_STEPS_PER_TICK = 8


class SimulationSession:
    def __init__(self, solver, publish):
        self.solver = solver
        self.publish = publish
        self.scene = None
        self.dt = None
        self._playing = False
        self._steps = 0
        self._acc = 0.0
        self._stats = None
        self._nanFree = True
        self._stableStep = -1

    @property
    def status(self):
        if self.scene is None:
            return "detached"
        return "playing" if self._playing else "ready"

    isPlaying = property(lambda self: self._playing)
    stepCount = property(lambda self: self._steps)
    lastStats = property(lambda self: self._stats)
    lastStepNaNFree = property(lambda self: self._nanFree)
    stableStep = property(lambda self: self._stableStep)

    def attach(self, scene, dt: float) -> None:
        self.scene = scene
        self.dt = float(dt)
        self.solver.initialize(scene)
        self._playing = False
        self._steps = 0
        self._acc = 0.0
        self._stats = None
        self._nanFree = True
        self._check(self.solver._lib.cs_session_reset(self.solver._h))
        self._stableStep = 0
        self.publish(scene.positions)

    def detach(self) -> None:
        self.scene = None
        self._playing = False
        self._steps = 0
        self._stats = None
        self._stableStep = -1

    def play(self):
        if self.scene is not None:
            self._playing = True

    def pause(self):
        self._playing = False

    def toggle(self):
        if self._playing:
            self.pause()
        else:
            self.play()
        return self._playing

    def stepOnce(self, count: int = 1) -> None:
        for _ in range(count):
            if not self._doStep():
                return

    def tick(self, realDtSeconds: float) -> None:
        if not self._playing or self.scene is None:
            return
        self._acc += max(0.0, min(realDtSeconds, 0.25))
        steps = 0
        while self._acc >= self.dt and steps < MAX_STEPS_PER_TICK:
            if not self._doStep():
                self._acc = 0.0
                return
            self._acc -= self.dt
            steps += 1
        if steps >= MAX_STEPS_PER_TICK:
            self._acc = 0.0

    def _check(self, rc):
        if rc == L.CS_E_NONFINITE:
            raise FloatingPointError(self.solver._lib.cs_last_error(self.solver._h).decode())
        if rc != L.CS_OK:
            raise RuntimeError(self.solver._lib.cs_last_error(self.solver._h).decode())

    def _doStep(self) -> bool:
        if self.scene is None:
            return False
        s = self.solver
        s._send_pins()
        ok = C.c_int32(0)
        self._check(s._lib.cs_session_step(s._h, self.dt, L.ptr(self.scene.positions), C.byref(ok)))
        s._check(s._lib.cs_get_velocities(s._h, L.ptr(self.scene.velocities)))
        s.lastStats = s._stats()
        self._steps += 1
        self._stats = s.lastStats
        self._nanFree = bool(ok.value)
        if self._nanFree:
            self._stableStep = self._steps
        self.publish(self.scene.positions)
        return self._nanFree

    def hasStableState(self) -> bool:
        return self._stableStep >= 0

    def restoreStable(self) -> bool:
        if self.scene is None or self._stableStep < 0:
            return False
        s = self.solver
        step = C.c_int32(-1)
        self._check(s._lib.cs_session_restore_stable(s._h, C.byref(step)))
        s._pull()
        self._acc = 0.0
        self._playing = False
        self._stats = None
        self._nanFree = True
        self.publish(self.scene.positions)
        return True
