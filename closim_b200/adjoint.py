"""Differentiable cloth rollout with torch.autograd.Function semantics.

    x_N = ClothRollout.apply(theta, v0, solver, x0, dt, steps, checkpointEvery)

theta = (C00, C11, G, k_bend) as a float64 tensor, v0 the initial velocities
(3n, float64). forward() sets the material and the initial state, runs the
rollout on the device (cs_forward) and returns the final positions;
backward() runs the implicit-function-theorem adjoint (cs_backward) and
returns dL/dtheta and dL/dv0. x0, dt, steps and the solver are not
differentiated. k_bend sets bendWarp = bendWeft.

The gradient is that of the converged step map: the solver's stepper options
must let every step converge (gradTol reached).
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import torch


class ClothRollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, v0, solver, x0, dt, steps, checkpointEvery=20):
        th = theta.detach().cpu().double().numpy()
        mat = replace(solver.scene.material, stretchWarp=float(th[0]), stretchWeft=float(th[1]), shear=float(th[2]),
                      bendWarp=float(th[3]), bendWeft=float(th[3]))
        solver.setMaterial(mat)
        sc = solver.scene
        sc.positions[:] = np.asarray(x0, np.float64)
        sc.velocities[:] = v0.detach().cpu().double().numpy()
        solver.push_state()
        xN = solver.forward(dt, int(steps), int(checkpointEvery)).copy()
        ctx.solver = solver
        return torch.from_numpy(xN)

    @staticmethod
    def backward(ctx, gxN):
        dtheta, dv0 = ctx.solver.backward(gxN.detach().cpu().double().numpy())
        gt = torch.tensor([dtheta["C00"], dtheta["C11"], dtheta["G"], dtheta["kBend"]], dtype=torch.float64)
        return gt, torch.from_numpy(dv0), None, None, None, None, None
