"""Regenerate tests/golden/adjoint_fd_12.npz: central finite differences of
the material-fit loss through the oracle's exact-Newton rollout.

Workload: closim_b200.configs.material_fit scaled down (12 x 12 vertices,
0.2 m, hung from two corners, 12 steps of 0.01 s), every step converged to
gradTol 1e-10 with PCG tolerance 1e-10. Loss = mean over vertices of
|x_N - x_N*|^2, x_N* the rollout at the ground-truth parameters.

Stored: x_N* and x_N at the start parameters theta0, the loss, dL/d(C00, C11,
G, k_bend) and the directional derivative along a seeded initial-velocity
direction u (numpy default_rng(7), standard normal times 1e-3, pinned dofs
zeroed), each by central differences with Richardson extrapolation over
relative steps 1e-2 and 5e-3 (1.0 and 0.5 along u). Runs in about 80 s.
Run from the repo root: python tests/golden/make_adjoint_fd.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from closim_b200 import configs  # noqa: E402
from tests.helpers import oracle_scene, oracle_step_kwargs  # noqa: E402

PCG_TOL = 1e-10


def small_fit():
    return configs.material_fit(nx=11, ny=11, w=0.2, hgt=0.2, steps=12, checkpoint_every=5, newton_iters=30,
                                pcg_max_iters=3000, grad_tol=1e-10)


def rollout(cfg, theta, v0=None):
    c = configs.with_theta(cfg, theta)
    if v0 is not None:
        c = dict(c, v=v0)
    osc = oracle_scene(c)
    kw = oracle_step_kwargs(c)
    conv = 0
    for k in range(c["steps"]):
        osc.set_pins(configs.pins_at(c, k))
        st = osc.step(c["h"], exact=True, pcg_tol=PCG_TOL, drift=True, **kw)
        conv += st["converged"] > 0
    assert conv == c["steps"], f"{conv} of {c['steps']} steps converged"
    return osc.positions


def direction(cfg):
    n = len(cfg["x"]) // 3
    u = np.random.default_rng(7).standard_normal(3 * n) * 1e-3
    for pid in cfg["fixed_pins"]:
        u[pid * 3:pid * 3 + 3] = 0
    return u


def richardson(f, h):
    def central(s):
        return (f(s) - f(-s)) / (2 * s)
    return (4 * central(h / 2) - central(h)) / 3


def main():
    cfg = small_fit()
    n = len(cfg["x"]) // 3
    xs = rollout(cfg, cfg["theta_gt"])
    th0 = cfg["theta0"].copy()
    x0 = rollout(cfg, th0)

    def loss(x):
        return float(np.sum((x - xs) ** 2) / n)

    fd = []
    for j in range(4):
        def f(dh, j=j):
            t = th0.copy()
            t[j] *= 1 + dh
            return loss(rollout(cfg, t))
        fd.append(richardson(f, 1e-2) / th0[j])
    u = direction(cfg)
    fd_u = richardson(lambda e: loss(rollout(cfg, th0, cfg["v"] + e * u)), 1.0)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "adjoint_fd_12.npz")
    np.savez_compressed(path, xs=xs, x0=x0, theta0=th0, loss=loss(x0), dL_dtheta=np.array(fd), dL_dv0_u=fd_u,
                        pcg_tol=PCG_TOL)
    print(f"wrote {path}: L0 {loss(x0):.6e}, dL/dtheta {np.array(fd)}, dL/dv0.u {fd_u:.8e}")


if __name__ == "__main__":
    main()
