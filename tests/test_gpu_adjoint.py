"""Adjoint of the rollout (cs_forward / cs_backward) against central finite
differences of the FP64 forward, through the C ABI.

Workload: the material-fit sheet scaled down (12 x 12 vertices, 0.2 m, hung
from two corners of one edge, 12 steps of 0.01 s, checkpoints every 5 steps so
the reverse sweep recomputes three segments). The forward runs with the
full-Hessian Newton solve (cs_set_newton_mode exact) to gradTol 1e-10 (its
FP64 floor is about 3e-11), so every step is converged and the
implicit-function theorem applies; the reference's own Newton budget leaves
these steps unconverged (gradient norms 7e-3..8e-2 measured), which makes any
finite difference of it noise. The finite differences are central with
Richardson extrapolation over relative steps of 1e-2 and 5e-3: a step of 1e-6
would move the positions by less than the converged solve's residual.

Target: relative agreement <= 1e-4 for dL/d(C00, C11, G, k_bend) and for a
directional derivative along a seeded random initial-velocity direction.

The same gradient is also checked against central differences through the
oracle's exact-Newton rollout, an implementation independent of the CUDA
forward (tests/golden/make_adjoint_fd.py writes them as a fixture).
"""
import os

import numpy as np
import pytest

import closim_b200 as cb
from closim_b200 import configs

pytestmark = pytest.mark.gpu

TOL = 1e-4


def small_fit():
    return configs.material_fit(nx=11, ny=11, w=0.2, hgt=0.2, steps=12, checkpoint_every=5, newton_iters=30,
                                pcg_max_iters=3000, grad_tol=1e-10)


def make_solver(cfg, theta):
    c = configs.with_theta(cfg, theta)
    sc = configs.make_scene(c)
    s = cb.CudaSolver("fp64", **c["options"])
    s.initialize(sc)
    s.setNewtonMode("exact", 1e-10)
    s.setAdjointOptions(4000, 1e-12)
    return s, sc


def rollout(cfg, theta, v0=None):
    s, sc = make_solver(cfg, theta)
    if v0 is not None:
        sc.velocities[:] = v0
        s.push_state()
    xN = s.forward(cfg["h"], cfg["steps"], cfg["checkpoint_every"]).copy()
    return xN, s


def test_adjoint_matches_central_differences():
    cfg = small_fit()
    xs, s_gt = rollout(cfg, cfg["theta_gt"])
    assert s_gt.adjointStats()["forwardConverged"] == cfg["steps"]
    th0 = cfg["theta0"].copy()
    x0, s = rollout(cfg, th0)
    st = s.adjointStats()
    assert st["forwardConverged"] == cfg["steps"], st
    n = len(x0) // 3

    def loss(x):
        return float(np.sum((x - xs) ** 2) / n)

    L0 = loss(x0)
    dth, dv0 = s.backward(2 * (x0 - xs) / n)
    ast = s.adjointStats()
    print(f"adjoint: L0 {L0:.6e}, {ast}")
    assert ast["solves"] == cfg["steps"] and ast["maxRelResidual"] < 1e-9
    # the state after the rollout is restored
    s.pull()
    assert np.array_equal(s.getPositions(), x0)
    adj = [dth["C00"], dth["C11"], dth["G"], dth["kBend"]]

    def central(f, h):
        return (f(h) - f(-h)) / (2 * h)

    def richardson(f, h):
        return (4 * central(f, h / 2) - central(f, h)) / 3

    for j, name in enumerate(["C00", "C11", "G", "kBend"]):
        def f(dh, j=j):
            t = th0.copy()
            t[j] *= 1 + dh
            return loss(rollout(cfg, t)[0])
        fd = richardson(f, 1e-2) / th0[j]
        rel = abs(adj[j] - fd) / max(abs(fd), 1e-300)
        print(f"dL/d{name}: adjoint {adj[j]:.8e}  FD {fd:.8e}  rel {rel:.2e}")
        assert rel <= TOL, (name, adj[j], fd)
    u = np.random.default_rng(7).standard_normal(3 * n) * 1e-3
    for pid in cfg["fixed_pins"]:
        u[pid * 3:pid * 3 + 3] = 0
    v0 = cfg["v"]
    fd = richardson(lambda e: loss(rollout(cfg, th0, v0 + e * u)[0]), 1.0)
    ad = float(dv0 @ u)
    rel = abs(ad - fd) / max(abs(fd), 1e-300)
    print(f"dL/dv0 . u: adjoint {ad:.8e}  FD {fd:.8e}  rel {rel:.2e}")
    assert rel <= TOL


GOLD_FD = os.path.join(os.path.dirname(__file__), "golden", "adjoint_fd_12.npz")


def test_adjoint_matches_central_differences_of_the_oracle():
    g = np.load(GOLD_FD)
    cfg = small_fit()
    assert np.array_equal(cfg["theta0"], g["theta0"])
    xs, _ = rollout(cfg, cfg["theta_gt"])
    x0, s = rollout(cfg, cfg["theta0"])
    n = len(x0) // 3
    # the forward rollouts themselves match the oracle's
    fwd = max(float(np.max(np.abs(xs - g["xs"])) / np.max(np.abs(g["xs"]))),
              float(np.max(np.abs(x0 - g["x0"])) / np.max(np.abs(g["x0"]))))
    dth, dv0 = s.backward(2 * (x0 - xs) / n)
    adj = np.array([dth["C00"], dth["C11"], dth["G"], dth["kBend"]])
    rel = np.abs(adj - g["dL_dtheta"]) / np.abs(g["dL_dtheta"])
    u = np.random.default_rng(7).standard_normal(3 * n) * 1e-3
    for pid in cfg["fixed_pins"]:
        u[pid * 3:pid * 3 + 3] = 0
    rel_u = abs(float(dv0 @ u) - float(g["dL_dv0_u"])) / abs(float(g["dL_dv0_u"]))
    print(f"adjoint vs oracle FD: forward {fwd:.2e}; dL/dtheta rel {rel}; dL/dv0.u rel {rel_u:.2e}")
    assert fwd <= 1e-9, fwd
    assert float(np.max(rel)) <= TOL and rel_u <= TOL, (rel, rel_u)


def test_autograd_function_semantics():
    """ClothRollout behaves as a torch.autograd.Function: loss.backward()
    fills theta.grad and v0.grad with the adjoint's values."""
    torch = pytest.importorskip("torch")
    from closim_b200.adjoint import ClothRollout
    cfg = small_fit()
    xs, _ = rollout(cfg, cfg["theta_gt"])
    s, sc = make_solver(cfg, cfg["theta0"])
    theta = torch.tensor(cfg["theta0"], dtype=torch.float64, requires_grad=True)
    v0 = torch.zeros(len(cfg["x"]), dtype=torch.float64, requires_grad=True)
    xN = ClothRollout.apply(theta, v0, s, cfg["x"], cfg["h"], cfg["steps"], cfg["checkpoint_every"])
    loss = ((xN - torch.from_numpy(xs)) ** 2).sum() / (len(xs) // 3)
    loss.backward()
    x_ref, s2 = rollout(cfg, cfg["theta0"])
    dth, dv0 = s2.backward(2 * (x_ref - xs) / (len(xs) // 3))
    assert np.allclose(theta.grad.numpy(), [dth["C00"], dth["C11"], dth["G"], dth["kBend"]], rtol=1e-9, atol=0)
    assert np.allclose(v0.grad.numpy(), dv0, rtol=1e-9, atol=1e-30)
