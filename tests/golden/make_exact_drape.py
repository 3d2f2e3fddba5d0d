"""Regenerate tests/golden/exact_drape_64.npz: the oracle's exact-Newton mode
on the 64x64 floor drape (closim_b200.configs.floor_drape: 4,096 vertices,
floor contact, mu 0.3, h = 1/120), 120 steps from rest at 0.3 m, at the
converging budget of the benchmark (40 Newton iterations, 3000 PCG
iterations, gradTol 1e-8, PCG tolerance 3e-4, the drift start).

Stored: positions after steps 30 (landing) and 120 as float64, and per step
the converged flag, Newton and PCG iteration counts. The oracle runs about
five minutes on one core. Run from the repo root:
python tests/golden/make_exact_drape.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from closim_b200 import configs  # noqa: E402
from tests.helpers import oracle_scene, oracle_step_kwargs  # noqa: E402

STEPS = 120
KEEP = (29, 119)
PCG_TOL = 3e-4
BUDGET = dict(newtonIters=40, pcgMaxIters=3000, gradTol=1e-8)


def main():
    cfg = configs.floor_drape()
    cfg["options"] = dict(cfg["options"], **BUDGET)
    osc = oracle_scene(cfg)
    kw = oracle_step_kwargs(cfg)
    out = {}
    conv, newton, pcg = [], [], []
    t0 = time.time()
    for s in range(STEPS):
        st = osc.step(cfg["h"], exact=True, pcg_tol=PCG_TOL, drift=True, **kw)
        conv.append(int(st["converged"]))
        newton.append(int(st["newtonItersUsed"]))
        pcg.append(int(st["pcgIters"]))
        if s in KEEP:
            out[f"x{s}"] = osc.positions
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "exact_drape_64.npz")
    np.savez_compressed(path, keep=np.array(KEEP), converged=np.array(conv, np.int8),
                        newton=np.array(newton, np.int16), pcg=np.array(pcg, np.int32),
                        pcg_tol=PCG_TOL, grad_tol=BUDGET["gradTol"], **out)
    print(f"wrote {path}: {sum(conv)}/{STEPS} converged, {sum(newton)} Newton, {sum(pcg)} PCG iterations, "
          f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
