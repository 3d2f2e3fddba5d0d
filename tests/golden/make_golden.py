"""Regenerate tests/golden/*.json from the reference checkout.

Reads the reference's published PCG iteration table
(G5_PRECONDITIONER_REPORT.md:65-76, produced by
tests/preconditioner-compare.test.ts) and writes g5_pcg_iters.json.
Run from the repo root: python tests/golden/make_golden.py <reference_dir>
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py <reference checkout>")
ref = sys.argv[1]
text = open(os.path.join(ref, "G5_PRECONDITIONER_REPORT.md")).read().splitlines()
rows = {}
start = None
for i, line in enumerate(text):
    if line.startswith("| cell | jacobi | block | schwarz1"):
        start = i
        break
assert start is not None, "table not found"
for line in text[start + 2:]:
    if not line.startswith("|"):
        break
    cells = [c.strip() for c in line.strip("|").split("|")]
    name = cells[0]
    vals = {}
    for key, c in zip(["jacobi", "block", "schwarz1", "mas2", "masX"], cells[1:]):
        m = re.match(r"(\d+)(✗)?\s*(\(([\d.e-]+)\))?", c)
        vals[key] = {"iters": int(m.group(1)), "capped": bool(m.group(2)),
                     "residual": float(m.group(4)) if m.group(4) else None}
    rows[name] = vals
out = {"source": "G5_PRECONDITIONER_REPORT.md:65-76 (tests/preconditioner-compare.test.ts)",
       "grid": [6, 6, 0.12, 0.12], "invH2": 3600, "tol": 1e-6, "maxIters": 200,
       "schwarz_domains": [16, 8, 32], "cells": rows}
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "g5_pcg_iters.json")
json.dump(out, open(path, "w"), indent=1)
print("wrote", path, len(rows), "cells")
