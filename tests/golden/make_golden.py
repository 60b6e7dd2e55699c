"""Writes the committed fixtures of tests/golden/ (run from the repository root:
``python -m tests.golden.make_golden``).

- kat.json: hand-derived known answers for the two projections.  Each value
  follows from the definitions (the derivation is in the comments below), not
  from running any code.
- potts_small.npz: a small seeded solve by the FP64 oracle (a regression pin of
  the oracle and a fixture the GPU tests can compare against).  The reference
  has no tests or golden vectors for this path and cannot be built here, so
  these fixtures pin the restatement to itself, not to the reference.
"""
from __future__ import annotations

import json
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent

# Simplex projection: p = max(q - theta, 0) with sum(p) = 1.
#  [2, 0]            theta = 1                          -> [1, 0]
#  [1, 1, 1]         theta = 2/3                        -> [1/3, 1/3, 1/3]
#  [0.3,-0.2,0.1,0]  theta = (0.3+0.1+0-1)/3 = -0.2     -> [0.5, 0, 0.3, 0.2]
#  [0, 0]            theta = -1/2                       -> [1/2, 1/2]
#  [-1]*5 + [5]      theta = 4                          -> [0]*5 + [1]
SIMPLEX = [
    {"q": [0.5, 0.5], "p": [0.5, 0.5]},
    {"q": [2.0, 0.0], "p": [1.0, 0.0]},
    {"q": [1.0, 1.0, 1.0], "p": [1 / 3, 1 / 3, 1 / 3]},
    {"q": [0.3, -0.2, 0.1, 0.0], "p": [0.5, 0.0, 0.3, 0.2]},
    {"q": [0.0, 0.0], "p": [0.5, 0.5]},
    {"q": [-1.0, -1.0, -1.0, -1.0, -1.0, 5.0], "p": [0.0, 0.0, 0.0, 0.0, 0.0, 1.0]},
]

# Dykstra onto {|q_i - q_j| <= 1}.  Two labels, |q2 - q1| = l > 1: sweep 1
# moves each end by (l-1)/2 towards the other (|q2 - q1| becomes 1), sweep 2
# reproduces the same correction, its step is 0, and the loop exits: 2 sweeps.
#  q1 = 0, q2 = (2,0,0):  -> (0.5,0,0), (1.5,0,0)
#  q1 = 0, q2 = (0,3,4):  l = 5, step (0,1.2,1.6) -> (0,1.2,1.6), (0,1.8,2.4)
# A feasible configuration is returned unchanged after 1 sweep.
PROJECT_K = [
    {"q": [[0, 0, 0], [2, 0, 0]], "p": [[0.5, 0, 0], [1.5, 0, 0]], "sweeps": 2},
    {"q": [[0, 0, 0], [0, 3, 4]], "p": [[0, 1.2, 1.6], [0, 1.8, 2.4]], "sweeps": 2},
    {"q": [[0, 0, 0], [0.5, 0, 0], [0, 0.5, 0]], "p": [[0, 0, 0], [0.5, 0, 0], [0, 0.5, 0]], "sweeps": 1},
]


def golden_case():
    """A 20 x 18 x 17 cylinder (r = 7.9), K = 3, blobs + noise; lam = 30, 25 iterations."""
    from oracle import oracle

    n, rows, cols, r, nstride = 20, 18, 17, 7.9, 32
    sr, bs, cb, ce, span = oracle.cylinder_mask(rows, cols, (cols - 1) / 2, (rows - 1) / 2, r, nstride)
    m = SimpleNamespace(n_images=n, rows=rows, cols=cols, nstride=nstride, col_begin=cb, col_end=ce,
                        start_row=sr, base=bs)
    rng = np.random.Generator(np.random.PCG64(2024))
    ci = [0.2, 0.45, 0.8]
    u = np.zeros(span, np.float32)
    lines = span // nstride
    lab = rng.integers(0, 3, size=(lines // 6 + 1, n // 5 + 1))
    for L in range(lines):
        vals = np.asarray(ci, np.float32)[lab[L // 6, np.arange(n) // 5]]
        u[L * nstride:L * nstride + n] = np.clip(vals + rng.normal(0, 0.1, n), 0, 1).astype(np.float32)
    return m, u, ci, {"lam": 30.0, "tau": float(np.float32(0.99) * np.sqrt(np.float32(1) / np.float32(12))),
                      "iters": 25}


def main():
    from oracle import oracle

    (HERE / "kat.json").write_text(json.dumps({"simplex": SIMPLEX, "project_K": PROJECT_K}, indent=1))
    m, u, ci, p = golden_case()
    r = oracle.solve(m, u, ci, p["lam"], p["tau"], p["tau"], p["iters"])
    np.savez_compressed(HERE / "potts_small.npz", u=u, labels=r.labels, V=r.V, Xi=r.Xi, dq_trace=r.dq_trace,
                        res=r.res, ci=np.asarray(ci, np.float32))


if __name__ == "__main__":
    main()
