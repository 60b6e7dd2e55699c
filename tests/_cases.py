"""Shared test inputs: cylinder volumes with seeded phantom or random intensities."""
from __future__ import annotations

import numpy as np

from segmentctscans_b200.layout import CylinderMapping
from segmentctscans_b200.potts import reference_tau

TAU = reference_tau()
TAU_BASELINE = float(np.float32(1.0) / np.sqrt(np.float32(12.0)))


def random_volume(n, rows, cols, r, K, seed=0, nstride=None, xc=None, yc=None):
    """Piecewise-constant blobs + noise so that all Dykstra/simplex branches occur."""
    rng = np.random.default_rng(seed)
    m = CylinderMapping.cylinder(n, rows, cols, r, xc=xc, yc=yc, nstride=nstride)
    ci = np.sort(rng.uniform(0.05, 0.95, K)).astype(np.float32)
    box = np.zeros((cols, rows, n), np.float32)
    lab = rng.integers(0, K, size=(max(cols // 4, 1) + 1, max(rows // 4, 1) + 1, max(n // 4, 1) + 1))
    cc, rr, nn = np.meshgrid(np.arange(cols) // 4, np.arange(rows) // 4, np.arange(n) // 4, indexing="ij")
    box[:] = ci[lab[cc, rr, nn]]
    box += rng.normal(0, 0.08, box.shape).astype(np.float32)
    box = np.clip(box, 0, 1)
    u = m.gather(box).astype(np.float32)
    return m, u, [float(c) for c in ci]


def phantom_volume(size=32, r=14.0, seed=0, k=3, radius_range=(2.0, 6.0)):
    from segmentctscans_b200.phantom import make_phantom

    ph = make_phantom(size, size, size, r, seed=seed, radius_range=radius_range, k=k, device="cpu")
    return ph.mapping, ph.u.numpy().copy(), ph.ci, ph
