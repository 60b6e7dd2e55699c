"""Seeded synthetic micro-CT phantoms in the cylinder layout.

The reference is run on the DRP-395 scans, which are not available here; these
phantoms stand in for them with the same structure: a glass matrix inside a
cylindrical core with random non-overlapping spherical pores (random
sequential addition) filled with brine or scCO2 (optionally a fourth phase),
partial-volume blur (Gaussian, sigma = 1 voxel), additive Gaussian noise, and
the intensity normalisation of the reference's ingest step
(transpose/transpose.cpp:253-285, transpose/convert_to_fp.cpp:35-43):
u = clamp((x - lo) / (hi - lo), 0, 1) with lo/hi the in-mask minimum/maximum,
and each label c_i mapped the same way (potts-model/potts-model.cpp:145-148).

Axis convention as in the reference: n (contiguous) runs along the cylinder
axis; the circular mask lies in the (row, col) plane.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from .layout import CylinderMapping

GLASS = 5.27e-2
BRINE = 4.09e-2
SCCO2 = 3.39e-2
PHASE4 = 4.6e-2


@dataclass
class Phantom:
    mapping: CylinderMapping
    u: "object"                # torch float32 tensor [span], normalised to [0, 1]
    truth: "object"            # torch uint8 tensor [span], index of the true phase in `labels`
    labels: list[float]        # raw phase intensities, ascending
    ci: list[float]            # labels in the units of u
    lo: float
    hi: float
    spheres: np.ndarray        # [m, 5]: n, row, col, radius, phase


def _rsa(rng: np.random.Generator, n: int, rows: int, cols: int, r_cyl: float, rmin: float, rmax: float,
         porosity: float, max_tries: int = 200000) -> np.ndarray:
    """Random sequential addition of non-overlapping spheres with centres in the cylinder."""
    yc, xc = (rows - 1) / 2.0, (cols - 1) / 2.0
    target = porosity * np.pi * r_cyl * r_cyl * n
    cs = np.zeros((0, 4))
    vol = 0.0
    tries = 0
    while vol < target and tries < max_tries:
        batch = 256
        tries += batch
        rad = rng.uniform(rmin, rmax, batch)
        rho = r_cyl * np.sqrt(rng.uniform(0, 1, batch))
        th = rng.uniform(0, 2 * np.pi, batch)
        cand = np.stack([rng.uniform(0, n, batch), yc + rho * np.sin(th), xc + rho * np.cos(th), rad], 1)
        for c in cand:
            if len(cs):
                d2 = ((cs[:, :3] - c[:3]) ** 2).sum(1)
                if np.any(d2 < (cs[:, 3] + c[3]) ** 2):
                    continue
            cs = np.vstack([cs, c[None]])
            vol += 4.0 / 3.0 * np.pi * c[3] ** 3
            if vol >= target:
                break
    return cs


def _blur_axis(x, axis: int, kernel):
    import torch
    import torch.nn.functional as F

    k = kernel.numel()
    xt = x.movedim(axis, -1)
    shp = xt.shape
    flat = xt.reshape(-1, 1, shp[-1])
    flat = F.pad(flat, (k // 2, k // 2), mode="replicate")
    out = F.conv1d(flat, kernel.view(1, 1, -1))
    return out.reshape(shp).movedim(-1, axis).contiguous()


def make_phantom(n: int, rows: int, cols: int, r: float, *, seed: int = 0, radius_range=(4.0, 12.0),
                 noise: float = 7e-3, porosity: float = 0.2, p_scco2: float = 0.4, k: int = 3,
                 p_phase4: float = 0.15, blur_sigma: float = 1.0, device="cpu",
                 mapping: Optional[CylinderMapping] = None) -> Phantom:
    """Build one phantom.  k = 3: scCO2 / brine / glass; k = 4 adds a phase at 4.6e-2 on
    p_phase4 of the pores.  Labels are returned in ascending intensity order.  ``mapping``
    (optional) is the cylinder mask of (n, rows, cols, r) built elsewhere; by default the
    native library builds it."""
    import torch

    if k not in (3, 4):
        raise ValueError("k must be 3 or 4")
    rng = np.random.Generator(np.random.PCG64(seed))
    if mapping is None:
        mapping = CylinderMapping.cylinder(n, rows, cols, r)
    elif (mapping.n_images, mapping.rows, mapping.cols) != (n, rows, cols):
        raise ValueError("mapping does not match the phantom's extents")
    labels = [SCCO2, BRINE, GLASS] if k == 3 else [SCCO2, BRINE, PHASE4, GLASS]
    glass_id = len(labels) - 1
    cs = _rsa(rng, n, rows, cols, r, radius_range[0], radius_range[1], porosity)
    ph = np.where(rng.uniform(0, 1, len(cs)) < p_scco2, 0, 1)
    if k == 4:
        ph = np.where(rng.uniform(0, 1, len(cs)) < p_phase4, 2, ph)
    spheres = np.concatenate([cs, ph[:, None].astype(np.float64)], 1) if len(cs) else np.zeros((0, 5))

    dev = torch.device(device)
    # phase id box [col, row, n]: n contiguous like the cylinder layout
    box = torch.full((cols, rows, n), glass_id, dtype=torch.uint8, device=dev)
    for cn, cr, cc, rad, p in spheres:
        n0, n1 = max(int(np.floor(cn - rad)), 0), min(int(np.ceil(cn + rad)) + 1, n)
        r0, r1 = max(int(np.floor(cr - rad)), 0), min(int(np.ceil(cr + rad)) + 1, rows)
        c0, c1 = max(int(np.floor(cc - rad)), 0), min(int(np.ceil(cc + rad)) + 1, cols)
        if n0 >= n1 or r0 >= r1 or c0 >= c1:
            continue
        gc = torch.arange(c0, c1, device=dev, dtype=torch.float32).view(-1, 1, 1) - cc
        gr = torch.arange(r0, r1, device=dev, dtype=torch.float32).view(1, -1, 1) - cr
        gn = torch.arange(n0, n1, device=dev, dtype=torch.float32).view(1, 1, -1) - cn
        inside = gc * gc + gr * gr + gn * gn < rad * rad
        sub = box[c0:c1, r0:r1, n0:n1]
        sub[inside] = int(p)

    lut = torch.tensor(labels, dtype=torch.float32, device=dev)
    x = lut[box.long()]
    if blur_sigma > 0:
        rad = int(np.ceil(4 * blur_sigma))
        t = torch.arange(-rad, rad + 1, dtype=torch.float64)
        kern = torch.exp(-0.5 * (t / blur_sigma) ** 2)
        kern = (kern / kern.sum()).to(torch.float32).to(dev)
        for ax in range(3):
            x = _blur_axis(x, ax, kern)
    if noise > 0:
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(seed) * 7919 + 17)
        x = x + noise * torch.randn(x.shape, generator=gen, device=dev, dtype=torch.float32)

    rows_l, cols_l = mapping.lines()
    li_r = torch.from_numpy(rows_l).to(dev)
    li_c = torch.from_numpy(cols_l).to(dev)
    lines = x[li_c, li_r, :]                     # [n_lines, n]
    truth_lines = box[li_c, li_r, :]
    del x, box
    lo = float(lines.min()) if lines.numel() else 0.0
    hi = float(lines.max()) if lines.numel() else 1.0
    if hi <= lo:
        hi = lo + 1.0
    # convert_to_fp: v <= lo -> 0, v >= hi -> 1, else (v - lo) / (hi - lo)
    norm = torch.where(lines <= lo, torch.zeros_like(lines),
                       torch.where(lines >= hi, torch.ones_like(lines), (lines - lo) / (hi - lo)))
    u = torch.zeros((mapping.n_lines, mapping.nstride), dtype=torch.float32, device=dev)
    u[:, :n] = norm
    truth = torch.zeros((mapping.n_lines, mapping.nstride), dtype=torch.uint8, device=dev)
    truth[:, :n] = truth_lines
    lo32, hi32 = np.float32(lo), np.float32(hi)
    ci = [float((np.float32(l) - lo32) / (hi32 - lo32)) for l in labels]
    return Phantom(mapping, u.reshape(-1), truth.reshape(-1), labels, ci, lo, hi, spheres)


def config0_phantom(seed: int = 0, device="cpu", size: int = 128, r: float = 60.0) -> Phantom:
    """128^3, cylinder radius 60, sphere radii U[4, 12], noise 7e-3, k = 3."""
    return make_phantom(size, size, size, r, seed=seed, radius_range=(4.0, 12.0), noise=7e-3, device=device)


def config1_phantom(seed: int = 0, device="cuda") -> Phantom:
    """768 x 768 x 1024 (rows x cols x n), radius 370, sphere radii U[6, 30], noise 7e-3, k = 3."""
    return make_phantom(1024, 768, 768, 370.0, seed=seed, radius_range=(6.0, 30.0), noise=7e-3, device=device)


def config2_phantom(seed: int = 0, device="cuda") -> Phantom:
    """Config-1 geometry with k = 4 (extra phase at 4.6e-2 on 15% of the pores)."""
    return make_phantom(1024, 768, 768, 370.0, seed=seed, radius_range=(6.0, 30.0), noise=7e-3, k=4,
                        device=device)


@dataclass
class BatchSpec:
    """One sub-volume of the batched sweep: geometry, seed and its own lambda and noise."""
    n: int
    rows: int
    cols: int
    radius: float
    sphere_radii: tuple
    lam: float
    noise: float
    seed: int


def config3_specs(count: int = 48, seed: int = 0) -> list[BatchSpec]:
    """The batched sweep: sides drawn uniformly from 64..256 per axis, the 128^3 recipe scaled to
    each size (cylinder radius 0.47 min(rows, cols), sphere radii U[4, 12] * side / 128 with
    side the mean of rows and cols), lambda log-uniform in [10, 100], noise U[4e-3, 1.2e-2]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        n, rows, cols = (int(x) for x in rng.integers(64, 257, size=3))
        side = 0.5 * (rows + cols)
        scale = side / 128.0
        lam = float(np.exp(rng.uniform(np.log(10.0), np.log(100.0))))
        noise = float(rng.uniform(4e-3, 1.2e-2))
        out.append(BatchSpec(n, rows, cols, 0.47 * min(rows, cols), (4.0 * scale, 12.0 * scale), lam, noise,
                             seed * 1000 + i))
    return out


def batch_phantom(spec: BatchSpec, device="cuda") -> Phantom:
    return make_phantom(spec.n, spec.rows, spec.cols, spec.radius, seed=spec.seed, radius_range=spec.sphere_radii,
                        noise=spec.noise, device=device)
