"""Seeded synthetic 10 m input planes in the format of the reference's static10 (domain.js:29-31), so synthetic
domains go through the same aggregation and build_domain rules as the real Ashburn input.

Terrain: a base elevation plus a sum of Gaussian hills (centres uniform in the box, sigma uniform 300-1200 m,
amplitudes scaled so the relief spans [0, relief_m]). Buildings: axis-aligned footprints (side lengths uniform in the
given range, heights uniform), placed without overlap by rejection while possible, rasterised on a 2 m sub-pixel grid
into building cover (frac x 25), mean height over covered sub-pixels and data-center roof area / 4 m^2. Land cover:
WorldCover class 50 (built-up, z0 0.5) where a 10 m cell is at least half covered, class 40 (z0 0.05) elsewhere.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .domain import Static10


@dataclass
class SynthSpec:
    ncols: int = 600              # 10 m cells (600 = the 6 km box)
    nrows: int = 600
    hills: int = 8
    relief_m: float = 30.0
    base_m: float = 60.0
    buildings: int = 1500
    side_m: tuple = (20.0, 120.0)
    height_m: tuple = (8.0, 30.0)
    dc_count: int = 60            # data-center roofs among the buildings (or added, see dc_side_m)
    dc_side_m: tuple = None       # if set, the data centers are separate footprints of this side range
    dc_height_m: tuple = (14.0, 25.0)
    seed: int = 1


# Benchmark configurations (the reference publishes no synthetic inputs; these are our seeded stand-ins)
C1 = SynthSpec(hills=8, relief_m=30.0, buildings=1500, side_m=(20.0, 120.0), height_m=(8.0, 30.0), dc_count=60,
               seed=1)
C2 = SynthSpec(hills=24, relief_m=40.0, buildings=4000, side_m=(15.0, 150.0), height_m=(8.0, 40.0), dc_count=211,
               dc_side_m=(60.0, 200.0), dc_height_m=(14.0, 25.0), seed=2)
# a quarter of the 600x600 box with the same densities (300x300x64 at 10 m): profiling-sized, state still >> L2
C2Q = SynthSpec(ncols=300, nrows=300, hills=6, relief_m=40.0, buildings=1000, side_m=(15.0, 150.0),
                height_m=(8.0, 40.0), dc_count=53, dc_side_m=(60.0, 200.0), dc_height_m=(14.0, 25.0), seed=3)


def _place(rng, n, side, box_w, box_h, occ, sub, allow_overlap_after=20):
    """n rectangles (x0, y0, w, h) in metres; rejection against the occupancy grid `occ` (sub-pixel size `sub`)."""
    out = []
    for _ in range(n):
        for attempt in range(allow_overlap_after + 1):
            w = rng.uniform(*side)
            h = rng.uniform(*side)
            x0 = rng.uniform(0, max(box_w - w, 1e-6))
            y0 = rng.uniform(0, max(box_h - h, 1e-6))
            a0, a1 = int(x0 / sub), int(np.ceil((x0 + w) / sub))
            b0, b1 = int(y0 / sub), int(np.ceil((y0 + h) / sub))
            if attempt == allow_overlap_after or not occ[b0:b1, a0:a1].any():
                occ[b0:b1, a0:a1] = True
                out.append((x0, y0, w, h))
                break
    return out


def make_static10(spec: SynthSpec) -> Static10:
    rng = np.random.default_rng(spec.seed)
    nx, ny = spec.ncols, spec.nrows
    W, H = nx * 10.0, ny * 10.0
    # terrain (north-up rows: row 0 north)
    yy, xx = np.mgrid[0:ny, 0:nx]
    X = (xx + 0.5) * 10.0
    Y = (yy + 0.5) * 10.0
    z = np.zeros((ny, nx))
    for _ in range(spec.hills):
        cx, cy = rng.uniform(0, W), rng.uniform(0, H)
        s = rng.uniform(300.0, 1200.0) * min(W, H) / 6000.0
        a = rng.uniform(0.3, 1.0)
        z += a * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
    if spec.hills and z.max() > z.min():
        z = (z - z.min()) / (z.max() - z.min()) * spec.relief_m
    demCm = np.round((spec.base_m + z) * 100).astype(np.int64).ravel()
    # buildings on a 2 m grid
    sub = 2.0
    sx, sy = int(W / sub), int(H / sub)
    hgt = np.zeros((sy, sx), np.float32)       # building height (m) per 2 m sub-pixel, 0 = none
    dcm = np.zeros((sy, sx), bool)
    occ = np.zeros((sy, sx), bool)
    scale = (nx * ny) / (600 * 600)
    nb = int(round(spec.buildings * scale))
    ndc = int(round(spec.dc_count * scale))
    rects = _place(rng, nb, spec.side_m, W, H, occ, sub)
    heights = rng.uniform(*spec.height_m, size=len(rects))
    if spec.dc_side_m is not None:
        dcs = _place(rng, ndc, spec.dc_side_m, W, H, occ, sub)
        dch = rng.uniform(*spec.dc_height_m, size=len(dcs))
        rects = rects + dcs
        heights = np.concatenate([heights, dch])
        is_dc = np.r_[np.zeros(len(rects) - len(dcs), bool), np.ones(len(dcs), bool)]
    else:
        is_dc = np.zeros(len(rects), bool)
        is_dc[rng.choice(len(rects), size=min(ndc, len(rects)), replace=False)] = True
    for (x0, y0, w, h), ht, dc in zip(rects, heights, is_dc):
        a0, a1 = int(x0 / sub), min(sx, int(np.ceil((x0 + w) / sub)))
        b0, b1 = int(y0 / sub), min(sy, int(np.ceil((y0 + h) / sub)))
        hgt[b0:b1, a0:a1] = ht
        if dc:
            dcm[b0:b1, a0:a1] = True
    cov = hgt > 0
    blk = lambda a: a.reshape(ny, 5, nx, 5)
    frac25 = blk(cov).sum(axis=(1, 3)).astype(np.int64)
    hsum_cm = blk(np.where(cov, np.round(hgt * 100), 0)).sum(axis=(1, 3))
    with np.errstate(invalid='ignore', divide='ignore'):
        hmeanCm = np.where(frac25 > 0, np.round(hsum_cm / np.maximum(frac25, 1)), 0).astype(np.uint16)
    dca4 = blk(dcm).sum(axis=(1, 3)).astype(np.uint8)
    lc = np.where(frac25 >= 13, 50, 40).astype(np.uint8)
    return Static10(nrows=ny, ncols=nx, demCm=demCm, lc=lc.ravel(), frac25=frac25.astype(np.uint8).ravel(),
                    hmeanCm=hmeanCm.ravel(), dca4=dca4.ravel(),
                    meta=dict(synthetic=True, seed=spec.seed, spec=spec.__dict__))


# scenario met for the configs (wind at 10 m, direction the wind blows from)
C1_MET = dict(u10=4.0, dirFrom=270.0, wstar=1.67, blh=903.0)
C2_MET = dict(u10=3.5, dirFrom=200.0, wstar=1.67, blh=903.0)
