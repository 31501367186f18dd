"""Live-solver domain: the packed 10 m static planes and the coarse solver geometry at dx = 20/30/40 m.

Host-side restatement of js/live/domain.js (reference) in numpy, with the same arithmetic order wherever the result is
rounded (the per-block drag coefficient sum is accumulated sequentially, row-major inside the block, as the reference
loop does), so the geometry handed to the device is the reference's bit for bit.

Conventions (domain.js:1-5): every 2-D array here is north-up, [row*nx + col], row 0 = north edge (scene z = -2995),
col 0 = west edge (scene x = -2995). The solver flips rows (j = 0 at the south edge) when it uploads them.
"""
from __future__ import annotations

import gzip
import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

# domain.js:7-10
SCENE_X0, SCENE_Z0, AOI_SIZE, BASE_ELEV = -2995.0, -2995.0, 6000, 83.53166
KAPPA = 0.4
Z0_BY_CLASS = {10: 1.0, 20: 0.3, 30: 0.03, 40: 0.05, 50: 0.5, 60: 0.01, 80: 0.0002, 90: 0.05}
Z0_DEFAULT = 0.1


class DomainError(ValueError):
    """A rejected domain request; the message is the reference's (domain.js:23,38,62,91)."""


@dataclass
class Static10:
    """Integer-exact 10 m planes (domain.js:29-31): dem in cm, WorldCover class, building cover fraction x 25,
    mean building height in cm, operational data-center roof area / 4 m^2."""
    nrows: int
    ncols: int
    demCm: np.ndarray      # int64 [nrows*ncols]
    lc: np.ndarray         # uint8
    frac25: np.ndarray     # uint8
    hmeanCm: np.ndarray    # uint16
    dca4: np.ndarray       # uint8
    meta: dict = field(default_factory=dict)


_cache: dict = {}


def load_static10(base: str) -> Static10:
    """Load and decode static10.json + static10.bin.gz from directory `base` (domain.js:32-69): the dem plane holds
    row-wise first differences of cm values as int16 split into a low-byte and a high-byte plane; checksums of all
    planes are verified."""
    base = os.path.abspath(base)
    if base in _cache:
        return _cache[base]
    try:
        meta = json.load(open(os.path.join(base, 'static10.json')))
        raw = open(os.path.join(base, meta.get('file', 'static10.bin.gz')), 'rb').read()
    except OSError as e:
        raise DomainError(f'live solver: cannot load {base} ({e})') from None
    if raw[:2] == b'\x1f\x8b':
        raw = gzip.decompress(raw)
    if len(raw) != meta['raw_bytes']:
        raise DomainError(f"live solver: static10 has {len(raw)} bytes, expected {meta['raw_bytes']}")
    ny, nx = meta['grid']['nrows'], meta['grid']['ncols']
    n = nx * ny
    P = meta['planes']
    b = np.frombuffer(raw, np.uint8)
    lo = b[P['dem']['offset']:P['dem']['offset'] + n].astype(np.int64)
    hi = b[P['dem']['offset'] + n:P['dem']['offset'] + 2 * n].astype(np.int64)
    d = lo | (hi << 8)
    d = np.where(d >= 32768, d - 65536, d).reshape(ny, nx)
    demCm = np.cumsum(d, axis=1).ravel()
    st = Static10(
        nrows=ny, ncols=nx, demCm=demCm,
        lc=b[P['lc']['offset']:P['lc']['offset'] + n].copy(),
        frac25=b[P['frac25']['offset']:P['frac25']['offset'] + n].copy(),
        hmeanCm=np.frombuffer(raw, '<u2', n, P['hmean']['offset']).copy(),
        dca4=b[P['dca4']['offset']:P['dca4']['offset'] + n].copy(),
        meta=meta,
    )
    ck = meta['checksums']
    got = dict(dem_sum_cm=int(st.demCm.sum()), lc_sum=int(st.lc.astype(np.int64).sum()),
               frac25_sum=int(st.frac25.astype(np.int64).sum()), hmean_sum_cm=int(st.hmeanCm.astype(np.int64).sum()),
               dca4_sum=int(st.dca4.astype(np.int64).sum()))
    for k, v in got.items():
        if v != ck[k]:
            raise DomainError(f'live solver: static10 checksum mismatch ({k})')
    _cache[base] = st
    return st


def round_half_even(x):
    """numpy-compatible rounding, half to even (domain.js:73-76)."""
    return np.rint(x)


def flip_rows(a: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """north-up [row][col] <-> solver orientation [j][i] with j = 0 at the south edge; its own inverse
    (domain.js:79-83)."""
    return np.ascontiguousarray(np.asarray(a).reshape(ny, nx)[::-1]).ravel()


@dataclass
class Aggregate:
    nx: int
    ny: int
    dx: float
    r: int
    dem: np.ndarray
    cnt: np.ndarray
    frac: np.ndarray
    hmean: np.ndarray
    dcarea: np.ndarray
    cd: np.ndarray


def aggregate(st: Static10, dx: float) -> Aggregate:
    """Block aggregation 10 m -> dx (domain.js:89-118): dem block mean; frac block mean of the integer counts; hmean
    area-weighted mean over covered sub-pixels; dcarea block sum; drag coefficient cd = (kappa/ln(0.5 dx/z0))^2 of
    every 10 m cell averaged over the block."""
    r = int(round(dx / 10))
    if abs(r * 10 - dx) > 1e-9 or st.ncols % r or st.nrows % r:
        raise DomainError(f'live solver: dx must be a multiple of 10 m dividing 6000 m (got {dx:g})')
    nx, ny, NC = st.ncols // r, st.nrows // r, st.ncols
    cdTab = np.empty(256, np.float64)
    for c in range(256):
        z0 = Z0_BY_CLASS.get(c, Z0_DEFAULT)
        v = KAPPA / math.log((0.5 * dx) / z0)
        cdTab[c] = v * v
    blk = lambda a: np.asarray(a).reshape(ny, r, nx, r)
    dem_b, f_b = blk(st.demCm).astype(np.int64), blk(st.frac25).astype(np.int64)
    h_b, a_b, lc_b = blk(st.hmeanCm).astype(np.int64), blk(st.dca4).astype(np.int64), blk(st.lc)
    sd = dem_b.sum(axis=(1, 3))                      # integer sums: exact in any order
    sc = f_b.sum(axis=(1, 3))
    sh = (f_b * h_b).sum(axis=(1, 3))
    sa = a_b.sum(axis=(1, 3))
    scd = np.zeros((ny, nx), np.float64)             # float sum: the reference's order (a outer, b inner)
    for a in range(r):
        for bb in range(r):
            scd = scd + cdTab[lc_b[:, a, :, bb]]
    dem = (sd / (100 * r * r)).ravel()
    frac = (sc / (25 * r * r)).ravel()
    with np.errstate(invalid='ignore', divide='ignore'):
        hmean = np.where(sc > 0, sh / np.maximum(sc, 1) / 100, 0.0).ravel()
    return Aggregate(nx=nx, ny=ny, dx=float(dx), r=r, dem=dem, cnt=sc.ravel(), frac=frac, hmean=hmean,
                     dcarea=(4 * sa).ravel().astype(np.float64), cd=(scd / (r * r)).ravel())


@dataclass
class Rasterized:
    newArea: np.ndarray
    heatW: np.ndarray
    info: list


def rasterize_campuses(lst, dx: float, nx: int, ny: int) -> Rasterized:
    """New campuses (domain.js:124-160): halls [x0, z0, x1, z1] in scene metres, exact area overlap with the coarse
    cells; each campus spreads mw over its total hall area; hall parts outside the box are dropped. Returns north-up
    per-cell new roof area (m^2, clipped to the cell area) and heat (W)."""
    n = nx * ny
    newArea = np.zeros(n, np.float64)
    heatW = np.zeros(n, np.float64)
    info = []
    X1, Z1, cellA = SCENE_X0 + nx * dx, SCENE_Z0 + ny * dx, dx * dx
    for cp in lst or []:
        per: dict = {}
        total = 0.0
        for h in cp.get('halls', []) or []:
            xa, xb = min(h[0], h[2]), max(h[0], h[2])
            za, zb = min(h[1], h[3]), max(h[1], h[3])
            if not (xb > xa and zb > za):
                continue
            total += (xb - xa) * (zb - za)
            x0, x1, z0, z1 = max(xa, SCENE_X0), min(xb, X1), max(za, SCENE_Z0), min(zb, Z1)
            if x1 <= x0 or z1 <= z0:
                continue
            c0 = max(0, math.floor((x0 - SCENE_X0) / dx)); c1 = min(nx - 1, math.floor((x1 - SCENE_X0) / dx))
            r0 = max(0, math.floor((z0 - SCENE_Z0) / dx)); r1 = min(ny - 1, math.floor((z1 - SCENE_Z0) / dx))
            for r in range(r0, r1 + 1):
                oz = min(z1, SCENE_Z0 + (r + 1) * dx) - max(z0, SCENE_Z0 + r * dx)
                if oz <= 0:
                    continue
                for c in range(c0, c1 + 1):
                    ox = min(x1, SCENE_X0 + (c + 1) * dx) - max(x0, SCENE_X0 + c * dx)
                    if ox <= 0:
                        continue
                    k = r * nx + c
                    per[k] = per.get(k, 0.0) + ox * oz
        mw = max(0.0, float(cp.get('mw') or 0))
        flux = mw * 1e6 / total if total > 0 else 0.0
        inDom = 0.0
        for k, a0 in per.items():
            a = min(a0, cellA)
            newArea[k] += a
            heatW[k] += a * flux
            inDom += a
        info.append(dict(id=cp.get('id'), mw=mw, roofArea_m2=total, inDomain_m2=inDom, flux_wm2=flux,
                         heatMW=inDom * flux / 1e6, cells=len(per)))
    newArea = np.minimum(newArea, cellA)
    return Rasterized(newArea=newArea, heatW=heatW, info=info)


@dataclass
class Domain:
    nx: int
    ny: int
    nz: int
    dx: float
    zbase: float
    kt: np.ndarray      # int32, north-up: terrain-solid cells per column
    nb: np.ndarray      # int32: building cells
    ktop: np.ndarray    # int32: first fluid level = kt + nb
    cd: np.ndarray      # float32 drag coefficient
    ktopMax: int
    nbCells: int
    dcarea: np.ndarray
    dem: np.ndarray


def build_domain(agg: Aggregate, heightM: float = 720, newArea=None, extraHeight: float = 14.0,
                 nzMin: int = 0) -> Domain:
    """lbm3d.build_domain on the aggregated grid (domain.js:166-190): zbase = floor(min dem) - dx;
    kt = max(1, ceil((dem - zbase)/dx - 0.5)); nb = round_half_even(hmean/dx) where frac >= 0.5; ktop = kt + nb;
    nz = round(heightM/dx), raised to ktopMax + 9 if ktopMax >= nz - 8. New campus area raises frac to area/dx^2 and
    hmean to at least extraHeight."""
    dx = agg.dx
    zbase = math.floor(float(agg.dem.min())) - dx
    frac, hmean = agg.frac.copy(), agg.hmean.copy()
    if newArea is not None:
        m = newArea > 0
        frac = np.where(m, np.maximum(frac, newArea / (dx * dx)), frac)
        hmean = np.where(m, np.maximum(hmean, extraHeight), hmean)
    kt = np.maximum(1, np.ceil((agg.dem - zbase) / dx - 0.5)).astype(np.int32)
    nb = np.where(frac >= 0.5, round_half_even(hmean / dx), 0).astype(np.int32)
    ktop = (kt + nb).astype(np.int32)
    ktopMax = int(ktop.max())
    nz = max(int(math.floor(heightM / dx + 0.5)), int(nzMin))     # Math.round
    if ktopMax >= nz - 8:
        nz = ktopMax + 9
    return Domain(nx=agg.nx, ny=agg.ny, nz=nz, dx=dx, zbase=zbase, kt=kt, nb=nb, ktop=ktop,
                  cd=agg.cd.astype(np.float32), ktopMax=ktopMax, nbCells=int(nb.sum()), dcarea=agg.dcarea,
                  dem=agg.dem)
