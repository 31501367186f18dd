"""Shared test helpers: solver factories over the CUDA backend or the CPU oracle, and comparison metrics."""
import os

import numpy as np

from ashburn_heat_twin_b200 import solver as S
from ashburn_heat_twin_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
# tests/live/validate.html:29 of the reference (KIAD 25 Aug 2024), with the explicit u* the parity runs used
MET_AUG25 = dict(u10=3.09, dirFrom=210, wstar=1.67, blh=903, ustar=0.32)
# the reference's hypothetical 120 MW campuses, scene metres (tests/live/validate.html:31-35)
CAMPUSES = {
    'A': dict(id='A', mw=120, halls=[[-205, 475, 175, 605], [-205, 635, 175, 765], [-205, 795, 175, 925]]),
    'B': dict(id='B', mw=120, halls=[[-2645, 1035, -2265, 1165], [-2645, 1195, -2265, 1325],
                                     [-2645, 1355, -2265, 1485]]),
    'C': dict(id='C', mw=120, halls=[[1555, -1495, 1935, -1365], [1555, -1335, 1935, -1205],
                                     [1555, -1175, 1935, -1045]]),
}


def campus_list(s):
    return [CAMPUSES[c] for c in (s or '') if c in CAMPUSES]


def oracle_backend(dtype=np.float32):
    from oracle.oracle import OracleDevice
    return lambda nx, ny, nz: OracleDevice(nx, ny, nz, dtype=dtype)


def cuda_backend(precision='fp32', arith='exact'):
    from ashburn_heat_twin_b200.cuda_device import CudaDevice
    return lambda nx, ny, nz: CudaDevice(nx, ny, nz, precision=precision, arith=arith)


def real_solver(backend, **kw):
    """createLiveSolver on the real Ashburn planes with the validation page's defaults (validate.html:61-75)."""
    o = dict(base=GOLDEN, dx=30, u10Max=8, heightM=720, met=MET_AUG25, existingFlux=400)
    o.update(kw)
    return S.create_live_solver(backend=backend, **o)


def small_static(seed=5, ncols=64, nrows=48, buildings=60):
    """A small seeded synthetic input (10 m cells) for quick parity runs."""
    spec = synth.SynthSpec(ncols=ncols, nrows=nrows, hills=3, relief_m=25.0, buildings=0, dc_count=0, seed=seed)
    st = synth.make_static10(spec)
    # buildings scaled to the small box explicitly (the default scales by area)
    spec2 = synth.SynthSpec(ncols=ncols, nrows=nrows, hills=3, relief_m=25.0,
                            buildings=int(buildings * 600 * 600 / (ncols * nrows)), side_m=(15, 60),
                            height_m=(8, 35), dc_count=int(8 * 600 * 600 / (ncols * nrows)), seed=seed)
    return synth.make_static10(spec2) if buildings else st


def small_solver(backend, seed=5, dx=10, heightM=300, met=None, ncols=64, nrows=48, **kw):
    st = small_static(seed=seed, ncols=ncols, nrows=nrows)
    o = dict(static=st, dx=dx, allowAnyDx=True, heightM=heightM, u10Max=8,
             met=met or dict(u10=4.0, dirFrom=250.0, wstar=1.2, blh=800.0), existingFlux=400)
    o.update(kw)
    return S.create_live_solver(backend=backend, **o)


def rel_l2(a, b):
    """tools/live/validate_live.py:146-149 of the reference."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def surf_stats(r):
    """surfStats of tests/live/validate.html:77-85."""
    s = r['surf'].astype(np.float64)
    ok = np.isfinite(s)
    out = dict(surfMax=float(s[ok].max()), surfMean=float(s[ok].sum() / s.size), nan=int((~ok).sum()))
    if r.get('u') is not None:
        sp = np.hypot(r['u'].astype(np.float64), r['v'].astype(np.float64))
        out['windMean'] = float(sp[np.isfinite(sp)].sum() / s.size)
    return out
