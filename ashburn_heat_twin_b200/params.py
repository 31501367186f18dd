"""Physical constants and the lattice parameter math of the live solver host (js/live/solver.js of the reference).

Everything here runs on the host in float64 and produces the exact byte images the reference uploads to the device:
the uniform parameter block (64 + 16*nz bytes, kernel.js:36-50 / solver.js:225-242) and the per-column record
vec4<u32>(kt, ktop, cd bits, q bits) (solver.js:359-376).
"""
from __future__ import annotations

import math

import numpy as np

from .domain import KAPPA

# solver.js:8-14 (lbm3d.py constants)
RHO_CP = 1.16 * 1005.0      # J m-3 K-1
T0 = 303.0                  # K, Boussinesq reference temperature
GRAV = 9.81
CS, PRT, NU0, KFLOOR, MOMFAC, ULAT, ALPHA, ZCAP, SPONGE_TAU_S = 0.16, 0.7, 0.2, 0.5, 1.0, 0.1, 0.14, 150.0, 60.0
U10_MIN = 0.5
DIR_TOL, CALM, ADJ_TAU_S = 30, 0.3, 300
DEFAULT_MET = dict(u10=3.09, dirFrom=210, wstar=1.67, blh=903)   # KIAD 25 Aug 2024 15:52 UTC


def params_bytes(nz: int) -> int:
    """byte size of the parameter block: 4 x vec4 of scalars + nz x vec4 profile (uin, vin, kbg, 0) (kernel.js:36)."""
    return 64 + 16 * nz


def wind_profile(U10, dirFrom, alpha, nz, dx, zcap=ZCAP):
    """Power law, constant above zcap, at z = (k + 0.5) dx; m/s arrays u (east), v (north), speed
    (solver.js:17-26)."""
    th = dirFrom * math.pi / 180
    sx, sy = -math.sin(th), -math.cos(th)
    u = np.empty(nz); v = np.empty(nz); sp = np.empty(nz)
    for k in range(nz):
        z = (k + 0.5) * dx
        sp[k] = U10 * math.pow(min(z, zcap) / 10.0, alpha)
        u[k] = sp[k] * sx
        v[k] = sp[k] * sy
    return u, v, sp


def kprofile(z, ustar, wstar, h):
    """Holtslag & Boville (1993) K = kappa w_m z (1 - z/h)^2, w_m = (u*^3 + 0.6 w*^3 min(z, 0.1h)/h)^(1/3)
    (solver.js:29-34)."""
    zz = min(z, 0.1 * h)
    wm = np.cbrt(ustar ** 3 + 0.6 * wstar ** 3 * zz / h)
    s = min(1.0, max(0.0, 1 - z / h))
    return KAPPA * wm * z * s * s


def default_ustar(u10):
    """kappa u10 / ln(10/0.2) (solver.js:36)."""
    return KAPPA * u10 / math.log(10 / 0.2)


def inflow_faces(dirFrom, side_deg=0.0):
    """The lbm3d eps rule for inflow faces from the wind direction only (solver.js:264-269)."""
    th = dirFrom * math.pi / 180
    ux, uy, eps = -math.sin(th), -math.cos(th), 1e-3
    side = math.sin(max(0.0, side_deg or 0.0) * math.pi / 180)
    return dict(w=int(ux > eps or abs(ux) < side), e=int(ux < -eps or abs(ux) < side),
                s=int(uy > eps or abs(uy) < side), n=int(uy < -eps or abs(uy) < side))


def pack_params(dx, dt, nz, inflow, nsp, nsw, oclip, ul, vl, kl) -> bytes:
    """The uniform parameter block (solver.js:225-242): f32 scalars derived in float64 and rounded once."""
    buf = np.zeros(params_bytes(nz) // 4, np.uint32)
    f = buf.view(np.float32)
    i = buf.view(np.int32)
    f[0] = 0.5 + 3 * NU0 * dt / (dx * dx)              # tau0
    f[1] = 18 * math.sqrt(2) * CS * CS                  # cs2smag
    f[2] = GRAV / T0 * dt * dt / dx                     # gbeta
    f[3] = PRT
    f[4] = KFLOOR * dt / (dx * dx)                      # kfloor
    f[5] = MOMFAC
    f[6] = 1.0                                          # srcscale (q is in K per step)
    f[7] = min(0.2, dt / SPONGE_TAU_S)                  # sigmax
    i[8], i[9], i[10], i[11] = inflow['w'], inflow['e'], inflow['s'], inflow['n']
    i[12], i[13], i[14], i[15] = nsp, nsw, oclip, 0
    prof = f[16:].reshape(nz, 4)
    prof[:, 0] = np.asarray(ul, np.float32)
    prof[:, 1] = np.asarray(vl, np.float32)
    prof[:, 2] = np.asarray(kl, np.float32)
    prof[:, 3] = 0
    return buf.tobytes()


def unpack_params(b: bytes, nz: int) -> dict:
    """Decode a parameter block (as the reference's _dbg.domain(), solver.js:529-535)."""
    a = np.frombuffer(b, np.uint32)
    f, i = a.view(np.float32), a.view(np.int32)
    return dict(tau0=float(f[0]), cs2smag=float(f[1]), gbeta=float(f[2]), prt=float(f[3]), kfloor=float(f[4]),
                momfac=float(f[5]), srcscale=float(f[6]), sigmax=float(f[7]),
                inflow=dict(w=int(i[8]), e=int(i[9]), s=int(i[10]), n=int(i[11])),
                nsp=int(i[12]), nsw=int(i[13]), oclip=int(i[14]),
                prof=f[16:16 + 4 * nz].reshape(nz, 4).copy())


def pack_columns(ktS, ktopS, cdS, dcarea_n, flux, heatW_n, nx, ny, dx, dt):
    """Per-column vec4<u32> (solver.js:359-376): kt, ktop, cd (f32 bits), source q in K per step (f32 bits),
    q = W dt/(rho cp dx^3) with W = dcarea*flux + campus W. Inputs kt/ktop/cd are in solver orientation (j = 0
    south), dcarea/heat north-up. Returns (colv uint32 [NXY, 4], total W, q float32 [NXY] solver orientation)."""
    kq = dt / (RHO_CP * dx * dx * dx)
    Wn = np.asarray(dcarea_n, np.float64) * flux + np.asarray(heatW_n, np.float64)
    W = Wn.reshape(ny, nx)[::-1].ravel()                 # north-up -> solver rows
    # sequential sum in the reference's order (solver rows, j outer); np.cumsum is a strict left-to-right scan
    totalW = float(np.cumsum(W)[-1]) if W.size else 0.0
    out = np.zeros((nx * ny, 4), np.uint32)
    out[:, 0] = np.asarray(ktS, np.uint32)
    out[:, 1] = np.asarray(ktopS, np.uint32)
    out[:, 2] = np.asarray(cdS, np.float32).view(np.uint32)
    q = (W * kq).astype(np.float32)
    out[:, 3] = q.view(np.uint32)
    return out, totalW, q
