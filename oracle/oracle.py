"""ORACLE — test infrastructure, not product code.

ctypes binding of liboracle.so (the CPU restatement of the reference's WGSL kernels, lbm_oracle.cpp) and a device
object with the same protocol as the product's CUDA device, so the product's host logic (solver.LiveSolver) can be
driven against the oracle in tests. Only tests/, the smoke check and the benchmark's CPU-baseline leg import this
module; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, 'liboracle.so')

_lib = None


def build(force=False):
    """Compile liboracle.so with the Makefile next to this file."""
    src = os.path.join(HERE, 'lbm_oracle.cpp')
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(['make', '-s', '-C', HERE], stdout=sys.stderr)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.orc_step_f32.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, i]
        L.orc_step_f64.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, i]
        L.orc_init_f32.argtypes = [i, i, i, vp, vp, vp, vp]
        L.orc_init_f64.argtypes = [i, i, i, vp, vp, vp, vp]
        L.orc_surf_f32.argtypes = [i, i, i, vp, vp, vp, vp, vp, f, vp]
        L.orc_vol_f32.argtypes = [i, i, i, vp, vp, vp, i, f, vp, vp]
        L.orc_reinit_f32.argtypes = [i, i, i, vp, vp, vp, vp]
        L.orc_stats_f32.argtypes = [i, i, i, vp, vp, vp, vp]
        L.orc_set_threads.argtypes = [i]
        L.orc_max_threads.restype = i
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def set_threads(n):
    lib().orc_set_threads(int(n))


def max_threads():
    return lib().orc_max_threads()


# ---------------------------------------------------------------- kernel-level calls (reference layout arrays)
def step(nx, ny, nz, params, colv, ktop, fA, gA, dbg=None, mode=0, dtype=np.float32):
    """One fused step; returns (fB, gB). params: bytes of the parameter block; colv uint32 [NXY, 4]."""
    N = nx * ny * nz
    pb = np.frombuffer(params, np.uint8).copy()
    fB = np.empty(19 * N, dtype)
    gB = np.empty(7 * N, dtype)
    # cells the kernel does not write (solid) keep the destination's previous content in the reference; ping-pong
    # buffers there are initialised identically, so solid cells carry the init values: mirror that by copying
    fB[:] = fA
    gB[:] = gA
    fn = lib().orc_step_f32 if dtype == np.float32 else lib().orc_step_f64
    fn(nx, ny, nz, _p(pb), _p(np.ascontiguousarray(colv, np.uint32)), _p(np.ascontiguousarray(ktop, np.uint32)),
       _p(fA), _p(fB), _p(gA), _p(gB), _p(dbg), int(mode))
    return fB, gB


def step_into(nx, ny, nz, params, colv, ktop, fA, fB, gA, gB, dbg=None, mode=0):
    """One fused step writing into preallocated fB/gB (the reference's ping-pong semantics)."""
    pb = np.frombuffer(params, np.uint8).copy()
    fn = lib().orc_step_f32 if fA.dtype == np.float32 else lib().orc_step_f64
    fn(nx, ny, nz, _p(pb), _p(np.ascontiguousarray(colv, np.uint32)), _p(np.ascontiguousarray(ktop, np.uint32)),
       _p(fA), _p(fB), _p(gA), _p(gB), _p(dbg), int(mode))


def init(nx, ny, nz, params, colv, dtype=np.float32):
    N = nx * ny * nz
    pb = np.frombuffer(params, np.uint8).copy()
    f = np.empty(19 * N, dtype)
    fn = lib().orc_init_f32 if dtype == np.float32 else lib().orc_init_f64
    fn(nx, ny, nz, _p(pb), _p(np.ascontiguousarray(colv, np.uint32)), _p(f), None)
    return f


def surf(nx, ny, nz, params, colv, ktop, fA, gA, conv):
    pb = np.frombuffer(params, np.uint8).copy()
    out = np.empty(3 * nx * ny, np.float32)
    lib().orc_surf_f32(nx, ny, nz, _p(pb), _p(np.ascontiguousarray(colv, np.uint32)),
                       _p(np.ascontiguousarray(ktop, np.uint32)), _p(fA), _p(gA), float(conv), _p(out))
    return out


def vol(nx, ny, nz, params, ktop, gA, nzv, volscale):
    pb = np.frombuffer(params, np.uint8).copy()
    nw = (nzv * nx * ny + 3) // 4
    out = np.empty(nw, np.uint32)
    tmax = np.zeros(1, np.float32)
    lib().orc_vol_f32(nx, ny, nz, _p(pb), _p(np.ascontiguousarray(ktop, np.uint32)), _p(gA), int(nzv),
                      float(volscale), _p(out), _p(tmax))
    return out, float(tmax[0])


def reinit(nx, ny, nz, ktop, oldk, f, g):
    lib().orc_reinit_f32(nx, ny, nz, _p(np.ascontiguousarray(ktop, np.uint32)),
                         _p(np.ascontiguousarray(oldk, np.uint32)), _p(f), _p(g))


def stats(nx, ny, nz, ktop, fA, gA):
    out = np.zeros(7, np.float64)
    lib().orc_stats_f32(nx, ny, nz, _p(np.ascontiguousarray(ktop, np.uint32)), _p(fA), _p(gA), _p(out))
    return dict(sumTheta=out[0], sumKE=out[1], sumRhoDev=out[2], count=int(out[3]), thetaMax=float(out[4]),
                nonFinite=int(out[5]), umax=float(out[6]))


class _Done:
    def __init__(self, value=None):
        self.value = value


class OracleDevice:
    """The device protocol of the product's CudaDevice, executed by the CPU oracle (synchronously)."""

    adapter = 'cpu-oracle'

    def __init__(self, nx, ny, nz, dtype=np.float32):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.N = nx * ny * nz
        self.dtype = dtype
        self.f = [np.zeros(19 * self.N, dtype), np.zeros(19 * self.N, dtype)]
        self.g = [np.zeros(7 * self.N, dtype), np.zeros(7 * self.N, dtype)]
        self.p = 0
        self.params = None
        self.colv = None
        self.ktop = None
        self.dbg = None
        self.steps_run = 0

    # host -> device images
    def set_params(self, b):
        self.params = bytes(b)

    def set_columns(self, colv):
        self.colv = np.ascontiguousarray(colv, np.uint32)

    def set_ktop(self, ktop, oldk):
        self.ktop = np.ascontiguousarray(ktop, np.uint32)
        if oldk is not None:
            reinit(self.nx, self.ny, self.nz, self.ktop, oldk, self.f[self.p], self.g[self.p])

    # state
    def init_flow(self):
        f = init(self.nx, self.ny, self.nz, self.params, self.colv, self.dtype)
        self.f[0][:] = f
        self.f[1][:] = f

    def clear_heat(self):
        self.g[0][:] = 0
        self.g[1][:] = 0

    def set_parity(self, p):
        self.p = p

    def parity(self):
        return self.p

    def step(self, n, mode):
        if mode and self.dbg is None:
            self.dbg = np.zeros(4 * self.N, self.dtype)
        for s in range(n):
            m = mode if (mode == 2 or s == n - 1) else 0
            a, b = self.p, 1 - self.p
            step_into(self.nx, self.ny, self.nz, self.params, self.colv, self.ktop, self.f[a], self.f[b],
                      self.g[a], self.g[b], self.dbg, m)
            self.p = b
            self.steps_run += 1

    def fence(self):
        from ashburn_heat_twin_b200.solver import Pending
        return Pending(value=None)

    def sync(self, timeout_s=None):
        pass

    def lost(self):
        return None

    def read(self, conv, volscale, nzv, want_vol, want_wind, finish):
        from ashburn_heat_twin_b200.solver import Pending
        nx, ny = self.nx, self.ny
        s = surf(nx, ny, self.nz, self.params, self.colv, self.ktop, self.f[self.p], self.g[self.p], conv)
        vw, tmax = vol(nx, ny, self.nz, self.params, self.ktop, self.g[self.p], nzv, volscale)
        NXY = nx * ny
        vb = vw.view(np.uint8)[:nzv * NXY].copy()
        return Pending(value=finish((s[:NXY].copy(), s[NXY:2 * NXY].copy(), s[2 * NXY:].copy(), vb, tmax)))

    def read_state(self):
        return self.f[self.p].copy(), self.g[self.p].copy()

    def write_state(self, f, g):
        if f is not None:
            self.f[self.p][:] = np.asarray(f, self.dtype).ravel()
        if g is not None:
            self.g[self.p][:] = np.asarray(g, self.dtype).ravel()

    def read_dbg(self):
        if self.dbg is None:
            self.dbg = np.zeros(4 * self.N, self.dtype)
        return self.dbg.copy()

    def clear_dbg(self):
        if self.dbg is None:
            self.dbg = np.zeros(4 * self.N, self.dtype)
        self.dbg[:] = 0

    def stats(self):
        return stats(self.nx, self.ny, self.nz, self.ktop, self.f[self.p], self.g[self.p])

    def destroy(self):
        self.f = self.g = None
