"""The live solver's domain builder on the GPU (ahx_static_* / ahx_domain_build in libahx.so).

The same images as domain.py + params.pack_columns (js/live/domain.js:32-190 and the column record of
js/live/solver.js:359-376 in the reference), built by kernels: the 10 m static planes go to the device once (the
dem's row-wise first differences are summed there), each grid spacing is block-aggregated once, and each request's
campus raster, building rule and column records are three small launches. Results are bit-identical to the host
restatement.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import domain as DM
from . import params as PM
from .cuda_device import AhxError, DomainOut, DomainSpec, _ptr, load_library


def raw_payload(st: DM.Static10):
    """(raw bytes, plane offsets) of a Static10 in the static10 payload layout: dem as row-wise int16 first differences
    (low-byte plane, then high-byte plane), lc u8, frac25 u8, hmean u16 little-endian, dca4 u8."""
    ny, nx = st.nrows, st.ncols
    n = nx * ny
    dem = np.asarray(st.demCm, np.int64).reshape(ny, nx)
    d = np.diff(dem, axis=1, prepend=0)
    if d.min() < -32768 or d.max() > 32767:
        raise DM.DomainError('live solver: dem steps exceed the int16 row-delta encoding')
    d16 = d.astype(np.int16).view(np.uint16).ravel()
    parts = [(d16 & 0xFF).astype(np.uint8).tobytes(), (d16 >> 8).astype(np.uint8).tobytes(),
             np.asarray(st.lc, np.uint8).tobytes(), np.asarray(st.frac25, np.uint8).tobytes(),
             np.asarray(st.hmeanCm, '<u2').tobytes(), np.asarray(st.dca4, np.uint8).tobytes()]
    offs = [0, 2 * n, 3 * n, 4 * n, 6 * n]
    return b''.join(parts), offs


def cd_table(dx: float) -> np.ndarray:
    """(kappa / ln(0.5 dx / z0))^2 per land-cover class, as domain.aggregate forms it (domain.js:96-101)."""
    t = np.empty(256, np.float64)
    for c in range(256):
        z0 = DM.Z0_BY_CLASS.get(c, DM.Z0_DEFAULT)
        v = DM.KAPPA / math.log((0.5 * dx) / z0)
        t[c] = v * v
    return t


class GpuDomain:
    """The static planes of one box on one device, and per-request builds of the solver geometry."""

    def __init__(self, st: DM.Static10, device=None):
        self.L = load_library()
        self.st = st
        raw, offs = raw_payload(st)
        self._raw = np.frombuffer(raw, np.uint8)
        o = (ctypes.c_size_t * 5)(*offs)
        h = ctypes.c_void_p()
        self._call('ahx_static_create', -1 if device is None else int(device), st.nrows, st.ncols,
                   self._raw.ctypes.data, self._raw.size, o, ctypes.byref(h))
        self.h = h

    def _call(self, name, *args):
        rc = getattr(self.L, name)(*args)
        if rc != 0:
            raise AhxError(rc, self.L.ahx_last_error().decode(errors='replace'))

    def checksums(self):
        """the reference's static10 checksums (static10.json 'checksums') computed on the device"""
        out = np.zeros(5, np.int64)
        self._call('ahx_static_checksums', self.h, _ptr(out))
        return dict(dem_sum_cm=int(out[0]), lc_sum=int(out[1]), frac25_sum=int(out[2]), hmean_sum_cm=int(out[3]),
                    dca4_sum=int(out[4]))

    def build(self, dx, heightM=720, campuses=(), flux=400.0, dt=None, nzMin=0, extraHeight=14.0):
        """One request's geometry: dict(nx, ny, nz, zbase, ktopMax, nbCells, colv (NXY x 4 u32, solver orientation),
        ktop (NXY u32, solver orientation), heatW and newArea (north-up, float64), campusFlux)."""
        r = int(round(dx / 10))
        nx, ny = self.st.ncols // r, self.st.nrows // r
        NXY = nx * ny
        mw = np.array([max(0.0, float(c.get('mw') or 0)) for c in campuses], np.float64)
        counts = np.array([len(c.get('halls') or []) for c in campuses], np.int32)
        halls = np.array([[float(v) for v in list(h)[:4]] for c in campuses for h in (c.get('halls') or [])],
                         np.float64).reshape(-1, 4)
        cflux = np.zeros(max(1, len(campuses)), np.float64)
        tab = cd_table(float(dx))
        kq = 0.0 if dt is None else dt / (PM.RHO_CP * dx * dx * dx)
        spec = DomainSpec(dx=float(dx), heightM=float(heightM), extra_height=float(extraHeight), nz_min=int(nzMin),
                          ncampus=len(campuses), campus_mw=mw.ctypes.data if len(campuses) else None,
                          hall_count=counts.ctypes.data if len(campuses) else None,
                          halls=halls.ctypes.data if halls.size else None, campus_flux=cflux.ctypes.data,
                          flux_existing=float(flux), kq=float(kq), cd_table=tab.ctypes.data)
        out = DomainOut()
        colv = np.empty((NXY, 4), np.uint32)
        ktop = np.empty(NXY, np.uint32)
        heat = np.empty(NXY, np.float64)
        area = np.empty(NXY, np.float64)
        self._call('ahx_domain_build', self.h, ctypes.byref(spec), ctypes.byref(out), _ptr(colv), _ptr(ktop),
                   _ptr(heat), _ptr(area))
        return dict(nx=out.nx, ny=out.ny, nz=out.nz, zbase=out.zbase, ktopMax=out.ktop_max, nbCells=out.nb_cells,
                    colv=colv, ktop=ktop, heatW=heat, newArea=area, campusFlux=cflux[:len(campuses)])

    def destroy(self):
        if self.h is not None:
            self._call('ahx_static_destroy', self.h)
            self.h = None
