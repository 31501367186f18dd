"""ctypes binding of libahx.so (include/ahx.h) and the CUDA device object the live solver host drives.

There is no fallback: if the library is missing, fails to load, or no CUDA device is present, constructing a
CudaDevice raises. The library is built in-tree by ashburn_heat_twin_b200._build (nvcc, sm_100a).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libahx.so')

PRECISIONS = {'fp32': 0, 'fp16': 1, 'bf16': 2, 'fp64': 3, 'fp16g32': 4, 'bf16g32': 5, 'fp16sr': 6}
ARITH = {'exact': 0, 'fast': 1}
STATUS = {0: 'AHX_OK', 1: 'AHX_EINVAL', 2: 'AHX_ENOMEM', 3: 'AHX_EDESTROYED', 4: 'AHX_EDEVICE', 5: 'AHX_ETIMEOUT',
          6: 'AHX_ENONFINITE', 7: 'AHX_EBUSY'}
MAX_READS = 8

# every symbol include/ahx.h declares
SYMBOLS = ('ahx_create', 'ahx_destroy', 'ahx_last_error', 'ahx_get_info', 'ahx_set_params', 'ahx_set_columns',
           'ahx_set_ktop', 'ahx_init_flow', 'ahx_clear_heat', 'ahx_set_parity', 'ahx_step', 'ahx_sync', 'ahx_fence',
           'ahx_fence_query', 'ahx_read_submit', 'ahx_read_wait', 'ahx_read_state', 'ahx_write_state',
           'ahx_read_state_f64', 'ahx_write_state_f64', 'ahx_read_dbg', 'ahx_clear_dbg', 'ahx_stats',
           'ahx_budget_enable', 'ahx_budget_read', 'ahx_set_launch', 'ahx_autotune', 'ahx_time_steps', 'ahx_stats_noalloc',
           'ahx_batch_create', 'ahx_batch_step', 'ahx_batch_time_steps', 'ahx_batch_sync', 'ahx_batch_set_launch',
           'ahx_batch_get_info', 'ahx_batch_destroy', 'ahx_batch_set_members', 'ahx_accum_enable', 'ahx_accum_read',
           'ahx_set_slab', 'ahx_row_bytes', 'ahx_row_pack', 'ahx_row_unpack', 'ahx_server_create',
           'ahx_server_submit', 'ahx_server_poll', 'ahx_server_stats', 'ahx_server_destroy', 'ahx_static_create',
           'ahx_static_checksums', 'ahx_static_destroy', 'ahx_domain_build', 'ahx_halo_bytes', 'ahx_halo_pack',
           'ahx_halo_unpack', 'ahx_step_rows')


class AhxError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class Dims(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('nz', ctypes.c_int32),
                ('precision', ctypes.c_int32), ('device_ordinal', ctypes.c_int32), ('arith', ctypes.c_int32)]


class InfoOut(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('nz', ctypes.c_int32), ('px', ctypes.c_int32),
                ('precision', ctypes.c_int32), ('arith', ctypes.c_int32), ('parity', ctypes.c_int32),
                ('device_ordinal', ctypes.c_int32), ('steps', ctypes.c_int64), ('state_bytes', ctypes.c_uint64),
                ('bytes_per_cell', ctypes.c_uint64), ('device_name', ctypes.c_char * 64)]


class StatsOut(ctypes.Structure):
    _fields_ = [('sum_theta', ctypes.c_double), ('sum_ke', ctypes.c_double), ('sum_rho_dev', ctypes.c_double),
                ('count', ctypes.c_double), ('theta_max', ctypes.c_float), ('umax', ctypes.c_float),
                ('non_finite', ctypes.c_uint32), ('pad', ctypes.c_uint32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [('device_ordinal', ctypes.c_int32), ('precision', ctypes.c_int32), ('arith', ctypes.c_int32),
                ('chunk', ctypes.c_int32), ('max_cells', ctypes.c_int64), ('hbm_budget_bytes', ctypes.c_uint64),
                ('batch_mode', ctypes.c_int32), ('tune', ctypes.c_int32), ('depth', ctypes.c_int32),
                ('pad', ctypes.c_int32)]


class RequestIn(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('nz', ctypes.c_int32), ('steps', ctypes.c_int32),
                ('params', ctypes.c_void_p), ('params_bytes', ctypes.c_size_t), ('colv', ctypes.c_void_p),
                ('ktop', ctypes.c_void_p), ('conv', ctypes.c_float), ('volscale', ctypes.c_float),
                ('nzv', ctypes.c_int32), ('want_vol', ctypes.c_int32), ('want_wind', ctypes.c_int32),
                ('pad', ctypes.c_int32), ('user_tag', ctypes.c_uint64)]


class ServerResult(ctypes.Structure):
    _fields_ = [('ticket', ctypes.c_uint64), ('user_tag', ctypes.c_uint64), ('nx', ctypes.c_int32),
                ('ny', ctypes.c_int32), ('nz', ctypes.c_int32), ('nzv', ctypes.c_int32), ('steps', ctypes.c_int32),
                ('status', ctypes.c_int32), ('submitted_s', ctypes.c_double), ('admitted_s', ctypes.c_double),
                ('done_s', ctypes.c_double), ('theta_max', ctypes.c_float), ('want_vol', ctypes.c_int32),
                ('want_wind', ctypes.c_int32), ('pad', ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ('submitted', 'admitted', 'completed', 'queued', 'active',
                                               'cell_updates', 'chunks', 'batch_steps', 'slots', 'idle_slots',
                                               'evictions', 'resident_cells')] + \
        [('slot_bytes', ctypes.c_uint64), ('hbm_budget_bytes', ctypes.c_uint64), ('elapsed_s', ctypes.c_double)]


class DomainSpec(ctypes.Structure):
    _fields_ = [('dx', ctypes.c_double), ('heightM', ctypes.c_double), ('extra_height', ctypes.c_double),
                ('nz_min', ctypes.c_int32), ('ncampus', ctypes.c_int32), ('campus_mw', ctypes.c_void_p),
                ('hall_count', ctypes.c_void_p), ('halls', ctypes.c_void_p), ('campus_flux', ctypes.c_void_p),
                ('flux_existing', ctypes.c_double), ('kq', ctypes.c_double), ('cd_table', ctypes.c_void_p)]


class DomainOut(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('nz', ctypes.c_int32), ('ktop_max', ctypes.c_int32),
                ('zbase', ctypes.c_double), ('nb_cells', ctypes.c_int64)]


class BudgetOut(ctypes.Structure):
    _fields_ = [('theta_sum', ctypes.c_double), ('src_sum', ctypes.c_double),
                ('face_theta_u', ctypes.c_double * 4), ('face_u', ctypes.c_double * 4), ('cells', ctypes.c_double),
                ('pad', ctypes.c_double * 5)]


class BatchInfoOut(ctypes.Structure):
    _fields_ = [('members', ctypes.c_int32), ('tiles', ctypes.c_int32), ('grid', ctypes.c_int32),
                ('minb', ctypes.c_int32), ('use_graph', ctypes.c_int32), ('zslab_max', ctypes.c_int32),
                ('pairs', ctypes.c_int32), ('pad', ctypes.c_int32), ('cells', ctypes.c_int64)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libahx.so and declare its signatures. Raises if the library is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise AhxError(-1, f'libahx.so not found at {path}: build it with ashburn_heat_twin_b200._build.build()')
    L = ctypes.CDLL(path)
    vp, i, u64p = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)
    H = ctypes.c_void_p
    sig = {
        'ahx_create': [ctypes.POINTER(Dims), ctypes.POINTER(H)],
        'ahx_destroy': [H],
        'ahx_get_info': [H, ctypes.POINTER(InfoOut)],
        'ahx_set_params': [H, vp, ctypes.c_size_t],
        'ahx_set_columns': [H, vp],
        'ahx_set_ktop': [H, vp, vp],
        'ahx_init_flow': [H],
        'ahx_clear_heat': [H],
        'ahx_set_parity': [H, i],
        'ahx_step': [H, i, i],
        'ahx_sync': [H, i],
        'ahx_time_steps': [H, i, i, i, ctypes.POINTER(ctypes.c_float)],
        'ahx_fence': [H, u64p],
        'ahx_fence_query': [H, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int)],
        'ahx_read_submit': [H, ctypes.c_float, ctypes.c_float, i, i, i, u64p],
        'ahx_read_wait': [H, ctypes.c_uint64, i, vp, vp, vp, vp, vp],
        'ahx_read_state': [H, vp, vp],
        'ahx_write_state': [H, vp, vp],
        'ahx_read_state_f64': [H, vp, vp],
        'ahx_write_state_f64': [H, vp, vp],
        'ahx_read_dbg': [H, vp],
        'ahx_clear_dbg': [H],
        'ahx_stats': [H, ctypes.POINTER(StatsOut)],
        'ahx_budget_enable': [H, i],
        'ahx_budget_read': [H, ctypes.POINTER(BudgetOut), i],
        'ahx_set_launch': [H, i, i],
        'ahx_autotune': [H, i, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                         ctypes.POINTER(ctypes.c_float)],
        'ahx_stats_noalloc': [i, i, i, vp, vp, vp, vp, vp],
        'ahx_batch_create': [ctypes.POINTER(H), i, ctypes.POINTER(H)],
        'ahx_batch_step': [H, i],
        'ahx_batch_time_steps': [H, i, i, ctypes.POINTER(ctypes.c_float)],
        'ahx_batch_sync': [H, i],
        'ahx_batch_set_launch': [H, i, i, i, i],
        'ahx_batch_set_members': [H, ctypes.POINTER(H), i],
        'ahx_accum_enable': [H, i],
        'ahx_set_slab': [H, i, i, i, i],
        'ahx_row_bytes': [H, ctypes.POINTER(ctypes.c_size_t)],
        'ahx_row_pack': [H, i, vp],
        'ahx_row_unpack': [H, i, vp],
        'ahx_halo_bytes': [H, ctypes.POINTER(ctypes.c_size_t)],
        'ahx_halo_pack': [H, i, i, i, vp],
        'ahx_halo_unpack': [H, i, i, vp],
        'ahx_step_rows': [H, i, i, i],
        'ahx_accum_read': [H, vp, vp, ctypes.POINTER(ctypes.c_int64), i],
        'ahx_batch_get_info': [H, ctypes.POINTER(BatchInfoOut)],
        'ahx_batch_destroy': [H],
        'ahx_server_create': [ctypes.POINTER(ServerConfig), ctypes.POINTER(H)],
        'ahx_server_submit': [H, ctypes.POINTER(RequestIn), u64p],
        'ahx_server_poll': [H, ctypes.c_uint64, i, ctypes.POINTER(ServerResult), vp, vp, vp, vp],
        'ahx_server_stats': [H, ctypes.POINTER(ServerStats)],
        'ahx_server_destroy': [H],
        'ahx_static_create': [i, i, i, vp, ctypes.c_size_t, vp, ctypes.POINTER(H)],
        'ahx_static_checksums': [H, vp],
        'ahx_static_destroy': [H],
        'ahx_domain_build': [H, ctypes.POINTER(DomainSpec), ctypes.POINTER(DomainOut), vp, vp, vp, vp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.ahx_last_error.argtypes = []
    L.ahx_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Handle:
    """Thin owner of one ahx_handle: raises AhxError on any nonzero status."""

    def __init__(self, nx, ny, nz, precision='fp32', device=None, arith='exact'):
        self.L = load_library()
        d = Dims(nx=nx, ny=ny, nz=nz, precision=PRECISIONS[precision], arith=ARITH[arith],
                 device_ordinal=-1 if device is None else int(device))
        h = ctypes.c_void_p()
        self._call('ahx_create', ctypes.byref(d), ctypes.byref(h))
        self.h = h
        self.nx, self.ny, self.nz = nx, ny, nz
        self.precision = precision

    def _call(self, name, *args):
        st = getattr(self.L, name)(*args)
        if st != 0:
            msg = self.L.ahx_last_error().decode(errors='replace')
            raise AhxError(st, msg or f'{name}: {STATUS.get(st, st)}')
        return st

    def call(self, name, *args):
        return self._call(name, self.h, *args)

    def info(self):
        o = InfoOut()
        self.call('ahx_get_info', ctypes.byref(o))
        return {k: (getattr(o, k).decode() if k == 'device_name' else getattr(o, k)) for k, _ in InfoOut._fields_}


class CudaDevice:
    """The live solver's device protocol (set_params, set_columns, set_ktop, init_flow, clear_heat, set_parity,
    step, fence, sync, read, read_state, write_state, read_dbg, clear_dbg, stats, lost, destroy) over libahx.so."""

    def __init__(self, nx, ny, nz, device=None, precision='fp32', arith='exact'):
        from .solver import Pending   # noqa: F401  (import check)
        self.hd = Handle(nx, ny, nz, precision=precision, device=device, arith=arith)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.N = nx * ny * nz
        self.precision = precision
        self.arith = arith
        info = self.hd.info()
        self.adapter = info['device_name']
        self._p = 0
        self._lost = None

    def _c(self, name, *args):
        try:
            return self.hd.call(name, *args)
        except AhxError as e:
            if e.status == 4:
                self._lost = str(e)
            raise

    # host images
    def set_params(self, b):
        buf = np.frombuffer(bytes(b), np.uint8)
        self._c('ahx_set_params', _ptr(buf), buf.nbytes)

    def set_columns(self, colv):
        a = np.ascontiguousarray(colv, np.uint32)
        self._c('ahx_set_columns', _ptr(a))

    def set_ktop(self, ktop, oldk):
        a = np.ascontiguousarray(ktop, np.uint32)
        o = None if oldk is None else np.ascontiguousarray(oldk, np.uint32)
        self._c('ahx_set_ktop', _ptr(a), _ptr(o))

    # state
    def init_flow(self):
        self._c('ahx_init_flow')

    def clear_heat(self):
        self._c('ahx_clear_heat')

    def set_parity(self, p):
        self._c('ahx_set_parity', int(p))
        self._p = int(p)

    def parity(self):
        return self._p

    def step(self, n, mode):
        self._c('ahx_step', int(n), int(mode))
        self._p ^= (int(n) & 1)

    def fence(self):
        from .solver import Pending
        t = ctypes.c_uint64()
        self._c('ahx_fence', ctypes.byref(t))
        ticket = t.value
        done = ctypes.c_int()

        def poll():
            self._c('ahx_fence_query', ctypes.c_uint64(ticket), ctypes.byref(done))
            return bool(done.value)

        def wait(timeout_s):
            import time
            t0 = time.perf_counter()
            while not poll():
                if timeout_s is not None and time.perf_counter() - t0 > timeout_s:
                    raise AhxError(5, 'live solver: timed out waiting for the GPU')
                time.sleep(0.0002)
            return None
        return Pending(poll=poll, wait=wait)

    def time_steps(self, n, mode=0, timeout_s=None):
        """queue n steps between two CUDA events on the handle's stream; returns their device time in ms"""
        ms = ctypes.c_float()
        self._c('ahx_time_steps', int(n), int(mode), -1 if timeout_s is None else int(timeout_s * 1000),
                ctypes.byref(ms))
        self._p ^= (int(n) & 1)
        return ms.value

    def sync(self, timeout_s=None):
        self._c('ahx_sync', -1 if timeout_s is None else int(timeout_s * 1000))

    def lost(self):
        return self._lost

    def read(self, conv, volscale, nzv, want_vol, want_wind, finish):
        from .solver import Pending
        t = ctypes.c_uint64()
        self._c('ahx_read_submit', ctypes.c_float(conv), ctypes.c_float(volscale), int(nzv), int(want_vol),
                int(want_wind), ctypes.byref(t))
        ticket = t.value
        NXY = self.nx * self.ny
        got = {}

        def fetch(timeout_ms):
            """copy the read-back out once it has arrived; False if it has not within timeout_ms"""
            surf = np.empty(NXY, np.float32)
            u = np.empty(NXY, np.float32) if want_wind else None
            v = np.empty(NXY, np.float32) if want_wind else None
            vb = np.empty(nzv * NXY, np.uint8) if want_vol else None
            tm = np.zeros(1, np.float32)
            try:
                self._c('ahx_read_wait', ctypes.c_uint64(ticket), int(timeout_ms), _ptr(surf), _ptr(u), _ptr(v),
                        _ptr(vb), _ptr(tm))
            except AhxError as e:
                if e.status == 5 and timeout_ms >= 0:    # not arrived yet: the read stays pending
                    return False
                raise
            got['res'] = finish((surf, u, v, vb, float(tm[0])))
            return True

        def poll():
            return 'res' in got or fetch(0)

        def wait(timeout_s):
            if 'res' not in got and not fetch(-1 if timeout_s is None else int(timeout_s * 1000)):
                raise AhxError(5, 'live solver: timed out waiting for the GPU')
            return got['res']
        return Pending(poll=poll, wait=wait)

    def read_state(self):
        f = np.empty(19 * self.N, np.float32)
        g = np.empty(7 * self.N, np.float32)
        self._c('ahx_read_state', _ptr(f), _ptr(g))
        return f, g

    def write_state(self, f, g):
        fa = None if f is None else np.ascontiguousarray(f, np.float32).ravel()
        ga = None if g is None else np.ascontiguousarray(g, np.float32).ravel()
        self._c('ahx_write_state', _ptr(fa), _ptr(ga))

    def read_state_f64(self):
        f = np.empty(19 * self.N, np.float64)
        g = np.empty(7 * self.N, np.float64)
        self._c('ahx_read_state_f64', _ptr(f), _ptr(g))
        return f, g

    def write_state_f64(self, f, g):
        fa = None if f is None else np.ascontiguousarray(f, np.float64).ravel()
        ga = None if g is None else np.ascontiguousarray(g, np.float64).ravel()
        self._c('ahx_write_state_f64', _ptr(fa), _ptr(ga))

    def read_dbg(self):
        d = np.empty(4 * self.N, np.float32)
        self._c('ahx_read_dbg', _ptr(d))
        return d

    def clear_dbg(self):
        self._c('ahx_clear_dbg')

    def stats(self):
        o = StatsOut()
        self._c('ahx_stats', ctypes.byref(o))
        return dict(sumTheta=o.sum_theta, sumKE=o.sum_ke, sumRhoDev=o.sum_rho_dev, count=int(o.count),
                    thetaMax=float(o.theta_max), nonFinite=int(o.non_finite), umax=float(o.umax))

    def budget_enable(self, on=True):
        self._c('ahx_budget_enable', int(bool(on)))

    def budget_read(self, reset=False):
        o = BudgetOut()
        self._c('ahx_budget_read', ctypes.byref(o), int(bool(reset)))
        return dict(theta_sum=o.theta_sum, src_sum=o.src_sum, face_theta_u=list(o.face_theta_u),
                    face_u=list(o.face_u), cells=o.cells)

    def set_launch(self, block_y=0, zslab=0):
        self._c('ahx_set_launch', int(block_y), int(zslab))
        prev = getattr(self, '_launch', (0, 0))
        self._launch = (int(block_y) or prev[0], int(zslab) or prev[1])

    def launch(self):
        """(block_y, zslab) in the ahx_set_launch encoding as last set or tuned; (0, 0) = the library's default."""
        return getattr(self, '_launch', (0, 0))

    def set_slab(self, jg0, nyg, jlo, jhi):
        self._c('ahx_set_slab', int(jg0), int(nyg), int(jlo), int(jhi))

    def row_bytes(self):
        b = ctypes.c_size_t()
        self._c('ahx_row_bytes', ctypes.byref(b))
        return b.value

    def row_pack(self, j, dst_ptr):
        """queue a copy of local row j (26 planes) of the current state into device memory at dst_ptr"""
        self._c('ahx_row_pack', int(j), ctypes.c_void_p(int(dst_ptr)))

    def row_unpack(self, j, src_ptr):
        self._c('ahx_row_unpack', int(j), ctypes.c_void_p(int(src_ptr)))

    def halo_bytes(self):
        b = ctypes.c_size_t()
        self._c('ahx_halo_bytes', ctypes.byref(b))
        return b.value

    def halo_pack(self, j, direction, dst_ptr, next_state=False):
        """queue a copy of the halo of local row j (the 6 planes with c_y = direction) into device memory at dst_ptr,
        from the current state or (next_state) from the one the step in progress writes"""
        self._c('ahx_halo_pack', int(j), int(direction), int(bool(next_state)), ctypes.c_void_p(int(dst_ptr)))

    def halo_unpack(self, j, direction, src_ptr):
        self._c('ahx_halo_unpack', int(j), int(direction), ctypes.c_void_p(int(src_ptr)))

    def step_rows(self, j0, j1, advance):
        """one step restricted to local rows [j0, j1); the call with advance completes the step"""
        self._c('ahx_step_rows', int(j0), int(j1), int(bool(advance)))
        if advance:
            self._p ^= 1

    def accum_enable(self, on=True):
        self._c('ahx_accum_enable', int(bool(on)))

    def accum_read(self, reset=False):
        """FP64 sums since enable / last reset: surf (3, ny, nx) = theta, ux, uy at the first fluid cell (solver
        orientation, lattice units), faces = dict(west, east: (2, nz, ny); south, north: (2, nz, nx)) of
        (theta, u_n), and the number of steps."""
        nx, ny, nz = self.nx, self.ny, self.nz
        surf = np.empty(3 * nx * ny, np.float64)
        faces = np.empty(2 * (2 * ny * nz + 2 * nx * nz), np.float64)
        n = ctypes.c_int64()
        self._c('ahx_accum_read', _ptr(surf), _ptr(faces), ctypes.byref(n), int(bool(reset)))
        fy, fx = ny * nz, nx * nz
        fc = faces.reshape(-1, 2)
        out = dict(west=fc[:fy], east=fc[fy:2 * fy], south=fc[2 * fy:2 * fy + fx], north=fc[2 * fy + fx:])
        out = {k: v.T.reshape(2, nz, -1) for k, v in out.items()}
        return surf.reshape(ny, nx, 3).transpose(2, 0, 1), out, n.value

    def autotune(self, steps_per_trial=4):
        by, zs, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        self._c('ahx_autotune', int(steps_per_trial), ctypes.byref(by), ctypes.byref(zs), ctypes.byref(ms))
        self._launch = (by.value, zs.value)
        return by.value, zs.value, ms.value

    def info(self):
        return self.hd.info()

    def destroy(self):
        if self.hd is not None:
            self.hd.call('ahx_destroy')   # refused while the handle belongs to a batch
            self.hd = None


class Batch:
    """Owner of one ahx_batch over the handles of several CudaDevice backends (same device, precision and
    arithmetic; grids may differ): each step of all members is one persistent launch, replayed from a CUDA graph."""

    def __init__(self, devices):
        self.L = load_library()
        self.devices = list(devices)
        arr = (ctypes.c_void_p * len(self.devices))(*[d.hd.h.value for d in self.devices])
        b = ctypes.c_void_p()
        self._call('ahx_batch_create', arr, len(self.devices), ctypes.byref(b))
        self.b = b

    def _call(self, name, *args):
        st = getattr(self.L, name)(*args)
        if st != 0:
            msg = self.L.ahx_last_error().decode(errors='replace')
            raise AhxError(st, msg or f'{name}: {STATUS.get(st, st)}')
        return st

    def _flip(self, n):
        for d in self.devices:
            d._p ^= (int(n) & 1)

    def step(self, n):
        self._call('ahx_batch_step', self.b, int(n))
        self._flip(n)

    def time_steps(self, n, timeout_s=None):
        """n batched steps between two CUDA events on the batch stream; returns their device time in ms"""
        ms = ctypes.c_float()
        self._call('ahx_batch_time_steps', self.b, int(n), -1 if timeout_s is None else int(timeout_s * 1000),
                   ctypes.byref(ms))
        self._flip(n)
        return ms.value

    def sync(self, timeout_s=None):
        self._call('ahx_batch_sync', self.b, -1 if timeout_s is None else int(timeout_s * 1000))

    def set_launch(self, minb=0, zslab=0, use_graph=True, pairs=None):
        """use_graph: True / 1 persistent launch replayed from a graph, False / 0 one persistent launch per step,
        'branches' / 2 each member's own step kernel on parallel graph branches"""
        g = 2 if use_graph in ('branches', 2) else (1 if use_graph else 0)
        self._call('ahx_batch_set_launch', self.b, int(minb), int(zslab), g, -1 if pairs is None else int(bool(pairs)))

    def set_members(self, devices):
        self.devices = list(devices)
        arr = (ctypes.c_void_p * max(1, len(self.devices)))(*[d.hd.h.value for d in self.devices])
        self._call('ahx_batch_set_members', self.b, arr, len(self.devices))

    def info(self):
        o = BatchInfoOut()
        self._call('ahx_batch_get_info', self.b, ctypes.byref(o))
        return {k: getattr(o, k) for k, _ in BatchInfoOut._fields_ if k != 'pad'}

    def destroy(self):
        if self.b is not None:
            self._call('ahx_batch_destroy', self.b)
            self.b = None


class Server:
    """Owner of one ahx_server (include/ahx.h): the continuous-batching scheduler thread inside libahx.so. submit()
    copies a request's byte images in and returns its ticket; poll() returns (result info, surf, u, v, vol) once the
    request is answered, or None while it is not (timeout)."""

    MODES = {'branches': 0, 'persistent': 1}

    def __init__(self, device=None, precision='fp32', arith='fast', chunk=256, max_cells=24_000_000,
                 hbm_budget_bytes=0, batch_mode='branches', tune=True, depth=2):
        self.L = load_library()
        cfg = ServerConfig(device_ordinal=-1 if device is None else int(device), precision=PRECISIONS[precision],
                           arith=ARITH[arith], chunk=int(chunk), max_cells=int(max_cells),
                           hbm_budget_bytes=int(hbm_budget_bytes or 0), batch_mode=self.MODES[batch_mode],
                           tune=int(bool(tune)), depth=int(depth), pad=0)
        h = ctypes.c_void_p()
        self._call('ahx_server_create', ctypes.byref(cfg), ctypes.byref(h))
        self.h = h
        self.cfg = cfg

    def _call(self, name, *args):
        st = getattr(self.L, name)(*args)
        if st != 0:
            raise AhxError(st, self.L.ahx_last_error().decode(errors='replace'))

    def submit(self, nx, ny, nz, steps, params, colv, ktop, conv, volscale, nzv, want_vol=True, want_wind=True,
               tag=0):
        pa = np.frombuffer(bytes(params), np.uint8)
        cv = np.ascontiguousarray(colv, np.uint32).ravel()
        kt = np.ascontiguousarray(ktop, np.uint32).ravel()
        if cv.size != 4 * nx * ny or kt.size != nx * ny:
            raise ValueError('column records or ktop plane of the wrong size')
        q = RequestIn(nx=int(nx), ny=int(ny), nz=int(nz), steps=int(steps), params=pa.ctypes.data,
                      params_bytes=pa.size, colv=cv.ctypes.data, ktop=kt.ctypes.data, conv=float(conv),
                      volscale=float(volscale), nzv=int(nzv), want_vol=int(bool(want_vol)),
                      want_wind=int(bool(want_wind)), pad=0, user_tag=int(tag))
        t = ctypes.c_uint64()
        self._call('ahx_server_submit', self.h, ctypes.byref(q), ctypes.byref(t))
        return t.value

    def poll(self, ticket, timeout_ms=0, nx=None, ny=None, nzv=None, want_vol=True, want_wind=True):
        NXY = int(nx) * int(ny)
        surf = np.empty(NXY, np.float32)
        u = np.empty(NXY, np.float32) if want_wind else None
        v = np.empty(NXY, np.float32) if want_wind else None
        vol = np.empty(int(nzv) * NXY, np.uint8) if want_vol else None
        info = ServerResult()
        st = self.L.ahx_server_poll(self.h, ctypes.c_uint64(ticket), int(timeout_ms), ctypes.byref(info), _ptr(surf),
                                    _ptr(u), _ptr(v), _ptr(vol))
        if st == 5:
            return None
        if st != 0:
            raise AhxError(st, self.L.ahx_last_error().decode(errors='replace'))
        return info, surf, u, v, vol

    def stats(self):
        o = ServerStats()
        self._call('ahx_server_stats', self.h, ctypes.byref(o))
        return {k: getattr(o, k) for k, _ in ServerStats._fields_}

    def destroy(self):
        if self.h is not None:
            self._call('ahx_server_destroy', self.h)
            self.h = None
