"""The Node backend (ashburn_heat_twin_b200/napi: live_cuda.js over the N-API addon ahx_napi.cc) cannot run here (no
Node). Its C-ABI traffic can: napi/call_sequences.json lists the calls each shim operation makes, and this test drives
the reference's api20 interface scenario (tests/live/validate.html `api`, archived in validation_summary.json) through
solver.py with a device that makes exactly those calls, in that order, via ctypes. The scenario's recorded answers
must come out as they do through the Python binding, and every operation's calls must match the listed sequence."""
import ctypes
import json
import os

import numpy as np
import pytest

from ashburn_heat_twin_b200 import cuda_device as CD
from ashburn_heat_twin_b200 import solver as S
from tests.helpers import campus_list, real_solver, surf_stats

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SEQ = {k: v for k, v in json.load(open(os.path.join(ROOT, 'ashburn_heat_twin_b200', 'napi',
                                                     'call_sequences.json'))).items() if not k.startswith('_')}


def matches(calls, pattern):
    """calls against a listed sequence (a trailing * repeats its call one or more times)"""
    i = 0
    for p in pattern:
        rep = p.endswith('*')
        name = p.rstrip('*')
        if i >= len(calls) or calls[i] != name:
            return False
        i += 1
        while rep and i < len(calls) and calls[i] == name:
            i += 1
    return i == len(calls)


class ShimReplay:
    """The device protocol solver.py drives, implemented with the C-ABI calls of live_cuda.js + ahx_napi.cc."""

    adapter = 'shim replay'

    def __init__(self, nx, ny, nz, arith='exact'):
        self.L = CD.load_library()
        self.nx, self.ny, self.nz = nx, ny, nz
        self.ops = []                     # (operation, [C-ABI calls])
        self._op('create')
        d = CD.Dims(nx=nx, ny=ny, nz=nz, precision=0, device_ordinal=-1, arith=CD.ARITH[arith])
        h = ctypes.c_void_p()
        self._call('ahx_create', ctypes.byref(d), ctypes.byref(h))
        self.h = h
        self._info()

    def _op(self, name):
        self.ops.append((name, []))

    def _call(self, fn, *args):
        self.ops[-1][1].append(fn)
        st = getattr(self.L, fn)(*args)
        if st != 0:
            raise CD.AhxError(st, self.L.ahx_last_error().decode())
        return st

    def _info(self):
        o = CD.InfoOut()
        self._call('ahx_get_info', self.h, ctypes.byref(o))
        return o

    # host images
    def set_params(self, b):
        self._op('setParams')
        a = np.frombuffer(bytes(b), np.uint8)
        self._call('ahx_set_params', self.h, a.ctypes.data, a.size)

    def set_columns(self, colv):
        self._op('setColumns')
        self._info()
        c = np.ascontiguousarray(colv, np.uint32)
        self._call('ahx_set_columns', self.h, c.ctypes.data)

    def set_ktop(self, ktop, old=None):
        self._op('setKtop')
        self._info()
        k = np.ascontiguousarray(ktop, np.uint32)
        o = None if old is None else np.ascontiguousarray(old, np.uint32)
        self._call('ahx_set_ktop', self.h, k.ctypes.data, None if o is None else o.ctypes.data)

    def init_flow(self):
        self._op('initFlow')
        self._call('ahx_init_flow', self.h)

    def clear_heat(self):
        self._op('clearHeat')
        self._call('ahx_clear_heat', self.h)

    def set_parity(self, p):
        self._op('setParity')
        self._call('ahx_set_parity', self.h, int(p))

    # stepping: the shim's step(n) queues the steps, records a fence and polls it
    def step(self, n, mode):
        self._op('step')
        self._call('ahx_step', self.h, int(n), int(mode))
        self._pending_step = True

    def fence(self):
        if not getattr(self, '_pending_step', False):
            self._op('step')
            self._call('ahx_step', self.h, 0, 0)
        self._pending_step = False
        t = ctypes.c_uint64()
        self._call('ahx_fence', self.h, ctypes.byref(t))
        ops = self.ops[-1][1]
        done = ctypes.c_int(0)
        while True:
            ops.append('ahx_fence_query')
            st = self.L.ahx_fence_query(self.h, t, ctypes.byref(done))
            if st != 0:
                raise CD.AhxError(st, self.L.ahx_last_error().decode())
            if done.value:
                return S.Pending(value=None)

    def sync(self):
        self._op('sync')
        self._call('ahx_sync', self.h, -1)

    def lost(self):
        return None

    def read(self, conv, volscale, nzv, want_vol, want_wind, finish):
        self._op('read')
        self._info()
        t = ctypes.c_uint64()
        self._call('ahx_read_submit', self.h, ctypes.c_float(conv), ctypes.c_float(volscale), int(nzv),
                   int(want_vol), int(want_wind), ctypes.byref(t))
        ops = self.ops[-1][1]
        NXY = self.nx * self.ny

        def wait(timeout_s):
            surf = np.empty(NXY, np.float32)
            u = np.empty(NXY, np.float32) if want_wind else None
            v = np.empty(NXY, np.float32) if want_wind else None
            vb = np.empty(nzv * NXY, np.uint8) if want_vol else None
            tm = np.zeros(1, np.float32)
            ops.append('ahx_read_wait')
            st = self.L.ahx_read_wait(self.h, t, -1, CD._ptr(surf), CD._ptr(u), CD._ptr(v), CD._ptr(vb), CD._ptr(tm))
            if st != 0:
                raise CD.AhxError(st, self.L.ahx_last_error().decode())
            return finish((surf, u, v, vb, float(tm[0])))
        return S.Pending(poll=lambda: False, wait=wait)

    def stats(self):
        self._op('stats')
        o = CD.StatsOut()
        self._call('ahx_stats', self.h, ctypes.byref(o))
        return dict(sumTheta=o.sum_theta, sumKE=o.sum_ke, sumRhoDev=o.sum_rho_dev, count=int(o.count),
                    thetaMax=float(o.theta_max), nonFinite=int(o.non_finite), umax=float(o.umax))

    def destroy(self):
        self._op('destroy')
        self._call('ahx_destroy', self.h)


def test_api20_through_the_shim_call_sequence(kat):
    k = kat['api20']
    devs = []

    def backend(nx, ny, nz):
        devs.append(ShimReplay(nx, ny, nz))
        return devs[-1]

    s = real_solver(backend, dx=20)
    ref = real_solver(lambda nx, ny, nz: CD.CudaDevice(nx, ny, nz, arith='exact'), dx=20)
    assert s.info['nFluid'] == k['info']['nFluid']
    for x in (s, ref):
        x.step(300).result()
    r0, q0 = s.read(vol=False, wind=False).result(), ref.read(vol=False, wind=False).result()
    assert r0['thetaMax'] == pytest.approx(k['readNoVolNoWind']['thetaMax'], rel=3e-6)
    assert np.array_equal(r0['surf'], q0['surf']) and r0['thetaMax'] == q0['thetaMax']
    ps = []
    for _ in range(8):                 # 8 reads submitted while stepping
        ps.append(s.read())
        s.step(5)
    assert [round(p.result()['simTime'], 2) for p in ps] == k['concurrentReads']
    s.setNewCampuses(campus_list('AB'))
    nf1, rA = s.info['nFluid'], s.read().result()
    s.step(1000).result()
    stA = s._dbg.stats()
    s.setNewCampuses([])
    nf2 = s.info['nFluid']
    s.step(1000).result()
    stB, rB = s._dbg.stats(), s.read().result()
    kc = k['campuses']
    assert (nf1, nf2) == (kc['nFluidWith'], kc['nFluidWithout'])
    assert rA['heatMW'] == pytest.approx(kc['heatMWwith'], rel=1e-12)
    assert rB['heatMW'] == pytest.approx(kc['heatMWwithout'], rel=1e-12)
    assert stA['nonFinite'] + stB['nonFinite'] == 0
    s.resetHeat()
    rH = s.read().result()
    assert rH['simTime'] == 0 and rH['thetaMax'] == 0
    assert surf_stats(rH)['windMean'] == pytest.approx(k['afterResetHeat']['windMean'], rel=1e-3)
    s.step(200).result()
    s.resetFlow()
    rF = s.read().result()
    assert surf_stats(rF)['windMean'] == pytest.approx(k['afterResetFlow']['windMean'], rel=1e-6)
    s.setMet(dict(u10=4, dirFrom=230))
    n1 = s.flowReinits
    s.setMet(dict(u10=4, dirFrom=30))
    assert dict(afterSmallTurn=n1, afterBigTurn=s.flowReinits) == k['flowReinits']
    s.destroy()
    ref.destroy()
    with pytest.raises(S.LiveSolverError) as e:
        s.step(1).result()
    assert 'rejected: ' + str(e.value) == k['afterDestroy']
    # every operation made exactly the C-ABI calls the shim makes for it
    seen = set()
    for op, calls in devs[0].ops:
        assert op in SEQ and matches(calls, SEQ[op]), (op, calls)
        seen.add(op)
    assert {'create', 'setParams', 'setColumns', 'setKtop', 'initFlow', 'clearHeat', 'setParity', 'step', 'sync',
            'read', 'stats', 'destroy'} <= seen
