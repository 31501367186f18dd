"""The live solver's host API: createLiveSolver() and the LiveSolver object of js/live/solver.js (reference), over the
CUDA backend (libahx.so, C ABI in include/ahx.h).

Method names, argument meaning, defaults, clamps and error messages follow the reference (solver.js:44-579) so code
written against the WebGPU solver reads the same here:

    s = create_live_solver(dx=30, u10Max=8)
    s.setMet(dict(u10=3.09, dirFrom=210, wstar=1.67, blh=903))
    s.setExistingFlux(400)
    s.setNewCampuses([dict(id='A', mw=120, halls=[[-205, 475, 175, 605]])])
    s.step(40).result()              # reference: await solver.step(40)
    r = s.read().result()            # reference: await solver.read()

`step()` and `read()` return a Pending (the reference returns Promises): `.result(timeout_s)` waits, `.done()` polls,
and it is awaitable from asyncio. The device work of `step(n)` is queued on the solver's CUDA stream and returns at
once; `read()` queues its two small kernels behind the steps already queued and copies on a second stream, so reads
never block stepping.

The host keeps all domain and parameter math (float64, rounded to f32 exactly as the reference) and hands the device
the same byte images WebGPU receives: the parameter block, the per-column records and the ktop plane.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import domain as D
from . import params as PM

_DXS = (20, 30, 40)


class LiveSolverError(RuntimeError):
    """Rejection with the reference's readable message (solver.js:47-54, 219-222)."""


def _jsnum(x):
    """Number formatting of a JS template literal (25 -> '25', 25.5 -> '25.5')."""
    try:
        xf = float(x)
    except (TypeError, ValueError):
        return str(x)
    if math.isfinite(xf) and xf == int(xf):
        return str(int(xf))
    return repr(xf)


def js_round(x):
    """Math.round: half toward +infinity."""
    return math.floor(x + 0.5)


def _mod360(x):
    """((x % 360) + 360) % 360 with JS remainder semantics."""
    return math.fmod(math.fmod(x, 360.0) + 360.0, 360.0)


class Pending:
    """Result of an asynchronous solver call (the reference's Promise)."""

    def __init__(self, poll=None, wait=None, value=None, error=None):
        self._poll, self._wait, self._value, self._error, self._resolved = poll, wait, value, error, poll is None

    def done(self):
        if not self._resolved and self._poll():
            self._finish(None)
        return self._resolved

    def _finish(self, timeout_s):
        if not self._resolved:
            try:
                v = self._wait(timeout_s)
                if v is not None:
                    self._value = v
            except Exception as e:          # the reference rejects the promise
                self._error = e
            self._resolved = True

    def result(self, timeout_s=None):
        self._finish(timeout_s)
        if self._error is not None:
            raise self._error
        return self._value

    def __await__(self):
        import asyncio
        while not self.done():
            yield from asyncio.sleep(0.0005).__await__()
        return self.result()


class LiveSolver:
    """The reference's LiveSolver (solver.js:103-579). Construct with create_live_solver()."""

    def __init__(self, o, st, agg, dom0, device_factory, prog):
        self._o, self._agg, self._dom, self._prog = o, agg, dom0, prog
        nx, ny, nz, dx = dom0.nx, dom0.ny, dom0.nz, dom0.dx
        self._alpha = float(o.get('alpha', PM.ALPHA))
        # dt fixed per instance from the profile maximum at u10Max (lbm3d.Sim: dt = ulat dx / Umax) (solver.js:107-110)
        Umax = float(PM.wind_profile(o['u10Max'], 0, self._alpha, nz, dx)[2].max())
        dt = PM.ULAT * dx / Umax
        self._dt, self._Umax, self._conv = dt, Umax, dx / dt
        self._nsp = int(o['nsp']) if o.get('nsp') is not None else max(1, js_round(120 / dx))
        self._nsw = int(o['nsw']) if o.get('nsw') is not None else max(1, js_round(160 / dx))
        self._oclip = 0 if o.get('outflowClip') is False else 1
        self.nzv = min(nz, js_round(420 / dx))
        nFluid = int((nz - dom0.ktop.astype(np.int64)).sum())
        dcRoof = float(np.cumsum(dom0.dcarea)[-1]) if dom0.dcarea.size else 0.0
        self._flux = float(o['existingFlux']) if o.get('existingFlux') is not None else 400.0
        self.info = dict(
            nx=nx, ny=ny, nz=nz, nzv=self.nzv, dx=dx, dt=dt, zbase=dom0.zbase, baseElev=D.BASE_ELEV,
            x0=D.SCENE_X0, z0=D.SCENE_Z0, adapter='unknown', heatExistingMW=dcRoof * self._flux / 1e6,
            dcRoofArea_m2=dcRoof,
            u10Max=o['u10Max'], Umax=Umax, convU=self._conv, nsp=self._nsp, nsw=self._nsw, nCells=nx * ny * nz,
            nFluid=nFluid, top=dom0.zbase + nz * dx)
        self.grid = None
        self.campusInfo = []
        self.flowReinits = 0
        self._met = None
        self._inflow = None
        self._prof = None
        self._flowRef = None
        self._applied = None
        self._campuses = []
        self._ras = D.rasterize_campuses([], dx, nx, ny)
        self._n = 0
        self._steps = 0
        self._destroyed = False
        self._params = None
        self._ktopS = None
        self._heatMW = 0.0
        self._dev = device_factory(nx, ny, nz)
        self.info['adapter'] = getattr(self._dev, 'adapter', 'unknown')
        self.__dbg = None

    @property
    def simTime(self):
        return self._n * self._dt

    # ------------------------------------------------------------------ set-up (solver.js:137-196)
    def _init(self):
        self._prog('Initialising the flow', 0.85)
        self._setGeometry(True)
        self.setMet(self._o.get('met') or PM.DEFAULT_MET)
        self.resetFlow()
        self._dev.sync()

    def _check(self):
        if self._destroyed:
            raise LiveSolverError('live solver: destroyed')
        lost = self._dev.lost() if self._dev is not None else None
        if lost:
            raise LiveSolverError(f'live solver: CUDA device lost ({lost})')

    # ------------------------------------------------------------------ parameters (solver.js:225-285)
    def _writeParams(self):
        d = self._dom
        self._params = PM.pack_params(d.dx, self._dt, d.nz, self._inflow, self._nsp, self._nsw, self._oclip,
                                      self._prof['ul'], self._prof['vl'], self._prof['kl'])
        self._dev.set_params(self._params)

    def setMet(self, m=None):
        """{ u10, dirFrom, wstar, blh, ustar (optional, default kappa u10 / ln(10/0.2)) }; applies from the next
        step (solver.js:245-285)."""
        self._check()
        m = dict(m or {})
        prev = self._met or PM.DEFAULT_MET
        pick = lambda k: float(m[k]) if m.get(k) is not None else float(prev[k])
        u10 = min(max(pick('u10'), PM.U10_MIN), float(self._o['u10Max']))
        dirFrom = _mod360(pick('dirFrom'))
        wstar = max(0.0, pick('wstar'))
        blh = min(max(pick('blh'), 50.0), 5000.0)
        ustar = max(0.0, float(m['ustar'])) if m.get('ustar') is not None else PM.default_ustar(u10)
        self._met = dict(u10=u10, dirFrom=dirFrom, wstar=wstar, blh=blh, ustar=ustar)
        nz, dx, dt = self._dom.nz, self._dom.dx, self._dt
        wu, wv, _ = PM.wind_profile(u10, dirFrom, self._alpha, nz, dx)
        kmaxLat = 1 / 6
        Kphys = np.array([PM.kprofile((k + 0.5) * dx, ustar, wstar, blh) for k in range(nz)])
        self._prof = dict(ul=(wu / self._conv).astype(np.float32), vl=(wv / self._conv).astype(np.float32),
                          kl=np.minimum(Kphys * dt / (dx * dx), kmaxLat).astype(np.float32), Kphys=Kphys)
        self._inflow = PM.inflow_faces(dirFrom, self._o.get('sideInflowDeg') or 0.0)
        self._writeParams()
        ref, applied = self._flowRef, self._applied
        reinit = False
        if ref and applied and self._o.get('metReinit') is not False:
            ang = lambda a, b: abs(math.fmod(a - b + 540, 360) - 180)
            turn = max(ang(dirFrom, ref['dir']), ang(dirFrom, applied['dir']))
            tol = self._o.get('dirTol') if self._o.get('dirTol') is not None else PM.DIR_TOL
            if u10 > PM.CALM and max(ref['u'], applied['u']) > PM.CALM and turn > tol:
                reinit = True
        self._applied = dict(dir=dirFrom, u=u10)
        if not ref or reinit:
            self._flowRef = dict(dir=dirFrom, u=u10)
        if reinit:
            self._reinitFlow()
            self.flowReinits += 1

    def _reinitFlow(self):
        """f -> equilibrium with the current inflow profile in both population buffers; theta kept."""
        self._dev.init_flow()

    def _advanceFlowRef(self, n):
        ref, ap = self._flowRef, self._applied
        if not ref or not ap:
            return
        a = 1 - math.exp(-n * self._dt / PM.ADJ_TAU_S)
        ref['dir'] = _mod360(ref['dir'] + (math.fmod(ap['dir'] - ref['dir'] + 540, 360) - 180) * a)
        ref['u'] += (ap['u'] - ref['u']) * a

    def setExistingFlux(self, wm2):
        """W per m^2 of operational data-center roof (solver.js:305-310)."""
        self._check()
        try:
            v = float(wm2)
        except (TypeError, ValueError):
            v = 0.0
        self._flux = max(0.0, v if math.isfinite(v) else 0.0)
        self.info['heatExistingMW'] = self.info['dcRoofArea_m2'] * self._flux / 1e6
        self._writeColumns()

    def setNewCampuses(self, lst):
        """[{ id, halls: [[x0, z0, x1, z1], ...] (scene metres), mw }] — replaces the previous list
        (solver.js:313-320)."""
        self._check()
        self._campuses = [dict(id=c.get('id'), mw=float(c.get('mw') or 0),
                               halls=[[float(v) for v in list(h)[:4]] for h in (c.get('halls') or [])])
                          for c in (lst or [])]
        d = self._dom
        self._ras = D.rasterize_campuses(self._campuses, d.dx, d.nx, d.ny)
        self.campusInfo = self._ras.info
        self._setGeometry(False)

    def _setGeometry(self, first):
        """geometry (kt/ktop with the campus rule of build_domain) + per-column source; uploads what changed
        (solver.js:323-356)."""
        nx, ny, nz = self._dom.nx, self._dom.ny, self._dom.nz
        dom = D.build_domain(self._agg, heightM=self._o['heightM'], newArea=self._ras.newArea, nzMin=nz)
        oldKtopS = self._ktopS
        self._ktS = D.flip_rows(dom.kt, nx, ny)
        self._ktopS = D.flip_rows(dom.ktop, nx, ny)
        self._cdS = D.flip_rows(dom.cd, nx, ny)
        self.grid = dict(ktop=dom.ktop, kt=dom.kt, nb=dom.nb, demMean=dom.dem.astype(np.float32), zbase=dom.zbase,
                         dx=dom.dx, nx=nx, ny=ny, nz=nz)
        changed = first or bool((self._ktopS != oldKtopS).any())
        if changed:
            oldk = None
            if not first and bool((self._ktopS < oldKtopS).any()):
                oldk = oldKtopS.astype(np.uint32)
            self._dev.set_ktop(self._ktopS.astype(np.uint32), oldk)
            self.info['nFluid'] = int((nz - self._ktopS.astype(np.int64)).sum())
        self._writeColumns()

    def _writeColumns(self):
        d = self._dom
        colv, totalW, q = PM.pack_columns(self._ktS, self._ktopS, self._cdS, self._agg.dcarea, self._flux,
                                          self._ras.heatW, d.nx, d.ny, d.dx, self._dt)
        self._colv, self._q = colv, q
        self._heatMW = totalW / 1e6
        self._dev.set_columns(colv)

    # ------------------------------------------------------------------ state (solver.js:380-427)
    def resetHeat(self):
        """theta -> 0 everywhere, flow kept, simTime -> 0."""
        self._check()
        self._dev.clear_heat()
        self._n = 0
        self._steps = 0

    def resetFlow(self):
        """full re-init: equilibrium with the inflow profile at the local height above terrain, theta -> 0,
        simTime -> 0."""
        self._check()
        self._dev.init_flow()
        self._dev.clear_heat()
        self._dev.set_parity(0)
        self._n = 0
        self._steps = 0
        if self._applied:
            self._flowRef = dict(self._applied)

    def step(self, n=1):
        """queue n steps; the Pending resolves when the device has finished them."""
        try:
            self._check()
        except LiveSolverError as e:
            return Pending(value=None, error=e)
        n = max(0, int(math.floor(n)))
        if n > 0:
            self._encodeSteps(n, 0)
        return self._dev.fence()

    def _encodeSteps(self, n, mode):
        self._dev.step(n, mode)
        self._n += n
        self._steps += n
        self._advanceFlowRef(n)

    # ------------------------------------------------------------------ read-back (solver.js:439-471)
    def read(self, vol=True, wind=True, volMax=3.0):
        """asynchronous snapshot of the current state; never blocks stepping."""
        self._check()
        vm = float(volMax) if (volMax is not None and float(volMax) > 0) else 3.0
        conv = np.float32(self._conv)
        volscale = np.float32(255 / vm)
        simTime, steps, heatMW = self.simTime, self._steps, self._heatMW
        nzv = self.nzv

        def finish(res):
            surf, u, v, vb, tmax = res
            return dict(simTime=simTime, surf=surf, u=u if wind else None, v=v if wind else None,
                        vol=vb if vol else None, volMax=vm, nzv=nzv, thetaMax=float(tmax), heatMW=heatMW,
                        steps=steps)
        return self._dev.read(conv, volscale, nzv, bool(vol), bool(wind), finish)

    def benchmark(self, nSteps=300):
        """steps the model (the state advances) and returns MLUPS (all nx*ny*nz cells) (solver.js:474-483)."""
        self._check()
        self.step(min(20, nSteps)).result()
        t0 = time.perf_counter()
        left = nSteps
        while left > 0:
            m = min(left, 500)
            self._encodeSteps(m, 0)
            left -= m
        self._dev.sync()
        ms = (time.perf_counter() - t0) * 1e3
        return self.info['nCells'] * nSteps / (ms * 1e3)

    def destroy(self):
        if self._destroyed:
            return
        if self._dev is not None:
            self._dev.destroy()     # raises, and the solver stays usable, while it belongs to a live batch
        self._destroyed = True
        self._dev = None

    # ------------------------------------------------------------------ validation hooks (solver.js:496-578)
    @property
    def _dbg(self):
        if self.__dbg is None:
            self.__dbg = _Dbg(self)
        return self.__dbg


class _Dbg:
    """The reference's _dbg hooks (not part of the app interface)."""

    def __init__(self, s: LiveSolver):
        self.s = s

    def domain(self):
        s = self.s
        p = PM.unpack_params(s._params, s._dom.nz)
        return dict(nx=s._dom.nx, ny=s._dom.ny, nz=s._dom.nz, dx=s._dom.dx, zbase=s._dom.zbase, dt=s._dt,
                    conv=s._conv,
                    params={k: p[k] for k in ('tau0', 'cs2smag', 'gbeta', 'prt', 'kfloor', 'momfac', 'srcscale',
                                              'sigmax', 'nsp', 'nsw', 'oclip')},
                    inflow=dict(s._inflow), met=dict(s._met), uin=s._prof['ul'], vin=s._prof['vl'],
                    kbg=s._prof['kl'], Kphys=list(s._prof['Kphys']),
                    kt=s._colv[:, 0].astype(np.int16), ktop=s._colv[:, 1].astype(np.int16),
                    cd=s._colv[:, 2].view(np.float32).copy(), q=s._colv[:, 3].view(np.float32).copy(),
                    heatMW=s._heatMW, parity=s._dev.parity(), steps=s._steps, campusInfo=s.campusInfo,
                    params_block=s._params, colv=s._colv, ktopS=s._ktopS.astype(np.uint32))

    def readState(self):
        self.s._check()
        f, g = self.s._dev.read_state()
        return dict(f=f, g=g)

    def writeState(self, f=None, g=None):
        self.s._check()
        self.s._dev.write_state(f, g)

    def readDbg(self):
        self.s._check()
        return self.s._dev.read_dbg()

    def clearDbg(self):
        self.s._check()
        self.s._dev.clear_dbg()

    def stepOut(self, n):
        """n steps; the last one writes (theta, ux, uy, uz) of every fluid cell to the debug buffer."""
        s = self.s
        s._check()
        if n > 1:
            s._encodeSteps(n - 1, 0)
        s._encodeSteps(1, 1)
        return s._dev.fence()

    def stepAcc(self, n):
        """n steps accumulating (theta, ux, uy, uz) into the debug buffer."""
        s = self.s
        s._check()
        s._encodeSteps(n, 2)
        return s._dev.fence()

    def stats(self):
        s = self.s
        s._check()
        st = s._dev.stats()
        nf = st['count']
        dx, c = s._dom.dx, s._conv
        return dict(simTime=s.simTime, steps=s._steps, nFluid=nf, nonFinite=st['nonFinite'],
                    thetaMax=st['thetaMax'], heatContentMJ=st['sumTheta'] * PM.RHO_CP * dx * dx * dx / 1e6,
                    keMean=st['sumKE'] / max(nf, 1) * c * c, rhoDevMean=st['sumRhoDev'] / max(nf, 1),
                    umax=st['umax'] * c)


def _validate(opts):
    """option defaults and checks of createLiveSolver (solver.js:44-54)."""
    o = dict(base=None, dx=30, u10Max=8, heightM=720, onProgress=lambda t, f: None, device=None)
    o.update({k: v for k, v in opts.items() if v is not None or k in ('nsp', 'nsw')})
    try:
        dx = float(o['dx'])
    except (TypeError, ValueError):
        dx = float('nan')
    if dx not in _DXS and not o.get('allowAnyDx'):
        raise LiveSolverError(f"live solver: dx must be 20, 30 or 40 m (got {_jsnum(opts.get('dx', o['dx']))})")
    o['dx'] = dx
    try:
        o['u10Max'] = float(o['u10Max'])
    except (TypeError, ValueError):
        o['u10Max'] = float('nan')
    try:
        o['heightM'] = float(o['heightM'])
    except (TypeError, ValueError):
        o['heightM'] = float('nan')
    if not (1 <= o['u10Max'] <= 20):
        raise LiveSolverError(f"live solver: u10Max must be within 1-20 m/s (got {_jsnum(opts.get('u10Max'))})")
    if not (300 <= o['heightM'] <= 2000):
        raise LiveSolverError(f"live solver: heightM must be within 300-2000 m (got {_jsnum(opts.get('heightM'))})")
    return o


def create_live_solver(backend=None, **opts):
    """createLiveSolver(opts) of the reference (solver.js:44-101). Options: base (directory of static10.json +
    static10.bin.gz), static (an in-memory Static10, e.g. a seeded synthetic domain, instead of base), dx, u10Max,
    heightM, onProgress, device (CUDA device ordinal), met, existingFlux, nsp, nsw, outflowClip, sideInflowDeg,
    metReinit, dirTol, allowAnyDx, alpha (power-law exponent; the reference's constant is 0.14), precision
    ('fp32' | 'fp16' | 'bf16' | 'fp64').

    `backend` (optional) is a factory (nx, ny, nz) -> device object implementing the device protocol of
    cuda_device.CudaDevice; by default the CUDA backend is used and an unavailable GPU or library is an error.
    """
    o = _validate(opts)
    prog = o['onProgress']

    def p(t, f):
        try:
            prog(t, f)
        except Exception:
            pass
    p('Loading terrain and buildings', 0.05)
    st = o.get('static')
    if st is None:
        if o.get('base') is None:
            raise LiveSolverError('live solver: no static10 input (pass base=<dir> or static=<Static10>)')
        st = D.load_static10(o['base'])
    dx = o['dx']
    p(f'Building the {_jsnum(dx)} m grid', 0.2)
    agg = D.aggregate(st, dx)
    dom0 = D.build_domain(agg, heightM=o['heightM'])
    if backend is None:
        from .cuda_device import CudaDevice

        def backend(nx, ny, nz):
            return CudaDevice(nx, ny, nz, device=o.get('device'), precision=o.get('precision', 'fp32'))
    s = LiveSolver(o, st, agg, dom0, backend, p)
    try:
        s._init()
    except Exception:
        s.destroy()
        raise
    p('Ready', 1)
    return s


# the reference's spelling
createLiveSolver = create_live_solver


class LiveBatch:
    """Steps several live solvers together: one persistent launch per step for all of them, replayed two steps at a
    time from a CUDA graph (libahx ahx_batch_*). No counterpart in the reference, which runs one solver per device;
    each member's state after batch.step(n) is bit-identical to member.step(n).

    Members must use the CUDA backend with the same device, precision and arithmetic; their grids may differ. They
    stay fully usable on their own (setMet, setExistingFlux, read, step ...), ordered against the batch's steps. A
    member cannot be destroyed while it belongs to a live batch: destroy the batch first."""

    def __init__(self, solvers):
        from .cuda_device import Batch, CudaDevice
        self.solvers = list(solvers)
        if not self.solvers:
            raise LiveSolverError('live solver: a batch needs at least one solver')
        for s in self.solvers:
            s._check()
            if not isinstance(s._dev, CudaDevice):
                raise LiveSolverError('live solver: batched stepping needs the CUDA backend')
        try:
            self._b = Batch([s._dev for s in self.solvers])
        except Exception as e:
            raise LiveSolverError(str(e)) from None

    @property
    def info(self):
        return self._b.info()

    def set_members(self, solvers):
        """replace the member list (possibly empty); ordered after the batch's queued steps, no synchronisation."""
        from .cuda_device import CudaDevice
        solvers = list(solvers)
        for s in solvers:
            s._check()
            if not isinstance(s._dev, CudaDevice):
                raise LiveSolverError('live solver: batched stepping needs the CUDA backend')
        try:
            self._b.set_members([s._dev for s in solvers])
        except Exception as e:
            raise LiveSolverError(str(e)) from None
        self.solvers = solvers

    def _advance(self, n):
        for s in self.solvers:
            s._n += n
            s._steps += n
            s._advanceFlowRef(n)

    def step(self, n=1):
        """queue n steps of every member; the Pending resolves when the device has finished them."""
        n = max(0, int(math.floor(n)))
        if self._b is None:
            return Pending(value=None, error=LiveSolverError('live solver: batch destroyed'))
        try:
            if n > 0 and self.solvers:
                self._b.step(n)
        except Exception as e:
            return Pending(value=None, error=LiveSolverError(str(e)))
        if not self.solvers:
            return Pending(value=None)
        self._advance(n)
        # every member's stream waits for the batch, so a fence on one member resolves after the batched steps
        return self.solvers[0]._dev.fence()

    def benchmark(self, n=50):
        """n batched steps timed on the device; returns aggregate MLUPS over all members' cells."""
        n = max(1, int(n))
        ms = self._b.time_steps(n)
        self._advance(n)
        return self._b.info()['cells'] * n / (ms * 1e-3) / 1e6

    def set_launch(self, minb=0, zslab=0, use_graph=True, pairs=None):
        """register-budget variant (4 / 5 / 6, 0 = keep), tile depth (levels, 0 = keep, -1 = whole columns), graph
        replay on or off, paired levels on packed f32x2 arithmetic (None = keep). use_graph='branches' steps each
        member with its own solo kernel and launch shape on parallel branches of one graph instead of the persistent
        launch."""
        self._b.set_launch(minb, zslab, use_graph, pairs)

    def autotune(self, steps_per_trial=4):
        """time the register-budget variants x tile depths on the batch itself and keep the fastest. Like
        benchmark(), the trials advance every member's state (by up to 25 x (2 + steps_per_trial) steps). The last
        candidate is the branch mode (each member's own launch shape, so tune the members first)."""
        paired = (False, True) if self.solvers[0]._dev.arith == 'fast' and self.solvers[0]._dev.precision != 'fp64' \
            else (False,)
        best = None
        for pr in paired:
            for minb in (4, 5, 6):
                for zs in (2, 4, 8, 16):
                    self._b.set_launch(minb, zs, True, pr)
                    self._b.time_steps(2)
                    ms = self._b.time_steps(steps_per_trial)
                    self._advance(2 + steps_per_trial)
                    if best is None or ms < best[0]:
                        best = (ms, minb, zs, pr)
        # each member's own tuned kernel on parallel graph branches
        self._b.set_launch(0, 0, 'branches', None)
        self._b.time_steps(2)
        ms = self._b.time_steps(steps_per_trial)
        self._advance(2 + steps_per_trial)
        if ms < best[0]:
            return dict(mode='branches', ms_per_step=ms / steps_per_trial)
        self._b.set_launch(best[1], best[2], True, best[3])
        return dict(mode='persistent', minb=best[1], zslab=best[2], pairs=best[3], ms_per_step=best[0] / steps_per_trial)

    def destroy(self):
        """release the batch (idempotent); the members stay alive."""
        if self._b is not None:
            self._b.destroy()
            self._b = None
