"""Serving loop with continuous batching over the live solver.

A request is one scenario of the live page (js/live.js drives one at a time: setMet, setExistingFlux,
setNewCampuses, then step until a simulated time, then read()). The server runs many at once on one device.

NativeServer (the default, `Server`): the scheduler is the C ABI server inside libahx.so (ahx_server_*). The host side
here builds each request's byte images exactly as a fresh solver would upload them (a LiveSolver over a recording
device replays setMet / setExistingFlux / setNewCampuses / resetFlow) and submits them when the request arrives; the
library admits requests under a resident-cell budget and the device-memory budget, steps the active ones together in
batched chunks (continuous batching: the member list changes between chunks) and answers each with its read-back.

HostServer: the same policy as a Python loop over LiveBatch (or any batch object with the LiveBatch protocol), for
backends without the C ABI server (the CPU oracle in host-logic tests):
- admission: an arrived request takes a solver slot of its grid class (a recycled one, or a new one while the
  device-memory budget allows) as long as the resident cells stay under `max_cells`; otherwise it queues (FIFO);
- a slot is configured exactly like a fresh page would be: setMet, setExistingFlux, setNewCampuses, resetFlow;
- the active slots are stepped together by one batch in chunks of at most `chunk` steps, never past any member's
  remaining steps; the member list follows the active slots at chunk boundaries;
- chunks are queued ahead (up to `depth` in flight) so admission, set-up uploads and read-back overlap the device;
- a finished request is answered with read() (surface theta, u, v and the u8 volume) and its slot returns to the
  pool of its class once that read has arrived.

Each request's answer is bit-identical to running its scenario alone on a fresh solver (the batched step is).
The reference has no server.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import domain as D
from . import solver as S


@dataclass
class Request:
    id: int
    arrival: float            # seconds after the trace start
    dx: float
    heightM: float
    met: dict
    flux: float
    campus: dict
    sim_s: float = 600.0
    steps: int = 0            # filled at admission from the slot's dt
    cells: int = 0            # nx * ny * nz of the request's grid, filled at admission
    # filled by the server
    admitted: float = math.nan
    done: float = math.nan
    result: dict = field(default=None, repr=False)


class _Slot:
    def __init__(self, solver, key):
        self.solver = solver
        self.key = key
        self.req = None
        self.left = 0
        self.bytes = 0


def _state_bytes(solver):
    try:
        return int(solver._dev.info()['state_bytes'])
    except Exception:
        return solver.info['nCells'] * 52 * 4


# launch of the serving batch on B200: each request's own tuned step kernel on parallel graph branches, measured
# 2-3 % above the best persistent launch (96-register variant, 8-level tiles) on the 40/40/20 % mix of 40 / 30 / 20 m
# requests
DEFAULT_BATCH_LAUNCH = dict(use_graph='branches')


class HostServer:
    """Continuous-batching server on one device, scheduled by this Python loop. `backend` builds a solver's device (CudaDevice by default);
    `batch_factory(solvers)` returns an object with step(n) -> Pending, set_members(solvers) and destroy()
    (LiveBatch by default); `batch_launch` holds its set_launch keywords (DEFAULT_BATCH_LAUNCH with LiveBatch, none
    with another factory unless given). `tune_slots` runs the launch-shape tuner on the first slot of each grid class
    and gives later slots of the class the same shape, which the branch mode of the batch steps them with (default:
    on in branch mode)."""

    def __init__(self, static, backend=None, batch_factory=None, max_cells=64_000_000, chunk=64, u10Max=8.0,
                 hbm_budget_bytes=None, depth=2, clock=time.perf_counter, sleep=time.sleep, batch_launch=None,
                 tune_slots=None):
        self.static = static
        self.class_launch: dict = {}
        self.backend = backend
        self.batch_factory = batch_factory or S.LiveBatch
        if batch_launch is None and batch_factory is None:
            batch_launch = DEFAULT_BATCH_LAUNCH
        self.batch_launch = dict(batch_launch) if batch_launch else None   # LiveBatch.set_launch keywords
        if tune_slots is None:
            tune_slots = bool(self.batch_launch) and self.batch_launch.get('use_graph') == 'branches'
        self.tune_slots = bool(tune_slots)   # tune the first slot of each grid class, reuse its launch shape
        self.max_cells = int(max_cells)
        self.chunk = int(chunk)
        self.depth = max(1, int(depth))
        self.u10Max = u10Max
        self.hbm_budget = hbm_budget_bytes
        self.clock, self.sleep = clock, sleep
        self.pool: dict = {}          # grid class -> idle slots
        self.slots: list = []         # every slot created
        self.active: list = []
        self.batch = None
        self.batch_members = None
        self.bytes_used = 0
        self.cell_updates = 0
        self.launch_chunks = 0
        self.rebuilds = 0
        self.evictions = 0
        self.batch_steps = 0
        self.chunk_log: list = []     # per chunk: [issued s, steps, resident cells, members, finished s (observed)]

    # ---------------------------------------------------------------- slots
    def _new_solver(self, r: Request):
        s = S.create_live_solver(backend=self.backend, static=self.static, dx=r.dx, allowAnyDx=True,
                                 heightM=r.heightM, u10Max=self.u10Max, met=r.met, existingFlux=r.flux)
        if self.tune_slots:
            key = (r.dx, r.heightM)
            if key not in self.class_launch:
                by, zs, _ = s._dev.autotune(3)          # trials run on a scratch copy of the state
                self.class_launch[key] = (by, zs)
            else:
                s._dev.set_launch(*self.class_launch[key])
        return s

    def _take_slot(self, r: Request):
        key = (r.dx, r.heightM)
        idle = self.pool.get(key)
        if idle:
            return idle.pop()
        if self.hbm_budget is not None:
            need = self._class_cells(r) * self._bytes_per_cell()
            while self.bytes_used + need > self.hbm_budget and self._evict_idle():
                pass
            if self.bytes_used + need > self.hbm_budget and self.slots:
                return None
        s = self._new_solver(r)
        slot = _Slot(s, key)
        slot.bytes = _state_bytes(s)
        self.bytes_used += slot.bytes
        self.slots.append(slot)
        return slot

    def prewarm(self, template: Request, n: int):
        """create n idle slots of template's grid class up front (solver, device buffers, read-back staging), as a
        server keeps a warm pool; stops early when the memory budget is reached."""
        made = 0
        for _ in range(int(n)):
            if self.hbm_budget is not None and self.slots:
                need = self._class_cells(template) * self._bytes_per_cell()
                if self.bytes_used + need > self.hbm_budget:
                    break
            s = self._new_solver(template)
            slot = _Slot(s, (template.dx, template.heightM))
            slot.bytes = _state_bytes(s)
            self.bytes_used += slot.bytes
            self.slots.append(slot)
            self.pool.setdefault(slot.key, []).append(slot)
            made += 1
        return made

    def _bytes_per_cell(self):
        for sl in self.slots:
            return sl.bytes / sl.solver.info['nCells']
        return 208.0

    def _evict_idle(self):
        """free one idle slot of any class (idle slots are never batch members: the member list follows the active
        slots as soon as requests finish)."""
        for key, idle in self.pool.items():
            if idle:
                sl = idle.pop()
                sl.solver.destroy()
                self.slots.remove(sl)
                self.bytes_used -= sl.bytes
                self.evictions += 1
                return True
        return False

    def _configure(self, slot: _Slot, r: Request):
        s = slot.solver
        s.setMet(r.met)
        s.setExistingFlux(r.flux)
        s.setNewCampuses([r.campus])
        s.resetFlow()
        r.steps = int(math.ceil(r.sim_s / s.info['dt'] - 1e-9))
        r.cells = int(s.info['nCells'])
        slot.req, slot.left = r, r.steps

    def _cells(self):
        return sum(sl.solver.info['nCells'] for sl in self.active)

    def _class_cells(self, r: Request):
        idle = self.pool.get((r.dx, r.heightM))
        if idle:
            return idle[-1].solver.info['nCells']
        for sl in self.slots:
            if sl.key == (r.dx, r.heightM):
                return sl.solver.info['nCells']
        nx = int(round(6000 / r.dx))
        return nx * nx * int(round(r.heightM / r.dx))

    # ---------------------------------------------------------------- batch
    def _sync_members(self):
        """keep the batch's member list equal to the active slots (stream-ordered; no synchronisation)."""
        members = [sl.solver for sl in self.active]
        if self.batch_members == members:
            return
        if self.batch is None:
            if not members:
                return
            self.batch = self.batch_factory(members)
            if self.batch_launch:
                self.batch.set_launch(**self.batch_launch)
        else:
            self.batch.set_members(members)
        self.batch_members = members
        self.rebuilds += 1

    def _poll(self, draining, done, t0, block=False):
        """retire finished requests whose read-back has arrived (all of them when block)."""
        keep = []
        for sl, p in draining:
            if block or p.done():
                sl.req.result = p.result()
                sl.req.done = self.clock() - t0
                done.append(sl.req)
                sl.req = None
                self.pool.setdefault(sl.key, []).append(sl)
            else:
                keep.append((sl, p))
        draining[:] = keep

    # ---------------------------------------------------------------- main loop
    def run(self, requests, timeout_s=None):
        """Serve `requests` in real time (arrival times relative to the call); returns the statistics dict. Raises
        TimeoutError if the trace is not finished within timeout_s seconds (None: no bound)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        queue: list = []
        nxt = 0
        t0 = self.clock()
        done: list = []
        inflight: list = []      # fences of queued chunks, oldest first
        draining: list = []      # (slot, read Pending) of finished requests
        while len(done) < len(reqs):
            now = self.clock() - t0
            if timeout_s is not None and now > timeout_s:
                raise TimeoutError(f'serving: {len(done)} of {len(reqs)} requests answered after {now:.1f} s')
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                queue.append(reqs[nxt])
                nxt += 1
            # admission (FIFO) while cells and memory allow; the first request is always admitted
            while queue:
                r = queue[0]
                if self.active and self._cells() + self._class_cells(r) > self.max_cells:
                    break
                slot = self._take_slot(r)
                if slot is None:
                    break
                queue.pop(0)
                self._configure(slot, r)
                r.admitted = self.clock() - t0
                self.active.append(slot)
            if self.active:
                self._sync_members()
                k = min(self.chunk, min(sl.left for sl in self.active))
                inflight.append(self.batch.step(k))
                self.chunk_log.append([self.clock() - t0, k, self._cells(), len(self.active), math.nan])
                inflight[-1].log = self.chunk_log[-1]
                self.launch_chunks += 1
                self.batch_steps += k
                self.cell_updates += k * self._cells()
                finished = [sl for sl in self.active if sl.left == k]
                for sl in self.active:
                    sl.left -= k
                for sl in finished:
                    # ordered after this chunk on the member's own stream
                    draining.append((sl, sl.solver.read(vol=True, wind=True)))
                    self.active.remove(sl)
                if finished:
                    self._sync_members()   # leavers are released now, so idle slots can be evicted safely
            # keep at most `depth` chunks queued; retire read-backs while waiting
            while inflight and (len(inflight) > self.depth or not self.active):
                if inflight[0].done():
                    p = inflight.pop(0)
                    p.result()
                    if getattr(p, 'log', None) is not None:
                        p.log[4] = self.clock() - t0
                    continue
                if timeout_s is not None and self.clock() - t0 > timeout_s:
                    raise TimeoutError(f'serving: a chunk did not finish within {timeout_s} s')
                self._poll(draining, done, t0)
                self.sleep(0.0002)
            self._poll(draining, done, t0)
            if not self.active:
                if draining:
                    self.sleep(0.0002)
                elif not queue and nxt < len(reqs):
                    self.sleep(max(0.0, min(0.01, reqs[nxt].arrival - (self.clock() - t0))))
        for p in inflight:
            p.result()
        makespan = self.clock() - t0
        return self._stats(reqs, makespan)

    def _stats(self, reqs, makespan):
        lat = np.array([r.done - r.arrival for r in reqs])
        qd = np.array([r.admitted - r.arrival for r in reqs])
        upd = self.cell_updates
        return dict(requests=len(reqs), makespan_s=makespan, cell_updates=int(upd),
                    glups=upd / makespan / 1e9 if makespan > 0 else 0.0,
                    latency_p50_s=float(np.percentile(lat, 50)), latency_p99_s=float(np.percentile(lat, 99)),
                    latency_mean_s=float(lat.mean()), queue_p50_s=float(np.percentile(qd, 50)),
                    queue_p99_s=float(np.percentile(qd, 99)), chunks=self.launch_chunks, batch_rebuilds=self.rebuilds,
                    slots=len(self.slots), slot_bytes=self.bytes_used, evictions=self.evictions,
                    batch_steps=self.batch_steps)

    def close(self):
        if self.batch is not None:
            self.batch.destroy()
            self.batch = None
        self.batch_members = None
        for sl in self.slots:
            sl.solver.destroy()
        self.slots, self.pool, self.active = [], {}, []


def requests_from_trace(trace, sim_s=600.0):
    """scenarios.serve_trace entries -> Request objects."""
    return [Request(id=t['id'], arrival=t['arrival'], dx=t['dx'], heightM=t['heightM'], met=dict(t['met']),
                    flux=t['flux'], campus=t['campus'], sim_s=sim_s) for t in trace]


def fifo_serial(requests, seconds_of):
    """Latencies of the same requests solved one after another in arrival order (a single FIFO server whose service
    time for request r is seconds_of(r)); returns (latencies, makespan)."""
    t = 0.0
    lat = []
    start = min(r.arrival for r in requests)
    for r in sorted(requests, key=lambda r: r.arrival):
        t = max(t, r.arrival) + seconds_of(r)
        lat.append(t - r.arrival)
    return np.array(lat), t - start


class SequentialBatch:
    """A stand-in batch that steps each member on its own (for backends without batched stepping, e.g. the CPU
    oracle in host-logic tests); same step(n) -> Pending / set_members / destroy() protocol as LiveBatch."""

    def __init__(self, solvers):
        self.solvers = list(solvers)

    def set_members(self, solvers):
        self.solvers = list(solvers)

    def step(self, n):
        p = S.Pending(value=None)
        for s in self.solvers:
            p = s.step(n)
            p.result()
        return p

    def destroy(self):
        self.solvers = []


class ImageRecorder:
    """A device for LiveSolver that keeps the byte images the solver uploads (parameter block, column records, ktop
    plane) instead of running anything: the host half of a request whose device half is the C ABI server."""

    adapter = 'image recorder (no device)'

    def __init__(self, nx, ny, nz):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.params = None
        self.colv = None
        self.ktop = None

    def set_params(self, b):
        self.params = bytes(b)

    def set_columns(self, colv):
        self.colv = np.array(colv, np.uint32, copy=True)

    def set_ktop(self, ktop, old=None):
        self.ktop = np.array(ktop, np.uint32, copy=True)

    def init_flow(self):
        pass

    def clear_heat(self):
        pass

    def set_parity(self, p):
        pass

    def sync(self):
        pass

    def lost(self):
        return None

    def fence(self):
        return S.Pending(value=None)

    def step(self, n, mode):
        raise S.LiveSolverError('live solver: an image recorder does not step')

    def destroy(self):
        pass


class NativeServer:
    """Continuous batching by the C ABI server (ahx_server_*). `run(requests)` replays a trace in real time: each
    request's images are built and submitted at its arrival time, answers are collected as the server finishes them.
    The request objects get `admitted` / `done` (seconds after the run started), `steps`, `cells` and `result` (the
    read() dict a solver would return: simTime, surf, u, v, vol, volMax, nzv, thetaMax, heatMW, steps)."""

    def __init__(self, static, precision='fp32', arith='fast', device=None, max_cells=24_000_000, chunk=256,
                 hbm_budget_bytes=None, batch_mode='branches', tune=True, depth=2, u10Max=8.0, volMax=3.0,
                 gpu_domain=True, clock=time.perf_counter, sleep=time.sleep):
        from .cuda_device import Server as CServer
        self.static = static
        self.u10Max = u10Max
        self.volMax = float(volMax)
        self.clock, self.sleep = clock, sleep
        self.srv = CServer(device=device, precision=precision, arith=arith, chunk=chunk, max_cells=max_cells,
                           hbm_budget_bytes=hbm_budget_bytes or 0, batch_mode=batch_mode, tune=tune, depth=depth)
        self.templates: dict = {}      # grid class -> LiveSolver over an ImageRecorder
        self.batch_launch = dict(mode=batch_mode, tune=bool(tune))
        self.max_cells, self.chunk = int(max_cells), int(chunk)
        self.hbm_budget = self.srv.stats()['hbm_budget_bytes']
        self.host_s = 0.0              # host time spent building images
        # per-request geometry (campus raster, building rule, column records) by the GPU domain builder; the
        # parameter block (met) stays on the host
        self.gdom = None
        if gpu_domain:
            from .gpu_domain import GpuDomain
            self.gdom = GpuDomain(static, device=device)

    def images(self, r: Request):
        """The byte images and read-back settings a fresh solver configured for r would use."""
        key = (r.dx, r.heightM)
        s = self.templates.get(key)
        if s is None:
            s = S.create_live_solver(backend=ImageRecorder, static=self.static, dx=r.dx, allowAnyDx=True,
                                     heightM=r.heightM, u10Max=self.u10Max, met=r.met, existingFlux=r.flux)
            self.templates[key] = s
        dt = s.info['dt']
        nx, ny, nz = s.info['nx'], s.info['ny'], s.info['nz']
        s.setMet(r.met)
        rec = s._dev
        if self.gdom is not None:
            g = self.gdom.build(r.dx, heightM=r.heightM, campuses=[r.campus], flux=r.flux, dt=dt, nzMin=nz)
            if g['nz'] == nz:
                # heat of the request: the sequential sum over solver rows of existing + campus W (solver.js:359-376)
                Wn = s._agg.dcarea * float(r.flux) + g['heatW']
                totalW = float(np.cumsum(D.flip_rows(Wn, nx, ny))[-1])
                return dict(nx=nx, ny=ny, nz=nz, params=rec.params, colv=g['colv'], ktop=g['ktop'],
                            conv=np.float32(s._conv), volscale=np.float32(255 / self.volMax), nzv=s.nzv, dt=dt,
                            heatMW=totalW / 1e6, steps=int(math.ceil(r.sim_s / dt - 1e-9)))
        s.setExistingFlux(r.flux)
        s.setNewCampuses([r.campus])
        s.resetFlow()
        return dict(nx=nx, ny=ny, nz=nz, params=rec.params, colv=rec.colv, ktop=rec.ktop, conv=np.float32(s._conv),
                    volscale=np.float32(255 / self.volMax), nzv=s.nzv, dt=dt, heatMW=s._heatMW,
                    steps=int(math.ceil(r.sim_s / dt - 1e-9)))

    def submit(self, r: Request):
        t = self.clock()
        im = self.images(r)
        self.host_s += self.clock() - t
        r.steps = im['steps']
        r.cells = im['nx'] * im['ny'] * im['nz']
        ticket = self.srv.submit(im['nx'], im['ny'], im['nz'], r.steps, im['params'], im['colv'], im['ktop'],
                                 im['conv'], im['volscale'], im['nzv'], True, True, tag=r.id)
        return ticket, im

    def _collect(self, ticket, im, r, t0, offset, timeout_ms=0):
        got = self.srv.poll(ticket, timeout_ms, im['nx'], im['ny'], im['nzv'], True, True)
        if got is None:
            return False
        info, surf, u, v, vol = got
        r.done = self.clock() - t0
        r.admitted = info.admitted_s - offset
        r.result = dict(simTime=r.steps * im['dt'], surf=surf, u=u, v=v, vol=vol, volMax=self.volMax, nzv=im['nzv'],
                        thetaMax=float(info.theta_max), heatMW=im['heatMW'], steps=r.steps)
        return True

    def run(self, requests, timeout_s=None):
        """Serve `requests` in real time (arrival times relative to the call); returns the statistics dict. Raises
        TimeoutError if the trace is not finished within timeout_s seconds (None: no bound)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        st0 = self.srv.stats()
        t0 = self.clock()
        offset = st0['elapsed_s'] + (self.clock() - t0)   # server clock at the run's start (to within a poll)
        nxt = 0
        open_: list = []
        done = 0
        while done < len(reqs):
            now = self.clock() - t0
            if timeout_s is not None and now > timeout_s:
                raise TimeoutError(f'serving: {done} of {len(reqs)} requests answered after {now:.1f} s')
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                r = reqs[nxt]
                ticket, im = self.submit(r)
                open_.append((ticket, im, r))
                nxt += 1
            keep = []
            for item in open_:
                if self._collect(item[0], item[1], item[2], t0, offset):
                    done += 1
                else:
                    keep.append(item)
            open_ = keep
            if done < len(reqs):
                wait = reqs[nxt].arrival - (self.clock() - t0) if nxt < len(reqs) else 0.002
                if open_ and not (nxt < len(reqs) and wait <= 0):
                    # block on the oldest open request until the next arrival (bounded)
                    ms = int(max(0.0, min(wait, 0.002)) * 1000)
                    ticket, im, r = open_[0]
                    if self._collect(ticket, im, r, t0, offset, timeout_ms=ms):
                        done += 1
                        open_.pop(0)
                elif not open_ and wait > 0:
                    self.sleep(min(wait, 0.01))
        makespan = self.clock() - t0
        st1 = self.srv.stats()
        lat = np.array([r.done - r.arrival for r in reqs])
        qd = np.array([r.admitted - r.arrival for r in reqs])
        upd = st1['cell_updates'] - st0['cell_updates']
        return dict(requests=len(reqs), makespan_s=makespan, cell_updates=int(upd),
                    glups=upd / makespan / 1e9 if makespan > 0 else 0.0,
                    latency_p50_s=float(np.percentile(lat, 50)), latency_p99_s=float(np.percentile(lat, 99)),
                    latency_mean_s=float(lat.mean()), queue_p50_s=float(np.percentile(qd, 50)),
                    queue_p99_s=float(np.percentile(qd, 99)), chunks=st1['chunks'] - st0['chunks'],
                    batch_steps=st1['batch_steps'] - st0['batch_steps'], slots=st1['slots'],
                    slot_bytes=st1['slot_bytes'], evictions=st1['evictions'] - st0['evictions'],
                    host_image_s=self.host_s)

    def stats(self):
        return self.srv.stats()

    def close(self):
        for s in self.templates.values():
            s.destroy()
        self.templates = {}
        if self.gdom is not None:
            self.gdom.destroy()
            self.gdom = None
        self.srv.destroy()


Server = NativeServer
