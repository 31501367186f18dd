#!/usr/bin/env python3
"""Benchmark of the fused D3Q19 + D3Q7 live-solver step on one B200 per rank.

Workload: the 600 x 600 x 64 domain at 10 m (23.04 M cells), seeded synthetic terrain and buildings (24 hills with
0-40 m relief, 4,000 buildings, 211 data-center roofs at 400 W/m^2), inflow 3.5 m/s from 200 deg with power-law
exponent 0.2, FP32 populations, pull scheme. Metric: GLUPS = all nx*ny*nz cells updated per second (the reference's
MLUPS convention, js/live/solver.js:482), whole job over all ranks.

`value` is device time (CUDA events on the solver's own stream) with the state resident in HBM; the state (4.8 GB)
is far larger than L2, so no flush is needed between steps. Warm-up is W untimed steps and then two more, so the
two-step CUDA graph the timed steps replay (one per starting parity) is captured before the clock starts. `e2e` runs the same stepping through the public API
(create_live_solver / setMet / step / read) with host buffers: every frame uploads a parameter block from host
memory, advances F steps and reads back the near-surface fields and the u8 volume, as the live app does.

--gpus N runs N independent replicas, one per rank (the path does not shard: "replicas only", weak scaling). Under
torchrun the ranks come from the environment; without it, --gpus N > 1 starts N ranks itself (torch.distributed.run
on 127.0.0.1, one process per GPU) and returns their exit status.
--impl reference times the CPU restatement of the reference kernels (the reference itself is WebGPU/WGSL and cannot
run here) on all host cores, rank 0 only; its line reports n_gpus 0 (no GPU takes part).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from ashburn_heat_twin_b200 import replicas as RP  # noqa: E402

WORKLOADS = {
    'c2': dict(desc='600x600x64 cells at 10 m (23.04 M), synthetic seed 2: 24 hills 0-40 m, 4000 buildings, '
                    '211 DC roofs', dx=10, heightM=640, met='C2_MET', spec='C2'),
    'c1': dict(desc='200x200x32 cells at 30 m (1.28 M), synthetic seed 1: 8 hills 0-30 m, 1500 buildings, '
                    '60 DC roofs', dx=30, heightM=960, met='C1_MET', spec='C1'),
    # the reference's own Ashburn planes (tests/golden/static10.*) at the grids its published step rates use
    # (js/live/README.md:226-238): 20 m 300x300x36, 30 m 200x200x24, 40 m 150x150x18; met of its validation page
    'r20': dict(desc='the Ashburn 6 km box at 20 m (300x300x36, 3.24 M cells), reference planes, validation met',
                dx=20, heightM=720, real=True, published_glups=4.28,
                published='RTX 4090 WebGPU 4,280 MLUPS, read() 4.2 / 9.9 ms median / max (js/live/README.md:232)'),
    'r30': dict(desc='the Ashburn 6 km box at 30 m (200x200x24, 0.96 M cells), reference planes, validation met',
                dx=30, heightM=720, real=True, published_glups=4.10,
                published='RTX 4090 WebGPU 4,100 MLUPS, read() 3.2 / 4.7 ms median / max (js/live/README.md:233)'),
    'r40': dict(desc='the Ashburn 6 km box at 40 m (150x150x18, 0.405 M cells), reference planes, validation met',
                dx=40, heightM=720, real=True, published_glups=6.60,
                published='RTX 4090 WebGPU 6,600 MLUPS, read() 3.0 / 5.3 ms median / max (js/live/README.md:234)'),
    'c2q': dict(desc='300x300x64 cells at 10 m (5.76 M), synthetic seed 3: 6 hills 0-40 m, 1000 buildings, '
                     '53 DC roofs', dx=10, heightM=640, met='C2_MET', spec='C2Q'),
    'c3': dict(desc='precision study on 600x600x64 at 10 m (config c2): FP32 / FP16 / BF16 / FP16 with stochastic '
                    'rounding / 16-bit f with f32 g storage against the FP64 build, cold start, 2 simulated minutes '
                    'of spin-up then a 10-minute mean', dx=10, heightM=640,
               met='C2_MET', spec='C2'),
    'c4': dict(desc='64 domains in one batch: 32 x 200x200x32 at 30 m + 32 x 150x150x24 at 40 m (58.2 M cells), '
                    'synthetic seed 1 box; per domain seeded wind (U[0,360) deg, U[2,8] m/s), roof flux U[200,600] '
                    'W/m2 and one 120 MW campus (300 x 300 m hall) at a building-free site', spec='C1'),
    'c5': dict(desc='serving: Poisson arrivals of live-solver requests, 40 % 150x150x24 at 40 m, 40 % 200x200x32 at '
                    '30 m, 20 % 300x300x48 at 20 m, 10 simulated minutes each (1,754 / 2,338 / 3,507 steps), seeded '
                    'wind, roof flux and one 120 MW campus per request, synthetic seed 1 box', spec='C1'),
}
METRIC = 'GLUPS (all cells) of the fused D3Q19+D3Q7 step, 600x600x64'
# algorithmic bytes per fluid-cell update: read + write of 19 f and 7 g populations at their storage widths
CELL_BYTES = {'fp32': 208, 'fp16': 104, 'bf16': 104, 'fp64': 416, 'fp16g32': 132, 'bf16g32': 132, 'fp16sr': 104}
DTYPE = {'fp32': 'f32', 'fp16': 'f16-store/f32', 'bf16': 'bf16-store/f32', 'fp64': 'f64',
         'fp16g32': 'f16-store f, f32-store g / f32', 'bf16g32': 'bf16-store f, f32-store g / f32',
         'fp16sr': 'f16-store (stochastic rounding) / f32'}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_solver(backend=None, device=None, precision='fp32', arith='exact', workload='c2'):
    from ashburn_heat_twin_b200 import solver as S
    from ashburn_heat_twin_b200 import synth
    w = WORKLOADS[workload]
    if w.get('real'):
        # the reference's validation settings (tests/live/validate.html:29,61-75): u10Max 8, alpha 0.14, flux 400
        kw = dict(base=os.path.join(ROOT, 'tests', 'golden'), dx=w['dx'], heightM=w['heightM'], u10Max=8,
                  met=dict(u10=3.09, dirFrom=210, wstar=1.67, blh=903, ustar=0.32), existingFlux=400)
    else:
        st = synth.make_static10(getattr(synth, w['spec']))
        kw = dict(static=st, dx=w['dx'], allowAnyDx=True, heightM=w['heightM'], u10Max=8, alpha=0.2,
                  met=getattr(synth, w['met']), existingFlux=400)
    if backend is None:
        from ashburn_heat_twin_b200.cuda_device import CudaDevice

        def backend(nx, ny, nz):
            return CudaDevice(nx, ny, nz, device=device, precision=precision, arith=arith)
    return S.create_live_solver(backend=backend, **kw)


def measured_peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        d = json.load(open(p))
        return float(d['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def profile_traffic(precision, launch, fluid):
    """DRAM bytes per launch of the step kernel from the committed ncu summaries of the same storage, arithmetic and
    launch shape (profiles/step_<precision>_traffic.json: one capture, or a list of captures of several launch
    shapes), scaled by fluid cells to this launch. Returns (bytes, source note); bytes is None when no capture of this
    launch shape exists."""
    p = os.path.join(ROOT, 'profiles', f'step_{precision}_traffic.json')
    try:
        caps = json.load(open(p))
    except Exception:
        return None, 'no ncu capture committed for this storage'
    caps = caps if isinstance(caps, list) else [caps]
    for d in caps:
        if launch is not None and tuple(launch) == (d.get('block_y'), d.get('zslab')):
            return d['dram_bytes_per_fluid_cell'] * fluid, (
                f"ncu dram__bytes_read.sum + dram__bytes_write.sum of the same launch shape on {d['grid']} "
                f"({d['dram_bytes_per_fluid_cell']:.1f} B per fluid cell), scaled by fluid cells")
    have = ', '.join(f"{d.get('block_y')} / zslab {d.get('zslab')}" for d in caps)
    return None, (f'the committed captures are of launch {have}, not the timed launch '
                  f'{launch[0] if launch else None} / zslab {launch[1] if launch else None}')


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile('w+', suffix='.csv', delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(['nvidia-smi', f'--query-gpu={self.Q}', '--format=csv,noheader,nounits',
                                       '-lms', '100', '-i', str(self.gpu)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        time.sleep(0.2)
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        try:
            rows = [r.split(',') for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        os.unlink(self.f.name)
        if not rows:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=['unsampled'])
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[5:9]) if v.strip() == 'Active'})
        return dict(sm_mhz=statistics.median(sm), sm_max_mhz=mx, reasons=reasons, samples=len(rows),
                    power_w_max=max(float(r[3]) for r in rows if r[3].strip().replace('.', '', 1).isdigit())
                    if any(r[3].strip().replace('.', '', 1).isdigit() for r in rows) else None)


def host_threads():
    """Host threads this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_baseline(seconds=10.0, max_steps=30, workload='c2'):
    """The oracle (CPU restatement of the reference kernels) on full steps of the workload, all host threads."""
    import numpy as np
    from oracle import oracle as O
    O.set_threads(host_threads())
    s = make_solver(backend=lambda nx, ny, nz: O.OracleDevice(nx, ny, nz), workload=workload)
    threads = O.max_threads()
    dev = s._dev
    t0 = time.perf_counter()
    dev.step(1, 0)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(max_steps, np.ceil(seconds / max(t1, 1e-3)))))
    t0 = time.perf_counter()
    dev.step(n, 0)
    t = time.perf_counter() - t0
    cells = s.info['nCells']
    s.destroy()
    return dict(value=cells * n / t / 1e9, unit='GLUPS', cores=threads, kind='port',
                sample=f'{n} full steps of the {s.info["nx"]}x{s.info["ny"]}x{s.info["nz"]} domain '
                       f'({cells * n / 1e6:.0f} M cell updates, {t:.1f} s)')


def bench_config(workload, precision, cells):
    """The config dict both arms print for a workload (identical keys and values for the same workload)."""
    return dict(workload=WORKLOADS[workload]['desc'], precision=precision, scheme='pull', parallelism='replicas',
                l2=f'inputs larger than L2, no flush: state {cells * CELL_BYTES[precision] / 1e9:.2f} GB per replica '
                   f'(both population buffers) against a 126 MB L2')


def run_reference(a, rank):
    if rank != 0:
        return 0
    import numpy as np
    from oracle import oracle as O
    O.set_threads(host_threads())   # every host thread, also under torchrun (which sets OMP_NUM_THREADS=1)
    s = make_solver(backend=lambda nx, ny, nz: O.OracleDevice(nx, ny, nz))
    dev = s._dev
    dev.step(a.warmup, 0)
    t0 = time.perf_counter()
    dev.step(a.steps, 0)
    t = time.perf_counter() - t0
    cells = s.info['nCells']
    v = cells * a.steps / t / 1e9
    out = dict(metric=METRIC, value=v, unit='GLUPS', n_gpus=0, steps=a.steps, warmup=a.warmup,
               ms_per_step=t / a.steps * 1e3, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f32',
               data='synthetic (seeded terrain and buildings; no public dataset involved)', impl='reference',
               devices=f'host CPU only ({O.max_threads()} threads, rank 0); no GPU takes part',
               config=bench_config('c2', 'fp32', cells),
               cpu_baseline=dict(value=v, unit='GLUPS', cores=O.max_threads(), kind='port',
                                 sample=f'{a.steps} full steps after {a.warmup} warm-up steps'),
               e2e=dict(value=v, unit='GLUPS', h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    s.destroy()
    del np
    print(json.dumps(out), flush=True)
    return 0


def warm_up(dev, n):
    """n untimed warm-up steps, then two more: the timed steps start at the parity (batch phase) the last two started
    at, so the two-step CUDA graph they replay is captured (a graph per starting parity) before the clock starts."""
    dev.time_steps(n)
    dev.time_steps(2)


def serial_time(solvers, steps):
    """Device time (ms) of `steps` steps of each solver, one solver after another: the serial arm of the batch
    comparisons. Each solver first takes two untimed steps from the parity its timed steps start at, so the two-step
    graph they replay is captured before its clock starts."""
    for s in solvers:
        s._dev.time_steps(2)
    return sum(s._dev.time_steps(steps) for s in solvers)


def secondary_rates(a, local):
    """Further device-timed measurements of the same run on one GPU, after the headline: the 16-bit storages on the
    same domain (FMA build, each on its own tuned launch; algorithmic bytes 104 B per fluid cell), and the 64-domain
    batched ensemble of the c4 workload (one batched launch sequence per step, against the same members stepped one
    after another)."""
    from ashburn_heat_twin_b200 import LiveBatch
    from ashburn_heat_twin_b200 import scenarios as SC
    from ashburn_heat_twin_b200 import solver as S
    from ashburn_heat_twin_b200 import synth
    from ashburn_heat_twin_b200.cuda_device import CudaDevice
    peak, peak_kind = measured_peaks()
    out = {}
    for p in ('fp16', 'fp16sr'):
        s = make_solver(device=local, precision=p, arith='fast', workload=a.workload)
        by, zs, _ = s._dev.autotune(3)
        warm_up(s._dev, a.warmup)
        ms = s._dev.time_steps(a.steps) / a.steps
        cells, fluid = s.info['nCells'], s.info['nFluid']
        traffic, traffic_src = profile_traffic(p, (by, zs), fluid)
        out[p] = dict(glups=cells / ms / 1e6, ms_per_step=ms, launch=dict(block_y=by, zslab=zs),
                      roofline=dict(bound='hbm', achieved=fluid * CELL_BYTES[p] / (ms / 1e3) / 1e9, peak=peak,
                                    unit='GB/s', frac=fluid * CELL_BYTES[p] / (ms / 1e3) / 1e9 / peak,
                                    traffic=traffic, traffic_source=traffic_src, peak_source=peak_kind),
                      dtype=DTYPE[p])
        s.destroy()
    st = synth.make_static10(synth.C1)
    scen = SC.batch64(st)

    def backend(nx, ny, nz):
        return CudaDevice(nx, ny, nz, device=local, precision='fp32', arith='fast')
    solvers = []
    for c in scen:
        s = S.create_live_solver(backend=backend, static=st, dx=c['dx'], heightM=c['heightM'], u10Max=8, met=c['met'],
                                 existingFlux=c['flux'])
        s.setNewCampuses([c['campus']])
        solvers.append(s)
    classes = {}
    for s in solvers:
        classes.setdefault((s.info['nx'], s.info['ny'], s.info['nz']), []).append(s)
    for members in classes.values():
        by, zs, _ = members[0]._dev.autotune(3)
        for m in members[1:]:
            m._dev.set_launch(by, zs)
    b = LiveBatch(solvers)
    btune = b.autotune(4)
    warm_up(b._b, a.warmup)
    ms = b._b.time_steps(a.steps) / a.steps
    serial_ms = serial_time(solvers, a.steps) / a.steps
    cells = sum(s.info['nCells'] for s in solvers)
    fluid = sum(s.info['nFluid'] for s in solvers)
    b.destroy()
    for s in solvers:
        s.destroy()
    out['batch64'] = dict(workload=WORKLOADS['c4']['desc'], glups=cells / ms / 1e6, ms_per_step=ms,
                          serial_glups=cells / serial_ms / 1e6, over_serial=serial_ms / ms, tuned=btune,
                          roofline_frac=fluid * 208 / (ms / 1e3) / 1e9 / peak, dtype='f32')
    return out


def main_batch(a, rank, world, local, dist, torch):
    """The batched workload: 64 seeded domains stepped by one persistent launch per step (a CUDA graph replays two
    steps); launch shapes tuned per grid class on scratch copies, then the batch's own variant and tile depth.
    Reports the aggregate rate, the same members stepped one after another (serial) for comparison, and an
    end-to-end frame rate through the public API."""
    from ashburn_heat_twin_b200 import LiveBatch
    from ashburn_heat_twin_b200 import scenarios as SC
    from ashburn_heat_twin_b200 import solver as S
    from ashburn_heat_twin_b200 import synth
    from ashburn_heat_twin_b200.cuda_device import CudaDevice
    st = synth.make_static10(synth.C1)
    scen = SC.batch64(st)
    if a.members < 64:   # a smaller batch with the same class mix (for profiling captures)
        half = a.members // 2
        scen = scen[:half] + scen[32:32 + a.members - half]

    def backend(nx, ny, nz):
        return CudaDevice(nx, ny, nz, device=local, precision=a.precision, arith=a.arith)

    solvers = []
    for c in scen:
        s = S.create_live_solver(backend=backend, static=st, dx=c['dx'], heightM=c['heightM'], u10Max=8,
                                 met=c['met'], existingFlux=c['flux'])
        s.setNewCampuses([c['campus']])
        solvers.append(s)
    classes = {}
    for s in solvers:
        classes.setdefault((s.info['nx'], s.info['ny'], s.info['nz']), []).append(s)
    tuned = {}
    for key, members in classes.items():
        if a.no_autotune:
            break
        by, zs, ms = members[0]._dev.autotune(3)
        for m in members[1:]:
            m._dev.set_launch(by, zs)
        tuned['x'.join(map(str, key))] = dict(block_y=by, zslab=zs, ms=round(ms, 4))
        log(f'[rank {rank}] autotune {key}: block_y {by} zslab {zs} {ms:.3f} ms/step')
    cells = sum(s.info['nCells'] for s in solvers)
    fluid = sum(s.info['nFluid'] for s in solvers)
    b = LiveBatch(solvers)
    btune = None
    if not a.no_autotune:
        btune = b.autotune(4)
        log(f'[rank {rank}] batch autotune: {btune}')
    warm_up(b._b, a.warmup)

    def barrier():
        RP.barrier(dist, lambda: torch.cuda.synchronize(local))

    barrier()
    with Clocks(local) as clk:
        barrier()
        ms = b._b.time_steps(a.steps)
        barrier()
    clocks = clk.summary()
    ms_all = RP.max_over_ranks(ms, dist, f'cuda:{local}')
    value = RP.aggregate_rate(cells * a.steps, world, ms_all / 1e3) / 1e9
    # the same members stepped one after another with their own tuned launches (no batch)
    serial_ms = serial_time(solvers, a.steps)
    bytes_launch = fluid * CELL_BYTES[a.precision]
    launch_ms = ms / a.steps
    achieved = bytes_launch / (launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    roof = dict(bound='hbm', achieved=achieved, peak=peak, unit='GB/s', frac=achieved / peak, traffic=None,
                peak_source=peak_kind, bytes_per_launch=bytes_launch, launch_ms=launch_ms,
                kernel='batch_kernel (one persistent launch per step over all 64 domains)')
    # end to end: per frame every member gets a new parameter block, the batch steps F, every member is read
    F = a.frame
    frames = max(3, a.steps // 4)
    mets = [dict(c['met']) for c in scen]
    b.step(F).result()
    barrier()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for fr in range(frames):
        for s, m in zip(solvers, mets):
            m['u10'] = min(8.0, m['u10'] + 0.01)
            s.setMet(m)
            h2d += len(s._params)
        b.step(F)
        pend = [s.read(vol=False, wind=True) for s in solvers]
        for s, p in zip(solvers, pend):
            p.result()
            d2h += 3 * s.info['nx'] * s.info['ny'] * 4 + 4
    barrier()
    e2e_s = RP.max_over_ranks(time.perf_counter() - t0, dist, f'cuda:{local}')
    e2e = dict(value=world * cells * F * frames / e2e_s / 1e9, unit='GLUPS', h2d_bytes_per_step=h2d / (F * frames),
               d2h_bytes_per_step=d2h / (F * frames), frame_steps=F, frames=frames,
               per_frame='setMet on all 64 members (parameter blocks H2D) + batch step(F) + read(wind) of every member '
                         '(surface theta, u, v D2H)')
    info = b.info
    b.destroy()
    for s in solvers:
        s.destroy()
    out = dict(metric='GLUPS (all cells) of the batched fused D3Q19+D3Q7 step, 64 domains (32 x 200x200x32 + '
                      '32 x 150x150x24)' if len(scen) == 64 else f'GLUPS of the batched step, {len(scen)} domains',
               value=value, unit='GLUPS', n_gpus=world, steps=a.steps, warmup=a.warmup,
               ms_per_step=ms_all / a.steps, higher_is_better=True, scaling='weak', vs_baseline=None,
               dtype=DTYPE[a.precision],
               data='synthetic (seeded terrain, buildings and scenarios; no public dataset involved)',
               config=dict(workload=WORKLOADS['c4']['desc'], precision=a.precision, arith=a.arith, scheme='pull',
                           parallelism=f'replicas x{world}', cells=cells, fluid_cells=fluid,
                           l2=f'state {cells * CELL_BYTES[a.precision] / 1e9:.1f} GB vs 126 MB L2', tuned=tuned,
                           batch=dict(tiles=info['tiles'], grid=info['grid'], minb=info['minb'],
                                      zslab_max=info['zslab_max'], graph=bool(info['use_graph']), tuned=btune)),
               serial=dict(value=world * cells * a.steps / (serial_ms / 1e3) / 1e9, unit='GLUPS',
                           ms_per_step=serial_ms / a.steps, what='the 64 members stepped one after another, each '
                                                                 'with its own tuned launch'),
               roofline=roof, cpu_baseline=None, e2e=e2e, gpu_launches=a.steps, clocks=clocks,
               glups_fluid=world * fluid * a.steps / (ms_all / 1e3) / 1e9)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def serve_serial(st, reqs, backend, tuned, clock=time.perf_counter):
    """The serial arm of the serving comparison, run for real: the same requests in arrival order, each solved alone
    end to end through the public API of one solver per grid class (setMet, setExistingFlux, setNewCampuses,
    resetFlow, step(n), read()), a request starting when it has arrived and the previous one has been answered.
    Returns (latencies, makespan, cell updates)."""
    from ashburn_heat_twin_b200 import solver as S
    solvers = {}
    for r in reqs:
        key = (r.dx, r.heightM)
        if key not in solvers:
            s = S.create_live_solver(backend=backend, static=st, dx=r.dx, allowAnyDx=True, heightM=r.heightM,
                                     u10Max=8, met=r.met, existingFlux=r.flux)
            if key in tuned:
                s._dev.set_launch(*tuned[key])
            solvers[key] = s
    lat, upd = [], 0
    t0 = clock()
    for r in sorted(reqs, key=lambda r: r.arrival):
        wait = r.arrival - (clock() - t0)
        if wait > 0:
            time.sleep(wait)
        s = solvers[(r.dx, r.heightM)]
        s.setMet(r.met)
        s.setExistingFlux(r.flux)
        s.setNewCampuses([r.campus])
        s.resetFlow()
        n = int(math.ceil(r.sim_s / s.info['dt'] - 1e-9))
        s.step(n)
        s.read(vol=True, wind=True).result()
        lat.append(clock() - t0 - r.arrival)
        upd += n * s.info['nCells']
    makespan = clock() - t0
    for s in solvers.values():
        s.destroy()
    return lat, makespan, upd


def main_serve(a, rank, world, local, dist, torch):
    """The serving workload: a seeded Poisson trace of requests served by the C ABI server (ahx_server_*: continuous
    batching, admission by resident cells and free HBM, chunks of --chunk steps; each request's own tuned step kernel
    on parallel graph branches, or --batch-mode persistent). The served rate is end to end (host image building,
    uploads, batched steps and read-back inside the wall clock). The serial arm runs the same trace for real: every
    request alone through the public solver API, back to back in arrival order, set-up and read-back included."""
    import numpy as np

    from ashburn_heat_twin_b200 import scenarios as SC
    from ashburn_heat_twin_b200 import serving as SV
    from ashburn_heat_twin_b200 import synth
    from ashburn_heat_twin_b200.cuda_device import CudaDevice
    st = synth.make_static10(synth.C1)

    def backend(nx, ny, nz):
        return CudaDevice(nx, ny, nz, device=local, precision=a.precision, arith=a.arith)

    free_b, _ = torch.cuda.mem_get_info(local)
    srv = SV.NativeServer(st, precision=a.precision, arith=a.arith, device=local, max_cells=a.max_cells,
                          chunk=a.chunk, hbm_budget_bytes=int(0.8 * free_b), batch_mode=a.batch_mode, tune=True)
    # warm-up through the same server: slots of every class, launch tuning, graph capture, read-back staging
    warm = SV.requests_from_trace(SC.serve_trace(st, 12, 1000.0, seed=a.seed + 100), sim_s=5.0)
    srv.run(warm, timeout_s=600)
    # each rank serves its own trace (replicas: seed + rank); the job's rate is all ranks' cell updates over the
    # longest makespan
    trace = SC.serve_trace(st, a.requests, a.rate, seed=a.seed + rank)
    reqs = SV.requests_from_trace(trace, sim_s=SC.SERVE_SIM_S)
    if dist is not None:
        dist.barrier()
    with Clocks(local) as clk:
        stats = srv.run(reqs, timeout_s=3600)
    clocks = clk.summary()
    makespan_all = RP.max_over_ranks(stats['makespan_s'], dist, f'cuda:{local}')
    job_glups = RP.aggregate_rate(stats['cell_updates'], world, makespan_all) / 1e9
    log(f'[rank {rank}] served {stats["requests"]} requests in {stats["makespan_s"]:.1f} s: {stats["glups"]:.2f} GLUPS, '
        f'p50 {stats["latency_p50_s"]:.2f} s, p99 {stats["latency_p99_s"]:.2f} s, {stats["chunks"]} chunks, '
        f'host image building {stats["host_image_s"]:.1f} s')
    srv.close()
    # the serial arm: the same trace, each request alone, launch shapes tuned per class first
    from ashburn_heat_twin_b200 import solver as S
    shapes = {}
    for r in reqs:
        key = (r.dx, r.heightM)
        if key not in shapes:
            s = S.create_live_solver(backend=backend, static=st, dx=r.dx, allowAnyDx=True, heightM=r.heightM, u10Max=8,
                                     met=r.met, existingFlux=r.flux)
            by, zs, _ = s._dev.autotune(3)
            shapes[key] = (by, zs)
            s.step(64).result()
            s.destroy()
    sreqs = SV.requests_from_trace(trace, sim_s=SC.SERVE_SIM_S)
    lat_ser, mk_ser, upd_ser = serve_serial(st, sreqs, backend, shapes)
    mk_ser_all = RP.max_over_ranks(mk_ser, dist, f'cuda:{local}')
    serial_glups = RP.aggregate_rate(upd_ser, world, mk_ser_all) / 1e9
    log(f'[rank {rank}] serial: {len(sreqs)} requests in {mk_ser:.1f} s: {upd_ser / mk_ser / 1e9:.2f} GLUPS, '
        f'p50 {np.percentile(lat_ser, 50):.2f} s, p99 {np.percentile(lat_ser, 99):.2f} s')
    upd = stats['cell_updates']
    h2d = sum(64 + 16 * int(round(r.heightM / r.dx)) + 20 * (6000 // int(r.dx)) ** 2 for r in reqs)
    d2h = sum((3 * 4 + min(int(round(r.heightM / r.dx)), int(round(420 / r.dx)))) * (6000 // int(r.dx)) ** 2
              for r in reqs)
    steps_total = sum(r.steps for r in reqs)
    out = dict(metric='GLUPS (all cells) served with continuous batching, Poisson trace of live-solver requests',
               value=job_glups, unit='GLUPS', n_gpus=world, steps=stats['batch_steps'], warmup=len(warm),
               ms_per_step=stats['makespan_s'] * 1e3 / max(1, stats['batch_steps']), higher_is_better=True,
               scaling='weak', vs_baseline=None, dtype=DTYPE[a.precision],
               data='synthetic (seeded terrain, buildings and request trace; no public dataset involved)',
               config=dict(workload=WORKLOADS['c5']['desc'], requests=a.requests, rate_hz=a.rate, seed=a.seed,
                           precision=a.precision, scheme='pull', parallelism='replicas',
                           l2='per-step state of the admitted requests >> 126 MB L2'),
               arith=a.arith, max_cells=a.max_cells, chunk=a.chunk, hbm_budget_bytes=srv.hbm_budget,
               batch_mode=a.batch_mode,
               serving=dict(latency_p50_s=stats['latency_p50_s'], latency_p99_s=stats['latency_p99_s'],
                            latency_mean_s=stats['latency_mean_s'], queue_p50_s=stats['queue_p50_s'],
                            queue_p99_s=stats['queue_p99_s'], makespan_s=stats['makespan_s'],
                            cell_updates=upd, chunks=stats['chunks'], slots=stats['slots'],
                            host_image_s=stats['host_image_s'], server='ahx_server_* (C ABI scheduler thread)'),
               serial=dict(value=serial_glups, unit='GLUPS', latency_p50_s=float(np.percentile(lat_ser, 50)),
                           latency_p99_s=float(np.percentile(lat_ser, 99)), makespan_s=mk_ser,
                           cell_updates=upd_ser,
                           what='the same trace run for real: each request alone through the public solver API '
                                '(setMet, setExistingFlux, setNewCampuses, resetFlow, step, read) back to back in '
                                'arrival order, set-up and read-back inside the wall clock'),
               served_over_serial=job_glups / serial_glups if serial_glups > 0 else None,
               roofline=None, cpu_baseline=None,
               e2e=dict(value=job_glups, unit='GLUPS', h2d_bytes_per_step=h2d / steps_total,
                        d2h_bytes_per_step=d2h / steps_total,
                        what='the served rate is end to end: request images, uploads, batched steps and read() '
                             'downloads are all inside the wall-clock makespan'),
               gpu_launches=stats['batch_steps'], clocks=clocks)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def main_precision(a, rank, world, local, dist, torch):
    """Storage precision study on the 600x600x64 domain: every storage (FP32, FP16, BF16 with the FMA build; FP64 with
    the exact build) runs the same cold start for --spin-s simulated seconds, then takes the --mean-s time means with
    the FP64 heat budget and the FP64 near-ground / lateral-face accumulators fused into the step. Reported per storage against FP64: rel-L2 of the mean
    near-ground theta (the first fluid cell of every column), peak mean warming, heat-closure terms, the rel-L2 of
    theta after one step from the FP64 state, and the step rate (GLUPS) on the tuned launch."""
    import numpy as np

    from ashburn_heat_twin_b200 import params as PM
    order = ['fp64', 'fp32', 'fp16', 'bf16', 'fp16g32', 'bf16g32', 'fp16sr']
    sol = {p: make_solver(device=local, precision=p, arith='exact' if p == 'fp64' else 'fast') for p in order}
    # sensitivity of the window means: FP64 runs whose flow populations get one seeded relative kick of size eps at
    # the end of the spin-up (the size of an f32 / a 16-bit rounding), nothing else changed
    kicks = {f'fp64 kick {e:g}': e for e in (a.kicks or ())}
    for p in kicks:
        sol[p] = make_solver(device=local, precision='fp64', arith='exact')
    s0 = sol['fp64']
    nx, ny, nz = s0.info['nx'], s0.info['ny'], s0.info['nz']
    N = nx * ny * nz
    dt, dx = s0.info['dt'], s0.info['dx']
    spin = int(round(a.spin_s / dt))
    mean = int(round(a.mean_s / dt))
    ktop = s0._ktopS.astype(np.int64)            # solver orientation, j = 0 south
    cols = np.nonzero(ktop < nz)[0]
    fluid = (np.arange(nz)[:, None] >= ktop[None, :]).reshape(-1)
    res = {}
    for p in order + list(kicks):
        s = sol[p]
        dev = s._dev
        t0 = time.perf_counter()
        s.step(spin).result()
        if p in kicks:
            f, g = dev.read_state_f64()
            rng = np.random.default_rng(11)
            f = f.reshape(19, N)
            f[:, fluid] *= 1.0 + kicks[p] * rng.uniform(-1.0, 1.0, (19, int(fluid.sum())))
            dev.write_state_f64(f, g)
            del f, g
        st0 = dev.stats()
        dev.budget_enable(True)
        dev.budget_read(reset=True)
        dev.accum_enable(True)
        dev.accum_read(reset=True)
        s.step(mean).result()
        bud = dev.budget_read(reset=True)
        surf, faces, nacc = dev.accum_read(reset=True)
        dev.budget_enable(False)
        dev.accum_enable(False)
        st1 = dev.stats()
        ng = surf[0].reshape(-1)[cols] / nacc                   # mean theta at each column's first fluid cell
        rc = PM.RHO_CP * dx ** 3 / (mean * dt) / 1e6          # K lattice units summed over the window -> MW
        ftu = bud['face_theta_u']                              # west, east, south, north sums of theta * u_n
        out_mw = rc * (ftu[1] - ftu[0] + ftu[3] - ftu[2])
        # the offline form (product of the time means on the faces)
        pm = {k: float((v[0] / nacc * v[1] / nacc).sum()) for k, v in faces.items()}
        out_pm_mw = PM.RHO_CP * dx ** 3 / dt / 1e6 * (pm['east'] - pm['west'] + pm['north'] - pm['south'])
        fu = bud['face_u']                                     # west, east, south, north sums of u_n
        mass_imb = abs(fu[0] - fu[1] + fu[2] - fu[3]) / max(sum(abs(x) for x in fu), 1e-300)
        res[p] = dict(ng=ng, peak=float(ng.max()), injected_mw=rc * bud['src_sum'], advected_out_mw=out_mw,
                      mass_imbalance=mass_imb,
                      advected_out_mean_product_mw=out_pm_mw,
                      content_rate_mw=rc * (st1['sumTheta'] - st0['sumTheta']), nonfinite=st1['nonFinite'],
                      wall_s=time.perf_counter() - t0)
        log(f'[rank {rank}] precision {p}: {spin}+{mean} steps in {res[p]["wall_s"]:.1f} s, peak {res[p]["peak"]:.4f} K')
    ref = res['fp64']

    def rel_l2(x, y):
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))

    sensitivity = {p: dict(kick=e, mean_ng_theta_rel_l2_vs_fp64=rel_l2(res[p]['ng'], ref['ng']),
                           peak_mean_warming_k=res[p]['peak']) for p, e in kicks.items()}
    for p in kicks:
        sol.pop(p).destroy()

    # one step from the FP64 state in every storage (theta of the fluid cells)
    f64, g64 = s0._dev.read_state_f64()
    s0._dbg.stepOut(1).result()
    th64 = s0._dbg.readDbg().reshape(N, 4)[fluid, 0].astype(np.float64)
    step_err = {}
    for p in order[1:]:
        sol[p]._dev.write_state(f64.astype(np.float32), g64.astype(np.float32))
        sol[p]._dbg.stepOut(1).result()
        th = sol[p]._dbg.readDbg().reshape(N, 4)[fluid, 0].astype(np.float64)
        step_err[p] = rel_l2(th, th64)
    # step rate of each storage on its tuned launch (after the study, so the runs share one start)
    rate = {}
    for p in order:
        dev = sol[p]._dev
        dev.autotune(3)
        warm_up(dev, a.warmup)
        ms = dev.time_steps(a.steps)
        rate[p] = N * a.steps / (ms / 1e3) / 1e9
    for s in sol.values():
        s.destroy()
    prec = {}
    for p in order:
        r = res[p]
        closure = (r['injected_mw'] - r['advected_out_mw'] - r['content_rate_mw']) / r['injected_mw']
        prec[p] = dict(glups=rate[p], speedup_vs_fp32=rate[p] / rate['fp32'],
                       mean_ng_theta_rel_l2_vs_fp64=None if p == 'fp64' else rel_l2(r['ng'], ref['ng']),
                       step_theta_rel_l2_vs_fp64=step_err.get(p), peak_mean_warming_k=r['peak'],
                       injected_mw=r['injected_mw'], advected_out_mw=r['advected_out_mw'],
                       advected_out_product_of_means_mw=r['advected_out_mean_product_mw'],
                       content_rate_mw=r['content_rate_mw'], closure_residual_frac=closure,
                       mass_imbalance=r['mass_imbalance'],
                       nonfinite=r['nonfinite'])
    # headline: FP16 storage with stochastic rounding, the 16-bit storage whose 10-minute mean stays within 1e-3
    out = dict(metric='GLUPS (all cells) of the FP16-storage step (stochastic rounding) on 600x600x64, with its '
                      '10-minute mean near-ground theta rel-L2 against the FP64 build', value=rate['fp16sr'],
               unit='GLUPS', n_gpus=world, steps=a.steps, warmup=a.warmup, ms_per_step=N / rate['fp16sr'] / 1e6,
               higher_is_better=True, scaling='weak', vs_baseline=None, dtype=DTYPE['fp16sr'],
               data='synthetic (seeded terrain and buildings; no public dataset involved)',
               config=dict(workload=WORKLOADS['c3']['desc'], spin_steps=spin, mean_steps=mean, dt_s=dt,
                           near_ground='first fluid cell of each column, mean over the window',
                           parallelism=f'replicas x{world}'),
               precision=prec, sensitivity=sensitivity or None, roofline=None, cpu_baseline=None, e2e=None,
               gpu_launches=a.steps)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def ranks_check(a, rank, world, local):
    """The multi-rank plumbing of the benchmark without the stepping: process group (NCCL on GPUs, gloo without
    CUDA), the barrier around the timed region and the max-over-ranks reduction. Rank 0 prints one JSON line."""
    import datetime

    import torch
    import torch.distributed as dist
    cuda = torch.cuda.is_available()
    if world > 1:
        if cuda:
            torch.cuda.set_device(local)
            dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=60),
                                    device_id=torch.device('cuda', local))
        else:
            dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=60))
    pg = dist if world > 1 else None
    RP.barrier(pg)
    top = RP.max_over_ranks(rank, pg, f'cuda:{local}' if cuda else 'cpu')
    out = dict(n_gpus=world if cuda else 0, ranks=world, max_rank_seen=int(top), backend=(
        'nccl' if cuda else 'gloo') if world > 1 else None)
    if pg is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--precision', default='fp32', choices=sorted(CELL_BYTES))
    ap.add_argument('--arith', default='fast', choices=['exact', 'fast'])
    ap.add_argument('--frame', type=int, default=10, help='steps per e2e frame (setMet + step(F) + read())')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-autotune', action='store_true')
    ap.add_argument('--no-secondary', action='store_true',
                    help='skip the further rates of the default run (16-bit storages, 64-domain batch)')
    ap.add_argument('--block-y', type=int, default=0, help='fix the launch shape instead of autotuning')
    ap.add_argument('--zslab', type=int, default=0)
    ap.add_argument('--workload', default='c2', choices=sorted(WORKLOADS),
                    help='c2 (the benchmark), c1 / c2q (smaller cases for profiling), r20 / r30 / r40 (the reference\'s '
                         'Ashburn planes at its published grids), c3 (storage precision study), c4 (64 domains in one '
                         'batch), c5 (serving)')
    ap.add_argument('--members', type=int, default=64, help='batch: scenarios in the batch (64 = the full set)')
    ap.add_argument('--requests', type=int, default=500, help='serving: requests in the trace')
    ap.add_argument('--rate', type=float, default=50.0, help='serving: mean arrival rate (requests/s)')
    ap.add_argument('--seed', type=int, default=5, help='serving: trace seed')
    ap.add_argument('--max-cells', type=int, default=24_000_000,
                    help='serving: resident cell budget (24 M: the served rate of 64 M at a lower p50)')
    ap.add_argument('--chunk', type=int, default=256, help='serving: steps per batched chunk')
    ap.add_argument('--batch-mode', default='branches', choices=['persistent', 'branches'],
                    help='serving: one persistent launch over tiles, or each request\'s own tuned kernel on parallel '
                         'graph branches')
    ap.add_argument('--spin-s', type=float, default=120.0, help='precision study: simulated spin-up seconds')
    ap.add_argument('--mean-s', type=float, default=600.0, help='precision study: simulated averaging seconds')
    ap.add_argument('--kicks', type=float, nargs='*', default=None,
                    help='precision study: also run FP64 with one relative kick of each size after the spin-up')
    ap.add_argument('--ranks-check', action='store_true',
                    help='start the ranks, run the barrier and the max-over-ranks reduction, print the rank count and '
                         'exit (no stepping; gloo when CUDA is unavailable)')
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)

    rank, world, local = RP.env_ranks()
    if a.impl == 'reference':
        return run_reference(a, rank)
    if a.gpus > 1 and 'WORLD_SIZE' not in os.environ:
        return RP.launch_ranks(os.path.abspath(__file__), sys.argv[1:], a.gpus)
    if 'WORLD_SIZE' in os.environ and world != a.gpus:
        log(f'bench.py: --gpus {a.gpus} but the launcher started {world} ranks')
        return 2
    if a.ranks_check:
        return ranks_check(a, rank, world, local)

    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device('cuda', local))
    from ashburn_heat_twin_b200 import _build
    _build.build()
    if a.workload == 'c4':
        return main_batch(a, rank, world, local, dist, torch)
    if a.workload == 'c5':
        return main_serve(a, rank, world, local, dist, torch)
    if a.workload == 'c3':
        return main_precision(a, rank, world, local, dist, torch)
    s = make_solver(device=local, precision=a.precision, arith=a.arith, workload=a.workload)
    dev = s._dev
    nx, ny, nz = s.info['nx'], s.info['ny'], s.info['nz']
    cells = nx * ny * nz
    fluid = s.info['nFluid']
    tune = None
    if a.block_y or a.zslab:
        dev.set_launch(a.block_y, a.zslab)
        tune = (a.block_y, a.zslab, None)
    elif not a.no_autotune:
        tune = dev.autotune(3)
        log(f'[rank {rank}] autotune: block_y {tune[0]} zslab {tune[1]} {tune[2]:.3f} ms/step')
    warm_up(dev, a.warmup)

    def barrier():
        RP.barrier(dist, lambda: torch.cuda.synchronize(local))

    barrier()
    with Clocks(local) as clk:
        barrier()
        ms = dev.time_steps(a.steps)
        barrier()
    clocks = clk.summary()
    ms_all = RP.max_over_ranks(ms, dist, f'cuda:{local}')
    value = RP.aggregate_rate(cells * a.steps, world, ms_all / 1e3) / 1e9

    # roofline of the step kernel (one launch per step): algorithmic bytes = fluid cells x (read + write of 19 f and
    # 7 g populations) at the storage width
    bytes_launch = fluid * CELL_BYTES[a.precision]
    launch_ms = ms / a.steps
    achieved = bytes_launch / (launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    launch_used = dev.launch()
    traffic, traffic_src = profile_traffic(a.precision, launch_used, fluid)
    roof = dict(bound='hbm', achieved=achieved, peak=peak, unit='GB/s', frac=achieved / peak,
                traffic=traffic, traffic_source=traffic_src, peak_source=peak_kind,
                bytes_per_launch=bytes_launch, launch_ms=launch_ms)

    # end to end through the public API with host buffers
    from ashburn_heat_twin_b200 import synth
    F = a.frame
    frames = max(10, 2 * a.steps)        # long enough that pipeline fill and drain stay a few per cent
    wl = WORKLOADS[a.workload]
    met = dict(u10=3.09, dirFrom=210, wstar=1.67, blh=903, ustar=0.32) if wl.get('real') else \
        dict(getattr(synth, wl['met']))
    u10_0 = met['u10']
    pend = []
    s.setMet(met)
    s.step(F)
    s.read().result()
    barrier()
    t0 = time.perf_counter()
    for fr in range(frames):
        met['u10'] = u10_0 + 0.01 * (fr % 5)        # a new parameter block every frame (host -> device)
        s.setMet(met)
        s.step(F)
        pend.append(s.read(vol=True, wind=True))
        if len(pend) > 2:
            pend.pop(0).result()
    for p in pend:
        p.result()
    barrier()
    e2e_s = RP.max_over_ranks(time.perf_counter() - t0, dist, f'cuda:{local}')
    NXY = nx * ny
    h2d = len(s._params)
    d2h = 3 * NXY * 4 + s.nzv * NXY + 4
    e2e = dict(value=world * cells * F * frames / e2e_s / 1e9, unit='GLUPS', h2d_bytes_per_step=h2d / F,
               d2h_bytes_per_step=d2h / F, frame_steps=F, frames=frames,
               per_frame='setMet (parameter block H2D) + step(F) + read(vol, wind) D2H')
    # read() latency on an idle device (the reference publishes its median / max, js/live/README.md:232-234)
    lat = []
    for _ in range(20):
        s.step(F).result()
        t1 = time.perf_counter()
        s.read(vol=True, wind=True).result()
        lat.append((time.perf_counter() - t1) * 1e3)
    lat.sort()
    read_ms = dict(median=lat[len(lat) // 2], max=lat[-1], reads=len(lat),
                   what='read(vol, wind) after the steps finished: surface and volume kernels, D2H, host arrays')
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        s_steps = s._steps
        cpu = cpu_baseline(workload=a.workload)
        del s_steps
    state_bytes = s._dev.info()['state_bytes']
    more = None
    if world == 1 and not a.no_secondary and a.workload == 'c2' and a.precision == 'fp32':
        s.destroy()
        s = None
        with Clocks(local) as clk2:
            more = secondary_rates(a, local)
        more['clocks'] = clk2.summary()
    metric = METRIC.replace('600x600x64', f'{nx}x{ny}x{nz}')
    vs = value / wl['published_glups'] if wl.get('published_glups') else None
    out = dict(metric=metric, value=value, unit='GLUPS', n_gpus=world, steps=a.steps, warmup=a.warmup,
               ms_per_step=ms_all / a.steps, higher_is_better=True, scaling='weak', vs_baseline=vs,
               dtype=DTYPE[a.precision],
               data=('the reference\'s own Ashburn planes (tests/golden/static10.*)' if wl.get('real') else
                     'synthetic (seeded terrain and buildings; no public dataset involved)'),
               config=bench_config(a.workload, a.precision, cells),
               arith=a.arith, fluid_cells=fluid, replicas=world, state_bytes=state_bytes,
               launch=dict(block_y=launch_used[0], zslab=launch_used[1], tuned=tune is not None and tune[2] is not None),
               published=wl.get('published'),
               roofline=roof, cpu_baseline=cpu, e2e=e2e, read_ms=read_ms, gpu_launches=a.steps, clocks=clocks,
               glups_fluid=world * fluid * a.steps / (ms_all / 1e3) / 1e9, secondary=more)
    if s is not None:
        s.destroy()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == '__main__':
    sys.exit(main())
