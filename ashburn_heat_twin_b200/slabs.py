"""One domain split into y-slabs (rows), one libahx handle per slab: the single-domain decomposition for grids beyond
one GPU's share (a 5 m grid, 1200x1200x128, needs ~100 GB in FP32).

The host builds the whole domain once (the live solver's own domain and parameter code, on a recording device that
only keeps the host images) and gives each slab its rows of the column records and the ktop plane, plus one ghost row
on each internal boundary. A neighbour's first row pulls from its ghost row only the populations that move toward it
(c_y = +1 northward, -1 southward: 5 flow and 1 temperature population), so each boundary exchanges a halo of 6 of the
26 planes per direction (ahx_halo_*). Every step is split (ahx_step_rows): a slab updates its boundary rows first,
packs their halos from the state being written, queues its interior rows, and only then waits for the packs, so the
transfer (device copies on one GPU; NCCL send / recv of 6 x nz x nx elements per direction across GPUs, one process
per slab) overlaps the interior update; the received halos are unpacked into the ghost rows behind the step. Faces and
sponges follow the global rows, so the stepped rows are bit-identical to the undivided domain's. A stochastic-rounding
state steps whole (its dithers count the step's blocks) and exchanges the same halos after the step.
"""
from __future__ import annotations

import numpy as np

from . import solver as S


class _Recorder:
    """A device that keeps the host images the live solver uploads and does nothing else."""

    def __init__(self, nx, ny, nz):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.params = self.colv = self.ktop = None
        self._p = 0
        self.adapter = 'host images'

    def set_params(self, b):
        self.params = bytes(b)

    def set_columns(self, colv):
        self.colv = np.array(colv, np.uint32).reshape(self.ny, self.nx, 4)

    def set_ktop(self, ktop, oldk):
        self.ktop = np.array(ktop, np.uint32).reshape(self.ny, self.nx)

    def set_parity(self, p):
        self._p = int(p)

    def parity(self):
        return self._p

    def init_flow(self):
        pass

    def clear_heat(self):
        pass

    def sync(self, timeout_s=None):
        pass

    def lost(self):
        return None

    def destroy(self):
        pass


def slab_rows(ny, nslabs):
    """Owned global rows [a, b) of each slab, as even as possible."""
    edges = np.linspace(0, ny, nslabs + 1).round().astype(int)
    return [(int(edges[r]), int(edges[r + 1])) for r in range(nslabs)]


class SlabDomain:
    """The domain of create_live_solver(**opts) split into `nslabs` y-slabs on one device (`device`), each a CudaDevice
    with precision / arithmetic as given. step(n) advances every slab n steps with a ghost-row exchange after each."""

    def __init__(self, nslabs, precision='fp32', arith='exact', device=None, **opts):
        from .cuda_device import CudaDevice
        rec = {}

        def recorder(nx, ny, nz):
            rec['dev'] = _Recorder(nx, ny, nz)
            return rec['dev']

        self.host = S.create_live_solver(backend=recorder, **opts)
        img = rec['dev']
        self.nx, self.ny, self.nz = img.nx, img.ny, img.nz
        self.rows = slab_rows(self.ny, nslabs)
        self.slabs = []
        for a, b in self.rows:
            ga, gb = int(a > 0), int(b < self.ny)
            jg0, nyl = a - ga, (b - a) + ga + gb
            d = CudaDevice(self.nx, nyl, self.nz, device=device, precision=precision, arith=arith)
            d.set_slab(jg0, self.ny, ga, ga + (b - a))
            d.set_params(img.params)
            d.set_columns(np.ascontiguousarray(img.colv[jg0:jg0 + nyl]).reshape(-1, 4))
            d.set_ktop(np.ascontiguousarray(img.ktop[jg0:jg0 + nyl]).reshape(-1), None)
            d.init_flow()
            d.clear_heat()
            self.slabs.append(dict(dev=d, a=a, b=b, jg0=jg0, ny=nyl, lo=ga, hi=ga + (b - a)))
        import torch
        nb = (self.slabs[0]['dev'].halo_bytes() + 255) // 256 * 256   # keep the second half 256-byte aligned
        self._buf = [torch.empty(2 * nb, dtype=torch.uint8, device=f'cuda:{device or 0}')
                     for _ in range(len(self.slabs) - 1)]
        self._nb = nb
        self.split = precision != 'fp16sr'
        self.steps = 0

    def step(self, n=1):
        """n steps; after each, every ghost row holds the neighbour's new halo (device copies)"""
        last = len(self.slabs) - 1
        for _ in range(int(n)):
            for r, s in enumerate(self.slabs):
                dev, south, north = s['dev'], r > 0, r < last
                bs = self._buf[r - 1].data_ptr() + self._nb if south else None   # my south-moving halo
                bn = self._buf[r].data_ptr() if north else None                   # my north-moving halo
                if self.split:
                    a = s['lo'] + int(south)
                    b = s['hi'] - int(north)
                    if south:
                        dev.step_rows(s['lo'], s['lo'] + 1, False)
                    if north and s['hi'] - 1 >= a:
                        dev.step_rows(s['hi'] - 1, s['hi'], False)
                    if south:
                        dev.halo_pack(s['lo'], -1, bs, next_state=True)
                    if north:
                        dev.halo_pack(s['hi'] - 1, 1, bn, next_state=True)
                    dev.step_rows(a, max(a, b), True)
                else:
                    dev.step(1, 0)
                    if south:
                        dev.halo_pack(s['lo'], -1, bs)
                    if north:
                        dev.halo_pack(s['hi'] - 1, 1, bn)
            for s in self.slabs:
                s['dev'].sync()
            for r in range(last):
                lo, hi = self.slabs[r], self.slabs[r + 1]
                p0, p1 = self._buf[r].data_ptr(), self._buf[r].data_ptr() + self._nb
                hi['dev'].halo_unpack(0, 1, p0)                 # into the north slab's ghost row 0
                lo['dev'].halo_unpack(lo['ny'] - 1, -1, p1)     # into the south slab's top ghost row
            self.steps += 1
        for s in self.slabs:
            s['dev'].sync()

    def read_state(self):
        """f (19, nz, ny, nx) and g (7, nz, ny, nx) of the whole domain, from the slabs' owned rows."""
        f = np.empty((19, self.nz, self.ny, self.nx), np.float32)
        g = np.empty((7, self.nz, self.ny, self.nx), np.float32)
        for s in self.slabs:
            fl, gl = s['dev'].read_state()
            fl = fl.reshape(19, self.nz, s['ny'], self.nx)
            gl = gl.reshape(7, self.nz, s['ny'], self.nx)
            f[:, :, s['a']:s['b']] = fl[:, :, s['lo']:s['hi']]
            g[:, :, s['a']:s['b']] = gl[:, :, s['lo']:s['hi']]
        return f, g

    def destroy(self):
        for s in self.slabs:
            s['dev'].destroy()
        self.slabs = []


class DistributedSlab:
    """One slab per process of a torch.distributed group: rank r owns rows slab_rows(ny, world)[r] of the domain of
    create_live_solver(**opts) and exchanges its boundary rows with ranks r - 1 and r + 1 after every step. With the
    NCCL backend the packed rows go device to device over NVLink; with gloo they are staged through host memory."""

    def __init__(self, dist, precision='fp32', arith='exact', device=None, **opts):
        import torch

        from .cuda_device import CudaDevice
        self.dist = dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        rec = {}

        def recorder(nx, ny, nz):
            rec['dev'] = _Recorder(nx, ny, nz)
            return rec['dev']

        S.create_live_solver(backend=recorder, **opts)
        img = rec['dev']
        self.nx, self.ny, self.nz = img.nx, img.ny, img.nz
        self.a, self.b = slab_rows(self.ny, self.world)[self.rank]
        ga, gb = int(self.a > 0), int(self.b < self.ny)
        self.jg0, self.nyl = self.a - ga, (self.b - self.a) + ga + gb
        self.lo, self.hi = ga, ga + (self.b - self.a)
        self.dev = CudaDevice(self.nx, self.nyl, self.nz, device=device, precision=precision, arith=arith)
        self.dev.set_slab(self.jg0, self.ny, self.lo, self.hi)
        self.dev.set_params(img.params)
        self.dev.set_columns(np.ascontiguousarray(img.colv[self.jg0:self.jg0 + self.nyl]).reshape(-1, 4))
        self.dev.set_ktop(np.ascontiguousarray(img.ktop[self.jg0:self.jg0 + self.nyl]).reshape(-1), None)
        self.dev.init_flow()
        self.dev.clear_heat()
        nb = (self.dev.halo_bytes() + 255) // 256 * 256
        dv = f'cuda:{device or 0}'
        self._nb = nb
        self._dv = dv
        self._send = torch.empty(2 * nb, dtype=torch.uint8, device=dv)
        self._recv = torch.empty(2 * nb, dtype=torch.uint8, device=dv)
        self._host = dist.get_backend() != 'nccl'
        self.split = precision != 'fp16sr'
        self.steps = 0

    def _step_and_pack(self):
        """this rank's part of one step up to the halos it sends: boundary rows, their halos from the state being
        written, then the interior rows queued behind them; returns once the halos are in the send buffers"""
        south, north = self.rank > 0, self.rank < self.world - 1
        s0, s1 = self._send.data_ptr(), self._send.data_ptr() + self._nb
        if self.split:
            a, b = self.lo + int(south), self.hi - int(north)
            if south:
                self.dev.step_rows(self.lo, self.lo + 1, False)
            if north and self.hi - 1 >= a:
                self.dev.step_rows(self.hi - 1, self.hi, False)
            if south:
                self.dev.halo_pack(self.lo, -1, s0, next_state=True)   # my first row's south-moving halo
            if north:
                self.dev.halo_pack(self.hi - 1, 1, s1, next_state=True)   # my last row's north-moving halo
            packed = self.dev.fence()
            self.dev.step_rows(a, max(a, b), True)                         # the interior overlaps the exchange
            packed.result()
        else:
            self.dev.step(1, 0)
            if south:
                self.dev.halo_pack(self.lo, -1, s0)
            if north:
                self.dev.halo_pack(self.hi - 1, 1, s1)
            self.dev.sync()

    def exchange(self):
        """send this rank's halos and unpack the neighbours' into the ghost rows (every rank takes the same steps in
        the same order)"""
        import torch
        south, north = self.rank > 0, self.rank < self.world - 1
        nb = self._nb
        send = self._send.cpu() if self._host else self._send
        recv = self._recv.cpu() if self._host else self._recv
        ops = []
        if south:
            ops += [self.dist.P2POp(self.dist.isend, send[:nb], self.rank - 1),
                    self.dist.P2POp(self.dist.irecv, recv[:nb], self.rank - 1)]
        if north:
            ops += [self.dist.P2POp(self.dist.isend, send[nb:], self.rank + 1),
                    self.dist.P2POp(self.dist.irecv, recv[nb:], self.rank + 1)]
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()
        if self._host:
            self._recv.copy_(recv)
        # the received halos are in place once torch's stream (NCCL's waits, the host copy) has run
        torch.cuda.current_stream(self._dv).synchronize()
        r0, r1 = self._recv.data_ptr(), self._recv.data_ptr() + nb
        if south:
            self.dev.halo_unpack(0, 1, r0)                  # the south neighbour's north-moving halo
        if north:
            self.dev.halo_unpack(self.nyl - 1, -1, r1)      # the north neighbour's south-moving halo
        self.dev.sync()

    def step(self, n=1):
        for _ in range(int(n)):
            self._step_and_pack()
            self.exchange()
            self.steps += 1

    def owned_state(self):
        """f (19, nz, rows, nx) and g (7, nz, rows, nx) of this rank's owned rows"""
        f, g = self.dev.read_state()
        f = f.reshape(19, self.nz, self.nyl, self.nx)[:, :, self.lo:self.hi]
        g = g.reshape(7, self.nz, self.nyl, self.nx)[:, :, self.lo:self.hi]
        return np.ascontiguousarray(f), np.ascontiguousarray(g)

    def destroy(self):
        self.dev.destroy()
