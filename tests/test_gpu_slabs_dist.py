"""The one-process-per-slab form of the y-slab decomposition (slabs.DistributedSlab) with two ranks of a gloo group,
both on the one GPU this run has: each rank steps its own slab and the ranks swap packed boundary rows through the
host after every step (the kernels of the two ranks never wait on each other). The owned rows of both ranks must be
bit-identical to the undivided domain."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300)]


def _opts():
    from tests.helpers import small_static
    return dict(static=small_static(seed=5), dx=10, allowAnyDx=True, heightM=300, u10Max=8,
                met=dict(u10=5.0, dirFrom=200.0, wstar=1.5, blh=700.0), existingFlux=400, nsw=6)


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from ashburn_heat_twin_b200.slabs import DistributedSlab
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s = DistributedSlab(dist, precision='fp32', arith='exact', device=0, **_opts())
        s.step(7)
        f, g = s.owned_state()
        out[rank] = dict(a=s.a, b=s.b, f=f.tobytes(), g=g.tobytes(), shape=(s.nz, s.b - s.a, s.nx))
        s.destroy()
    except Exception as e:
        out[rank] = dict(error=repr(e)[:300])
    dist.destroy_process_group()


def test_two_slab_ranks_match_the_undivided_domain():
    with socket.socket() as so:
        so.bind(('127.0.0.1', 0))
        port = so.getsockname()[1]
    ctx = mp.get_context('spawn')
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method='spawn')
        res = dict(out)
    assert all('error' not in v for v in res.values()), res
    from ashburn_heat_twin_b200 import solver as S
    from tests.helpers import cuda_backend
    whole = S.create_live_solver(backend=cuda_backend('fp32', 'exact'), **_opts())
    whole.step(7).result()
    nx, ny, nz = whole.info['nx'], whole.info['ny'], whole.info['nz']
    f0, g0 = whole._dev.read_state()
    f0 = f0.reshape(19, nz, ny, nx)
    g0 = g0.reshape(7, nz, ny, nx)
    assert res[0]['a'] == 0 and res[1]['b'] == ny and res[0]['b'] == res[1]['a']
    for r in (0, 1):
        nzr, rows, nxr = res[r]['shape']
        f = np.frombuffer(res[r]['f'], np.float32).reshape(19, nzr, rows, nxr)
        g = np.frombuffer(res[r]['g'], np.float32).reshape(7, nzr, rows, nxr)
        assert np.array_equal(f.view(np.uint32), f0[:, :, res[r]['a']:res[r]['b']].view(np.uint32))
        assert np.array_equal(g.view(np.uint32), g0[:, :, res[r]['a']:res[r]['b']].view(np.uint32))
    whole.destroy()
