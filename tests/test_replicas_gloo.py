"""The N>1 path of bench.py on the CPU: two ranks over gloo (127.0.0.1), each stepping its own replica domain with
the oracle device, a barrier around the timed region, the max over ranks of the time and the whole-job rate. Each
rank's state must equal the same domain stepped in a single process (replicas share nothing), and a rank that
raises before the collective makes the other rank's collective end with an error within the process-group timeout
instead of waiting for ever."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ashburn_heat_twin_b200 import replicas as RP


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _replica(rank):
    from tests.helpers import oracle_backend, small_solver
    s = small_solver(oracle_backend(), seed=5 + rank)
    return s


def _worker(rank, world, port, out, fail_rank):
    import time

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r, w, _ = RP.env_ranks()
    dist.init_process_group('gloo', rank=r, world_size=w, timeout=datetime.timedelta(seconds=10))
    try:
        s = _replica(r)
        if r == fail_rank:
            raise RuntimeError('injected failure on the host before the timed region')
        RP.barrier(dist)
        t0 = time.perf_counter()
        s.step(3).result()
        RP.barrier(dist)
        secs = RP.max_over_ranks(time.perf_counter() - t0, dist)
        f, g = s._dev.read_state()
        out[r] = dict(secs=secs, cells=s.info['nCells'], crc=float(np.float64(f).sum() + np.float64(g).sum()),
                      rate=RP.aggregate_rate(s.info['nCells'] * 3, w, secs))
        s.destroy()
        dist.destroy_process_group()
    except Exception as e:   # the surviving rank records how its collective ended
        out[r] = dict(error=type(e).__name__ + ': ' + str(e)[:200])


@pytest.mark.timeout(240)
def test_two_replicas_over_gloo():
    ctx = mp.get_context('spawn')
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, _free_port(), out, -1), nprocs=2, join=True, start_method='spawn')
        res = dict(out)
    assert set(res) == {0, 1} and all('error' not in v for v in res.values()), res
    assert res[0]['secs'] == res[1]['secs']                   # both ranks report the max over ranks
    assert res[0]['rate'] == pytest.approx(2 * res[0]['cells'] * 3 / res[0]['secs'])
    for r in (0, 1):                                          # replicas are independent: same as a lone run
        s = _replica(r)
        s.step(3).result()
        f, g = s._dev.read_state()
        assert res[r]['crc'] == float(np.float64(f).sum() + np.float64(g).sum())
        s.destroy()


@pytest.mark.timeout(240)
def test_a_failed_rank_ends_the_other_ranks_collective():
    ctx = mp.get_context('spawn')
    with ctx.Manager() as m:
        out = m.dict()
        ctx_ = mp.start_processes(_worker, args=(2, _free_port(), out, 1), nprocs=2, join=False,
                                  start_method='spawn')
        while not ctx_.join(timeout=60):
            pass
        res = dict(out)
    assert 'injected failure' in res[1]['error']
    assert 'error' in res[0]                                  # rank 0's barrier did not wait for ever


def test_bench_gpus_flag_starts_that_many_ranks():
    """`python bench.py --gpus 2` (the driver's command form, no torchrun around it) starts two ranks itself; the
    ranks check runs the benchmark's barrier and max-over-ranks reduction (gloo here, no CUDA) and reports both."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ('RANK', 'WORLD_SIZE', 'LOCAL_RANK', 'MASTER_ADDR',
                                                            'MASTER_PORT')}
    r = subprocess.run([sys.executable, os.path.join(root, 'bench.py'), '--gpus', '2', '--ranks-check'],
                       capture_output=True, text=True, timeout=240, env=env, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [x for x in r.stdout.splitlines() if x.startswith('{')]
    assert len(line) == 1, r.stdout
    d = json.loads(line[0])
    assert d['ranks'] == 2 and d['max_rank_seen'] == 1


def test_bench_rejects_a_rank_count_other_than_gpus():
    """Under a launcher whose world size differs from --gpus the benchmark refuses to run instead of reporting a
    device count it did not use."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, RANK='0', WORLD_SIZE='1', LOCAL_RANK='0')
    r = subprocess.run([sys.executable, os.path.join(root, 'bench.py'), '--gpus', '2', '--ranks-check'],
                       capture_output=True, text=True, timeout=120, env=env, cwd=root)
    assert r.returncode == 2 and 'ranks' in r.stderr
