"""Serving loop host logic on the CPU: admission under a cell budget (FIFO queueing), chunked continuous batching that
never steps a request past its simulated time, slot recycling across requests of one grid class, eviction under a
memory budget, and answers identical to each scenario run alone on a fresh solver (the CPU oracle stands in for the
device and a sequential stand-in for the batch)."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import scenarios as SC
from ashburn_heat_twin_b200 import serving as SV
from ashburn_heat_twin_b200 import solver as S
from tests.helpers import oracle_backend, small_static


def make_requests(st, n=5, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        dx = (40, 20)[i % 2]
        out.append(SV.Request(id=i, arrival=0.0, dx=dx, heightM=320, met=SC.random_met(rng),
                              flux=float(rng.uniform(200, 600)),
                              campus=dict(id=f'R{i}', mw=30.0, halls=[SC.free_site(st, rng, side_m=60.0)]),
                              sim_s=0.0))
    return out


def fresh(st, r):
    return S.create_live_solver(backend=oracle_backend(), static=st, dx=r.dx, allowAnyDx=True, heightM=r.heightM,
                                u10Max=8, met=r.met, existingFlux=r.flux)


def solo(st, r, steps):
    s = fresh(st, r)
    s.setMet(r.met)
    s.setExistingFlux(r.flux)
    s.setNewCampuses([r.campus])
    s.resetFlow()
    s.step(steps).result()
    out = s.read(vol=True, wind=True).result()
    s.destroy()
    return out


@pytest.fixture(scope='module')
def st():
    return small_static(seed=9)


def test_serving_answers_match_solo_runs(st):
    reqs = make_requests(st)
    for r in reqs:                                   # 3 / 5 steps of simulated time per request
        r.sim_s = fresh(st, r).info['dt'] * (3 if r.dx == 40 else 5)
    c40 = fresh(st, reqs[0]).info['nCells']
    # cell budget of two 40 m grids: later requests queue and slots are recycled
    srv = SV.HostServer(st, backend=oracle_backend(), batch_factory=SV.SequentialBatch, max_cells=2 * c40, chunk=2)
    stats = srv.run(reqs, timeout_s=120)
    assert stats['requests'] == 5 and all(r.result is not None for r in reqs)
    assert [r.steps for r in reqs] == [3, 5, 3, 5, 3]
    assert stats['chunks'] >= 5 and stats['batch_rebuilds'] >= 3
    assert len(srv.slots) <= 3                      # recycled, not one solver per request
    assert all(r.admitted >= r.arrival and r.done >= r.admitted for r in reqs)
    assert stats['latency_p99_s'] >= stats['latency_p50_s'] >= 0
    assert stats['cell_updates'] == sum(r.steps * r.cells for r in reqs)
    for r in reqs:
        ref = solo(st, r, r.steps)
        for k in ('surf', 'u', 'v', 'vol'):
            assert np.array_equal(r.result[k], ref[k]), (r.id, k)
        assert r.result['thetaMax'] == ref['thetaMax'] and r.result['steps'] == r.steps
    srv.close()


def test_serving_evicts_idle_slots_under_a_memory_budget(st):
    reqs = make_requests(st, n=4, seed=4)
    for r in reqs:
        r.sim_s = 1e-6                               # one step each
    c20 = fresh(st, reqs[1]).info['nCells']
    budget = c20 * 208                               # one resident slot at a time: classes alternate, so evict
    srv = SV.HostServer(st, backend=oracle_backend(), batch_factory=SV.SequentialBatch, max_cells=10**9,
                    hbm_budget_bytes=budget)
    stats = srv.run(reqs, timeout_s=120)
    assert stats['requests'] == 4 and all(r.result is not None for r in reqs)
    assert srv.bytes_used <= budget and stats['evictions'] >= 2 and stats['slots'] == 1
    srv.close()


def test_fifo_serial_reference():
    reqs = [SV.Request(id=i, arrival=a, dx=40, heightM=960, met={}, flux=0, campus={}) for i, a in
            enumerate((0.0, 0.5, 3.0))]
    lat, mk = SV.fifo_serial(reqs, lambda r: 1.0)
    assert list(lat) == [1.0, 1.5, 1.0] and mk == 4.0
