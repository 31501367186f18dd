"""The serving loop on the GPU through the C ABI server (ahx_server_*): requests of three grid classes arriving over
time, admitted under a cell budget and stepped together in batched chunks whose member list changes as requests join
and leave, must be answered exactly as each scenario run alone on a fresh CUDA solver (read() fields bit-identical),
in both batch modes (each request's own tuned step kernel on graph branches; one persistent launch)."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import scenarios as SC
from ashburn_heat_twin_b200 import serving as SV
from ashburn_heat_twin_b200 import solver as S
from tests.helpers import cuda_backend, small_static

pytestmark = pytest.mark.gpu


def _requests(st, n=7, seed=11):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        dx = (40, 20, 30)[i % 3]
        reqs.append(SV.Request(id=i, arrival=0.002 * i, dx=dx, heightM=320, met=SC.random_met(rng),
                               flux=float(rng.uniform(200, 600)),
                               campus=dict(id=f'R{i}', mw=40.0, halls=[SC.free_site(st, rng, side_m=80.0)]),
                               sim_s=float(rng.uniform(4.0, 12.0))))
    return reqs


def _solo(st, r, be):
    s = S.create_live_solver(backend=be, static=st, dx=r.dx, allowAnyDx=True, heightM=r.heightM, u10Max=8,
                             met=r.met, existingFlux=r.flux)
    s.setMet(r.met)
    s.setExistingFlux(r.flux)
    s.setNewCampuses([r.campus])
    s.resetFlow()
    s.step(r.steps).result()
    ref = s.read(vol=True, wind=True).result()
    s.destroy()
    return ref


@pytest.mark.parametrize('mode', ['branches', 'persistent'])
def test_served_answers_match_solo_runs(mode):
    st = small_static(seed=9, ncols=120, nrows=96)
    reqs = _requests(st)
    srv = SV.NativeServer(st, precision='fp32', arith='fast', max_cells=60_000, chunk=8, batch_mode=mode)
    stats = srv.run(reqs, timeout_s=120)
    assert stats['requests'] == 7 and stats['chunks'] >= 3 and stats['batch_steps'] > 0
    assert stats['cell_updates'] == sum(r.steps * r.cells for r in reqs)
    assert all(r.done >= r.admitted >= r.arrival - 1e-3 for r in reqs)
    be = cuda_backend('fp32', 'fast')
    for r in reqs:
        ref = _solo(st, r, be)
        for k in ('surf', 'u', 'v', 'vol'):
            assert np.array_equal(r.result[k], ref[k]), (mode, r.id, k)
        assert r.result['thetaMax'] == ref['thetaMax'] and r.result['simTime'] == ref['simTime']
        assert r.result['heatMW'] == ref['heatMW']
    srv.close()


def test_server_recycles_slots_and_handles_zero_step_requests():
    """A request with no steps is answered with its initial state; requests of one grid reuse slots when the cell
    budget forces them to run one after another; polling an unfinished request times out without consuming it."""
    st = small_static(seed=9, ncols=120, nrows=96)
    reqs = _requests(st, n=4, seed=3)
    for r in reqs:
        r.dx, r.arrival = 40, 0.0
    reqs[0].sim_s = 0.0
    srv = SV.NativeServer(st, precision='fp32', arith='fast', max_cells=1, chunk=4, tune=False)
    im = srv.images(reqs[1])
    t = srv.srv.submit(im['nx'], im['ny'], im['nz'], 10 ** 6, im['params'], im['colv'], im['ktop'], im['conv'],
                       im['volscale'], im['nzv'])
    assert srv.srv.poll(t, 0, im['nx'], im['ny'], im['nzv']) is None       # long request still running
    srv.close()                                                            # destroy drops it
    srv = SV.NativeServer(st, precision='fp32', arith='fast', max_cells=1, chunk=4, tune=False)
    stats = srv.run(reqs, timeout_s=120)
    # one request at a time: a finished request's slot is still draining its read-back when the next one is admitted,
    # so the four requests alternate between two slots instead of creating four
    assert stats['slots'] == 2 and stats['requests'] == 4
    be = cuda_backend('fp32', 'fast')
    for r in reqs:
        ref = _solo(st, r, be)
        assert np.array_equal(r.result['surf'], ref['surf']) and r.result['steps'] == r.steps
    assert reqs[0].steps == 0
    srv.close()


def test_gpu_built_request_images_equal_the_host_images():
    """The serving loop builds each request's geometry with the GPU domain builder: its column records, ktop plane and
    heat equal what a solver configured on the host uploads, for every grid class of the mix."""
    st = small_static(seed=9, ncols=120, nrows=96)
    reqs = _requests(st, n=6, seed=5)
    g = SV.NativeServer(st, precision='fp32', arith='fast', tune=False)
    h = SV.NativeServer(st, precision='fp32', arith='fast', tune=False, gpu_domain=False)
    for r in reqs:
        a, b = g.images(r), h.images(r)
        assert a['params'] == b['params'] and (a['nx'], a['ny'], a['nz']) == (b['nx'], b['ny'], b['nz'])
        assert np.array_equal(np.asarray(a['colv']).ravel(), np.asarray(b['colv']).ravel())
        assert np.array_equal(a['ktop'], b['ktop']) and a['heatMW'] == b['heatMW'] and a['steps'] == b['steps']
    g.close()
    h.close()
