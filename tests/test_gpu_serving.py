"""The serving loop on the GPU: requests of three grid classes, admitted under a cell budget and stepped by the
batched launch in chunks (membership changing between chunks), must be answered exactly as each scenario run alone
on a fresh CUDA solver (read() fields bit-identical)."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import scenarios as SC
from ashburn_heat_twin_b200 import serving as SV
from ashburn_heat_twin_b200 import solver as S
from tests.helpers import cuda_backend, small_static

pytestmark = pytest.mark.gpu


def test_served_answers_match_solo_runs():
    st = small_static(seed=9, ncols=120, nrows=96)
    rng = np.random.default_rng(11)
    be = cuda_backend('fp32', 'fast')
    reqs = []
    for i in range(7):
        dx = (40, 20, 30)[i % 3]
        reqs.append(SV.Request(id=i, arrival=0.002 * i, dx=dx, heightM=320, met=SC.random_met(rng),
                               flux=float(rng.uniform(200, 600)),
                               campus=dict(id=f'R{i}', mw=40.0, halls=[SC.free_site(st, rng, side_m=80.0)]),
                               sim_s=float(rng.uniform(4.0, 12.0))))
    srv = SV.Server(st, backend=be, max_cells=60_000, chunk=8)
    stats = srv.run(reqs, timeout_s=120)
    assert stats['requests'] == 7 and stats['batch_rebuilds'] >= 3 and stats['batch_steps'] > 0
    for r in reqs:
        s = S.create_live_solver(backend=be, static=st, dx=r.dx, allowAnyDx=True, heightM=r.heightM, u10Max=8,
                                 met=r.met, existingFlux=r.flux)
        s.setMet(r.met)
        s.setExistingFlux(r.flux)
        s.setNewCampuses([r.campus])
        s.resetFlow()
        s.step(r.steps).result()
        ref = s.read(vol=True, wind=True).result()
        s.destroy()
        for k in ('surf', 'u', 'v', 'vol'):
            assert np.array_equal(r.result[k], ref[k]), (r.id, k)
        assert r.result['thetaMax'] == ref['thetaMax']
    srv.close()
