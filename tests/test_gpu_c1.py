"""The 200x200x32 workload at its own size (30 m cells, seeded synthetic terrain and buildings, 4 m/s from 270 deg,
alpha 0.2): 600 steps of the exact CUDA build against the CPU oracle, bit-identical in the final state, in the
600-step accumulated (theta, u, v, w) of every cell (so in the 600-step mean near-ground theta) and in read();
and one step of the FMA build from the oracle's state within the single-step theta rel-L2 bar of 1e-5."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import solver as S
from ashburn_heat_twin_b200 import synth
from tests.helpers import cuda_backend, oracle_backend, rel_l2

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(900)]


def c1_solver(backend):
    st = synth.make_static10(synth.C1)
    return S.create_live_solver(backend=backend, static=st, dx=30, allowAnyDx=True, heightM=960, u10Max=8,
                                alpha=0.2, met=synth.C1_MET, existingFlux=400)


def test_c1_600_steps_bit_exact_and_mean_near_ground_theta():
    g = c1_solver(cuda_backend('fp32', 'exact'))
    o = c1_solver(oracle_backend())
    assert (g.info['nx'], g.info['ny'], g.info['nz']) == (200, 200, 32)
    for s in (g, o):
        s._dbg.clearDbg()
        s._dbg.stepAcc(600).result()
    sg, so = g._dbg.readState(), o._dbg.readState()
    assert np.array_equal(sg['f'], so['f']) and np.array_equal(sg['g'], so['g'])
    dg, do = g._dbg.readDbg().reshape(-1, 4), o._dbg.readDbg().reshape(-1, 4)
    assert np.array_equal(dg, do)
    # the 600-step mean near-ground theta (first fluid cell of each column) is therefore identical; check its scale
    ktop = g._ktopS.astype(np.int64)
    cols = np.nonzero(ktop < g.info['nz'])[0]
    ng = dg[ktop[cols] * 200 * 200 + cols, 0] / 600.0
    assert np.isfinite(ng).all() and ng.max() > 0.05
    rg, ro = g.read().result(), o.read().result()
    for key in ('surf', 'u', 'v', 'vol'):
        assert np.array_equal(rg[key], ro[key]), key
    # the FMA build: one step from the oracle's state
    f = c1_solver(cuda_backend('fp32', 'fast'))
    f._dbg.writeState(so['f'], so['g'])
    f._dbg.stepOut(1).result()
    o._dbg.stepOut(1).result()
    a, b = f._dbg.readDbg().reshape(-1, 4), o._dbg.readDbg().reshape(-1, 4)
    fl = b[:, 0] != 0
    assert rel_l2(a[fl, 0], b[fl, 0]) <= 1e-5
    for s in (g, o, f):
        s.destroy()
