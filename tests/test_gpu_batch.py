"""Batched stepping (ahx_batch_*, LiveBatch): several domains of different grid sizes stepped by one persistent launch
per step must leave every member's state bit-identical to stepping it alone, through the graph and the plain launch
paths, across odd step counts, solo steps between batched ones, and parameter changes between batched steps.

The reference has no batched path (one solver per device); the oracle for a member is the same member stepped solo,
itself pinned bit-exactly against the CPU restatement by the parity tests."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import LiveBatch, LiveSolverError
from ashburn_heat_twin_b200 import solver as S
from ashburn_heat_twin_b200 import synth
from tests.helpers import cuda_backend

pytestmark = pytest.mark.gpu

# (columns, rows, seed, dx, heightM): three unequal grids
SCENARIOS = [(64, 48, 5, 10, 300), (40, 56, 6, 10, 320), (72, 40, 7, 20, 420)]
METS = [dict(u10=4.0, dirFrom=250.0, wstar=1.2, blh=800.0), dict(u10=6.5, dirFrom=35.0, wstar=0.4, blh=600.0),
        dict(u10=2.5, dirFrom=160.0, wstar=1.8, blh=1200.0)]


def scenario(i, precision='fp32', arith='exact'):
    ncols, nrows, seed, dx, hm = SCENARIOS[i]
    spec = synth.SynthSpec(ncols=ncols, nrows=nrows, hills=3, relief_m=25.0, buildings=int(60 * 600 * 600 / (ncols * nrows)),
                           side_m=(15, 60), height_m=(8, 35), dc_count=int(8 * 600 * 600 / (ncols * nrows)), seed=seed)
    st = synth.make_static10(spec)
    return S.create_live_solver(backend=cuda_backend(precision, arith), static=st, dx=dx, allowAnyDx=True,
                                heightM=hm, u10Max=8, met=METS[i], existingFlux=400)


def state(s):
    f, g = s._dev.read_state()
    return f.view(np.uint32), g.view(np.uint32)


def same(a, b):
    fa, ga = state(a)
    fb, gb = state(b)
    assert np.array_equal(fa, fb) and np.array_equal(ga, gb)


@pytest.mark.parametrize('precision,arith', [('fp32', 'exact'), ('fp32', 'fast'), ('fp16', 'fast'),
                                            ('fp16sr', 'fast')])
def test_batch_matches_solo(precision, arith):
    solo = [scenario(i, precision, arith) for i in range(3)]
    mem = [scenario(i, precision, arith) for i in range(3)]
    b = LiveBatch(mem)
    info = b.info
    assert info['members'] == 3 and info['tiles'] > 0 and info['grid'] > 0 and info['use_graph'] == 1
    # odd count: graph pairs plus one plain launch
    for s in solo:
        s.step(7).result()
    b.step(7).result()
    for a, m in zip(solo, mem):
        same(a, m)
        assert m.simTime == a.simTime
    # parameters change between batched steps; one member steps on its own in between
    for s in (solo[1], mem[1]):
        s.setMet(dict(u10=5.0, dirFrom=60.0, wstar=0.8, blh=700.0))
    for s in (solo[2], mem[2]):
        s.setExistingFlux(550)
    solo[0].step(3).result()
    mem[0].step(3).result()
    for s in solo:
        s.step(6).result()
    b.step(6).result()
    for a, m in zip(solo, mem):
        same(a, m)
    # the plain-launch path gives the same bits as the graph
    b.set_launch(use_graph=False)
    for s in solo:
        s.step(5).result()
    b.step(5).result()
    for a, m in zip(solo, mem):
        same(a, m)
    r1, r2 = solo[1].read().result(), mem[1].read().result()
    assert np.array_equal(r1['surf'], r2['surf']) and r1['steps'] == r2['steps']
    b.destroy()
    for s in solo + mem:
        s.destroy()


def test_batch_variants_agree():
    mem = [scenario(i) for i in range(3)]
    ref = [scenario(i) for i in range(3)]
    b = LiveBatch(mem)
    b.set_launch(minb=4, zslab=8)
    b.step(4).result()
    b.destroy()
    b2 = LiveBatch(ref)
    b2.set_launch(minb=6, zslab=-1)
    b2.step(4).result()
    with pytest.raises(Exception, match='paired levels need the FMA build'):
        b2.set_launch(pairs=True)                  # exact build: no paired variant
    b2.destroy()
    for a, m in zip(ref, mem):
        same(a, m)
    for s in mem + ref:
        s.destroy()


def test_batch_membership_rules():
    a, c = scenario(0), scenario(1)
    h = scenario(2, 'fp16', 'fast')
    with pytest.raises(LiveSolverError, match='share device, precision and arithmetic'):
        LiveBatch([a, h])
    b = LiveBatch([a, c])
    with pytest.raises(Exception, match='belongs to a batch'):
        a.destroy()
    b.destroy()
    b.destroy()                                  # idempotent
    with pytest.raises(LiveSolverError, match='batch destroyed'):
        b.step(2).result()                       # a destroyed batch rejects steps
    a.destroy()
    c.destroy()
    h.destroy()


def test_batch_membership_changes_match_solo():
    solo = [scenario(i, 'fp32', 'fast') for i in range(3)]
    mem = [scenario(i, 'fp32', 'fast') for i in range(3)]
    b = LiveBatch(mem[:2])
    b.step(5)
    b.set_members([mem[1], mem[2]])      # member 0 leaves, member 2 joins: no synchronisation in between
    b.step(4)
    b.set_members([mem[2], mem[0], mem[1]])
    b.step(3).result()
    for s, n in zip(solo, (8, 12, 7)):
        s.step(n).result()
    for a, m in zip(solo, mem):
        same(a, m)
    b.set_members([mem[1]])
    mem[0].destroy()                     # a member that left may be destroyed while the batch lives
    b.step(2).result()
    solo[1].step(2).result()
    same(solo[1], mem[1])
    b.destroy()
    for s in solo + mem[1:]:
        s.destroy()


def test_batch_paired_levels_match_solo():
    solo = [scenario(i, 'fp16', 'fast') for i in range(3)]
    mem = [scenario(i, 'fp16', 'fast') for i in range(3)]
    b = LiveBatch(mem)
    b.set_launch(minb=4, zslab=8, pairs=True)
    assert b.info['pairs'] == 1
    b.step(7).result()
    for s in solo:
        s.step(7).result()
    for a, m in zip(solo, mem):
        same(a, m)
    b.destroy()
    for s in solo + mem:
        s.destroy()


@pytest.mark.parametrize('precision', ['fp32', 'fp16sr'])
def test_batch_branches_match_solo(precision):
    """Branch mode: each member's own solo kernel (its own launch shape) on parallel graph branches, with odd step
    counts (a one-step graph), membership changes and solo steps in between, leaves every member bit-identical to
    stepping it alone."""
    solo = [scenario(i, precision, 'fast') for i in range(3)]
    mem = [scenario(i, precision, 'fast') for i in range(3)]
    for a, m, shape in zip(solo, mem, ((2504, 3), (604, 2), (404, 0))):
        for s in (a, m):
            s._dev.set_launch(*shape)
    b = LiveBatch(mem)
    b.set_launch(use_graph='branches')
    assert b.info['use_graph'] == 2
    b.step(7).result()
    for s in solo:
        s.step(7).result()
    for a, m in zip(solo, mem):
        same(a, m)
    mem[1].step(3).result()
    solo[1].step(3).result()
    b.set_members([mem[2], mem[1]])
    b.step(4).result()
    for s in (solo[2], solo[1]):
        s.step(4).result()
    for a, m in zip(solo, mem):
        same(a, m)
    b.destroy()
    for s in solo + mem:
        s.destroy()

