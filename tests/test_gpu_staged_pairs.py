"""The TMA-staged paired step of the 16-bit storages (launch shapes 2000 + 1000 + 100 x depth + rows: the interior
pairs' pull sources staged into shared memory by tensor-map box copies, tma_pairs.cuh) leaves exactly the state of the
plain paired step (2504) it restates: same relaxation, same stores, same stochastic-rounding dithers. Checked on the
small synthetic domain with whole columns and with even and odd z-slabs, and on the 600x600x64 benchmark domain in
the shapes the benchmark tries."""
import numpy as np
import pytest

import bench
from tests.helpers import cuda_backend, small_solver

pytestmark = pytest.mark.gpu

SHAPES = ((3204, 0), (3304, 8), (3404, 6), (3304, 7), (3208, 4), (3308, 0))


def _state_bits(s):
    f, g = s._dev.read_state()
    return f.view(np.uint32).copy(), g.view(np.uint32).copy()


@pytest.mark.parametrize('precision', ['fp16', 'bf16', 'fp16sr'])
def test_staged_pairs_bit_identical_small(precision):
    met = dict(u10=5.0, dirFrom=300.0, wstar=1.5, blh=700.0)
    ref = small_solver(cuda_backend(precision, 'fast'), met=met)
    ref._dev.set_launch(2504, 4)
    ref.step(9).result()
    fr, gr = _state_bits(ref)
    ref.destroy()
    for shape, zs in SHAPES:
        s = small_solver(cuda_backend(precision, 'fast'), met=met)
        s._dev.set_launch(shape, zs)
        s.step(9).result()
        f, g = _state_bits(s)
        assert np.array_equal(f, fr) and np.array_equal(g, gr), (shape, zs)
        s.destroy()


@pytest.mark.parametrize('precision', ['fp16', 'fp16sr'])
def test_staged_pairs_bit_identical_c2(precision):
    ref = bench.make_solver(backend=cuda_backend(precision, 'fast'), workload='c2')
    ref._dev.set_launch(2504, 4)
    ref.step(4).result()
    fr, gr = _state_bits(ref)
    ref.destroy()
    for shape, zs in ((3304, 0), (3404, 32), (3208, 16)):
        s = bench.make_solver(backend=cuda_backend(precision, 'fast'), workload='c2')
        s._dev.set_launch(shape, zs)
        s.step(4).result()
        f, g = _state_bits(s)
        assert np.array_equal(f, fr) and np.array_equal(g, gr), (shape, zs)
        s.destroy()


def test_staged_pairs_rejects_other_storages():
    s = small_solver(cuda_backend('fp32', 'fast'))
    with pytest.raises(Exception):
        s._dev.set_launch(3404, 0)
    s.destroy()
