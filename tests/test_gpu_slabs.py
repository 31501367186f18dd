"""Single-domain y-slab decomposition (ahx_set_slab, the 6-plane halos ahx_halo_*, the split step ahx_step_rows,
slabs.SlabDomain): the domain split into row slabs, each stepping its boundary rows, packing their halos and then
stepping its interior rows, with ghost rows refreshed after every step, must leave the owned rows bit-identical to the
undivided domain and, in the exact build, to the CPU oracle, with the wind crossing the slab boundaries (inflow on the
south and west faces, outflow and its sponge on the north and east faces)."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import solver as S
from ashburn_heat_twin_b200.slabs import SlabDomain
from tests.helpers import cuda_backend, oracle_backend, small_static

pytestmark = pytest.mark.gpu


def opts():
    return dict(static=small_static(seed=5), dx=10, allowAnyDx=True, heightM=300, u10Max=8,
                met=dict(u10=5.0, dirFrom=200.0, wstar=1.5, blh=700.0), existingFlux=400, nsw=6)


@pytest.mark.parametrize('nslabs,precision,arith', [(2, 'fp32', 'exact'), (3, 'fp32', 'exact'), (3, 'fp32', 'fast'),
                                                    (2, 'fp16', 'fast'), (3, 'fp16sr', 'fast')])
def test_slabs_match_the_undivided_domain(nslabs, precision, arith):
    whole = S.create_live_solver(backend=cuda_backend(precision, arith), **opts())
    sd = SlabDomain(nslabs, precision=precision, arith=arith, **opts())
    nx, ny, nz = whole.info['nx'], whole.info['ny'], whole.info['nz']
    assert (sd.nx, sd.ny, sd.nz) == (nx, ny, nz)
    f0, g0 = whole._dev.read_state()
    f1, g1 = sd.read_state()
    assert np.array_equal(f0.reshape(19, nz, ny, nx), f1) and np.array_equal(g0.reshape(7, nz, ny, nx), g1)
    whole.step(9).result()
    sd.step(9)
    f0, g0 = whole._dev.read_state()
    f1, g1 = sd.read_state()
    assert np.array_equal(f0.reshape(19, nz, ny, nx).view(np.uint32), f1.view(np.uint32))
    assert np.array_equal(g0.reshape(7, nz, ny, nx).view(np.uint32), g1.view(np.uint32))
    whole.destroy()
    sd.destroy()


def test_exact_slabs_match_the_oracle():
    """Three slabs of the exact build against the CPU oracle on the same domain, directly (not through the undivided
    CUDA domain)."""
    o = S.create_live_solver(backend=oracle_backend(), **opts())
    sd = SlabDomain(3, precision='fp32', arith='exact', **opts())
    o.step(6).result()
    sd.step(6)
    nx, ny, nz = o.info['nx'], o.info['ny'], o.info['nz']
    st = o._dbg.readState()
    f1, g1 = sd.read_state()
    assert np.array_equal(st['f'].reshape(19, nz, ny, nx).view(np.uint32), f1.view(np.uint32))
    assert np.array_equal(st['g'].reshape(7, nz, ny, nx).view(np.uint32), g1.view(np.uint32))
    o.destroy()
    sd.destroy()


@pytest.mark.parametrize('nslabs', [24, 33])
def test_thin_slabs_of_one_and_two_rows(nslabs):
    """Slabs of one or two owned rows: the split step's boundary and interior parts degenerate (a row is both
    boundaries, the interior is empty) and the result stays the undivided domain's."""
    whole = S.create_live_solver(backend=cuda_backend('fp32', 'fast'), **opts())
    sd = SlabDomain(nslabs, precision='fp32', arith='fast', **opts())
    assert min(b - a for a, b in sd.rows) == (2 if nslabs == 24 else 1)
    whole.step(4).result()
    sd.step(4)
    nx, ny, nz = whole.info['nx'], whole.info['ny'], whole.info['nz']
    f0, g0 = whole._dev.read_state()
    f1, g1 = sd.read_state()
    assert np.array_equal(f0.reshape(19, nz, ny, nx).view(np.uint32), f1.view(np.uint32))
    assert np.array_equal(g0.reshape(7, nz, ny, nx).view(np.uint32), g1.view(np.uint32))
    whole.destroy()
    sd.destroy()


def test_step_in_row_bands_equals_one_step():
    """ahx_step_rows over bands covering all rows, the last one advancing, is one step, bit for bit; a
    stochastic-rounding state refuses it; a halo is 6 of a row's 26 planes."""
    a = S.create_live_solver(backend=cuda_backend('fp32', 'fast'), **opts())
    b = S.create_live_solver(backend=cuda_backend('fp32', 'fast'), **opts())
    ny = a.info['ny']
    for _ in range(3):
        a._dev.step(1, 0)
        b._dev.step_rows(0, 7, False)
        b._dev.step_rows(30, ny, False)
        b._dev.step_rows(7, 30, True)
    fa, ga = a._dev.read_state()
    fb, gb = b._dev.read_state()
    assert np.array_equal(fa.view(np.uint32), fb.view(np.uint32)) and np.array_equal(ga.view(np.uint32),
                                                                                   gb.view(np.uint32))
    nx, nz, px = a.info['nx'], a.info['nz'], None
    assert b._dev.halo_bytes() == 6 * nz * nx * 4
    sr = S.create_live_solver(backend=cuda_backend('fp16sr', 'fast'), **opts())
    from ashburn_heat_twin_b200.cuda_device import AhxError
    with pytest.raises(AhxError):
        sr._dev.step_rows(0, 5, False)
    for s in (a, b, sr):
        s.destroy()
