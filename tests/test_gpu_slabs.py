"""Single-domain y-slab decomposition (ahx_set_slab, ahx_row_pack / ahx_row_unpack, slabs.SlabDomain): the domain
split into 2 or 3 row slabs, each stepping its own rows with ghost rows refreshed after every step, must leave the
owned rows bit-identical to the undivided domain, with the wind crossing the slab boundaries (inflow on the south
and west faces, outflow and its sponge on the north and east faces)."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import solver as S
from ashburn_heat_twin_b200.slabs import SlabDomain
from tests.helpers import cuda_backend, small_static

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
