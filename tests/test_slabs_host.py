"""Host side of the y-slab decomposition: the row split covers the domain exactly, and the recording device keeps the
same host images the live solver uploads to a real device."""
import numpy as np

from ashburn_heat_twin_b200 import slabs as SL
from ashburn_heat_twin_b200 import solver as S
from tests.helpers import oracle_backend, small_static


def test_slab_rows_partition_the_domain():
    for ny, n in ((48, 2), (48, 3), (50, 3), (7, 7)):
        rows = SL.slab_rows(ny, n)
        assert rows[0][0] == 0 and rows[-1][1] == ny and all(a < b for a, b in rows)
        assert all(rows[r][1] == rows[r + 1][0] for r in range(n - 1))


def test_recorder_keeps_the_uploaded_images():
    st = small_static(seed=5)
    o = dict(static=st, dx=10, allowAnyDx=True, heightM=300, u10Max=8,
             met=dict(u10=5.0, dirFrom=200.0, wstar=1.5, blh=700.0), existingFlux=400)
    rec = {}

    def recorder(nx, ny, nz):
        rec['d'] = SL._Recorder(nx, ny, nz)
        return rec['d']

    h = S.create_live_solver(backend=recorder, **o)
    ref = S.create_live_solver(backend=oracle_backend(), **o)
    d = rec['d']
    assert d.params == bytes(ref._params)
    assert np.array_equal(d.ktop.reshape(-1), ref._ktopS.astype(np.uint32))
    assert np.array_equal(d.colv.reshape(-1, 4), np.asarray(ref._colv, np.uint32).reshape(-1, 4))
    h.destroy()
    ref.destroy()
