"""The domain builder on the GPU (ahx_static_* / ahx_domain_build) against the host restatement of js/live/domain.js
(domain.py) and the column record of js/live/solver.js:359-376 (params.pack_columns): on the reference's own Ashburn
planes at 20, 30 and 40 m, with and without the validation page's campuses A and B, the ktop plane, the packed column
records (kt, ktop, cd bits, source bits), the campus heat and roof area, nz and zbase are bit-identical; the device's
plane checksums equal static10.json's; and the A+B campus delta at 20 m is the reference's 828 columns
(js/live/README.md:163-164). A synthetic box (row-delta encoded here) is checked the same way."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import domain as D
from ashburn_heat_twin_b200 import gpu_domain as GD
from ashburn_heat_twin_b200 import params as PM
from ashburn_heat_twin_b200 import synth
from tests.helpers import GOLDEN, campus_list

pytestmark = pytest.mark.gpu


def host_images(st, dx, campuses, flux, dt, heightM=720):
    agg = D.aggregate(st, dx)
    ras = D.rasterize_campuses(campuses, dx, agg.nx, agg.ny)
    dom = D.build_domain(agg, heightM=heightM, newArea=ras.newArea)
    ktS = D.flip_rows(dom.kt, agg.nx, agg.ny)
    ktopS = D.flip_rows(dom.ktop, agg.nx, agg.ny)
    cdS = D.flip_rows(dom.cd, agg.nx, agg.ny)
    colv, totalW, q = PM.pack_columns(ktS, ktopS, cdS, agg.dcarea, flux, ras.heatW, agg.nx, agg.ny, dx, dt)
    return dom, ras, colv, ktopS.astype(np.uint32)


@pytest.fixture(scope='module')
def real():
    st = D.load_static10(GOLDEN)
    g = GD.GpuDomain(st)
    yield st, g
    g.destroy()


def test_checksums_match_static10(real):
    st, g = real
    want = {k: st.meta['checksums'][k] for k in ('dem_sum_cm', 'lc_sum', 'frac25_sum', 'hmean_sum_cm', 'dca4_sum')}
    assert g.checksums() == want


@pytest.mark.parametrize('dx', [20, 30, 40])
@pytest.mark.parametrize('which', ['', 'AB', 'ABC'])
def test_images_bit_identical_to_host(real, dx, which):
    st, g = real
    camp = campus_list(which)
    dt = 0.1 * dx / 11.0
    dom, ras, colv, ktop = host_images(st, dx, camp, 400.0, dt)
    out = g.build(dx, heightM=720, campuses=camp, flux=400.0, dt=dt)
    assert (out['nx'], out['ny'], out['nz']) == (dom.nx, dom.ny, dom.nz)
    assert out['zbase'] == dom.zbase and out['ktopMax'] == dom.ktopMax and out['nbCells'] == dom.nbCells
    assert np.array_equal(out['ktop'], ktop)
    assert np.array_equal(out['colv'], colv)
    assert np.array_equal(out['heatW'].view(np.uint64), ras.heatW.view(np.uint64))
    assert np.array_equal(out['newArea'].view(np.uint64), ras.newArea.view(np.uint64))
    for c, info in zip(out['campusFlux'], ras.info):
        assert c == info['flux_wm2']


def test_campus_delta_at_20m_is_the_reference_828(real):
    st, g = real
    a = g.build(20, campuses=campus_list('AB'), dt=0.1)
    b = g.build(20, campuses=[], dt=0.1)
    assert int((a['ktop'] != b['ktop']).sum()) == 828


def test_synthetic_box_bit_identical():
    st = synth.make_static10(synth.C1)
    g = GD.GpuDomain(st)
    rng = np.random.default_rng(2)
    from ashburn_heat_twin_b200 import scenarios as SC
    camp = [dict(id='S', mw=120.0, halls=[SC.free_site(st, rng)])]
    for dx in (30, 40, 20):
        dt = 0.1 * dx / 13.0
        dom, ras, colv, ktop = host_images(st, dx, camp, 350.0, dt, heightM=960)
        out = g.build(dx, heightM=960, campuses=camp, flux=350.0, dt=dt)
        assert out['nz'] == dom.nz and np.array_equal(out['colv'], colv) and np.array_equal(out['ktop'], ktop)
    g.destroy()
