"""Host-side restatement of js/live/domain.js and the parameter code of js/live/solver.js, pinned against the
reference's archived known answers (tests/live/validation_summary.json)."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import domain as D
from ashburn_heat_twin_b200 import params as PM
from ashburn_heat_twin_b200 import solver as S
from tests.helpers import GOLDEN, MET_AUG25, campus_list


@pytest.fixture(scope='module')
def st():
    return D.load_static10(GOLDEN)


@pytest.mark.parametrize('tag,dx', [('p30a', 30), ('p20', 20), ('p40', 40)])
def test_build_domain_matches_reference(st, kat, tag, dx):
    dom = kat[tag]['domain']
    d = D.build_domain(D.aggregate(st, dx))
    assert d.zbase == dom['zbase_js']
    assert d.nz == dom['nz']
    assert int((d.nb > 0).sum()) == dom['building_columns']
    assert [int(d.kt.min()), int(d.kt.max())] == dom['kt_range']


def test_fluid_counts(st, kat):
    # info.nFluid without campuses (api20 / api30 / p40) and with A+B at 20 m (p20)
    for dx, want in ((20, kat['api20']['info']['nFluid']), (30, kat['api30']['info']['nFluid']),
                     (40, kat['p40']['info']['nFluid'])):
        d = D.build_domain(D.aggregate(st, dx))
        assert int((d.nz - d.ktop).sum()) == want
    agg = D.aggregate(st, 20)
    ras = D.rasterize_campuses(campus_list('AB'), 20, agg.nx, agg.ny)
    d = D.build_domain(agg, newArea=ras.newArea)
    assert int((d.nz - d.ktop).sum()) == kat['p20']['info']['nFluid']
    d0 = D.build_domain(agg)
    assert int((d.ktop != d0.ktop).sum()) == 828          # js/live/README.md:163-164


@pytest.mark.parametrize('tag', ['p30b', 'p20', 'p40', 'p40w'])
def test_campus_rasterisation(st, kat, tag):
    k = kat[tag]
    dx = k['info']['dx']
    agg = D.aggregate(st, dx)
    ras = D.rasterize_campuses(campus_list(k['campus']), dx, agg.nx, agg.ny)
    for got, want in zip(ras.info, k['campusInfo']):
        assert got['cells'] == want['cells']
        assert got['roofArea_m2'] == pytest.approx(want['roofArea_m2'], rel=1e-12)
        assert got['flux_wm2'] == want['flux_wm2']
        assert got['heatMW'] == pytest.approx(want['heatMW'], rel=1e-12)


def test_static10_checksum_rejects_corruption(tmp_path):
    import json
    import shutil
    shutil.copy(f'{GOLDEN}/static10.bin.gz', tmp_path / 'static10.bin.gz')
    meta = json.load(open(f'{GOLDEN}/static10.json'))
    meta['checksums']['lc_sum'] += 1
    json.dump(meta, open(tmp_path / 'static10.json', 'w'))
    with pytest.raises(D.DomainError, match='checksum mismatch'):
        D.load_static10(str(tmp_path))


@pytest.mark.parametrize('tag', ['p30a', 'p30b', 'p20', 'p40', 'p40w'])
def test_params_block_bit_exact(kat, tag):
    """The f32 parameter block, dt, conv, nsp, nsw and inflow faces equal the reference's for each validation run."""
    k = kat[tag]
    info = k['info']
    kw = dict(base=GOLDEN, dx=info['dx'], met=MET_AUG25, existingFlux=400, nsw=k['params']['nsw'],
              outflowClip=bool(k['params']['oclip']))
    if tag == 'p40':
        kw['met'] = dict(u10=6, dirFrom=75, wstar=MET_AUG25['wstar'], blh=MET_AUG25['blh'])
    if tag == 'p40w':
        kw['met'] = dict(u10=1, dirFrom=300, wstar=0, blh=MET_AUG25['blh'])
        kw['existingFlux'] = 800
    o = S._validate(kw)
    st = D.load_static10(GOLDEN)
    agg = D.aggregate(st, o['dx'])
    dom0 = D.build_domain(agg, heightM=o['heightM'])
    s = S.LiveSolver(o, st, agg, dom0, lambda nx, ny, nz: _NullDevice(), lambda t, f: None)
    s._setGeometry(True)
    s.setMet(o['met'])
    d = s._dbg.domain()
    assert s.info['dt'] == info['dt']
    assert s.info['convU'] == pytest.approx(info['convU'], rel=1e-15)
    assert s.info['nzv'] == info['nzv']
    for key in ('tau0', 'cs2smag', 'gbeta', 'prt', 'kfloor', 'momfac', 'srcscale', 'sigmax', 'nsp', 'nsw',
                'oclip'):
        assert d['params'][key] == k['params'][key], key
    assert d['inflow'] == k['inflow']
    if tag in ('p30a', 'p30b', 'p20'):
        s.setNewCampuses(campus_list(k['campus']))
        assert s._heatMW == k['heatMW']


class _NullDevice:
    adapter = 'none'

    def __getattr__(self, name):
        return lambda *a, **k: None


def test_create_rejections():
    """validate.html api: bad dx and u10Max reject with the reference's messages (validation_summary api30)."""
    with pytest.raises(S.LiveSolverError, match=r'^live solver: dx must be 20, 30 or 40 m \(got 25\)$'):
        S._validate(dict(dx=25))
    with pytest.raises(S.LiveSolverError, match=r'^live solver: u10Max must be within 1-20 m/s \(got 0\)$'):
        S._validate(dict(u10Max=0))
    with pytest.raises(S.LiveSolverError, match='heightM must be within 300-2000 m'):
        S._validate(dict(heightM=100))
    assert S._validate(dict(dx=10, allowAnyDx=True))['dx'] == 10


def test_wind_profile_and_kprofile():
    u, v, sp = PM.wind_profile(8, 0, 0.14, 24, 30)
    assert sp.max() == 8 * (150 / 10) ** 0.14
    assert np.allclose(u, 0) and np.all(v < 0)          # wind from the north blows south
    assert PM.kprofile(0.0, 0.3, 1.0, 900) == 0.0
    assert PM.default_ustar(3.09) == pytest.approx(0.3159, abs=1e-4)
    assert PM.inflow_faces(210) == dict(w=1, e=0, s=1, n=0)
    assert PM.inflow_faces(75) == dict(w=0, e=1, s=0, n=1)
    assert PM.inflow_faces(180) == dict(w=0, e=0, s=1, n=0)


def test_raw_payload_encoding_reproduces_static10(st):
    """The payload the GPU domain builder uploads (gpu_domain.raw_payload) is, for the reference's own planes, byte for
    byte the static10 payload: the dem as row-wise int16 first differences in low / high byte planes, then lc,
    frac25, hmean (u16), dca4 at the offsets static10.json lists."""
    import gzip
    import os

    from ashburn_heat_twin_b200 import gpu_domain as GD
    raw, offs = GD.raw_payload(st)
    ref = gzip.decompress(open(os.path.join(GOLDEN, 'static10.bin.gz'), 'rb').read())
    P = st.meta['planes']
    assert offs == [P[k]['offset'] for k in ('dem', 'lc', 'frac25', 'hmean', 'dca4')]
    assert raw == ref[:len(raw)]
