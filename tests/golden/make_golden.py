"""Regenerate the golden fixtures under tests/golden/ from a checkout of the reference repository.

The reference (alanhuang116/ashburn-heat-twin) ships its real Ashburn input planes (data/live/static10.json +
static10.bin.gz) and the archived results of its validation runs (tests/live/validation_summary.json). This script
copies the two input files unchanged (the checksums in static10.json are verified on load by the domain builder) and
extracts the scalar known answers the tests use into kat_live.json, so the tests run without the reference checkout
(it does not exist on the GPU machines).

usage: python tests/golden/make_golden.py <reference checkout>
"""
import gzip
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _pick(d, keys):
    return {k: d[k] for k in keys if k in d}


def main(ref):
    live = os.path.join(ref, 'data', 'live')
    for nm in ('static10.json', 'static10.bin.gz'):
        shutil.copyfile(os.path.join(live, nm), os.path.join(HERE, nm))
    meta = json.load(open(os.path.join(HERE, 'static10.json')))
    raw = gzip.decompress(open(os.path.join(HERE, 'static10.bin.gz'), 'rb').read())
    assert len(raw) == meta['raw_bytes'], 'static10 size mismatch'

    summ = json.load(open(os.path.join(ref, 'tests', 'live', 'validation_summary.json')))
    kat = {'source': 'tests/live/validation_summary.json of the reference'}
    # short parity runs (tests/live/validate.html `short`): real domain, met of 25 Aug 2024, flux 400 W/m2
    for tag in ('p30a', 'p30b', 'p20', 'p40', 'p40w'):
        e = summ[tag]
        r = e['result']
        rec = dict(
            steps=r['steps'], pre=r['pre'], inflow=r['inflow'], params=r['params'], info=r['info'],
            thetaMax=r['thetaMax'], heatMW=r['heatMW'], surfMax=r['surfMax'], surfMean=r['surfMean'],
            windMean=r['windMean'], campusInfo=r['campusInfo'],
            campus=''.join(c['id'] for c in r['campusInfo']),
            theta_max_numba=e['short_report']['theta_max_ref'],
            fluid_cells=e['short_report']['fluid_cells'],
            init_state_vs_lbm3d=e['short_report'].get('init_state_vs_lbm3d'),
        )
        if 'domain_report' in e:
            rec['domain'] = _pick(e['domain_report'], ('zbase_js', 'ktop_max', 'building_columns', 'nz', 'kt_range',
                                                       'ktop_mismatch'))
        kat[tag] = rec
    # long run (25 Aug 2024 at 30 m, 2200 s spin-up + 600 s mean, outlet clip, nsw 5)
    L = summ['L30c']
    rep = L['long_refauto_report']
    kat['L30c'] = dict(
        nspin=rep['nspin'], navg=rep['navg'], dt=rep['dt'], nsw=rep['nsw_webgpu'], oclip=rep['oclip_webgpu'],
        surface_mean_theta_webgpu=rep['surface_mean_theta']['webgpu'],
        surface_mean_theta_numba=rep['surface_mean_theta']['numba'],
        surface_mean_wind=rep['surface_mean_wind'],
        heat_budget_webgpu=rep['heat_budget_webgpu'], heat_budget_numba=rep['heat_budget_numba'],
        plume_webgpu=rep['plume_webgpu'], plume_numba=rep['plume_numba'],
        final=L['result']['final'],
    )
    # interface test (validate.html `api`) at 20 and 30 m: default settings, cold start
    for tag in ('api20', 'api30'):
        r = summ[tag]['result']
        kat[tag] = _pick(r, ('badDx', 'badU10Max', 'info', 'readNoVolNoWind', 'concurrentReads', 'campuses',
                             'heatExistingMW800', 'afterResetHeat', 'afterResetFlow', 'flowReinits', 'afterDestroy'))
    # stability matrix and direction scan: only the pass/fail outcome and the bounded maxima
    st = summ['stab']['result']['results']
    kat['stab'] = [dict(dx=r['dx'], name=r['name'], ok=r['ok'], umaxDomain=r.get('umaxDomain')) for r in st]
    kat['bench_rtx4090'] = [_pick(r, ('dx', 'wg', 'cells', 'fluid', 'median', 'msPerStep'))
                            for r in summ['benchF']['result']['results']]
    json.dump(kat, open(os.path.join(HERE, 'kat_live.json'), 'w'), indent=1)
    print('wrote', os.path.join(HERE, 'kat_live.json'))


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else '/root/reference')
