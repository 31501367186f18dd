"""The 10-minute mean of the 16-bit storage with stochastic rounding against the FP64 build, at the 200x200x32
workload's own size (30 m cells, seeded synthetic terrain and buildings, 4 m/s from 270 deg, alpha 0.2).

Both runs start cold, spin up for 2 simulated minutes, then take a 10-minute window with the FP64 heat budget and
the FP64 near-ground / lateral-face time accumulators fused into the step. Against the FP64 build (exact arithmetic):
  - FP16 storage with stochastic rounding (AHX_FP16_SR, the FMA build a deployment runs): mean near-ground theta
    (the first fluid cell of every column) within rel-L2 1e-3, peak mean warming within 1e-3 relative, and the heat
    closure (injected - advected out - content change, as a fraction of the injected heat) within 2e-3 of FP64's
    (measured 1.2e-3: the temperature populations are stored in 16 bits too);
  - FP32 storage (FMA build): the mean within rel-L2 1e-4 (the 10-minute-mean bar for f32).
The metric definitions follow tools/live/validate_live.py:226-240 (heat budget) and :146-154 (rel-L2) of the
reference; the advected heat here is the mean of theta * u_n summed over the lateral faces (the fused budget)."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import params as PM
from tests.helpers import cuda_backend, rel_l2
from tests.test_gpu_c1 import c1_solver

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(900)]


def _window(precision, arith, spin_s=120.0, mean_s=600.0):
    s = c1_solver(cuda_backend(precision, arith))
    dev = s._dev
    dt, dx, nz = s.info['dt'], s.info['dx'], s.info['nz']
    spin, mean = int(round(spin_s / dt)), int(round(mean_s / dt))
    s.step(spin).result()
    st0 = dev.stats()
    dev.budget_enable(True)
    dev.budget_read(reset=True)
    dev.accum_enable(True)
    dev.accum_read(reset=True)
    s.step(mean).result()
    bud = dev.budget_read(reset=True)
    surf, _, n = dev.accum_read(reset=True)
    dev.budget_enable(False)
    dev.accum_enable(False)
    st1 = dev.stats()
    assert n == mean and st1['nonFinite'] == 0
    ktop = s._ktopS.astype(np.int64)
    cols = np.nonzero(ktop < nz)[0]
    ng = surf[0].reshape(-1)[cols] / n
    rc = PM.RHO_CP * dx ** 3 / (mean * dt) / 1e6          # lattice K summed over the window -> MW
    ftu = bud['face_theta_u']                              # west, east, south, north
    inj = rc * bud['src_sum']
    adv = rc * (ftu[1] - ftu[0] + ftu[3] - ftu[2])
    content = rc * (st1['sumTheta'] - st0['sumTheta'])
    s.destroy()
    return dict(ng=ng, peak=float(ng.max()), closure=(inj - adv - content) / inj, injected=inj)


@pytest.fixture(scope='module')
def fp64_window():
    return _window('fp64', 'exact')


def test_fp16_stochastic_rounding_ten_minute_mean_within_1e3(fp64_window):
    r = _window('fp16sr', 'fast')
    ref = fp64_window
    err = rel_l2(r['ng'], ref['ng'])
    assert err <= 1e-3, err
    assert abs(r['peak'] / ref['peak'] - 1) <= 1e-3, (r['peak'], ref['peak'])
    assert abs(r['closure'] - ref['closure']) <= 2e-3, (r['closure'], ref['closure'])
    assert r['injected'] == pytest.approx(ref['injected'], rel=1e-5)


def test_fp32_ten_minute_mean_within_1e4(fp64_window):
    r = _window('fp32', 'fast')
    err = rel_l2(r['ng'], fp64_window['ng'])
    assert err <= 1e-4, err
    assert abs(r['closure'] - fp64_window['closure']) <= 1e-4, (r['closure'], fp64_window['closure'])
