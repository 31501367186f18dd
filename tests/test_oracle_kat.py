"""The CPU oracle (oracle/lbm_oracle.cpp) pinned against the reference's archived results on the real Ashburn
domain: the WebGPU solver's read() after 300 cold-start steps (validation_summary.json p30a and api30)."""
import numpy as np
import pytest

from tests.helpers import oracle_backend, real_solver, surf_stats


def test_oracle_p30a(kat):
    """Cold start, 30 m, prototype outlet (oclip 0), sponge width 16, 300 steps (validate.html `short`, tag p30a).
    The published WebGPU-vs-numba agreement is ~3e-6 relative; the f32 oracle must land within that band."""
    k = kat['p30a']
    s = real_solver(oracle_backend(), dx=30, nsw=16, outflowClip=False)
    s.setNewCampuses([])
    s._dbg.stepOut(k['steps']).result()
    r = s.read(vol=True, wind=True, volMax=3).result()
    ss = surf_stats(r)
    assert r['thetaMax'] == pytest.approx(k['thetaMax'], rel=3e-6)
    assert ss['surfMax'] == pytest.approx(k['surfMax'], rel=3e-6)
    assert ss['surfMean'] == pytest.approx(k['surfMean'], rel=3e-6)
    assert ss['windMean'] == pytest.approx(k['windMean'], rel=3e-6)
    assert r['heatMW'] == k['heatMW']
    assert ss['nan'] == 0
    # the numba reference's own theta max lies within the same band
    assert r['thetaMax'] == pytest.approx(k['theta_max_numba'], rel=5e-6)
    # the step output (theta of all fluid cells) is finite and its surface maximum matches the read-back
    dbg = s._dbg.readDbg().reshape(-1, 4)
    assert np.isfinite(dbg).all()
    s.destroy()


def test_oracle_api30(kat):
    """Default live settings at 30 m (outlet clip on, sponge width 5): read().thetaMax after 300 steps
    (validate.html `api`, tag api30)."""
    k = kat['api30']
    s = real_solver(oracle_backend(), dx=30)
    s.step(300).result()
    r = s.read(vol=False, wind=False).result()
    assert r['u'] is None and r['v'] is None and r['vol'] is None
    assert r['surf'].size == k['readNoVolNoWind']['surf']
    assert r['thetaMax'] == pytest.approx(k['readNoVolNoWind']['thetaMax'], rel=3e-6)
    assert r['simTime'] == pytest.approx(k['readNoVolNoWind']['simTime'], rel=1e-12)
    s.destroy()


def test_oracle_restores_the_callers_floating_point_mode():
    """The oracle flushes f32 subnormals inside its own parallel regions only (as the CUDA build's -ftz=true does);
    the calling thread keeps gradual underflow afterwards, so host-side metrics computed next to it are unaffected."""
    from tests.helpers import small_solver
    tiny = np.array([1e-40], np.float32)
    assert (tiny * np.float32(1.0))[0] != 0          # subnormals survive before the oracle runs
    s = small_solver(oracle_backend())
    s._dbg.stepOut(2).result()
    s.read(vol=True, wind=True).result()
    s._dbg.stats()
    s.destroy()
    assert (tiny * np.float32(1.0))[0] != 0          # ... and after it
    assert np.float64(5e-324) * 1.0 != 0
