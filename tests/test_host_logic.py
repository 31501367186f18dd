"""Host behaviour of the live solver (js/live/solver.js semantics) driven against the CPU oracle device on a small
synthetic domain: controls, clamps, flow re-initialisation, campus geometry changes, resets, destroy."""
import numpy as np
import pytest

from ashburn_heat_twin_b200 import solver as S
from tests.helpers import oracle_backend, small_solver


@pytest.fixture()
def s():
    x = small_solver(oracle_backend())
    yield x
    x.destroy()


def test_setmet_clamps(s):
    s.setMet(dict(u10=50, dirFrom=-30, wstar=-1, blh=1e6))
    m = s._met
    assert m['u10'] == 8 and m['dirFrom'] == 330 and m['wstar'] == 0 and m['blh'] == 5000
    s.setMet(dict(u10=0.1))
    assert s._met['u10'] == 0.5
    assert s._met['dirFrom'] == 330     # unspecified fields keep the previous value


def test_flow_reinit_on_big_turn_only(s):
    n0 = s.flowReinits
    s.setMet(dict(u10=4, dirFrom=270))     # 20 degrees from 250: applied directly
    assert s.flowReinits == n0
    s.setMet(dict(u10=4, dirFrom=70))      # 200 degrees: flow re-initialised
    assert s.flowReinits == n0 + 1


def test_lagged_reference_direction(s):
    s.setMet(dict(u10=4, dirFrom=275))     # 25 deg, below the 30 deg tolerance
    s.step(int(600 / s.info['dt'])).result()   # the interior adjusts toward 275 with a 300 s lag
    assert s._flowRef['dir'] == pytest.approx(275 - 25 * np.exp(-600 * 1 / 300) * 1, abs=1.0)


def test_resets_and_simtime(s):
    s.step(10).result()
    assert s.simTime == pytest.approx(10 * s.info['dt'])
    s.resetHeat()
    assert s.simTime == 0
    r = s.read().result()
    assert r['thetaMax'] == 0
    s.step(5).result()
    s.resetFlow()
    st = s._dbg.stats()
    assert st['steps'] == 0 and st['nonFinite'] == 0 and st['thetaMax'] == 0


def test_campus_add_remove_reinitialises_uncovered_cells():
    s = small_solver(oracle_backend(), dx=10)
    nf0 = s.info['nFluid']
    # a 200 m x 150 m hall inside the small box (scene origin is the west/north corner)
    campus = [dict(id='X', mw=50, halls=[[-2995 + 100, -2995 + 100, -2995 + 300, -2995 + 250]])]
    s.setNewCampuses(campus)
    assert s.info['nFluid'] < nf0
    assert s.campusInfo[0]['heatMW'] == pytest.approx(50)
    s.step(3).result()
    s.setNewCampuses([])
    assert s.info['nFluid'] == nf0
    # cells uncovered again hold rest equilibrium and theta 0 until the next step
    f, g = s._dbg.readState()['f'], s._dbg.readState()['g']
    N = s.info['nCells']
    ktop_now = s._ktopS
    assert np.isfinite(f).all() and np.isfinite(g).all() and f.size == 19 * N and ktop_now.size * s.info['nz'] == N
    s.destroy()


def test_destroy_is_idempotent_and_rejects_later_calls(s):
    s.destroy()
    s.destroy()
    with pytest.raises(S.LiveSolverError, match='^live solver: destroyed$'):
        s.setMet(dict(u10=3))
    with pytest.raises(S.LiveSolverError, match='destroyed'):
        s.step(1).result()


def test_existing_flux_updates_heat(s):
    s.setExistingFlux(800)
    h800 = s.info['heatExistingMW']
    s.setExistingFlux(400)
    assert h800 == pytest.approx(2 * s.info['heatExistingMW'])
    s.setExistingFlux('junk')
    assert s.info['heatExistingMW'] == 0
