"""Seeded scenario sets for batched and served runs of the live solver.

A scenario is what one createLiveSolver + setMet + setExistingFlux + setNewCampuses sequence needs: grid spacing and
domain height, a met state, the operational roof flux and one new campus. The reference drives one such scenario per
page (js/live.js); ensembles and the serving loop run many on one device.

- batch64: 32 scenarios on the 6 km box at 30 m (200x200x32) and 32 at 40 m (150x150x24); wind direction
  U[0, 360), 10 m speed U[2, 8] m/s, roof flux U[200, 600] W/m^2, one 120 MW campus (a 300 x 300 m hall, 1,333 W/m^2)
  at a random building-free site.
- serving mix: 40 % 40 m (150x150x24), 40 % 30 m (200x200x32), 20 % 20 m (300x300x48), each run for 10 simulated
  minutes.
"""
from __future__ import annotations

import math

import numpy as np

from . import domain as DM
from . import params as PM

HALL_M = 300.0
CAMPUS_MW = 120.0


def free_site(static: DM.Static10, rng: np.random.Generator, side_m: float = HALL_M, tries: int = 200):
    """A side_m x side_m square (scene metres, [x0, z0, x1, z1]) inside the box whose 10 m cells carry no building
    cover (the least-covered of `tries` random candidates if none is entirely free)."""
    n10 = int(round(side_m / 10.0))
    frac = static.frac25.reshape(static.nrows, static.ncols)
    best, best_cov = None, None
    for _ in range(tries):
        c0 = int(rng.integers(2, static.ncols - n10 - 2))
        r0 = int(rng.integers(2, static.nrows - n10 - 2))
        cov = int(frac[r0:r0 + n10, c0:c0 + n10].sum())
        if best is None or cov < best_cov:
            best, best_cov = (c0, r0), cov
            if cov == 0:
                break
    c0, r0 = best
    x0, z0 = DM.SCENE_X0 + c0 * 10.0, DM.SCENE_Z0 + r0 * 10.0
    return [x0, z0, x0 + side_m, z0 + side_m]


def random_met(rng: np.random.Generator, speed=(2.0, 8.0)):
    return dict(u10=float(rng.uniform(*speed)), dirFrom=float(rng.uniform(0.0, 360.0)), wstar=1.67, blh=903.0)


def batch64(static: DM.Static10, seed: int = 4):
    """The 64 seeded scenarios of the batched workload (32 at 30 m, then 32 at 40 m)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(64):
        dx = 30 if i < 32 else 40
        out.append(dict(id=i, dx=dx, heightM=960, met=random_met(rng), flux=float(rng.uniform(200.0, 600.0)),
                        campus=dict(id=f'S{i}', mw=CAMPUS_MW, halls=[free_site(static, rng)])))
    return out


# the serving mix: (share, dx, heightM); 10 simulated minutes each
SERVE_MIX = ((0.4, 40, 960), (0.4, 30, 960), (0.2, 20, 960))
SERVE_SIM_S = 600.0


def steps_for(dx: float, heightM: float = 960, sim_s: float = SERVE_SIM_S, u10max: float = 8.0,
              alpha: float = PM.ALPHA):
    """Steps of one request: sim_s / dt with the solver's dt = 0.1 dx / Umax, Umax the profile maximum at u10Max
    (solver.js:107-112)."""
    nz = int(round(heightM / dx))
    umax = float(PM.wind_profile(u10max, 0, alpha, nz, dx)[2].max())
    return int(math.ceil(sim_s / (0.1 * dx / umax)))


def serve_trace(static: DM.Static10, n: int, rate_hz: float, seed: int = 5):
    """n requests with Poisson arrivals at rate_hz: arrival time (s), grid class, met, flux and one campus."""
    rng = np.random.default_rng(seed)
    t = 0.0
    shares = np.cumsum([m[0] for m in SERVE_MIX])
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate_hz))
        cls = int(np.searchsorted(shares, rng.uniform(0.0, shares[-1]), side='right'))
        cls = min(cls, len(SERVE_MIX) - 1)
        _, dx, hm = SERVE_MIX[cls]
        out.append(dict(id=i, arrival=t, dx=dx, heightM=hm, met=random_met(rng),
                        flux=float(rng.uniform(200.0, 600.0)),
                        campus=dict(id=f'R{i}', mw=CAMPUS_MW, halls=[free_site(static, rng)])))
    return out
