"""B200-native (sm_100a) coupled D3Q19 flow + D3Q7 heat lattice-Boltzmann step of the ashburn-heat-twin live solver,
behind the live solver's host API (createLiveSolver) and a C ABI (include/ahx.h, libahx.so)."""
from .solver import (LiveBatch, LiveSolver, LiveSolverError, Pending, createLiveSolver,  # noqa: F401
                     create_live_solver)
