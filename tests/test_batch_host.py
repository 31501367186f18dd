"""Host-side rules of LiveBatch that need no GPU: members must use the CUDA backend, a batch needs members."""
import pytest

from ashburn_heat_twin_b200 import LiveBatch, LiveSolverError
from tests.helpers import oracle_backend, small_solver


def test_batch_needs_members_and_the_cuda_backend():
    with pytest.raises(LiveSolverError, match='at least one solver'):
        LiveBatch([])
    s = small_solver(oracle_backend())
    with pytest.raises(LiveSolverError, match='needs the CUDA backend'):
        LiveBatch([s])
    s.destroy()
