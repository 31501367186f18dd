"""ahx_stats_noalloc: diagnostics for callers that cannot allocate device memory when they ask for them (an engine
whose device memory all belongs to its own pool, or a latency-critical path where an allocation would synchronise). The caller owns every buffer; the entry
point keeps its per-block partial sums in a fixed scratch array inside the library.

Checked through the C ABI against ahx_stats on the same state, on two calls in a row, with the tolerance the other
diagnostics tests use (FP64 sums 1e-12 relative; maxima and counts exact). Runs alone in a fresh process as well as
after the rest of the suite (this file sorts last so a failure here never hides another test's).
"""
import ctypes

import numpy as np
import pytest

from ashburn_heat_twin_b200 import cuda_device as CD
from tests.helpers import cuda_backend, real_solver

pytestmark = pytest.mark.gpu


def _noalloc_stats(lib, s, torch):
    """Copy the solver's state into caller-owned device buffers (reference layout) and run ahx_stats_noalloc."""
    f, g = s._dev.read_state()
    ktop = s._ktopS.astype(np.uint32)
    tf = torch.from_numpy(f).cuda()
    tg = torch.from_numpy(g).cuda()
    tk = torch.from_numpy(ktop.view(np.int32)).cuda()
    out = torch.zeros(ctypes.sizeof(CD.StatsOut), dtype=torch.uint8, device='cuda')
    stream = torch.cuda.current_stream()
    st = lib.ahx_stats_noalloc(s.info['nx'], s.info['ny'], s.info['nz'], ctypes.c_void_p(tf.data_ptr()),
                               ctypes.c_void_p(tg.data_ptr()), ctypes.c_void_p(tk.data_ptr()),
                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert st == 0, lib.ahx_last_error()
    stream.synchronize()
    return CD.StatsOut.from_buffer_copy(out.cpu().numpy().tobytes())


def _same(a, b):
    assert a.count == b['count'] and a.non_finite == b['nonFinite']
    assert a.theta_max == np.float32(b['thetaMax']) and a.umax == np.float32(b['umax'])
    assert a.sum_theta == pytest.approx(b['sumTheta'], rel=1e-12)
    assert a.sum_ke == pytest.approx(b['sumKE'], rel=1e-12)
    assert a.sum_rho_dev == pytest.approx(b['sumRhoDev'], rel=1e-12, abs=1e-15)


def test_stats_noalloc_matches_handle_stats():
    import torch
    lib = CD.load_library()
    s = real_solver(cuda_backend('fp32', 'exact'), dx=30)
    s.step(120).result()
    a1 = _noalloc_stats(lib, s, torch)
    _same(a1, s._dev.stats())
    assert a1.count > 0 and a1.sum_theta > 0
    s.step(60).result()
    a2 = _noalloc_stats(lib, s, torch)          # second call in a row, on the advanced state
    _same(a2, s._dev.stats())
    assert a2.sum_theta != a1.sum_theta
    a3 = _noalloc_stats(lib, s, torch)          # same state again: the fixed-order reduction repeats exactly
    assert bytes(a3) == bytes(a2)
    s.destroy()


def test_stats_noalloc_rejects_oversize_grid():
    lib = CD.load_library()
    dummy = ctypes.c_void_p(16)
    st = lib.ahx_stats_noalloc(4096, 4096, 16, dummy, dummy, dummy, dummy, None)
    assert st == 1
    assert b'at most 134217728 cells' in lib.ahx_last_error()
