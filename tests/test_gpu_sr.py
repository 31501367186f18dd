"""FP16 storage with stochastic rounding (AHX_FP16_SR): the step's 16-bit stores round up with probability equal to
the dropped fraction, from a dither keyed on the cell's global index and the handle's step counter.

No reference counterpart (the reference stores f32); the checks are against the FP64 build and between runs of the
same storage: the dither sequence is a function of the step history only (not of launch shapes, graph replay, the
tuner's trials or batching), the rounding is unbiased where round-to-nearest stagnates (a heat source increment
below half an ulp of a 16-bit temperature population), and the error stays within the 16-bit bar."""
import numpy as np
import pytest

from tests.helpers import cuda_backend, rel_l2, small_solver

pytestmark = pytest.mark.gpu

MET = dict(u10=5.0, dirFrom=250.0, wstar=1.5, blh=700.0)


def bits(s):
    f, g = s._dev.read_state()
    return f.view(np.uint32), g.view(np.uint32)


def same(a, b):
    fa, ga = bits(a)
    fb, gb = bits(b)
    return np.array_equal(fa, fb) and np.array_equal(ga, gb)


def test_dithers_follow_the_step_history_only():
    """Two handles stepped through different call patterns, launch shapes and a tuner run end bit-identical; a
    handle that took one step more differs (the counter advances the dithers)."""
    a = small_solver(cuda_backend('fp16sr', 'fast'), met=MET)
    b = small_solver(cuda_backend('fp16sr', 'fast'), met=MET)
    a.step(10).result()                        # graph pairs
    b._dev.autotune(2)                         # trials on scratch copies with a scratch counter
    b._dev.set_launch(2504, 5)
    for n in (1, 3, 1, 5):                     # plain launches and graph pairs of another shape
        b.step(n).result()
    assert same(a, b)
    a.step(1).result()
    c = small_solver(cuda_backend('fp16sr', 'fast'), met=MET)
    c.step(11).result()
    assert same(a, c)
    d = small_solver(cuda_backend('fp16', 'fast'), met=MET)
    d.step(11).result()
    assert not same(a, d)                      # the storages share a format but not the rounding
    for s in (a, b, c, d):
        s.destroy()


W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def test_rounding_is_unbiased():
    """From one state on the 16-bit grid, a step's f32 results (the FP32 storage's step, same FMA arithmetic) are
    rounded to nearest by FP16 storage and stochastically by FP16_SR: every SR draw lies within one 16-bit step of
    the f32 value, and the mean of 32 draws (the step counter advances the dithers) is far closer to it than the
    round-to-nearest result."""
    h16 = small_solver(cuda_backend('fp16', 'fast'), met=MET)
    h16.step(40).result()
    X = h16._dev.read_state()                            # decoded 16-bit values: exactly representable again
    ref = small_solver(cuda_backend('fp32', 'fast'), met=MET)
    ref._dev.write_state(*X)
    ref.step(1).result()
    f32, g32 = (a.astype(np.float64) for a in ref._dev.read_state())
    h16._dev.write_state(*X)
    h16.step(1).result()
    frn, grn = (a.astype(np.float64) for a in h16._dev.read_state())
    nx, ny, nz = ref.info['nx'], ref.info['ny'], ref.info['nz']
    ktop = ref._ktopS.astype(np.int64)
    fluid = (np.arange(nz)[:, None] >= ktop[None, :]).reshape(-1)
    sr = small_solver(cuda_backend('fp16sr', 'fast'), met=MET)
    n = 32
    fsum, gsum = np.zeros_like(f32), np.zeros_like(g32)
    # one 16-bit step of each f32 value, in population units: spacing of the stored (f - w) * 16 or g * 16
    wq = np.repeat(W19, f32.size // 19)
    uf = np.spacing(np.abs((f32 - wq) * 16).astype(np.float16)).astype(np.float64) / 16
    ug = np.spacing(np.abs(g32 * 16).astype(np.float16)).astype(np.float64) / 16
    for _ in range(n):
        sr._dev.write_state(*X)
        sr.step(1).result()
        f, g = (a.astype(np.float64) for a in sr._dev.read_state())
        assert (np.abs(f - f32).reshape(19, -1)[:, fluid] <= 2 * uf.reshape(19, -1)[:, fluid] + 1e-12).all()
        assert (np.abs(g - g32).reshape(7, -1)[:, fluid] <= 2 * ug.reshape(7, -1)[:, fluid] + 1e-12).all()
        fsum += f
        gsum += g

    def rms(d, q):
        return float(np.sqrt(np.mean(d.reshape(q, -1)[:, fluid] ** 2)))

    e_rn = rms(frn - f32, 19), rms(grn - g32, 7)
    e_sr = rms(fsum / n - f32, 19), rms(gsum / n - g32, 7)
    assert e_sr[0] < 0.4 * e_rn[0] and e_sr[1] < 0.4 * e_rn[1], (e_rn, e_sr)
    for s in (h16, ref, sr):
        s.destroy()


def test_stochastic_rounding_error_vs_fp64():
    """theta after 300 steps (FMA build) within the 16-bit bar of the FP64 build, and every value finite."""
    h = small_solver(cuda_backend('fp16sr', 'fast'), met=MET)
    d = small_solver(cuda_backend('fp64', 'exact'), met=MET)
    for s in (h, d):
        s._dbg.stepOut(300).result()
    a, b = h._dbg.readDbg().reshape(-1, 4), d._dbg.readDbg().reshape(-1, 4)
    fl = b[:, 0] != 0
    assert np.isfinite(a).all()
    assert rel_l2(a[fl, 0], b[fl, 0]) <= 2e-3
    h.destroy()
    d.destroy()
