"""The stochastic-rounding dither of AHX_FP16_SR, restated on the CPU (numpy) from its definition: a per-cell seed
(an xorshift-multiply integer finaliser of the global cell index mixed with the step key), population slot p's
dither = bits 16-28 of seed x M_p (M_p odd), which the kernel hands to the stochastic-rounding conversion
(cvt.rs.f16x2.f32: a two-value instruction that adds its low half's dither from bits 0-12 and its high half's from
bits 16-28 of the random operand, below the 13 mantissa bits an f32 -> f16 conversion drops, then truncates the
magnitude). The kernel moves bits 16-31 of each cell's product into the half the conversion reads, so a cell's
dither is the same whether it is converted alone or paired with the level above. Checks: each slot's dither is
uniform, slots are uncorrelated, and dither + truncation is unbiased in the f16 normal range. (The device code
itself is checked on the GPU in test_gpu_sr.py.)"""
import numpy as np

M32 = 0xFFFFFFFF


def mix32(x):
    x = np.asarray(x, dtype=np.uint64) & M32
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(0x7feb352d)) & M32
    x ^= x >> np.uint64(15)
    x = (x * np.uint64(0x846ca68b)) & M32
    x ^= x >> np.uint64(16)
    return x


def slot_mul(p):
    return int(mix32((0x2545f491 + 0x9e3779b9 * p) & M32)) | 1


def dithers(seeds, p):
    return (((seeds * np.uint64(slot_mul(p))) & M32) >> np.uint64(16)) & np.uint64(0x1FFF)


def rbits_pair(seed_lo, seed_hi, p):
    """The random operand of one paired conversion: bits 16-31 of the low cell's product in its low half, of the high
    cell's in its high half (a byte permutation in the kernel)."""
    m = np.uint64(slot_mul(p))
    lo = ((np.asarray(seed_lo, np.uint64) * m) & M32) >> np.uint64(16)
    hi = ((np.asarray(seed_hi, np.uint64) * m) & M32) >> np.uint64(16)
    return lo | (hi << np.uint64(16))


def test_paired_operand_gives_each_cell_its_own_dither():
    """The conversion reads bits 0-12 (low value) and 16-28 (high value) of the operand: those are exactly the two
    cells' single-cell dithers."""
    rng = np.random.default_rng(5)
    a = rng.integers(0, 2 ** 32, 1000, dtype=np.uint64)
    b = rng.integers(0, 2 ** 32, 1000, dtype=np.uint64)
    for p in (0, 7, 25):
        r = rbits_pair(a, b, p)
        assert np.array_equal(r & np.uint64(0x1FFF), dithers(a, p))
        assert np.array_equal((r >> np.uint64(16)) & np.uint64(0x1FFF), dithers(b, p))


def test_slot_multipliers_are_odd_and_distinct():
    ms = [slot_mul(p) for p in range(26)]
    assert all(m & 1 for m in ms) and len(set(ms)) == 26


def test_dithers_uniform_and_uncorrelated():
    rng = np.random.default_rng(3)
    gid = rng.integers(0, 23_040_000, 200_000, dtype=np.uint64)
    key = int(mix32(17 * 0x9e3779b9 + 0x632be5ab))
    seeds = mix32(gid ^ np.uint64(key))
    d = np.stack([dithers(seeds, p).astype(np.float64) for p in range(26)])
    assert d.min() >= 0 and d.max() < 8192
    # uniform on [0, 8192): mean 4095.5, variance 8192^2/12
    assert np.allclose(d.mean(axis=1), 4095.5, rtol=0.01)
    assert np.allclose(d.var(axis=1), 8192 ** 2 / 12, rtol=0.02)
    c = np.corrcoef(d)
    off = c[~np.eye(26, dtype=bool)]
    assert np.abs(off).max() < 0.02
    # 16 equal bins per slot, chi-square well inside the 99.9 % bound for 15 degrees of freedom
    for row in d:
        h = np.bincount((row // 512).astype(np.int64), minlength=16)
        e = row.size / 16
        assert ((h - e) ** 2 / e).sum() < 37.7


def test_dither_then_truncate_is_unbiased():
    rng = np.random.default_rng(4)
    v = rng.uniform(-4.0, 4.0, 4000).astype(np.float32)
    v = v[np.abs(v) > 2.0 ** -13]                       # f16 normal range
    bits = v.view(np.uint32).astype(np.uint64)
    all_d = np.arange(8192, dtype=np.uint64)
    # every dither value once: the expectation of the stochastic rounding exactly
    trunc = ((bits[:, None] + all_d[None, :]) & np.uint64(0xFFFFE000)).astype(np.uint32).view(np.float32)
    mean = trunc.astype(np.float64).mean(axis=1)
    assert np.allclose(mean, v.astype(np.float64), rtol=0, atol=1e-12 * np.abs(v).max())
    # and round-to-nearest is not: its error is a fixed function of the value
    rn = v.astype(np.float16).astype(np.float64)
    assert np.abs(rn - v).max() > 1e-5
