"""The number format of the FP32-arithmetic spread (k_spread_fx), restated on
the host: a float contribution v becomes q = round(v 2^38) (the float
product v 2^38 is exact, then rounded to the nearest integer), split into a
20-bit low part lo = q mod 2^20 and a high part hi = floor(q / 2^20); the
cell sums the low parts in an unsigned 32-bit word and the high parts in a
signed 32-bit word, and reads hi 2^20 + lo.  The checks: the split is exact,
the sum does not depend on the order of the terms, and the stated limits
(at most 4,096 terms a cell and sweep, one per list entry; sums below 2^13
in magnitude) keep the low word from wrapping and the high word's sum in
range (its intermediate sums may wrap: two's complement addition modulo
2^32 still ends exact)."""
import numpy as np

LO_BITS = 20
SCALE = np.float32(2.0 ** 38)


def quant(v):
    return np.rint(np.float32(v) * SCALE).astype(np.int64)


def split(q):
    return (q & ((1 << LO_BITS) - 1)).astype(np.uint64), (q >> LO_BITS).astype(np.int64)


def cell_sum(values):
    """The cell's two words after adding every value, with 32-bit wrapping."""
    lo, hi = split(quant(values))
    lo_w = int(lo.sum()) % (1 << 32)
    hi_w = int(hi.sum())
    hi_w = (hi_w + (1 << 31)) % (1 << 32) - (1 << 31)
    return lo_w, hi_w


def value(lo_w, hi_w):
    return (hi_w * (1 << LO_BITS) + lo_w) * 2.0 ** -38


def test_split_is_exact():
    rng = np.random.default_rng(1)
    v = (rng.standard_normal(10000) * 10.0 ** rng.uniform(-9, -1, 10000)).astype(np.float32)
    q = quant(v)
    lo, hi = split(q)
    assert np.all(lo < (1 << LO_BITS))
    assert np.array_equal(hi * (1 << LO_BITS) + lo.astype(np.int64), q)


def test_sum_is_exact_and_order_free():
    rng = np.random.default_rng(2)
    v = (rng.standard_normal(300) * 1e-4).astype(np.float32)
    a = cell_sum(v)
    b = cell_sum(v[rng.permutation(v.size)])
    assert a == b
    assert value(*a) == float(quant(v).sum()) * 2.0 ** -38
    # against the float64 sum of the float32 terms: within the resolution
    # per term
    assert abs(value(*a) - float(np.sum(v.astype(np.float64)))) <= v.size * 2.0 ** -38


def test_limits_keep_the_words_from_wrapping():
    # 4,096 terms whose low parts are all at their maximum stay below 2^32
    # (one more would not: the cap on a tile's list is what bounds them)
    assert 4096 * ((1 << LO_BITS) - 1) < (1 << 32) < 4097 * ((1 << LO_BITS) - 1)
    # a cell sum just below 2^13, and one just above -2^13, in 4,096 terms:
    # exact
    for sign in (1.0, -1.0):
        v = np.full(4096, np.float32(sign * 0.999 * 2.0 ** 13 / 4096))
        lo_w, hi_w = cell_sum(v)
        assert value(lo_w, hi_w) == float(quant(v).sum()) * 2.0 ** -38
    # intermediate wrapping of the high word: terms of both signs whose
    # running sum leaves int32 but whose total does not
    v = np.concatenate([np.full(2048, np.float32(12000.0 / 2048)),
                        np.full(2048, np.float32(-11999.0 / 2048))])
    hi = split(quant(v))[1]
    assert np.max(np.abs(np.cumsum(hi))) >= (1 << 31)      # the running sum leaves int32
    assert value(*cell_sum(v)) == float(quant(v).sum()) * 2.0 ** -38
    # resolution
    assert 2.0 ** -38 < 3.7e-12
