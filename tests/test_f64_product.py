"""The FP64 Montgomery product (csrc/field.cuh mont_mul_f64) restated step by
step over Python integers, with the IEEE bit patterns of the split halves
taken from real doubles: checks the exponent-bias bookkeeping of the column
sums, the carry shortcut for the cancelled low half of q_i p_0, the 16 a
pre-scaling that turns R' = 2^260 into R = 2^256, and the bounds the kernel
relies on (columns below 2^57, result below 1.19 p before the one
conditional subtraction).  The device code itself is checked bit-exactly
against Python integers by the product tests on the GPU."""
import random
import struct

import pytest

FR = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
FQ = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
M52 = (1 << 52) - 1
M64 = (1 << 64) - 1
EXP_LO, EXP_HI = 0x4330000000000000, 0x4670000000000000


def bits(x):
    """Bit pattern of the double nearest to integer x (exact for the values used)."""
    d = float(x)
    assert int(d) == x, "value not exactly representable"
    return struct.unpack("<Q", struct.pack("<d", d))[0]


def split(a, b):
    """fma_rz(a, b, 2^104) and fma(a, b, 2^104 + 2^52 - h) for a, b < 2^52."""
    assert a < 1 << 52 and b < 1 << 52
    ab = a * b
    h = (1 << 104) + ((ab >> 52) << 52)          # round toward zero at ulp 2^52
    s = (1 << 104) + (1 << 52) - h               # exact difference
    assert int(float(s)) == s
    l_ = ab + s                                  # in [2^52, 2^53): exact
    assert 1 << 52 <= l_ < 1 << 53
    return bits(h), bits(l_)


def bias(k):
    nl = nh = 0
    for i in range(5):
        for j in range(5):
            nl += i + j == k
            nh += 2 * (i + j + 1 == k)
            nl += j > 0 and i + j == k
    return (nl * EXP_LO + nh * EXP_HI) & M64


def limbs52(x, shift=0):
    x <<= shift
    return [(x >> (52 * i)) & M52 for i in range(5)]


def mont_mul_f64(a, b, p, stats):
    np52 = (-pow(p, -1, 1 << 64)) % (1 << 64) & M52
    pl = limbs52(p)
    A, B = limbs52(a, 4), limbs52(b)
    assert (a << 4) < 1 << 260
    col = [(-bias(k)) & M64 for k in range(10)]
    for i in range(5):
        for j in range(5):
            h, l_ = split(A[i], B[j])
            col[i + j] = (col[i + j] + l_) & M64
            col[i + j + 1] = (col[i + j + 1] + h) & M64
    for i in range(5):
        t = col[i]
        stats["max_col"] = max(stats["max_col"], t)
        tl = t & M52
        q = (tl * np52) & M52
        assert (tl + ((q * pl[0]) & M52)) & M52 == 0, "q_i must cancel the low digit"
        h0, _ = split(q, pl[0])
        carry = (t >> 52) + (1 if tl else 0)
        col[i + 1] = (col[i + 1] + carry + h0) & M64
        for j in range(1, 5):
            h, l_ = split(q, pl[j])
            col[i + j] = (col[i + j] + l_) & M64
            col[i + j + 1] = (col[i + j + 1] + h) & M64
    for k in range(5, 10):
        stats["max_col"] = max(stats["max_col"], col[k])
    r = sum(col[5 + k] << (52 * k) for k in range(5))
    stats["max_ratio"] = max(stats["max_ratio"], r / p)
    return r - p if r >= p else r


@pytest.mark.parametrize("p", [FR, FQ], ids=["fr", "fq"])
def test_f64_product_restatement(p):
    rng = random.Random(p & 0xFFFF)
    rinv = pow(1 << 256, -1, p)
    edges = [0, 1, 2, p - 1, p - 2, (1 << 253) - 1, p >> 1, (p >> 1) + 1, 1 << 252, p - (1 << 200),
             (1 << 256) % p, (1 << 52) - 1, 1 << 52, (1 << 208) - 1, p - (1 << 52)]
    cases = [(x, y) for x in edges for y in edges] + [(rng.randrange(p), rng.randrange(p)) for _ in range(3000)]
    stats = {"max_col": 0, "max_ratio": 0.0}
    for a, b in cases:
        got = mont_mul_f64(a, b, p, stats)
        assert got == a * b * rinv % p, (hex(a), hex(b))
    assert stats["max_col"] < 1 << 57
    assert stats["max_ratio"] < 1.19


def test_bias_is_the_term_count():
    # 25 product splits put a low half in column i + j and a high half in
    # i + j + 1; reduction step i puts a high half of q_i p_0 in i + 1 and,
    # for j = 1..4, low and high halves of q_i p_j in i + j and i + j + 1:
    # 45 low and 50 high halves over the ten columns
    lo, hi = [0] * 10, [0] * 10
    for i in range(5):
        for j in range(5):
            lo[i + j] += 1
            hi[i + j + 1] += 1
        hi[i + 1] += 1
        for j in range(1, 5):
            lo[i + j] += 1
            hi[i + j + 1] += 1
    assert (sum(lo), sum(hi)) == (45, 50)
    for k in range(10):
        assert bias(k) == (lo[k] * EXP_LO + hi[k] * EXP_HI) & M64
