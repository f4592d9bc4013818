"""The value bounds behind the lazy accumulation forms (csrc/lazy.cuh with
csrc/curve.cuh xyzzz_madd / xyzzz_dbl_affine, R = 2^261; csrc/lazy64.cuh with
xyzzd_madd / xyzzd_dbl_affine, R' = 2^260), re-derived with exact rational
arithmetic: every subtraction a - b + K p must see b below (K - 0.001) p,
every product input must keep the column sums exact, and the accumulator
bounds (R = 2^261: X < 5.39p, Y < 3.34p, ZZ, ZZZ < 2p; R' = 2^260: X < 5.4p,
Y < 3.45p, ZZ, ZZZ < 1.2p) must be stable from one addition to the next.
Also checks the borrow-adjusted K p limbs of the 29-bit form and the K p
limbs of the 52-bit form."""
from fractions import Fraction as Q

P = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 1 << 261
EPS = Q(P, R)                   # product of a p and b p is below (1 + EPS a b) p


EPS_260 = Q(P, 1 << 260)        # the FP64 form's R'
_eps = [EPS]


def mul(a, b):
    return 1 + _eps[0] * a * b


def sub(a, b, K):
    assert b < K - Q(1, 1000), f"subtrahend bound {float(b)} needs K > {float(b)}, got {K}"
    return a + K


def madd(X1, Y1, ZZ1, ZZZ1, qx, qy):
    U2, S2 = mul(qx, ZZ1), mul(qy, ZZZ1)
    P_ = sub(U2, X1, 6)
    R_ = sub(S2, Y1, 4)
    PP, RR = mul(P_, P_), mul(R_, R_)
    PPP, Qv = mul(P_, PP), mul(X1, PP)
    X3 = sub(RR, PPP + 2 * Qv, 4)
    w = sub(Qv, X3, 6)
    Y3 = sub(mul(R_, w), mul(Y1, PPP), 2)
    return X3, Y3, mul(ZZ1, PP), mul(ZZZ1, PPP), (U2, S2, P_, R_, PP, RR, PPP, Qv, w)


def dbl_affine(qx, qy):
    U = qy + qy
    V, xx = mul(U, U), mul(qx, qx)
    W, S = mul(U, V), mul(qx, V)
    M = 3 * xx
    MM, Wy = mul(M, M), mul(W, qy)
    X3 = sub(MM, 2 * S, 3)
    Y3 = sub(mul(M, sub(S, X3, 5)), Wy, 2)
    return X3, Y3, V, W


def test_madd_bounds_are_stable():
    qx, qy = Q(101, 100), Q(2)          # canonical or times beta; canonical or negated (2p - y)
    X, Y, ZZ, ZZZ = Q(539, 100), Q(334, 100), Q(2), Q(2)
    X3, Y3, ZZ3, ZZZ3, inner = madd(X, Y, ZZ, ZZZ, qx, qy)
    assert X3 <= X and Y3 <= Y and ZZ3 <= ZZ and ZZZ3 <= ZZZ
    # the infinity start (acc = q, ZZ = ZZZ = 1 < p) is inside the same bounds
    assert qx <= X and qy <= Y
    # every product input stays well inside the column-sum budget (values below 16 p)
    assert max(inner) < 16


def test_doubling_path_bounds():
    X3, Y3, ZZ3, ZZZ3 = dbl_affine(Q(101, 100), Q(2))
    assert X3 < Q(539, 100) and Y3 < Q(334, 100) and ZZ3 < 2 and ZZZ3 < 2


def test_store_product_below_2p():
    # the store multiplies each coordinate by 2^256 mod p (< p): result < 2p
    for bound in (Q(539, 100), Q(334, 100), Q(2)):
        assert mul(bound, 1) < 2


def _p29(i):
    return (P >> (29 * i)) & ((1 << 29) - 1) if i < 8 else P >> 232


def _kp29(K, i):
    v = K * P
    return (v >> (29 * i)) & ((1 << 29) - 1) if i < 8 else v >> 232


def test_borrow_adjusted_limbs():
    for K in (2, 3, 4, 5, 6):
        limbs = [_kp29(K, i) + ((1 << 30) if i < 8 else 0) - (2 if i > 0 else 0) for i in range(9)]
        assert sum(l << (29 * i) for i, l in enumerate(limbs)) == K * P
        assert all(l >= (1 << 30) - 2 for l in limbs[:8])
        assert all(l < (1 << 32) for l in limbs)
        # an almost-normalised b < (K - 0.001) p keeps the top limb difference non-negative
        b_top_max = (K * P - P // 1000) >> 232
        assert limbs[8] >= b_top_max
        # a + L - b stays below 2^32 per limb for a, b limbs below 2^29 + 8
        assert max(limbs[:8]) + (1 << 29) + 8 < (1 << 32)


def test_column_sums_fit_64_bits():
    lim = (1 << 29) + 8                 # almost-normalised limb
    assert 9 * lim * lim + 9 * ((1 << 29) - 1) ** 2 + (1 << 35) < 1 << 64
    # squares use doubled limbs (2 a_j < 2^30.1)
    assert 5 * lim * (2 * lim) + lim * lim + 9 * ((1 << 29) - 1) ** 2 + (1 << 35) < 1 << 64
    assert _p29(8) < (1 << 29)


def test_fp64_form_bounds_are_stable():
    _eps[0] = EPS_260
    try:
        qx, qy = Q(1), Q(2)              # canonical (halved from the stored form); negated 2p - y
        B = (Q(54, 10), Q(345, 100), Q(12, 10), Q(12, 10))
        X3, Y3, ZZ3, ZZZ3, inner = madd(*B, qx, qy)
        assert all(a <= b for a, b in zip((X3, Y3, ZZ3, ZZZ3), B))
        assert qx <= B[0] and qy <= B[1]  # the infinity start (acc = q, ZZ = ZZZ = 1)
        assert max(inner) < Q(72, 10)     # largest product input, below 2^257 / p
        assert max(inner) * P < 1 << 257
        dX, dY, dZZ, dZZZ = dbl_affine(qx, qy)
        assert dX <= B[0] and dY <= B[1] and dZZ <= B[2] and dZZZ <= B[3]
        assert mul(B[0], 1) < 2          # the store product by 2^256 mod p
    finally:
        _eps[0] = EPS


def _p52(i):
    return (P >> (52 * i)) & ((1 << 52) - 1)


def test_fp64_form_limbs():
    # K p in the 52-bit grid (kp52): normalised, the top limb holding the rest
    for K in (2, 3, 4, 5, 6):
        limbs = [((K * P) >> (52 * i)) & ((1 << 52) - 1) if i < 4 else (K * P) >> 208 for i in range(5)]
        assert sum(l << (52 * i) for i, l in enumerate(limbs)) == K * P
        assert limbs[4] < 1 << 52
    # every lazy value stays below 2^257, so its top limb is below 2^49 and
    # the signed limb sums of a - b + K p stay far inside 64 bits
    assert 8 * P < 1 << 257
    assert sum(_p52(i) << (52 * i) for i in range(5)) == P


def test_ntt_residues_below_2p():
    """The radix-4 NTT pass keeps values in [0, 2p) (field.cuh: mont_mul_f64_lazy,
    add2p, sub2p, canon2p): for both BN254 moduli a product of operands below
    2p leaves (16 a b + Q p) / 2^260 < (64 p / 2^260 + 1) p < 1.76 p < 2p
    (Q < 2^260), a sum of two such values is below 4p < 2^256 (no carry out of
    the 8 words), one subtraction of 2p brings a sum or a borrowed difference
    back below 2p, and one subtraction of p makes a value below 2p canonical.
    Exhaustive over the interval ends with exact integers."""
    r = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
    for m in (P, r):
        assert Q(64 * m, 1 << 260) + 1 < Q(176, 100)
        assert 4 * m < 1 << 256
        two = 2 * m
        words = [(two >> (32 * w)) & 0xFFFFFFFF for w in range(8)]
        # m2word<C>(w): (m_w << 1) | (m_{w-1} >> 31), as the device computes it
        mw = [(m >> (32 * w)) & 0xFFFFFFFF for w in range(8)]
        dev = [((mw[w] << 1) & 0xFFFFFFFF) | (mw[w - 1] >> 31 if w else 0) for w in range(8)]
        assert dev == words
        for a in (0, 1, m - 1, m, two - 1):
            for b in (0, 1, m - 1, m, two - 1):
                s = a + b
                assert s < 1 << 256
                s = s - two if s >= two else s
                assert 0 <= s < two and s % m == (a + b) % m
                d = a - b
                d = d + two if d < 0 else d
                assert 0 <= d < two and d % m == (a - b) % m
            c = a - m if a >= m else a
            assert 0 <= c < m and c == a % m
