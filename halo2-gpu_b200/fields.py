"""Host-side BN254 constants and conversions (Python integers).

Launch-time constants only: domain roots of unity, coset factors, Montgomery
conversions of small inputs, and the affine table 2^j G used to build a
synthetic SRS on the device.  Per-element field work never runs here.

Constants: moduli and Montgomery radix from
halo2_proofs/cuda/include/field/alt_bn128.hpp:15-43; zeta (the coset generator
g_coset) from halo2_proofs/cuda/include/kernel/zeta.h:19-28; the 2-adic root
of unity is 7^((r-1)/2^28) (generator 7, S = 28, the halo2curves bn256::Fr
convention) and DELTA = 7^(2^28).  EvaluationDomain follows halo2's
EvaluationDomain::new(j, k).
"""
import numpy as np

R_MOD = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
Q_MOD = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
RADIX = 1 << 256
S = 28
GENERATOR = 7
ROOT_OF_UNITY = pow(GENERATOR, (R_MOD - 1) >> S, R_MOD)
DELTA = pow(GENERATOR, 1 << S, R_MOD)
# zeta.h stores zeta in Montgomery form; this is its plain value.
ZETA = 0x30644E72E131A029048B6E193FD84104CC37A73FEC2BC5E9B8CA0B2D36636F23


_RINV = {R_MOD: pow(RADIX, -1, R_MOD), Q_MOD: pow(RADIX, -1, Q_MOD)}


def to_mont(x, m=R_MOD):
    return (x % m) * RADIX % m


def from_mont(x, m=R_MOD):
    return x * _RINV[m] % m


def ints_to_limbs(xs):
    """list of ints (< 2^256) -> (n, 4) uint64 little-endian limbs."""
    xs = list(xs)
    out = np.zeros((len(xs), 4), dtype=np.uint64)
    for i, x in enumerate(xs):
        for k in range(4):
            out[i, k] = (x >> (64 * k)) & 0xFFFFFFFFFFFFFFFF
    return out


def limbs_to_ints(a):
    a = np.asarray(a, dtype=np.uint64).reshape(-1, 4)
    return [int(r[0]) | (int(r[1]) << 64) | (int(r[2]) << 128) | (int(r[3]) << 192) for r in a]


def fr_mont_limbs(xs):
    return ints_to_limbs([to_mont(x, R_MOD) for x in xs])


def fq_mont_limbs(xs):
    return ints_to_limbs([to_mont(x, Q_MOD) for x in xs])


def fr_from_mont_limbs(a):
    return [from_mont(x, R_MOD) for x in limbs_to_ints(a)]


def fr_scalar(x):
    """One Fr element as 32 Montgomery bytes (for host-scalar arguments)."""
    return fr_mont_limbs([x]).tobytes()


class EvaluationDomain:
    """Constants of halo2's EvaluationDomain::new(j, k) (plain integers)."""

    def __init__(self, j, k):
        self.k = k
        self.n = 1 << k
        self.quotient_poly_degree = j - 1
        ek = k
        while (1 << ek) < self.n * self.quotient_poly_degree:
            ek += 1
        self.extended_k = ek
        self.extended_omega = pow(ROOT_OF_UNITY, 1 << (S - ek), R_MOD)
        self.extended_omega_inv = pow(self.extended_omega, -1, R_MOD)
        self.omega = pow(self.extended_omega, 1 << (ek - k), R_MOD)
        self.omega_inv = pow(self.omega, -1, R_MOD)
        self.g_coset = ZETA
        self.g_coset_inv = ZETA * ZETA % R_MOD
        self.ifft_divisor = pow(1 << k, -1, R_MOD)
        self.extended_ifft_divisor = pow(1 << ek, -1, R_MOD)
        orig = pow(ZETA, self.n, R_MOD)
        step = pow(self.extended_omega, self.n, R_MOD)
        t, cur = [], orig
        while True:
            t.append(cur)
            cur = cur * step % R_MOD
            if cur == orig:
                break
        self.t_evaluations = [pow((x - 1) % R_MOD, -1, R_MOD) for x in t]

    def extended_len(self):
        return 1 << self.extended_k


# --- G1 affine arithmetic over Fq (setup tables only) ------------------------

G1_GENERATOR = (1, 2)


def g1_add(P, Q):
    if P is None:
        return Q
    if Q is None:
        return P
    (x1, y1), (x2, y2) = P, Q
    if x1 == x2:
        if (y1 + y2) % Q_MOD == 0:
            return None
        lam = 3 * x1 * x1 * pow(2 * y1, -1, Q_MOD) % Q_MOD
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, Q_MOD) % Q_MOD
    x3 = (lam * lam - x1 - x2) % Q_MOD
    return (x3, (lam * (x1 - x3) - y1) % Q_MOD)


def g1_mul(P, s):
    R, A = None, P
    while s:
        if s & 1:
            R = g1_add(R, A)
        A = g1_add(A, A)
        s >>= 1
    return R


def g1_pow2_table(count=256):
    """Affine 2^j G for j < count, Montgomery limbs, shape (count, 8)."""
    pts, P = [], G1_GENERATOR
    for _ in range(count):
        pts.append(P)
        P = g1_add(P, P)
    xs = fq_mont_limbs([p[0] for p in pts])
    ys = fq_mont_limbs([p[1] for p in pts])
    return np.concatenate([xs, ys], axis=1)


def jac_to_affine_ints(j):
    """96-byte Jacobian image (12 uint64, Montgomery) -> plain (x, y) or None."""
    v = limbs_to_ints(np.asarray(j, dtype=np.uint64).reshape(3, 4))
    if v[2] == 0:
        return None
    x, y, z = (from_mont(t, Q_MOD) for t in v)
    zi = pow(z, -1, Q_MOD)
    return (x * zi * zi % Q_MOD, y * zi * zi * zi % Q_MOD)
