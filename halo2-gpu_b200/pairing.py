"""BN254 optimal ate pairing on the host (Python integers), for the KZG
verifier's final check.

The reference ends every KZG verification with one pairing product
(halo2_proofs/src/poly/kzg/msm.rs:159-176, `DualMSM::check`):

    e(left, [s]_2) * e(right, -[1]_2) == 1

with `left` and `right` the two G1 sums the multi-open verifier accumulates
and [1]_2, [s]_2 = s [1]_2 the SRS's G2 elements (poly/kzg/commitment.rs:
188-189).  halo2curves computes it for BN254; this module restates the
published construction (Vercauteren's optimal ate pairing for
Barreto-Naehrig curves, with the usual D-type sextic twist) from the curve's
parameters alone:

* BN parameter x = 0x44E992B44A6909F1: p = 36x^4 + 36x^3 + 24x^2 + 6x + 1 and
  r = 36x^4 + 36x^3 + 18x^2 + 6x + 1 (checked against the field moduli).
* Fq2 = Fq[u] / (u^2 + 1); xi = 9 + u; G2 lives on the twist
  E': y^2 = x^3 + 3 / xi over Fq2.
* Fq12 = Fq[w] / (w^12 - 18 w^6 + 82), i.e. w^6 = xi, held as 12
  coefficients; the untwisting map is (x, y) -> (x w^2, y w^3).
* Miller loop over 6x + 2 (binary, most significant bit first) with affine
  line functions evaluated at P (vertical lines omitted: they lie in a
  subfield that the final exponentiation sends to 1), then the two lines
  through pi(Q) and -pi^2(Q), pi the p-power Frobenius on the twist
  (x, y) -> (conj(x) xi^((p-1)/3), conj(y) xi^((p-1)/2)).
* Final exponentiation (p^12 - 1) / r as (p^6 - 1)(p^2 + 1) by Frobenius
  and one inversion, then the hard part (p^4 - p^2 + 1) / r by
  square-and-multiply.

Points are affine tuples, None for infinity: G1 (x, y) with ints, G2
((x0, x1), (y0, y1)) with x = x0 + x1 u.
"""
from . import fields as F

Q = F.Q_MOD
R = F.R_MOD
BN_X = 0x44E992B44A6909F1
ATE_LOOP = 6 * BN_X + 2

assert Q == 36 * BN_X**4 + 36 * BN_X**3 + 24 * BN_X**2 + 6 * BN_X + 1
assert R == 36 * BN_X**4 + 36 * BN_X**3 + 18 * BN_X**2 + 6 * BN_X + 1

# The standard generator of G2 (the one halo2curves' G2Affine::generator()
# returns; published with the curve in EIP-197).
G2_GENERATOR = (
    (10857046999023057135944570762232829481370756359578518086990519993285655852781,
     11559732032986387107991004021392285783925812861821192530917403151452391805634),
    (8495653923123431417604973247489272438418190587263600148770280649306958101930,
     4082367875863433681332203403145435568316851327593401208105741076214120093531),
)


# --- Fq2 --------------------------------------------------------------------------

def f2_add(a, b):
    return ((a[0] + b[0]) % Q, (a[1] + b[1]) % Q)


def f2_sub(a, b):
    return ((a[0] - b[0]) % Q, (a[1] - b[1]) % Q)


def f2_neg(a):
    return ((-a[0]) % Q, (-a[1]) % Q)


def f2_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % Q, (a[0] * b[1] + a[1] * b[0]) % Q)


def f2_scale(a, k):
    return (a[0] * k % Q, a[1] * k % Q)


def f2_inv(a):
    n = (a[0] * a[0] + a[1] * a[1]) % Q
    if n == 0:
        raise ZeroDivisionError("inverse of 0 in Fq2")
    ni = pow(n, -1, Q)
    return (a[0] * ni % Q, (-a[1]) * ni % Q)


def f2_conj(a):
    return (a[0], (-a[1]) % Q)


def f2_pow(a, e):
    r = (1, 0)
    while e:
        if e & 1:
            r = f2_mul(r, a)
        a = f2_mul(a, a)
        e >>= 1
    return r


XI = (9, 1)
TWIST_B = f2_mul((3, 0), f2_inv(XI))
FROB_X = f2_pow(XI, (Q - 1) // 3)
FROB_Y = f2_pow(XI, (Q - 1) // 2)


# --- G2 (affine, on the twist) --------------------------------------------------

def g2_on_curve(P):
    if P is None:
        return True
    x, y = P
    return f2_sub(f2_mul(y, y), f2_add(f2_mul(f2_mul(x, x), x), TWIST_B)) == (0, 0)


def g2_neg(P):
    return None if P is None else (P[0], f2_neg(P[1]))


def _g2_add_slope(P, Qp):
    """(P + Q, slope of the line through them), or (P + Q, None) when the line
    is vertical (the sum is infinity)."""
    if P is None:
        return Qp, None
    if Qp is None:
        return P, None
    (x1, y1), (x2, y2) = P, Qp
    if x1 == x2:
        if f2_add(y1, y2) == (0, 0):
            return None, None
        lam = f2_mul(f2_scale(f2_mul(x1, x1), 3), f2_inv(f2_scale(y1, 2)))
    else:
        lam = f2_mul(f2_sub(y2, y1), f2_inv(f2_sub(x2, x1)))
    x3 = f2_sub(f2_sub(f2_mul(lam, lam), x1), x2)
    y3 = f2_sub(f2_mul(lam, f2_sub(x1, x3)), y1)
    return (x3, y3), lam


def g2_add(P, Qp):
    return _g2_add_slope(P, Qp)[0]


def g2_mul(P, s):
    s %= R
    acc = None
    while s:
        if s & 1:
            acc = g2_add(acc, P)
        P = g2_add(P, P)
        s >>= 1
    return acc


def g2_frobenius(P):
    if P is None:
        return None
    return (f2_mul(f2_conj(P[0]), FROB_X), f2_mul(f2_conj(P[1]), FROB_Y))


# --- Fq12 = Fq[w] / (w^12 - 18 w^6 + 82) ----------------------------------------

ONE12 = [1] + [0] * 11


def f12_mul(a, b):
    c = [0] * 23
    for i, ai in enumerate(a):
        if ai:
            for j, bj in enumerate(b):
                if bj:
                    c[i + j] += ai * bj
    for i in range(22, 11, -1):
        t = c[i]
        if t:
            c[i - 6] += 18 * t
            c[i - 12] -= 82 * t
    return [x % Q for x in c[:12]]


def f12_pow(a, e):
    r = ONE12
    for bit in bin(e)[2:]:
        r = f12_mul(r, r)
        if bit == "1":
            r = f12_mul(r, a)
    return r


def f12_inv(a):
    """a^-1 by solving a * v = 1 (a 12 x 12 linear system over Fq)."""
    cols = []
    wj = ONE12
    wshift = [0, 1] + [0] * 10
    for _ in range(12):
        cols.append(f12_mul(a, wj))
        wj = f12_mul(wj, wshift)
    m = [[cols[j][i] for j in range(12)] + [1 if i == 0 else 0] for i in range(12)]
    for c in range(12):
        piv = next((r for r in range(c, 12) if m[r][c] % Q), None)
        if piv is None:
            raise ZeroDivisionError("inverse of 0 in Fq12")
        m[c], m[piv] = m[piv], m[c]
        inv = pow(m[c][c], -1, Q)
        m[c] = [x * inv % Q for x in m[c]]
        for r in range(12):
            if r != c and m[r][c]:
                k = m[r][c]
                m[r] = [(x - k * y) % Q for x, y in zip(m[r], m[c])]
    return [m[i][12] for i in range(12)]


def _embed(a, k, out):
    """out += a * w^k for a in Fq2 (a0 + a1 u = (a0 - 9 a1) + a1 w^6), k < 6."""
    out[k] = (out[k] + a[0] - 9 * a[1]) % Q
    out[k + 6] = (out[k + 6] + a[1]) % Q


_FROB = None


def _frob_table():
    """(w^p)^i for i < 12: the p-power Frobenius is linear over Fq."""
    global _FROB
    if _FROB is None:
        wp = f12_pow([0, 1] + [0] * 10, Q)
        t, acc = [], ONE12
        for _ in range(12):
            t.append(acc)
            acc = f12_mul(acc, wp)
        _FROB = t
    return _FROB


def f12_frobenius(a, times=1):
    tab = _frob_table()
    for _ in range(times):
        r = [0] * 12
        for ai, col in zip(a, tab):
            if ai:
                for j in range(12):
                    r[j] += ai * col[j]
        a = [x % Q for x in r]
    return a


# --- Miller loop and final exponentiation ---------------------------------------

def _line(T, lam, P):
    """The line through untwisted T with twist slope lam, at P = (xP, yP):
    yP - lam xP w + (lam xT - yT) w^3."""
    xP, yP = P
    out = [0] * 12
    out[0] = yP % Q
    _embed(f2_neg(f2_scale(lam, xP)), 1, out)
    _embed(f2_sub(f2_mul(lam, T[0]), T[1]), 3, out)
    return out


def _step(f, T, S, P):
    """f * line(T, S)(P), T + S."""
    T2, lam = _g2_add_slope(T, S)
    if lam is None:
        raise ValueError("degenerate Miller loop step (a point of small order)")
    return f12_mul(f, _line(T, lam, P)), T2


def miller_loop(P, Qp):
    """f_{6x+2,Q}(P) times the lines through pi(Q) and -pi^2(Q); 1 when
    either point is infinity."""
    if P is None or Qp is None:
        return ONE12
    f, T = ONE12, Qp
    for bit in bin(ATE_LOOP)[3:]:
        f = f12_mul(f, f)
        f, T = _step(f, T, T, P)
        if bit == "1":
            f, T = _step(f, T, Qp, P)
    q1 = g2_frobenius(Qp)
    q2 = g2_neg(g2_frobenius(q1))
    f, T = _step(f, T, q1, P)
    f, _ = _step(f, T, q2, P)
    return f


_HARD = (Q**4 - Q**2 + 1) // R
assert _HARD * R == Q**4 - Q**2 + 1


def final_exponentiation(f):
    f = f12_mul(f12_frobenius(f, 6), f12_inv(f))      # f^(p^6 - 1)
    f = f12_mul(f12_frobenius(f, 2), f)                # ^(p^2 + 1)
    return f12_pow(f, _HARD)


def pairing(P, Qp):
    """e(P, Q) in Fq12 (12 coefficients)."""
    return final_exponentiation(miller_loop(P, Qp))


def pairing_check(pairs):
    """True when prod_i e(P_i, Q_i) == 1 (one final exponentiation for the
    product of the Miller loops, as multi_miller_loop does)."""
    f = ONE12
    for P, Qp in pairs:
        f = f12_mul(f, miller_loop(P, Qp))
    return final_exponentiation(f) == ONE12
