"""Montgomery product parity on the device: every product implementation
(mad.lo/mad.hi CIOS, mad.wide CIOS, 29-bit column products and squares, and
the FP64 product over 52-bit limbs, for Fr and Fq) against Python integers, on random and boundary operands (the
reference's field arithmetic is Montgomery multiplication with R = 2^256,
halo2_proofs/cuda/include/field/alt_bn128.hpp:15-43)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RADIX = 1 << 256


def _edge_ints(p):
    r = RADIX % p
    return [0, 1, 2, p - 1, p - 2, r, p - r, (RADIX * RADIX) % p, (p - 1) // 2, (p + 1) // 2,
            (1 << 255) % p, ((1 << 254) - 1) % p, p - (1 << 32), (1 << 232) - 1, p - (1 << 232), (1 << 29) - 1]


@pytest.mark.parametrize("impl", [0, 1, 2, 3, 4, 5, 6, 7])
def test_product_impls(h2b, orc, cuda, impl):
    f = h2b.fields
    p = f.Q_MOD if impl in (4, 5, 7) else f.R_MOD
    square = impl in (3, 5)
    n = 1 << 16
    rng = np.random.default_rng(impl)
    a = orc.chacha_fr(11, n)
    b = orc.chacha_fr(12, n)
    if p == f.Q_MOD:  # uniform below q from random 256-bit words
        a = f.ints_to_limbs([x % p for x in f.limbs_to_ints(rng.integers(0, 2**63, (n, 4), dtype=np.uint64) * 2)])
        b = f.ints_to_limbs([x % p for x in f.limbs_to_ints(rng.integers(0, 2**63, (n, 4), dtype=np.uint64) * 2 + 1)])
    edges = [x % p for x in _edge_ints(p)]
    ea = f.ints_to_limbs([x for x in edges for _ in edges])
    eb = f.ints_to_limbs([y for _ in edges for y in edges])
    a = np.concatenate([a, ea])
    b = np.concatenate([b, eb])
    m = a.shape[0]
    d_a, d_b, d_o = h2b.to_dev(a), h2b.to_dev(b), h2b.dev_empty(32 * m)
    h2b.call("h2b_fr_mul_batch", impl, h2b.ptr(d_a), h2b.ptr(d_b), h2b.ptr(d_o), m, h2b.stream_handle())
    got = f.limbs_to_ints(h2b.to_host(d_o))
    rinv = pow(RADIX, -1, p)
    ai, bi = f.limbs_to_ints(a), f.limbs_to_ints(b)
    bad = [i for i in range(m) if got[i] != ai[i] * (ai[i] if square else bi[i]) * rinv % p]
    assert not bad, f"impl {impl}: {len(bad)} wrong products, first at {bad[0]}"
