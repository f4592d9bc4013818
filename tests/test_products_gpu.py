"""Batch inversion, grand-product scan and the lookup / permutation products
against the oracle (reference tests: halo2_proofs/src/cuda/tests.rs:39-50,
978-1565)."""
import numpy as np
import pytest

from conftest import assert_limbs_equal

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 7, 2048, 2049, 10000, 1 << 16])
@pytest.mark.parametrize("field_type", [0, 1])
def test_batch_invert(h2b, orc, cuda, n, field_type):
    x = orc.chacha_fr(n + field_type, n)
    if field_type == 1:
        # reduce Fr-random limbs below q: they are < r < q already
        pass
    x[::13] = 0
    want = orc.batch_invert(x, field_type)
    d = h2b.to_dev(x)
    h2b.batch_invert_device(d, n, field_type)
    assert_limbs_equal(h2b.to_host(d), want, "batch_invert")
    d2 = h2b.to_dev(x)
    h2b.batch_invert_device_scratch(d2, n, field_type)
    assert_limbs_equal(h2b.to_host(d2), want, "batch_invert (scratch)")


def test_batch_invert_full_size_property(h2b, orc, cuda):
    """x * x^-1 == 1 over 2^24 nonzero uniform Fr (checked on the device with
    the product's own multiply, then every row compared to one)."""
    n = 1 << 24
    d = h2b.random_fr_device(n, 77)
    d_inv = d.clone()
    h2b.batch_invert_device_scratch(d_inv, n, 0)
    d_prod = h2b.dev_empty(32 * n)
    h2b.call("_halo2_poly_elementwise_multiply", h2b.ptr(d_prod), h2b.ptr(d), h2b.ptr(d_inv), n, h2b.stream_handle())
    one = h2b.fields.fr_mont_limbs([1])[0]
    prod = h2b.to_host(d_prod)
    assert (prod == one).all()
    # spot-check against the oracle
    x = h2b.to_host(d)
    sel = np.r_[0:2048, n - 2048:n]
    assert_limbs_equal(h2b.to_host(d_inv)[sel], orc.batch_invert(x[sel]), "spot")


@pytest.mark.parametrize("n", [1, 5, 2048, 4096, 100000, (1 << 20)])
def test_grand_product(h2b, orc, cuda, n):
    x = orc.chacha_fr(900 + n, n)
    pre = orc.chacha_fr(901, 1)
    want = orc.grand_product(x, pre)
    assert_limbs_equal(h2b.grand_product(x, pre), want, "host grand product")
    d = h2b.to_dev(x)
    h2b.grand_product_device(d, h2b.to_dev(pre), n)
    assert_limbs_equal(h2b.to_host(d), want, "device grand product")


def test_grand_product_offset_chunk(h2b, orc, cuda):
    n, off, ln = 50000, 12345, 20000
    x = orc.chacha_fr(5, n)
    pre = h2b.fields.fr_mont_limbs([1])
    want = orc.grand_product(x[off:off + ln], pre)
    got = h2b.grand_product(x, pre, offset=off, length=ln)
    assert_limbs_equal(got[off:off + ln], want, "offset chunk")
    d = h2b.to_dev(x)
    h2b.grand_product_device(d, h2b.to_dev(pre), ln, offset=off)
    host = h2b.to_host(d)
    assert_limbs_equal(host[off:off + ln], want, "device offset chunk")
    assert_limbs_equal(host[:off], x[:off], "outside chunk untouched")


@pytest.mark.parametrize("n", [3, 4096, 70000])
def test_lookup_product(h2b, orc, cuda, n):
    arrs = [orc.chacha_fr(40 + i, n) for i in range(4)]
    beta, gamma = orc.chacha_fr(50, 1), orc.chacha_fr(51, 1)
    want = orc.lookup_product(*arrs, beta, gamma)
    got = h2b.lookup_product(*arrs, beta, gamma)
    assert_limbs_equal(got, want, "host lookup product")
    d = [h2b.to_dev(a) for a in arrs]
    d_out = h2b.dev_empty(32 * n)
    h2b.lookup_product_device(d_out, *d, h2b.to_dev(beta), h2b.to_dev(gamma), n)
    assert_limbs_equal(h2b.to_host(d_out), want, "device lookup product")


@pytest.mark.parametrize("n,cols", [(5, 1), (4096, 2), (30000, 3)])
def test_permutation_product(h2b, orc, cuda, n, cols):
    f = h2b.fields
    mod = orc.chacha_fr(60, n)
    vals = [orc.chacha_fr(61 + c, n) for c in range(cols)]
    perms = [orc.chacha_fr(71 + c, n) for c in range(cols)]
    omega = f.fr_mont_limbs([f.EvaluationDomain(4, 20).omega])
    beta, gamma = orc.chacha_fr(80, 1), orc.chacha_fr(81, 1)
    delta = f.fr_mont_limbs([f.DELTA])
    dw = orc.chacha_fr(82, 1)
    want, want_dw = orc.permutation_product(mod, vals, perms, omega, beta, gamma, delta, dw)
    got, got_dw = h2b.permutation_product(mod, perms, vals, beta, gamma, delta, omega, dw)
    assert_limbs_equal(got, want, "host permutation product")
    assert_limbs_equal(got_dw.reshape(1, 4), want_dw.reshape(1, 4), "deltaomega advance")
    d_mod = h2b.to_dev(mod)
    d_dw = h2b.to_dev(dw)
    h2b.permutation_product_device(d_mod, [h2b.to_dev(p) for p in perms], [h2b.to_dev(v) for v in vals],
                                   h2b.to_dev(beta), h2b.to_dev(gamma), h2b.to_dev(delta), h2b.to_dev(omega), d_dw, n)
    assert_limbs_equal(h2b.to_host(d_mod), want, "device permutation product")
    assert_limbs_equal(h2b.to_host(d_dw), want_dw.reshape(1, 4), "device deltaomega")
