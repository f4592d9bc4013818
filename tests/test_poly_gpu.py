"""Element-wise polynomial entry points against plain big-integer arithmetic
(reference equivalence tests: halo2_proofs/tests/{divide_by_vanishing,
distribute_powers_zeta,extended_from_lagrange_vec,poly_multiply_add}_device_equivalence.rs)."""
import numpy as np
import pytest

from conftest import assert_limbs_equal

pytestmark = pytest.mark.gpu


def ints(h2b, a):
    return h2b.fields.fr_from_mont_limbs(a)


def mont(h2b, xs):
    return h2b.fields.fr_mont_limbs(xs)


def test_elementwise_ops(h2b, orc, cuda):
    f = h2b.fields
    R = f.R_MOD
    n = 3000
    a, b = orc.chacha_fr(1, n), orc.chacha_fr(2, n)
    ia, ib = ints(h2b, a), ints(h2b, b)
    da, db, dout = h2b.to_dev(a), h2b.to_dev(b), h2b.dev_empty(32 * n)
    sh = h2b.stream_handle()
    h2b.call("_halo2_poly_elementwise_multiply", h2b.ptr(dout), h2b.ptr(da), h2b.ptr(db), n, sh)
    assert_limbs_equal(h2b.to_host(dout), mont(h2b, [x * y % R for x, y in zip(ia, ib)]), "mul")
    k = orc.chacha_fr(3, 1)
    h2b.call("_halo2_poly_multiply_add", h2b.ptr(da), h2b.ptr(db), h2b.ptr(h2b.to_dev(k)), n, sh)
    ik = ints(h2b, k)[0]
    assert_limbs_equal(h2b.to_host(da), mont(h2b, [(x + y * ik) % R for x, y in zip(ia, ib)]), "mul_add")
    h2b.call("_halo2_poly_fill_one", h2b.ptr(dout), n, sh)
    assert_limbs_equal(h2b.to_host(dout), mont(h2b, [1] * n), "fill one")
    da = h2b.to_dev(a)
    h2b.call("_halo2_poly_sub_short_inplace", h2b.ptr(da), h2b.ptr(db), 1000, sh)
    want = [(x - y) % R if i < 1000 else x for i, (x, y) in enumerate(zip(ia, ib))]
    assert_limbs_equal(h2b.to_host(da), mont(h2b, want), "sub short")
    da = h2b.to_dev(a)
    h2b.call("_halo2_poly_sub_short_out_of_place", h2b.ptr(dout), h2b.ptr(da), h2b.ptr(db), 1000, n, sh)
    assert_limbs_equal(h2b.to_host(dout), mont(h2b, want), "sub short oop")
    h2b.call("_halo2_poly_sub_scalar_at_zero", h2b.ptr(da), h2b.ptr(h2b.to_dev(k)), sh)
    got = h2b.to_host(da)
    assert ints(h2b, got[:1])[0] == (ia[0] - ik) % R


def test_vanishing_zeta_and_interleave(h2b, orc, cuda):
    f = h2b.fields
    R = f.R_MOD
    d = f.EvaluationDomain(5, 8)
    N = d.extended_len()
    a = orc.chacha_fr(5, N)
    ia = ints(h2b, a)
    t = d.t_evaluations
    da = h2b.to_dev(a)
    sh = h2b.stream_handle()
    h2b.call("_halo2_divide_by_vanishing_poly", h2b.ptr(da), h2b.ptr(h2b.to_dev(mont(h2b, t))), len(t), N, sh)
    assert_limbs_equal(h2b.to_host(da), mont(h2b, [x * t[i % len(t)] % R for i, x in enumerate(ia)]), "vanishing")
    da = h2b.to_dev(a)
    cp = [d.g_coset_inv, d.g_coset]
    h2b.call("_halo2_distribute_powers_zeta", h2b.ptr(da), h2b.ptr(h2b.to_dev(mont(h2b, cp))), 2, N, sh)
    want = [x if i % 3 == 0 else x * cp[i % 3 - 1] % R for i, x in enumerate(ia)]
    assert_limbs_equal(h2b.to_host(da), mont(h2b, want), "distribute zeta")
    parts = [orc.chacha_fr(10 + p, 256) for p in range(4)]
    dparts = [h2b.to_dev(p) for p in parts]
    table = h2b.to_dev(np.array([t.data_ptr() for t in dparts], dtype=np.uint64))
    dout = h2b.dev_empty(32 * 1024)
    h2b.call("_halo2_extended_from_lagrange_vec_device", h2b.ptr(dout), h2b.ptr(table), 4, 256, sh)
    want = np.stack(parts, axis=1).reshape(-1, 4)
    assert_limbs_equal(h2b.to_host(dout), want, "interleave")
