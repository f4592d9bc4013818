"""NTT parity: every `_halo2_fft_*` entry point against the oracle, bit-exact,
plus size-independent round trips at the full k=22 -> 24 extension.
Shapes follow the reference's tests (halo2_proofs/src/cuda/tests.rs:110-347)."""
import numpy as np
import pytest

from conftest import assert_limbs_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[0, 1], ids=["radix2", "radix4"], autouse=True)
def pass_kind(request, h2b):
    """Every NTT test runs with the radix-2 and the radix-4 pass kernels."""
    L = h2b.lib()
    before = L.h2b_ntt_get_radix4()
    L.h2b_ntt_set_radix4(request.param)
    yield request.param
    L.h2b_ntt_set_radix4(before)


def mont(h2b, x):
    return h2b.fields.fr_mont_limbs([x])


@pytest.mark.parametrize("k", [1, 2, 3, 5, 8, 9, 10, 11, 12, 16])
def test_fft_normal_all_types(h2b, orc, cuda, k):
    f = h2b.fields
    d = f.EvaluationDomain(3, k)
    a = orc.chacha_fr(100 + k, 1 << k)
    c = d.g_coset * d.extended_omega % f.R_MOD
    cases = [(1, d.omega, 1), (2, d.omega_inv, d.ifft_divisor), (6, d.omega, c), (3, d.omega, 1),
             (4, d.omega_inv, d.ifft_divisor)]
    for t, om, dv in cases:
        got = h2b.fft_normal(t, k, a, om, dv)
        want = orc.ntt(t, k, k, a, mont(h2b, om), mont(h2b, dv))
        assert_limbs_equal(got, want, f"type {t} k={k}")


@pytest.mark.parametrize("k", [4, 12, 18])
def test_fft_normal_to_device_aliasing(h2b, orc, cuda, k):
    f = h2b.fields
    d = f.EvaluationDomain(4, k)
    a = orc.chacha_fr(7 + k, 1 << k)
    c = d.g_coset * pow(d.extended_omega, 3, f.R_MOD) % f.R_MOD
    for t, om, dv in ((1, d.omega, 1), (2, d.omega_inv, d.ifft_divisor), (6, d.omega, c)):
        want = orc.ntt(t, k, k, a, mont(h2b, om), mont(h2b, dv))
        d_in = h2b.to_dev(a)
        d_out = h2b.dev_empty(32 << k)
        h2b.fft_normal_to_device(t, k, d_in, d_out, om, dv)
        assert_limbs_equal(h2b.to_host(d_out), want, f"oop type {t}")
        assert_limbs_equal(h2b.to_host(d_in), a, "input untouched")
        h2b.fft_normal_to_device(t, k, d_in, d_in, om, dv)   # aliased in place
        assert_limbs_equal(h2b.to_host(d_in), want, f"aliased type {t}")


@pytest.mark.parametrize("k,ek", [(2, 4), (10, 12), (16, 18)])
def test_cosetfft_extension(h2b, orc, cuda, k, ek):
    f = h2b.fields
    we = pow(f.ROOT_OF_UNITY, 1 << (28 - ek), f.R_MOD)
    a = orc.chacha_fr(9 + k, 1 << k)
    got = h2b.cosetfft(k, ek, a, we)
    want = orc.ntt(3, k, ek, a, mont(h2b, we), mont(h2b, 1))
    assert_limbs_equal(got, want, "coset extension")


@pytest.mark.parametrize("k,ek", [(3, 5), (10, 12), (13, 16)])
def test_coset_extension_device_input(h2b, orc, cuda, k, ek):
    """Device-input coeff_to_extended (the spread path that skips the first
    ek-k broadcast stages) against the oracle."""
    f = h2b.fields
    we = pow(f.ROOT_OF_UNITY, 1 << (28 - ek), f.R_MOD)
    a = orc.chacha_fr(40 + k, 1 << k)
    d_out = h2b.dev_empty(32 << ek)
    h2b.fft_many_to_device(3, k, ek, [h2b.to_dev(a)], [d_out], we, 1, input_on_device=True)
    assert_limbs_equal(h2b.to_host(d_out), orc.ntt(3, k, ek, a, mont(h2b, we), mont(h2b, 1)), "spread coset")


@pytest.mark.parametrize("k", [10, 14])
def test_fft_many_host_and_device(h2b, orc, cuda, k):
    f = h2b.fields
    d = f.EvaluationDomain(4, k)
    polys = [orc.chacha_fr(30 + i, 1 << k) for i in range(3)]
    for j in range(1 << (d.extended_k - k)):
        c = d.g_coset * pow(d.extended_omega, j, f.R_MOD) % f.R_MOD
        want = [orc.ntt(6, k, k, p, mont(h2b, d.omega), mont(h2b, c)) for p in polys]
        got = h2b.fft_many(6, k, k, polys, d.omega, c)
        for g, w in zip(got, want):
            assert_limbs_equal(g, w, f"fft_many part {j}")
        d_in = [h2b.to_dev(p) for p in polys]
        d_out = [h2b.dev_empty(32 << k) for _ in polys]
        h2b.fft_many_to_device(6, k, k, d_in, d_out, d.omega, c, input_on_device=True)
        for g, w in zip(d_out, want):
            assert_limbs_equal(h2b.to_host(g), w, f"fft_many_to_device part {j}")
    # host inputs into device outputs, plain iFFT
    d_out = [h2b.dev_empty(32 << k) for _ in polys]
    h2b.fft_many_to_device(2, k, k, polys, d_out, d.omega_inv, d.ifft_divisor, input_on_device=False)
    for g, p in zip(d_out, polys):
        assert_limbs_equal(h2b.to_host(g), orc.ntt(2, k, k, p, mont(h2b, d.omega_inv), mont(h2b, d.ifft_divisor)),
                           "fft_many_to_device host input")


def test_full_size_roundtrip_k22_ext24(h2b, orc, cuda):
    """coeff_to_extended 2^22 -> 2^24, then the inverse transform at 2^24
    returns the zeta-twisted input followed by zero padding (size-independent
    property at the benchmark size)."""
    f = h2b.fields
    k, ek = 22, 24
    d = f.EvaluationDomain(5, k)
    assert d.extended_k == ek
    n, N = 1 << k, 1 << ek
    d_a = h2b.random_fr_device(n, 1234)
    d_ext = h2b.dev_empty(32 * N)
    h2b.fft_many_to_device(3, k, ek, [d_a], [d_ext], d.extended_omega, 1, input_on_device=True)
    d_back = h2b.dev_empty(32 * N)
    h2b.fft_normal_to_device(2, ek, d_ext, d_back, d.extended_omega_inv, d.extended_ifft_divisor)
    a = h2b.to_host(d_a)
    back = h2b.to_host(d_back)
    assert not back[n:].any()
    zi = [1, f.ZETA * f.ZETA % f.R_MOD, f.ZETA]  # zeta^-(i mod 3)
    sel = np.r_[0:64, n // 2: n // 2 + 64, n - 64:n]
    got = [f.from_mont(v) * zi[i % 3] % f.R_MOD for v, i in zip(f.limbs_to_ints(back[sel]), sel)]
    want = [f.from_mont(v) for v in f.limbs_to_ints(a[sel])]
    assert got == want


def test_full_size_coset_extension_k22_ext24_against_cpu(h2b, orc, cuda):
    """coeff_to_extended 2^22 -> 2^24 (the k=22 benchmark's coset NTT) checked
    against the CPU, not against a device inverse: output i is the input
    polynomial at zeta * w_ext^i, evaluated by the oracle's Horner at 259
    indices -- 0, 1, 2, N/2 and N-1, and one seeded index in every 2^16 block
    of the output.  Bit-exact."""
    import random
    f = h2b.fields
    k, ek = 22, 24
    d = f.EvaluationDomain(5, k)
    n, N = 1 << k, 1 << ek
    d_a = h2b.random_fr_device(n, 4321)
    d_ext = h2b.dev_empty(32 * N)
    h2b.fft_many_to_device(3, k, ek, [d_a], [d_ext], d.extended_omega, 1, input_on_device=True)
    rng = random.Random(22)
    idx = sorted({0, 1, 2, N // 2, N - 1} | {b + rng.randrange(1 << 16) for b in range(0, N, 1 << 16)})
    pts = [f.ZETA * pow(d.extended_omega, i, f.R_MOD) % f.R_MOD for i in idx]
    want = orc.fr_eval_many(h2b.to_host(d_a), f.fr_mont_limbs(pts))
    ext = h2b.to_host(d_ext)
    assert_limbs_equal(ext[np.array(idx)], want, "coset extension 2^22 -> 2^24 vs CPU evaluation")
