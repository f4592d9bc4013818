"""MSM parity against the oracle (bit-exact 96-byte Jacobian images), the
reference's edge-case families (halo2_proofs/tests/multiexp_dense_bucket_edge_equivalence.rs:104-280,
halo2_proofs/src/cuda/tests.rs:390-585) and the KZG property
MSM(s, [tau^i]G) = [sum s_i tau^i] G at the full 2^22 size."""
import numpy as np
import pytest

from conftest import assert_limbs_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def srs_small(h2b, orc):
    tau = h2b.fields.fr_mont_limbs([0x1234567890ABCDEF1234567890ABCDEF])
    return tau, orc.srs(tau, 1 << 12)


def all_variants(h2b, sc, bases):
    n = sc.shape[0]
    out = [h2b.multiexp_gpu(sc, bases)]
    d_b = h2b.to_dev(bases)
    out.append(h2b.multiexp_gpu_device_bases(sc, d_b))
    d_s = h2b.to_dev(sc)
    out.append(h2b.multiexp_gpu_device_scalars_device_bases(d_s, d_b, n))
    assert_limbs_equal(h2b.to_host(d_s), sc, "device scalars must not be mutated")
    return out


@pytest.mark.parametrize("n", [1, 2, 3, 20, 100, 1000, 4096])
def test_msm_uniform_small(h2b, orc, cuda, srs_small, n):
    _, srs = srs_small
    bases = srs[:n]
    sc = orc.chacha_fr(500 + n, n)
    want = orc.msm(sc, bases)
    for got in all_variants(h2b, sc, bases):
        assert_limbs_equal(got, want, f"msm n={n}")


def test_msm_edge_cases(h2b, orc, cuda, srs_small):
    _, srs = srs_small
    n = 2048
    bases = srs[:n].copy()
    sc = orc.chacha_fr(77, n)
    # zero scalars and infinity bases
    sc[::5] = 0
    bases[::7] = 0
    want = orc.msm(sc, bases)
    for got in all_variants(h2b, sc, bases):
        assert_limbs_equal(got, want, "zeros / infinity")
    # all zero -> (0, 1, 0)
    z = np.zeros((n, 4), np.uint64)
    got = h2b.multiexp_gpu(z, srs[:n])
    assert not got[0:4].any() and not got[8:12].any()
    assert_limbs_equal(got, orc.msm(z, srs[:n]), "all zero")
    # dense buckets: the first half share one constant scalar (reference's K)
    K = h2b.fields.fr_mont_limbs([0x022B5F6A3C1D0E8F94D049BB133111EBBF58476D1CE4E5B99E3779B97F4A7C15])
    sc2 = orc.chacha_fr(78, n)
    sc2[: n // 2] = K
    assert_limbs_equal(h2b.multiexp_gpu(sc2, srs[:n]), orc.msm(sc2, srs[:n]), "dense constant")
    # every scalar 1 and every scalar -1 (one bucket per window, all points)
    ones = h2b.fields.fr_mont_limbs([1] * n)
    assert_limbs_equal(h2b.multiexp_gpu(ones, srs[:n]), orc.msm(ones, srs[:n]), "all ones")
    negs = h2b.fields.fr_mont_limbs([h2b.fields.R_MOD - 1] * n)
    assert_limbs_equal(h2b.multiexp_gpu(negs, srs[:n]), orc.msm(negs, srs[:n]), "all minus one")
    # P + (-P) cancellation inside a bucket
    b3 = srs[:n].copy()
    b3[1::2] = b3[0::2]
    sc3 = np.tile(h2b.fields.fr_mont_limbs([5, h2b.fields.R_MOD - 5]), (n // 2, 1))
    got = h2b.multiexp_gpu(sc3, b3)
    assert not got[8:12].any(), "sum must be infinity"


def test_msm_all_bases_generator(h2b, orc, cuda):
    n = 1 << 14
    g = orc.g1_generator()
    bases = np.tile(g, (n, 1))
    sc = orc.chacha_fr(3, n)
    total = h2b.fields.fr_mont_limbs([sum(h2b.fields.fr_from_mont_limbs(sc)) % h2b.fields.R_MOD])
    want = orc.g1_mul(total, g)
    assert_limbs_equal(h2b.multiexp_gpu(sc, bases), want, "(sum s) G")


def test_msm_config1_k16_and_mix(h2b, orc, cuda):
    n = 1 << 16
    tau = h2b.fields.fr_mont_limbs([0xC0FFEE])
    srs = h2b.to_host(h2b.srs_device(0xC0FFEE, n), (n, 8))
    # device SRS generator agrees with the oracle at sampled indices
    for i in (0, 1, 2, 777, n - 1):
        p = orc.g1_mul(h2b.fields.fr_mont_limbs([pow(0xC0FFEE, i, h2b.fields.R_MOD)]), orc.g1_generator())
        assert_limbs_equal(srs[i], p[:8], f"srs[{i}]")
    del tau
    for mix in (0, 1):
        sc = h2b.to_host(h2b.random_fr_device(n, 42 + mix, mix))
        want = orc.msm(sc, srs)
        assert_limbs_equal(h2b.multiexp_gpu_device_bases(sc, h2b.to_dev(srs)), want, f"k=16 mix={mix}")


def test_msm_n65540_ten_dense_buckets(h2b, orc, cuda):
    """n = 65540 with ten distinct constants each on 10% of the rows
    (the reference's ten-dense-buckets-per-window case)."""
    n = 65540
    srs = h2b.to_host(h2b.srs_device(99, n), (n, 8))
    sc = orc.chacha_fr(11, n)
    ks = orc.chacha_fr(12, 10)
    for j in range(10):
        sc[j * (n // 10):(j + 1) * (n // 10)] = ks[j]
    assert_limbs_equal(h2b.multiexp_gpu(sc, srs), orc.msm(sc, srs), "ten dense")


def test_msm_kzg_property_k22(h2b, orc, cuda):
    """MSM over [tau^i]G with the 50/30/20 scalar mix at n = 2^22 equals
    [f(tau)] G with f(tau) = sum s_i tau^i computed on the CPU."""
    f = h2b.fields
    n = 1 << 22
    tau = 0x2A2B2C2D2E2F
    d_srs = h2b.srs_device(tau, n)
    d_sc = h2b.random_fr_device(n, 2022, 1)
    got = h2b.multiexp_gpu_device_scalars_device_bases(d_sc, d_srs, n)
    sc = h2b.to_host(d_sc)
    ft = orc.fr_eval(sc, f.fr_mont_limbs([tau]))
    want = orc.g1_mul(ft, orc.g1_generator())
    assert_limbs_equal(got, want, "KZG property at 2^22")
    # the device SRS agrees with the oracle at sampled indices
    srs = h2b.to_host(d_srs[: 64 * 4], (4, 8))
    for i in range(4):
        p = orc.g1_mul(f.fr_mont_limbs([pow(tau, i, f.R_MOD)]), orc.g1_generator())
        assert_limbs_equal(srs[i], p[:8], f"srs[{i}]")
    # host scalars (copied in pieces that overlap the split) give the same point
    assert_limbs_equal(h2b.multiexp_gpu_device_bases(sc, d_srs, n), want, "host scalars at 2^22")


@pytest.mark.parametrize("n", [(1 << 18) - 1, 1 << 18, (1 << 18) + 5, 300007])
def test_msm_host_scalars_in_pieces(h2b, orc, cuda, n):
    """_halo2_multiexp_device_bases copies host scalars in pieces from 2^18
    points on; ragged piece boundaries against the device-scalar path."""
    d_srs = h2b.srs_device(0x51CE5, n)
    d_sc = h2b.random_fr_device(n, 77 + n, 1)
    want = h2b.multiexp_gpu_device_scalars_device_bases(d_sc, d_srs, n)
    got = h2b.multiexp_gpu_device_bases(h2b.to_host(d_sc), d_srs, n)
    assert_limbs_equal(got, want, f"host scalars n={n}")


@pytest.mark.parametrize("rounds", [1, 2, 3])
def test_msm_pairing_rounds(h2b, orc, cuda, srs_small, rounds):
    """The batch-affine pairing rounds (h2b_msm_set_pair_rounds, off by
    default) give the same bytes: uniform scalars, zeros, infinity bases,
    equal points in a bucket (doubling), P + (-P), a dense constant and the
    witness-like mix."""
    f = h2b.fields
    _, srs = srs_small
    n = 4096
    L = h2b.lib()
    L.h2b_msm_set_pair_rounds(rounds)
    if L.h2b_msm_get_pair_rounds() != rounds:
        pytest.skip("pairing rounds are built only with H2B_EXPERIMENTS=1")
    try:
        cases = []
        sc = orc.chacha_fr(90 + rounds, n)
        b = srs[:n].copy()
        sc[::5] = 0
        b[::7] = 0
        cases.append((sc, b))
        b2 = srs[:n].copy()
        b2[1::2] = b2[0::2]                      # equal points -> doubling in the pair formula
        cases.append((np.tile(f.fr_mont_limbs([5, 5]), (n // 2, 1)), b2))
        cases.append((np.tile(f.fr_mont_limbs([5, f.R_MOD - 5]), (n // 2, 1)), b2))  # P + (-P)
        sc4 = orc.chacha_fr(95, n)
        sc4[: n // 2] = f.fr_mont_limbs([0x022B5F6A3C1D0E8F94D049BB133111EBBF58476D1CE4E5B99E3779B97F4A7C15])
        cases.append((sc4, srs[:n]))
        mix = f.fr_mont_limbs([v % f.R_MOD for v in ([0x1F2E3D4C5B6A7988 * (i + 1) for i in range(n // 4)] +
                                                     [i % 2 for i in range(n // 4)] +
                                                     [f.limbs_to_ints(orc.chacha_fr(96, n // 2))[i] for i in
                                                      range(n // 2)])])
        cases.append((mix, srs[:n]))
        for sc_, b_ in cases:
            want = orc.msm(sc_, b_)
            for got in all_variants(h2b, sc_, b_):
                assert_limbs_equal(got, want, f"pairing rounds {rounds}")
    finally:
        L.h2b_msm_set_pair_rounds(0)


@pytest.mark.parametrize("variant", [0, 5, 6, 7])
def test_msm_accumulate_forms(h2b, orc, cuda, srs_small, variant):
    """Every bucket-accumulation form (h2b_msm_set_accumulate_variant: 0 =
    29-bit lazy R = 2^261, 5 = normalised R = 2^256, 6 = FP64 lazy R' =
    2^260) gives the oracle's bytes on the edge families: zero scalars and
    infinity bases, equal points in a bucket (the doubling branch), P + (-P)
    (infinity inside a bucket), a dense constant and the witness-like mix;
    and over a window table."""
    f = h2b.fields
    _, srs = srs_small
    n = 4096
    L = h2b.lib()
    before = L.h2b_msm_get_accumulate_variant()
    L.h2b_msm_set_accumulate_variant(variant)
    if L.h2b_msm_get_accumulate_variant() != variant:
        pytest.skip(f"accumulation form {variant} is built only with H2B_EXPERIMENTS=1")
    try:
        cases = []
        sc = orc.chacha_fr(190 + variant, n)
        b = srs[:n].copy()
        sc[::5] = 0
        b[::7] = 0
        cases.append((sc, b))
        b2 = srs[:n].copy()
        b2[1::2] = b2[0::2]
        cases.append((np.tile(f.fr_mont_limbs([5, 5]), (n // 2, 1)), b2))
        cases.append((np.tile(f.fr_mont_limbs([5, f.R_MOD - 5]), (n // 2, 1)), b2))
        sc4 = orc.chacha_fr(195, n)
        sc4[: n // 2] = f.fr_mont_limbs([0x022B5F6A3C1D0E8F94D049BB133111EBBF58476D1CE4E5B99E3779B97F4A7C15])
        cases.append((sc4, srs[:n]))
        mix = f.fr_mont_limbs([v % f.R_MOD for v in ([0x1F2E3D4C5B6A7988 * (i + 1) for i in range(n // 4)] +
                                                     [i % 2 for i in range(n // 4)] +
                                                     [f.limbs_to_ints(orc.chacha_fr(196, n // 2))[i] for i in
                                                      range(n // 2)])])
        cases.append((mix, srs[:n]))
        for sc_, b_ in cases:
            want = orc.msm(sc_, b_)
            for got in all_variants(h2b, sc_, b_):
                assert_limbs_equal(got, want, f"accumulate variant {variant}")
        # over a window table (tables use the lazy forms 0 or 6)
        table = h2b.msm_table_precompute(h2b.to_dev(srs[:n]), n)
        out = h2b.dev_empty(96)
        h2b.msm_device_table(h2b.to_dev(mix), table, n, out, n)
        assert_limbs_equal(h2b.to_host(out, (12,)), orc.msm(mix, srs[:n]), f"table, variant {variant}")
    finally:
        L.h2b_msm_set_accumulate_variant(before)
