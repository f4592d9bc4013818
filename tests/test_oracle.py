"""Pins the CPU oracle against the golden vectors (pure-Python big-integer
restatement in tests/golden/make_golden.py) and against the reference's
known-answer shapes.  CPU only."""
import json
import os

import numpy as np
import pytest

from conftest import assert_limbs_equal

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def L(hexes):
    return np.array([[int(h, 16) for h in x] for x in hexes], dtype=np.uint64)


def one(hexes):
    return L([hexes])


def jac(img):
    return np.concatenate([L([img[0]]), L([img[1]]), L([img[2]])]).reshape(12)


def test_field_ops(orc):
    lib = orc.lib()
    for case in GOLDEN["fr_ops"]:
        a, b = one(case["a"]), one(case["b"])
        r = np.zeros((1, 4), np.uint64)
        lib.o_field_mul(0, a.ctypes.data, b.ctypes.data, r.ctypes.data)
        assert_limbs_equal(r, one(case["ab"]), "fr mul")
        lib.o_field_add(0, a.ctypes.data, b.ctypes.data, r.ctypes.data)
        assert_limbs_equal(r, one(case["a_plus_b"]), "fr add")
        lib.o_field_sub(0, a.ctypes.data, b.ctypes.data, r.ctypes.data)
        assert_limbs_equal(r, one(case["a_minus_b"]), "fr sub")
        lib.o_field_inv(0, a.ctypes.data, r.ctypes.data)
        assert_limbs_equal(r, one(case["inv_a"]), "fr inv")
    for case in GOLDEN["fq_ops"]:
        a, b = one(case["a"]), one(case["b"])
        r = np.zeros((1, 4), np.uint64)
        lib.o_field_mul(1, a.ctypes.data, b.ctypes.data, r.ctypes.data)
        assert_limbs_equal(r, one(case["ab"]), "fq mul")
        lib.o_field_inv(1, a.ctypes.data, r.ctypes.data)
        assert_limbs_equal(r, one(case["inv_a"]), "fq inv")


def test_zeta_and_root_constants(h2b):
    f = h2b.fields
    assert pow(f.ZETA, 3, f.R_MOD) == 1 and f.ZETA != 1
    assert pow(f.ROOT_OF_UNITY, 1 << 28, f.R_MOD) == 1
    assert pow(f.ROOT_OF_UNITY, 1 << 27, f.R_MOD) == f.R_MOD - 1
    # zeta.h stores zeta in Montgomery form; the product's constant matches it
    z_mont = [244305545194690131, 8351807910065594880, 14266533074055306532, 404339206190769364]
    assert f.to_mont(f.ZETA) == sum(v << (64 * i) for i, v in enumerate(z_mont))


@pytest.mark.parametrize("case", GOLDEN["ntt"], ids=lambda c: f"k{c['k']}")
def test_ntt_golden(orc, case):
    k = case["k"]
    a = L(case["input"])
    assert_limbs_equal(orc.ntt(1, k, k, a, one(case["omega"]), one(case["divisor"])), L(case["fft"]), "fft")
    assert_limbs_equal(orc.ntt(2, k, k, a, one(case["omega_inv"]), one(case["divisor"])), L(case["ifft"]), "ifft")
    assert_limbs_equal(orc.ntt(6, k, k, a, one(case["omega"]), one(case["coset_factor"])), L(case["coset_part"]),
                       "coset part")


def test_coset_extension_golden(orc):
    c = GOLDEN["coset_ext"]
    out = orc.ntt(3, c["k"], c["ek"], L(c["input"]), one(c["omega_ext"]), one(c["omega_ext"]))
    assert_limbs_equal(out, L(c["output"]), "coset ext")


def test_ntt_roundtrip_and_coset_inverse(orc, h2b):
    f = h2b.fields
    for k in (5, 9, 12):
        d = f.EvaluationDomain(4, k)
        a = orc.chacha_fr(11 + k, 1 << k)
        fw = orc.ntt(1, k, k, a, f.fr_mont_limbs([d.omega]), f.fr_mont_limbs([1]))
        back = orc.ntt(2, k, k, fw, f.fr_mont_limbs([d.omega_inv]), f.fr_mont_limbs([d.ifft_divisor]))
        assert_limbs_equal(back, a, f"roundtrip k={k}")
        ek = d.extended_k
        ext = orc.ntt(3, k, ek, a, f.fr_mont_limbs([d.extended_omega]), f.fr_mont_limbs([1]))
        coeffs = orc.ntt(4, ek, ek, ext, f.fr_mont_limbs([d.extended_omega_inv]),
                         f.fr_mont_limbs([d.extended_ifft_divisor]))
        assert_limbs_equal(coeffs[: 1 << k], a, "coset ext inverse")
        assert not coeffs[1 << k:].any()
        # the extension's parts equal coset_part NTTs at zeta * w_ext^j
        for j in range(1 << (ek - k)):
            c = d.g_coset * pow(d.extended_omega, j, f.R_MOD) % f.R_MOD
            part = orc.ntt(6, k, k, a, f.fr_mont_limbs([d.omega]), f.fr_mont_limbs([c]))
            assert_limbs_equal(part, ext[j::1 << (ek - k)], f"part {j}")


def test_msm_golden(orc):
    m = GOLDEN["msm"]
    bases = np.concatenate([L([p[0] for p in m["bases"]]), L([p[1] for p in m["bases"]])], axis=1)
    sc = L(m["scalars"])
    assert_limbs_equal(orc.msm(sc, bases, threads=1), jac(m["result"]), "msm")
    assert_limbs_equal(orc.msm_naive(sc, bases), jac(m["result"]), "msm naive")


def test_msm_all_bases_g(orc):
    m = GOLDEN["msm_all_g"]
    g = orc.g1_generator()
    sc = L(m["scalars"])
    bases = np.tile(g, (sc.shape[0], 1))
    assert_limbs_equal(orc.msm(sc, bases), jac(m["result"]), "(sum s) G")


def test_msm_reference_fixed_scalar(orc, h2b):
    if "reference_fixed_scalar" not in GOLDEN:
        pytest.skip("reference tree absent when the golden file was made")
    c = GOLDEN["reference_fixed_scalar"]
    raw = sum(int(h, 16) << (64 * i) for i, h in enumerate(c["raw_limbs"]))
    s = h2b.fields.fr_mont_limbs([raw])
    assert_limbs_equal(orc.g1_mul(s, orc.g1_generator()), jac(c["times_g"]), "K * G")


def test_msm_threaded_matches_serial_and_edges(orc, h2b):
    f = h2b.fields
    n = 300
    tau = f.fr_mont_limbs([123456789])
    bases = orc.srs(tau, n)
    sc = orc.chacha_fr(5, n)
    ref = orc.msm_naive(sc, bases)
    assert_limbs_equal(orc.msm(sc, bases, threads=1), ref, "serial")
    assert_limbs_equal(orc.msm(sc, bases, threads=7), ref, "threaded")
    zero = np.zeros((n, 4), np.uint64)
    inf = orc.msm(zero, bases)
    assert inf[8:].sum() == 0 and int(inf[4]) != 0  # (0, 1, 0)
    b2 = bases.copy()
    b2[::3] = 0  # infinity bases are skipped
    assert_limbs_equal(orc.msm(sc, b2, threads=3), orc.msm_naive(sc, b2), "inf bases")


def test_batch_invert_golden(orc):
    c = GOLDEN["batch_invert"]
    assert_limbs_equal(orc.batch_invert(L(c["input"])), L(c["output"]), "batch invert")
    assert_limbs_equal(orc.batch_invert_par(L(c["input"]), threads=3), L(c["output"]), "batch invert par")


def test_grand_product_golden(orc):
    c = GOLDEN["grand_product"]
    assert_limbs_equal(orc.grand_product(L(c["input"]), one(c["prefix"])), L(c["output"]), "grand product")


def test_permute_pair_golden(orc):
    c = GOLDEN["permute_pair"]
    pin, ptab = orc.permute_pair(L(c["input"]), L(c["table"]), c["n"], c["usable"])
    assert_limbs_equal(pin, L(c["permuted_input"]), "A'")
    assert_limbs_equal(ptab, L(c["permuted_table"]), "S'")


def test_permute_pair_rejects_missing_value(orc):
    a = orc.chacha_fr(1, 8)
    t = orc.chacha_fr(2, 8)
    with pytest.raises(ValueError):
        orc.permute_pair(a, t, 8, 6)


def test_chacha_fr_is_canonical(orc, h2b):
    xs = orc.chacha_fr(0, 64)
    ints = h2b.fields.limbs_to_ints(xs)
    assert all(x < h2b.fields.R_MOD for x in ints)
    assert len(set(ints)) == 64


def test_quotient_interpreter_matches_direct_gate_evaluation(orc, h2b):
    """The oracle's rule interpreter, fed the reference's 128-bit encoding of
    the config-3 gates, equals the gates evaluated directly with integers."""
    import rules as R
    f = h2b.fields
    P = f.R_MOD
    g = R.Graph()
    parts = R.plonk_and_fibonacci(g)
    nq, rs = 64, 2
    fixed = [orc.chacha_fr(10 + i, nq) for i in range(3)]
    inst = [orc.chacha_fr(20, nq)]
    adv = [orc.chacha_fr(30 + i, nq) for i in range(4)]
    chal = orc.chacha_fr(40, 1)
    y = 987654321
    ec = f.fr_mont_limbs([0, 1, P - 1, 2, y])
    got = orc.quotient(fixed, inst, adv, chal, f.fr_mont_limbs(g.constants), ec, np.array(g.rules, np.uint64),
                       np.array(parts, np.uint64), nq, rs, 0, nq)
    I = lambda a: f.fr_from_mont_limbs(a)
    F, IN, A, C = [I(c) for c in fixed], I(inst[0]), [I(c) for c in adv], I(chal)[0]
    for r in range(nq):
        at = lambda k: (r + k * rs) % nq
        g1 = (A[0][r] * F[0][r] + A[1][r] * F[1][r] + A[0][r] * A[1][r] * F[2][r] + A[2][r] * 7 + 12345) % P
        g2 = (A[3][at(2)] - A[3][at(1)] - A[3][r]) % P
        g3 = IN[at(-1)] * C % P
        want = ((g1 * y + g2) * y + g3) % P
        assert I(got[r:r + 1])[0] == want, f"row {r}"
