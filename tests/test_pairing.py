"""The host BN254 optimal ate pairing (halo2-gpu_b200/pairing.py) that ends
the KZG verifier's check (poly/kzg/msm.rs:159-176 in the reference): the
curve parameters, the G2 generator, non-degeneracy, order r, bilinearity in
both arguments, the product check the verifier runs, the Frobenius map and
the inversion it is built from."""
import importlib
import random

import pytest


@pytest.fixture(scope="module")
def E(h2b):
    return importlib.import_module(h2b.__name__ + ".pairing")


def test_bn_parameter_gives_the_moduli(h2b, E):
    x = E.BN_X
    assert h2b.fields.Q_MOD == 36 * x**4 + 36 * x**3 + 24 * x**2 + 6 * x + 1
    assert h2b.fields.R_MOD == 36 * x**4 + 36 * x**3 + 18 * x**2 + 6 * x + 1
    assert E.ATE_LOOP == 6 * x + 2


def test_g2_generator_on_twist_with_order_r(E):
    g = E.G2_GENERATOR
    assert E.g2_on_curve(g)
    assert E.g2_add(E.g2_mul(g, E.R - 1), g) is None           # r G2 = infinity
    assert E.g2_mul(g, 2) == E.g2_add(g, g)
    assert E.g2_on_curve(E.g2_frobenius(g))
    # pi acts on G2 as multiplication by p (mod r)
    assert E.g2_frobenius(g) == E.g2_mul(g, E.Q % E.R)


def test_fq12_frobenius_and_inverse(E):
    rng = random.Random(3)
    a = [rng.randrange(E.Q) for _ in range(12)]
    b = [rng.randrange(E.Q) for _ in range(12)]
    assert E.f12_frobenius(E.f12_mul(a, b)) == E.f12_mul(E.f12_frobenius(a), E.f12_frobenius(b))
    assert E.f12_frobenius(a, 12) == a
    assert E.f12_frobenius(a) == E.f12_pow(a, E.Q)
    assert E.f12_mul(a, E.f12_inv(a)) == E.ONE12


def test_pairing_is_bilinear_and_non_degenerate(h2b, E):
    F = h2b.fields
    g1, g2 = F.G1_GENERATOR, E.G2_GENERATOR
    rng = random.Random(11)
    a, b = rng.randrange(1, E.R), rng.randrange(1, E.R)
    e = E.pairing(g1, g2)
    assert e != E.ONE12
    assert E.f12_pow(e, E.R) == E.ONE12
    ab = E.pairing(F.g1_mul(g1, a), E.g2_mul(g2, b))
    assert ab == E.f12_pow(e, a * b % E.R)
    assert E.pairing(F.g1_mul(g1, a * b % E.R), g2) == ab
    assert E.pairing(None, g2) == E.ONE12 and E.pairing(g1, None) == E.ONE12


def test_product_check_as_the_verifier_runs_it(h2b, E):
    """e(W', [s]_2) e(R, -[1]_2) == 1 exactly when R = s W'."""
    F = h2b.fields
    rng = random.Random(17)
    s, k = rng.randrange(2, E.R), rng.randrange(2, E.R)
    g2, s_g2 = E.G2_GENERATOR, E.g2_mul(E.G2_GENERATOR, s)
    left = F.g1_mul(F.G1_GENERATOR, k)
    right = F.g1_mul(left, s)
    assert E.pairing_check([(left, s_g2), (right, E.g2_neg(g2))])
    assert not E.pairing_check([(left, s_g2), (F.g1_add(right, F.G1_GENERATOR), E.g2_neg(g2))])
    assert not E.pairing_check([(left, E.g2_mul(g2, s + 1)), (right, E.g2_neg(g2))])
