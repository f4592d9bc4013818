"""GLV constants of the MSM (halo2-gpu_b200/csrc/glv.cuh), checked with exact
integer arithmetic on the CPU: the endomorphism, the lattice basis, the
fixed-point rounding constants, and a proof that the split of every scalar
k < r has |k1|, |k2| < 2^127 (the window count of the MSM relies on it)."""
import random
import re
from fractions import Fraction
from pathlib import Path

import pytest

import importlib.util
import sys

ROOT = Path(__file__).resolve().parents[1]
GLV = (ROOT / "halo2-gpu_b200" / "csrc" / "glv.cuh").read_text()


def _fields():
    spec = importlib.util.spec_from_file_location("h2b_fields", ROOT / "halo2-gpu_b200" / "fields.py")
    m = importlib.util.module_from_spec(spec)
    sys.modules.setdefault("h2b_fields", m)
    spec.loader.exec_module(m)
    return m


F = _fields()
r, q = F.R_MOD, F.Q_MOD


def _limbs(name, width):
    m = re.search(name + r"\[\d+\]\s*=\s*\{([^}]*)\}", GLV)
    vals = [int(x.strip().rstrip("ul"), 16) for x in m.group(1).split(",")]
    return sum(v << (width * i) for i, v in enumerate(vals))


G1 = _limbs("G1c", 64)
G2 = _limbs("G2c", 64)
A1 = _limbs("A1c", 64)
B2 = _limbs("B2c", 64)
A2 = int(re.search(r"A2\s*=\s*(0x[0-9a-f]+)ull", GLV).group(1), 16)
BETA = sum(int(v, 16) << (32 * int(i)) for i, v in re.findall(r"b\.v\[(\d)\]\s*=\s*(0x[0-9a-f]+)u", GLV))
B1 = -A2
LAMBDA = F.ZETA
M = 1 << 256


def decompose(k):
    """Python restatement of glv::decompose (two's complement mod 2^256)."""
    c1 = (k * G1) >> 256
    c2 = (k * G2) >> 256
    k1 = (k - c1 * A1 - c2 * A2) % M
    k2 = (c1 * A2 - c2 * B2) % M
    return (k1 - M if k1 >> 255 else k1), (k2 - M if k2 >> 255 else k2)


def test_endomorphism():
    beta = F.from_mont(BETA, q)
    assert beta != 1 and pow(beta, 3, q) == 1
    assert LAMBDA != 1 and pow(LAMBDA, 3, r) == 1
    g = (1, 2)
    assert F.g1_mul(g, LAMBDA) == (beta * g[0] % q, g[1])
    p = F.g1_mul(g, 0x1234567890ABCDEF)
    assert F.g1_mul(p, LAMBDA) == (beta * p[0] % q, p[1])


def test_lattice_and_rounding_constants():
    assert (A1 + B1 * LAMBDA) % r == 0
    assert (A2 + B2 * LAMBDA) % r == 0
    assert A1 * B2 - A2 * B1 == r
    assert G1 == (B2 << 256) // r
    assert G2 == (-B1 << 256) // r
    # the kernel keeps c1 in two and c2 in one 64-bit limb
    assert ((r - 1) * G1) >> 256 < 1 << 128 and ((r - 1) * G2) >> 256 < 1 << 64


def test_split_bound_for_every_scalar():
    """c_i = x_i - d_i with x_1 = k b2 / r, x_2 = -k b1 / r and
    0 <= d_i < 1 + (r / 2^256) frac(2^256 b_i / r).  Since x_1 a1 + x_2 a2 = k
    and x_1 a2 - x_2 b2 = 0 exactly, k1 = d1 a1 + d2 a2 and k2 = d2 b2 - d1 a2,
    so the bounds below hold for all k < r."""
    e1 = Fraction((B2 << 256) % r, r)
    e2 = Fraction((-B1 << 256) % r, r)
    d1 = 1 + Fraction(r, M) * e1
    d2 = 1 + Fraction(r, M) * e2
    assert d1 * A1 + d2 * A2 < 1 << 127
    assert d2 * B2 < 1 << 127 and d1 * A2 < 1 << 127


@pytest.mark.parametrize("seed", [1, 2])
def test_decompose_samples(seed):
    rng = random.Random(seed)
    ks = [0, 1, 2, r - 1, r - 2, LAMBDA, r - LAMBDA, (r - 1) // 2, A1, B2] + [rng.randrange(r) for _ in range(3000)]
    for k in ks:
        k1, k2 = decompose(k)
        assert (k1 + k2 * LAMBDA - k) % r == 0
        assert abs(k1) < 1 << 127 and abs(k2) < 1 << 127
