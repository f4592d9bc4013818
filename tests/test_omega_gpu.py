"""Twiddle-table entry points against Python integers (the reference's tests:
halo2_proofs/src/poly/domain.rs:1226-1352 test_power_of_omega,
test_omega_powers_generation, test_omega_lookup_table_generation, which
compare with omega.pow_vartime and generate_omega_lut_cpu)."""
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ints(h2b, limbs):
    f = h2b.fields
    return [f.from_mont(x) for x in f.limbs_to_ints(limbs)]


def test_power_of_omega_max_pow(h2b, cuda):
    """log_n = 31 and pow = u32::MAX >> 1, as in domain.rs:1227-1253."""
    f = h2b.fields
    omega = random.Random(5).randrange(1, f.R_MOD)
    log_n, pw = 31, (1 << 32) - 1 >> 1
    res, lut = h2b.power_of_omega_gpu(omega, log_n, pw)
    assert _ints(h2b, res) == [pow(omega, pw, f.R_MOD)]
    assert _ints(h2b, lut) == [1] + [pow(omega, 1 << i, f.R_MOD) for i in range(log_n)]


@pytest.mark.parametrize("log_n,pw", [(0, 0), (1, 1), (5, 17), (22, 0x2aaaaa)])
def test_power_of_omega_domain(h2b, cuda, log_n, pw):
    f = h2b.fields
    omega = f.EvaluationDomain(1, max(log_n, 1)).omega
    res, lut = h2b.power_of_omega_gpu(omega, log_n, pw)
    assert _ints(h2b, res) == [pow(omega, pw, f.R_MOD)]
    assert len(lut) == log_n + 1


@pytest.mark.parametrize("log_n", [1, 5, 8, 9, 10, 13, 16])
def test_generate_omega_powers(h2b, cuda, log_n):
    """domain.rs:1255-1318: omega^i for i < 2^log_n, first 2^log_n - 13 compared (all here)."""
    f = h2b.fields
    omega = f.EvaluationDomain(1, log_n).omega
    got = _ints(h2b, h2b.generate_omega_powers_gpu(omega, log_n))
    want, cur = [], 1
    for _ in range(1 << log_n):
        want.append(cur)
        cur = cur * omega % f.R_MOD
    assert got == want


def test_generate_omega_powers_k20_properties(h2b, cuda):
    """At 2^20: spot values against pow, and the cycle closes (omega^(n/2) = -1)."""
    f = h2b.fields
    log_n = 20
    omega = f.EvaluationDomain(1, log_n).omega
    got = h2b.generate_omega_powers_gpu(omega, log_n)
    ints = f.limbs_to_ints(got)
    rng = random.Random(3)
    for i in [0, 1, 255, 256, 4095, 4096, (1 << 19), (1 << 20) - 1] + [rng.randrange(1 << 20) for _ in range(200)]:
        assert f.from_mont(ints[i]) == pow(omega, i, f.R_MOD), i
    assert f.from_mont(ints[1 << 19]) == f.R_MOD - 1


@pytest.mark.parametrize("log_n", [10, 11, 14, 20])
def test_generate_omega_lut(h2b, cuda, log_n):
    """generate_omega_lut_cpu (halo2_proofs/src/cpu/arithmetic.rs:199-220)."""
    f = h2b.fields
    omega = f.EvaluationDomain(1, log_n).omega
    got = _ints(h2b, h2b.generate_omega_lut_gpu(omega, log_n))
    low = [pow(omega, i, f.R_MOD) for i in range(1 << 10)]
    s = pow(omega, 1 << 10, f.R_MOD)
    high = [pow(s, i, f.R_MOD) for i in range(1 << (log_n - 10))]
    assert got == low + high


@pytest.mark.parametrize("log_n,colnum,start,end", [(10, 1, 0, 1023), (12, 5, 100, 3000), (16, 8, 0, 65535)])
def test_generate_omegadelta(h2b, cuda, log_n, colnum, start, end):
    """out[i] = omega^row * delta^col over the (col, row) mapping (kernel/omega.h cukernel_generate_omegadelta)."""
    f = h2b.fields
    n = 1 << log_n
    omega = f.EvaluationDomain(1, log_n).omega
    rng = random.Random(log_n)
    ncols_table = 1 << max(0, (colnum - 1).bit_length())
    mapping = np.zeros((n, 2), dtype=np.uint32)
    mapping[:, 0] = [rng.randrange(ncols_table) for _ in range(n)]
    mapping[:, 1] = [rng.randrange(n) for _ in range(n)]
    d_map = h2b.to_dev(mapping)
    d_out = h2b.dev_empty(32 * (end - start + 1))
    h2b.generate_omegadelta_device(d_out, d_map, omega, f.DELTA, log_n, start, end, colnum)
    got = _ints(h2b, h2b.to_host(d_out))
    want = [pow(omega, int(mapping[i, 1]), f.R_MOD) * pow(f.DELTA, int(mapping[i, 0]), f.R_MOD) % f.R_MOD
            for i in range(start, end + 1)]
    assert got == want
