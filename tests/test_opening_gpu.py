"""Opening-phase kernels against the oracle and Python integers: Horner
evaluation (halo2_proofs/src/poly/domain.rs eval tests, polynomial_ops.rs
eval_polynomial_gpu), Kate division q = (a - a(u)) / (X - u)
(kate_division.cu; checked directly for small n and by the identity
q(x)(x - u) = a(x) - a(u) at a random x for large n), the multiopen
calculation (multiopen.cu) and the Assigned<F> decode (decode_assigned.cu)."""
import numpy as np
import pytest

from conftest import assert_limbs_equal

pytestmark = pytest.mark.gpu


def _ints(f, limbs):
    return [f.from_mont(x) for x in f.limbs_to_ints(limbs)]


def _synthetic_division(a, u, p):
    """q_{n-2} = a_{n-1}; q_{j-1} = a_j + u q_j (Python integers)."""
    n = len(a)
    q = [0] * (n - 1)
    acc = 0
    for j in range(n - 1, 0, -1):
        acc = (a[j] + u * acc) % p
        q[j - 1] = acc
    return q


@pytest.mark.parametrize("n", [1, 2, 7, 4095, 4096, 4097, 100003, 1 << 20])
def test_eval_polynomial(h2b, orc, cuda, n):
    f = h2b.fields
    a = orc.chacha_fr(700 + n % 97, n)
    for z in (0, 1, 0x1234567890ABCDEF1122334455667788):
        zl = f.fr_mont_limbs([z])
        got = h2b.eval_polynomial_device(h2b.to_dev(a), n, zl)
        assert_limbs_equal(got.reshape(1, 4), orc.fr_eval(a, zl), f"eval n={n} z={z}")


def test_eval_polynomial_batch_chunks(h2b, orc, cuda):
    f = h2b.fields
    n = 5000
    polys = [orc.chacha_fr(800 + i, n) for i in range(3)]
    pts = f.fr_mont_limbs([3, 0xDEADBEEF, f.R_MOD - 2])
    for off, ln in ((0, n), (1000, 2345), (4999, 1)):
        got = h2b.batch_eval_polynomial_gpu(polys, pts, off, ln)
        for i in range(3):
            assert_limbs_equal(got[i:i + 1], orc.fr_eval(polys[i][off:off + ln], pts[i:i + 1]), f"batch {off},{ln}")


@pytest.mark.parametrize("n", [2, 3, 9, 2048, 2049, 2050, 5001])
def test_kate_division_small(h2b, orc, cuda, n):
    f = h2b.fields
    p = f.R_MOD
    a = orc.chacha_fr(900 + n, n)
    for u in (0, 5, 0xABCDEF0123456789ABCDEF):
        want = _synthetic_division(_ints(f, a), u, p)
        d_q = h2b.dev_empty(32 * (n - 1))
        h2b.kate_division_device(h2b.to_dev(a), d_q, h2b.to_dev(f.fr_mont_limbs([u])), n)
        assert _ints(f, h2b.to_host(d_q)) == want, f"kate n={n} u={u}"


def test_kate_division_padded(h2b, orc, cuda):
    f = h2b.fields
    p = f.R_MOD
    n = 3000
    a = orc.chacha_fr(950, n)
    u = 77
    want = _synthetic_division(_ints(f, a), u, p)
    for out_len in (n - 1, n + 500, 1000):
        d_q = h2b.to_dev(np.full((out_len, 4), 0xFFFFFFFFFFFFFFFF, np.uint64))
        h2b.kate_division_device(h2b.to_dev(a), d_q, h2b.to_dev(f.fr_mont_limbs([u])), n, out_len=out_len)
        got = _ints(f, h2b.to_host(d_q))
        k = min(n - 1, out_len)
        assert got[:k] == want[:k] and all(x == 0 for x in got[k:]), f"padded out_len={out_len}"
    # n < 2: zeros only
    d_q = h2b.to_dev(np.full((8, 4), 0xFFFFFFFFFFFFFFFF, np.uint64))
    h2b.kate_division_device(h2b.to_dev(a[:1]), d_q, h2b.to_dev(f.fr_mont_limbs([u])), 1, out_len=8)
    assert not h2b.to_host(d_q).any()


@pytest.mark.parametrize("n", [1 << 20, (1 << 22) + 5])
def test_kate_division_identity_large(h2b, orc, cuda, n):
    """Two and three scan levels: q(x)(x - u) = a(x) - a(u) at a random x."""
    f = h2b.fields
    p = f.R_MOD
    a = orc.chacha_fr(990, n)
    u, x = 0x5EED5EED5EED, 0xC0FFEE1234567
    d_q = h2b.dev_empty(32 * (n - 1))
    h2b.kate_division_device(h2b.to_dev(a), d_q, h2b.to_dev(f.fr_mont_limbs([u])), n)
    q = h2b.to_host(d_q)
    xl, ul = f.fr_mont_limbs([x]), f.fr_mont_limbs([u])
    qx = _ints(f, orc.fr_eval(q, xl))[0]
    ax, au = _ints(f, orc.fr_eval(a, xl))[0], _ints(f, orc.fr_eval(a, ul))[0]
    assert qx * (x - u) % p == (ax - au) % p


def test_multiopen_poly_calculation(h2b, orc, cuda):
    f = h2b.fields
    p = f.R_MOD
    n, batch = 4000, 4
    polys = [orc.chacha_fr(1100 + i, n) for i in range(batch)]
    ch = f.fr_mont_limbs([2, 3, p - 1, 0x123456789])
    pts = f.fr_mont_limbs([7, 11, 13, 0xFEDCBA])
    for off, ln in ((0, n), (1500, 1200)):
        acc = np.full((n, 4), 0x55, np.uint64)
        acc_before = acc.copy()
        res = h2b.multiopen_poly_calculation(polys, acc, ch, pts, off, ln)
        for i in range(batch):
            assert_limbs_equal(res[i:i + 1], orc.fr_eval(polys[i][off:off + ln], pts[i:i + 1]), "multiopen eval")
        ci = _ints(f, ch)
        P = [_ints(f, q[off:off + ln]) for q in polys]
        want = [sum(ci[i] * P[i][k] for i in range(batch)) % p for k in range(ln)]
        assert _ints(f, acc[off:off + ln]) == want, "multiopen accumulator"
        # only the chunk is written
        assert (acc[:off] == acc_before[:off]).all() and (acc[off + ln:] == acc_before[off + ln:]).all()


def test_decode_assigned(h2b, orc, cuda):
    """Assigned<F> as the Rust side lays it out: tag byte, then the payloads
    at 8-byte-aligned offsets (stride 72 = 8 + 32 + 32)."""
    f = h2b.fields
    n = 3001
    stride, no, do = 72, 8, 40
    nums = orc.chacha_fr(1200, n)
    dens = orc.chacha_fr(1201, n)
    tags = np.arange(n) % 3
    raw = np.zeros(n * stride, np.uint8)
    for i in range(n):
        raw[i * stride] = tags[i]
        raw[i * stride + 1:i * stride + 8] = 0xAB   # padding bytes are ignored
        if tags[i] >= 1:
            raw[i * stride + no:i * stride + no + 32] = nums[i].view(np.uint8)
        if tags[i] == 2:
            raw[i * stride + do:i * stride + do + 32] = dens[i].view(np.uint8)
    d_n, d_d = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
    h2b.decode_assigned_device(d_n, d_d, h2b.to_dev(raw), n, stride, no, do)
    one = f.fr_mont_limbs([1])[0]
    want_n = np.where((tags >= 1)[:, None], nums, 0).astype(np.uint64)
    want_d = np.where((tags == 2)[:, None], dens, one).astype(np.uint64)
    assert_limbs_equal(h2b.to_host(d_n), want_n, "numerators")
    assert_limbs_equal(h2b.to_host(d_d), want_d, "denominators")


def _assigned_records(orc, n, seed, stride=72, no=8, do=40):
    """Random Assigned<F> records (tags Zero/Trivial/Rational) with some zero
    numerators and zero denominators; returns (raw bytes, tags, nums, dens)."""
    rng = np.random.default_rng(seed)
    tags = rng.integers(0, 3, n)
    nums = orc.chacha_fr(seed, n)
    dens = orc.chacha_fr(seed + 1, n)
    nums[rng.random(n) < 0.05] = 0
    dens[rng.random(n) < 0.05] = 0
    raw = np.zeros((n, stride), np.uint8)
    raw[:, 0] = tags
    raw[:, 1:no] = 0xCD                              # padding bytes are ignored
    raw[:, no:no + 32] = nums.view(np.uint8).reshape(n, 32)
    raw[:, do:do + 32] = dens.view(np.uint8).reshape(n, 32)
    return raw.reshape(-1), tags, nums, dens


def _assigned_values(f, tags, nums, dens, rows):
    p = f.R_MOD
    N, D = _ints(f, nums[rows]), _ints(f, dens[rows])
    out = []
    for t, a, b in zip(tags[rows], N, D):
        out.append(0 if t == 0 else (a if t == 1 else (a * pow(b, -1, p) % p if b else 0)))
    return out


@pytest.mark.parametrize("n,ncols", [(5000, 3), (1 << 20, 2)])
def test_batch_invert_assigned(h2b, orc, cuda, n, ncols):
    """batch_invert_assigned_device (halo2_proofs/src/poly.rs:364-420) as one
    entry point: every column's records decoded, denominators inverted
    together (a zero denominator gives 0), numerators multiplied; checked
    against Python integers (all rows at 5000, 4096 sampled rows at 2^20)."""
    f = h2b.fields
    cols = [_assigned_records(orc, n, 3000 + 7 * c) for c in range(ncols)]
    d_raw = [h2b.to_dev(c[0]) for c in cols]
    d_out = [h2b.dev_empty(32 * n) for _ in cols]
    h2b.batch_invert_assigned_device(d_out, d_raw, n, 72, 8, 40)
    rng = np.random.default_rng(n)
    rows = np.arange(n) if n <= 5000 else np.unique(np.r_[0, n - 1, rng.integers(0, n, 4094)])
    for (raw, tags, nums, dens), d in zip(cols, d_out):
        got = _ints(f, h2b.to_host(d)[rows])
        assert got == _assigned_values(f, tags, nums, dens, rows)


def test_batch_invert_assigned_rejects_bad_layouts(h2b, cuda):
    d = h2b.dev_empty(32 * 8)
    for stride, no, do in ((72, 8, 41), (70, 8, 40), (72, 8, 48), (72, 0, 40)):
        with pytest.raises(h2b.Halo2GpuError, match="layout"):
            h2b.batch_invert_assigned_device([d], [d], 8, stride, no, do)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 1000, (1 << 16) + 3])
def test_eval_many_device_matches_single_evaluations(h2b, orc, cuda, n):
    """h2b_eval_many_device over 64 device polynomials (points 0, 1, -1 and
    random) gives the bytes of _halo2_eval_polynomial per polynomial; more
    than 64 is an error."""
    import ctypes
    import random
    f = h2b.fields
    rng = random.Random(n)
    polys = [h2b.to_dev(orc.chacha_fr(500 + i, n)) for i in range(64)]
    pts = [0, 1, f.R_MOD - 1] + [rng.randrange(f.R_MOD) for _ in range(61)]
    got = h2b.to_host(h2b.eval_many_device(polys, pts, n))
    ws = h2b.dev_empty(h2b.lib()._halo2_eval_polynomial_workspace_size(n))
    for i, (d, z) in enumerate(zip(polys, pts)):
        res = ctypes.c_void_p()
        h2b.call("_halo2_eval_polynomial", h2b.ptr(d), ctypes.byref(h2b.host_ffi(f.fr_mont_limbs([z]))),
                 ctypes.byref(res), n, h2b.ptr(ws), ws.numel(), h2b.stream_handle())
        off = res.value - ws.data_ptr()
        assert h2b.to_host(ws[off:off + 32]).tobytes() == got[i].tobytes(), i
    with pytest.raises(h2b.Halo2GpuError, match="more than 64"):
        h2b.eval_many_device(polys + polys[:1], pts + [5], n)


@pytest.mark.gpu
@pytest.mark.parametrize("count", [0, 1, 7, 64])
def test_linear_combination_matches_multiply_add(h2b, orc, cuda, count):
    """h2b_poly_linear_combination (accumulating or not) gives the bytes of
    one _halo2_poly_multiply_add per term; more than 64 terms is an error."""
    import random
    f = h2b.fields
    n = 5000
    rng = random.Random(count)
    polys = [h2b.to_dev(orc.chacha_fr(700 + i, n)) for i in range(count)]
    coeffs = [rng.randrange(f.R_MOD) for _ in range(count)]
    start = orc.chacha_fr(699, n)
    want = h2b.to_dev(start)
    for d, c in zip(polys, coeffs):
        h2b.call("_halo2_poly_multiply_add", h2b.ptr(want), h2b.ptr(d), h2b.ptr(h2b.to_dev(f.fr_mont_limbs([c]))), n,
                 h2b.stream_handle())
    acc = h2b.to_dev(start)
    h2b.linear_combination_device(acc, polys, coeffs, n, accumulate=True)
    assert h2b.to_host(acc).tobytes() == h2b.to_host(want).tobytes()
    fresh = h2b.to_dev(orc.chacha_fr(698, n))          # overwritten: starts from zero
    h2b.linear_combination_device(fresh, polys, coeffs, n, accumulate=False)
    zero = h2b.to_dev(np.zeros((n, 4), np.uint64))
    for d, c in zip(polys, coeffs):
        h2b.call("_halo2_poly_multiply_add", h2b.ptr(zero), h2b.ptr(d), h2b.ptr(h2b.to_dev(f.fr_mont_limbs([c]))), n,
                 h2b.stream_handle())
    assert h2b.to_host(fresh).tobytes() == h2b.to_host(zero).tobytes()
    if count == 64:
        with pytest.raises(h2b.Halo2GpuError, match="more than 64"):
            h2b.linear_combination_device(acc, polys + polys[:1], coeffs + [1], n)
