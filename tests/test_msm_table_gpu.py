"""Precomputed window tables (SRS kept resident with [2^(c w)] P_i): the table
entries (stored as x * 2^261 mod p) against Python curve arithmetic, and MSMs over a table against the
oracle and the plain MSM, including zero scalars, infinity bases, n below the
table size, and batched jobs over a shared table."""
import numpy as np
import pytest
import torch

from conftest import assert_limbs_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def table4k(h2b, orc, cuda):
    tau = h2b.fields.fr_mont_limbs([0x7AB1E5])
    srs = orc.srs(tau, 1 << 12)
    srs[5] = 0                                   # an infinity base
    d_srs = h2b.to_dev(srs)
    table = h2b.msm_table_precompute(d_srs, 1 << 12)
    torch.cuda.synchronize()
    return srs, d_srs, table


def test_table_entries(h2b, table4k):
    f = h2b.fields
    srs, _, table = table4k
    tn = 1 << 12
    pts = h2b.lib().h2b_msm_table_points(tn)
    W = pts // (2 * tn)                          # W slices, then their phi images
    t = h2b.to_host(table, (pts, 8))
    # the 2^12-point plan uses 10-bit windows: 13 of them cover the 127-bit GLV halves plus the digit carry
    c = 10
    assert W == 13
    for i in (0, 1, 5, 77, tn - 1):
        x = f.from_mont(f.limbs_to_ints(srs[i][:4].reshape(1, 4))[0], f.Q_MOD)
        y = f.from_mont(f.limbs_to_ints(srs[i][4:].reshape(1, 4))[0], f.Q_MOD)
        P = (x, y)
        for w in (0, 1, W - 1):
            got = t[w * tn + i]
            if i == 5:
                assert not got.any() and not t[W * tn + w * tn + i].any(), "infinity stays (0, 0)"
                continue
            want = f.g1_mul(P, 1 << (c * w))
            # stored as x * 2^261 mod p, the form the accumulation reads
            r261 = pow(2, 261, f.Q_MOD)
            assert f.limbs_to_ints(got[:4].reshape(1, 4))[0] == want[0] * r261 % f.Q_MOD
            assert f.limbs_to_ints(got[4:].reshape(1, 4))[0] == want[1] * r261 % f.Q_MOD
            # phi image W tn points later: (beta x, y), beta a cube root of unity mod p
            ph = t[W * tn + w * tn + i]
            px = f.limbs_to_ints(ph[:4].reshape(1, 4))[0] * pow(r261, -1, f.Q_MOD) % f.Q_MOD
            assert px != want[0] and pow(px * pow(want[0], -1, f.Q_MOD) % f.Q_MOD, 3, f.Q_MOD) == 1
            assert f.limbs_to_ints(ph[4:].reshape(1, 4))[0] == want[1] * r261 % f.Q_MOD


@pytest.mark.parametrize("n", [1, 2, 100, 3000, 4096])
def test_msm_over_table(h2b, orc, cuda, table4k, n):
    srs, d_srs, table = table4k
    tn = 1 << 12
    sc = orc.chacha_fr(300 + n, n)
    sc[::7] = 0
    want = orc.msm(sc, srs[:n])
    d_sc = h2b.to_dev(sc)
    out = h2b.dev_empty(96)
    h2b.msm_device_table(d_sc, table, tn, out, n)
    assert_limbs_equal(h2b.to_host(out, (12,)), want, f"table msm n={n}")
    # the plain device MSM gives the same bytes
    out2 = h2b.dev_empty(96)
    ws = h2b.msm_workspace(n)
    h2b.msm_device(d_sc, d_srs, out2, n, ws)
    assert out.cpu().numpy().tobytes() == out2.cpu().numpy().tobytes()


def test_msm_over_table_k16_mix_and_batch(h2b, orc, cuda):
    """2^16 table, witness-like scalars; then 6 batched jobs over the shared
    table next to the same jobs over plain bases."""
    n = 1 << 16
    d_srs = h2b.srs_device(0x7AB1E, n)
    table = h2b.msm_table_precompute(d_srs, n)
    d_sc = h2b.random_fr_device(n, 31, 1)
    out_t, out_p = h2b.dev_empty(96), h2b.dev_empty(96)
    h2b.msm_device_table(d_sc, table, n, out_t, n)
    h2b.msm_device(d_sc, d_srs, out_p, n, h2b.msm_workspace(n))
    torch.cuda.synchronize()
    assert out_t.cpu().numpy().tobytes() == out_p.cpu().numpy().tobytes()
    lengths = [n, 1 << 14, 1000, 1, 1 << 15, 77]
    scs = [h2b.random_fr_device(m, 40 + i, i % 2) for i, m in enumerate(lengths)]
    outs_t = [h2b.dev_empty(96) for _ in lengths]
    outs_p = [h2b.dev_empty(96) for _ in lengths]
    jt = h2b.msm_batch_jobs(scs, [table] * len(lengths), outs_t, lengths, table_n=n)
    jp = h2b.msm_batch_jobs(scs, [d_srs] * len(lengths), outs_p, lengths)
    h2b.msm_batch(jt, len(lengths), 4, h2b.msm_batch_workspace(jt, len(lengths), 4))
    h2b.msm_batch(jp, len(lengths), 4, h2b.msm_batch_workspace(jp, len(lengths), 4))
    torch.cuda.synchronize()
    assert [o.cpu().numpy().tobytes() for o in outs_t] == [o.cpu().numpy().tobytes() for o in outs_p]


def test_table_argument_errors(h2b, cuda, table4k):
    _, _, table = table4k
    d_sc = h2b.dev_empty(32 * 8192)
    with pytest.raises(h2b.Halo2GpuError):   # n above the table size
        h2b.msm_device_table(d_sc, table, 1 << 12, h2b.dev_empty(96), 8192, ws=h2b.dev_empty(1 << 20))
    assert h2b.lib().h2b_msm_table_points(1 << 28) == 0


def _bytes(t):
    return t.cpu().numpy().tobytes()


def test_merged_jobs_over_one_table(h2b, orc, cuda, table4k):
    """h2b_msm_merged: jobs of different lengths (full, partial, one point, an
    empty job, a repeated scalar vector) over the shared 2^12 table give the
    oracle's MSM per job and the bytes of h2b_msm_device_table."""
    srs, _, table = table4k
    tn = 1 << 12
    lengths = [tn, 3000, 100, 1, 0, tn, 517]
    scs = []
    for i, m in enumerate(lengths):
        sc = orc.chacha_fr(700 + i, max(m, 1))[:m] if m else np.zeros((0, 4), np.uint64)
        if m > 10:
            sc[::5] = 0
        scs.append(sc)
    scs[5] = scs[0].copy()                       # two jobs with the same scalars
    d_scs = [h2b.to_dev(s) if len(s) else h2b.dev_empty(32) for s in scs]
    outs = [h2b.dev_empty(96) for _ in lengths]
    jobs = h2b.msm_batch_jobs(d_scs, [table] * len(lengths), outs, lengths, table_n=tn)
    ws = h2b.dev_empty(h2b.msm_merged_workspace_bytes(jobs, len(lengths)))
    h2b.msm_merged(jobs, len(lengths), ws)
    for i, (m, sc) in enumerate(zip(lengths, scs)):
        got = h2b.to_host(outs[i], (12,))
        if m == 0:
            assert_limbs_equal(got, h2b.to_host(_inf_image(h2b), (12,)), "empty job")
            continue
        assert_limbs_equal(got, orc.msm(sc, srs[:m]), f"merged job {i} (n={m})")
        one = h2b.dev_empty(96)
        h2b.msm_device_table(d_scs[i], table, tn, one, m)
        assert _bytes(one) == _bytes(outs[i])


def _inf_image(h2b):
    """(0, 1, 0): the reference's image of the point at infinity."""
    f = h2b.fields
    img = np.zeros(12, np.uint64)
    img[4:8] = f.fq_mont_limbs([1])[0]
    return h2b.to_dev(img)


def test_merged_64_jobs_k16_match_the_batch(h2b, cuda):
    """The 64-job maximum at mixed lengths over a 2^16 table, witness-like and
    uniform scalars: the same bytes as h2b_msm_batch over that table."""
    n = 1 << 16
    d_srs = h2b.srs_device(0x7AB1E, n)
    table = h2b.msm_table_precompute(d_srs, n)
    lengths = [n if i % 9 == 0 else (1 << (8 + i % 8)) + i for i in range(64)]
    scs = [h2b.random_fr_device(m, 900 + i, i % 2) for i, m in enumerate(lengths)]
    outs_m = [h2b.dev_empty(96) for _ in lengths]
    outs_b = [h2b.dev_empty(96) for _ in lengths]
    jm = h2b.msm_batch_jobs(scs, [table] * 64, outs_m, lengths, table_n=n)
    jb = h2b.msm_batch_jobs(scs, [table] * 64, outs_b, lengths, table_n=n)
    h2b.msm_merged(jm, 64, h2b.dev_empty(h2b.msm_merged_workspace_bytes(jm, 64)))
    h2b.msm_batch(jb, 64, 8, h2b.msm_batch_workspace(jb, 64, 8))
    torch.cuda.synchronize()
    assert [_bytes(o) for o in outs_m] == [_bytes(o) for o in outs_b]


def test_merged_argument_errors(h2b, cuda, table4k):
    srs, d_srs, table = table4k
    tn = 1 << 12
    sc = h2b.dev_empty(32 * tn)
    out = h2b.dev_empty(96)
    L = h2b.lib()
    other = h2b.msm_table_precompute(d_srs, tn)
    bad = [h2b.msm_batch_jobs([sc, sc], [table, other], [out, out], [10, 10], table_n=tn),   # two tables
           h2b.msm_batch_jobs([sc], [d_srs], [out], [10], table_n=0),                       # plain bases
           h2b.msm_batch_jobs([sc], [table], [out], [tn + 1], table_n=tn)]                  # longer than table
    for jobs in bad:
        assert L.h2b_msm_merged_workspace_size(jobs, len(jobs)) == 0
        with pytest.raises(h2b.Halo2GpuError, match="h2b_msm_merged"):
            h2b.msm_merged(jobs, len(jobs), h2b.dev_empty(1 << 20))
    many = h2b.msm_batch_jobs([sc] * 65, [table] * 65, [out] * 65, [1] * 65, table_n=tn)
    assert L.h2b_msm_merged_workspace_size(many, 65) == 0
    with pytest.raises(h2b.Halo2GpuError, match="1 to 64 jobs"):
        h2b.msm_merged(many, 65, h2b.dev_empty(1 << 20))
    ok = h2b.msm_batch_jobs([sc], [table], [out], [tn], table_n=tn)
    need = L.h2b_msm_merged_workspace_size(ok, 1)
    with pytest.raises(h2b.Halo2GpuError):
        h2b.msm_merged(ok, 1, h2b.dev_empty(need - 256))


def test_wide_windows_split_bit_sums(h2b, orc, cuda):
    """Window widths 17-19 give bucket reductions whose bit sums span more
    than 4096 segment sums, split over several CTAs and summed by a second
    kernel: a table MSM and a plain MSM at those widths equal the oracle."""
    L = h2b.lib()
    n = 1 << 12
    tau = h2b.fields.fr_mont_limbs([0x51DE])
    srs = orc.srs(tau, n)
    d_srs = h2b.to_dev(srs)
    sc = orc.chacha_fr(77, n)
    sc[::5] = 0
    want = orc.msm(sc, srs)
    d_sc = h2b.to_dev(sc)
    try:
        for c in (17, 19):
            L.h2b_msm_set_tuning(c, 0)
            assert L.h2b_msm_window_bits(n) == c
            table = h2b.msm_table_precompute(d_srs, n)
            out = h2b.dev_empty(96)
            h2b.msm_device_table(d_sc, table, n, out, n)
            assert_limbs_equal(h2b.to_host(out, (12,)), want, f"table msm at {c} bits")
            out2 = h2b.dev_empty(96)
            h2b.msm_device(d_sc, d_srs, out2, n, h2b.msm_workspace(n))
            assert_limbs_equal(h2b.to_host(out2, (12,)), want, f"plain msm at {c} bits")
    finally:
        L.h2b_msm_set_tuning(0, 0)
