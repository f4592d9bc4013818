"""Quotient evaluator parity against the oracle's rule interpreter, plus the
permutation and lookup constraint kernels (reference equivalence tests:
halo2_proofs/src/cpu/evaluator.rs:1045-1439, halo2_proofs/src/cuda/tests.rs:1570,1895)."""
import random

import numpy as np
import pytest

from conftest import assert_limbs_equal
import rules as R

pytestmark = pytest.mark.gpu


def columns(orc, seed, count, n):
    return [orc.chacha_fr(seed + i, n) for i in range(count)]


def run_both(h2b, orc, g, parts, nf, ni, na, nch, nq, rot_scale, row_start, row_end, prev=None, seed=0):
    f = h2b.fields
    fixed = columns(orc, 1000 + seed, nf, nq)
    inst = columns(orc, 2000 + seed, ni, nq)
    adv = columns(orc, 3000 + seed, na, nq)
    chal = orc.chacha_fr(4000 + seed, nch) if nch else np.zeros((0, 4), np.uint64)
    consts = f.fr_mont_limbs(g.constants)
    y = 0x1234567 + seed
    rules = np.array(g.rules, dtype=np.uint64)
    vp = np.array(parts, dtype=np.uint64)
    ec = f.fr_mont_limbs([0, 1, f.R_MOD - 1, 2, y])
    want = orc.quotient(fixed, inst, adv, chal if nch else np.zeros((1, 4), np.uint64), consts, ec, rules, vp, nq,
                        rot_scale, row_start, row_end, prev)
    d_out = h2b.dev_empty(32 * (row_end - row_start))
    d_prev = h2b.to_dev(prev) if prev is not None else None
    h2b.quotient_device([h2b.to_dev(c) for c in fixed], [h2b.to_dev(c) for c in inst], [h2b.to_dev(c) for c in adv],
                        chal, consts, y, rules, vp, nq, rot_scale, row_start, row_end, d_out, d_prev)
    assert_limbs_equal(h2b.to_host(d_out), want, "device quotient")
    # the host-column entry point has no prev seed (quotient.cu:309-440)
    if prev is not None:
        want = orc.quotient(fixed, inst, adv, chal if nch else np.zeros((1, 4), np.uint64), consts, ec, rules, vp,
                            nq, rot_scale, row_start, row_end, None)
    got = h2b.quotient_host(fixed, inst, adv, chal, consts, y, rules, vp, nq, rot_scale, row_start, row_end)
    assert_limbs_equal(got, want, "host quotient")


@pytest.mark.parametrize("nq,rot_scale", [(1 << 10, 1), (1 << 12, 4), (1 << 16, 4), (1 << 18, 1)])
def test_plonk_fibonacci_gates(h2b, orc, cuda, nq, rot_scale):
    g = R.Graph()
    parts = R.plonk_and_fibonacci(g)
    run_both(h2b, orc, g, parts, 3, 1, 4, 1, nq, rot_scale, 0, nq)


def test_chunked_rows_and_prev_seed(h2b, orc, cuda):
    g = R.Graph()
    parts = R.plonk_and_fibonacci(g)
    nq = 1 << 12
    prev = orc.chacha_fr(77, 1000)
    # a chunk in the middle, one wrapping past the end via negative / positive rotations
    run_both(h2b, orc, g, parts, 3, 1, 4, 1, nq, 4, 1500, 2500, prev=prev)
    run_both(h2b, orc, g, parts, 3, 1, 4, 1, nq, 4, nq - 1000, nq, prev=prev)


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_random_expression_graphs(h2b, orc, cuda, seed):
    rng = random.Random(seed)
    nops = [20, 60, 150, 400][seed - 1]
    g, parts = R.random_graph(rng, nops, num_fixed=5, num_instance=2, num_advice=7, num_challenges=3)
    run_both(h2b, orc, g, parts, 5, 2, 7, 3, 1 << 11, 2, 0, 1 << 11, seed=seed)


def test_degenerate_zero_columns(h2b, orc, cuda):
    """No instance columns, no challenges, a constant-only value part."""
    g = R.Graph()
    a = g.add("store", R.vs(R.ADVICE, 0, 0))
    b = g.add("square", a)
    parts = [b, g.const(99), R.vs(R.CONST, 0)]
    run_both(h2b, orc, g, parts, 1, 0, 1, 0, 1 << 9, 1, 0, 1 << 9)


@pytest.mark.parametrize("n", [1 << 14, 1 << 20])
def test_lookup_quotient(h2b, orc, cuda, n):
    arrs = [orc.chacha_fr(10 + i, n) for i in range(8)]
    beta, gamma, y = (orc.chacha_fr(30 + i, 1) for i in range(3))
    want = orc.quotient_lookups(*arrs, beta, gamma, y)
    d = [h2b.to_dev(a) for a in arrs]
    h2b.quotient_lookups_device(*d, h2b.to_dev(beta), h2b.to_dev(gamma), h2b.to_dev(y), n)
    assert_limbs_equal(h2b.to_host(d[0]), want, "lookup quotient")


@pytest.mark.parametrize("ncols,chunk_len,n", [(4, 2, 1 << 12), (5, 2, 1 << 12), (3, 3, 1 << 12), (4, 2, 1 << 20)])
def test_permutation_quotient(h2b, orc, cuda, ncols, chunk_len, n):
    """Up to one full extended part of the k = 20 proof (2^20 rows, 4 columns in 2 sets)."""
    f = h2b.fields
    nsets = (ncols + chunk_len - 1) // chunk_len
    values = orc.chacha_fr(1, n)
    cols = [orc.chacha_fr(10 + i, n) for i in range(ncols)]
    perms = [orc.chacha_fr(20 + i, n) for i in range(ncols)]
    prods = [orc.chacha_fr(30 + i, n) for i in range(nsets)]
    l0, ll, la = (orc.chacha_fr(40 + i, n) for i in range(3))
    dom = f.EvaluationDomain(4, 10)
    y, beta, gamma = (orc.chacha_fr(50 + i, 1) for i in range(3))
    delta = f.fr_mont_limbs([f.DELTA])
    delta_start = orc.chacha_fr(60, 1)
    ext_omega = f.fr_mont_limbs([pow(dom.extended_omega, 3, f.R_MOD)])
    omega = f.fr_mont_limbs([dom.extended_omega])
    last_rotation, rot_scale = -5, 4
    want = orc.permutation_quotient(values, 0, rot_scale, n, last_rotation, chunk_len, cols, prods, perms, l0, ll, la,
                                    y, beta, gamma, delta, delta_start, ext_omega, omega)
    d_vals = h2b.to_dev(values)
    h2b.quotient_permutation_device(d_vals, h2b.to_dev(l0), h2b.to_dev(ll), h2b.to_dev(la),
                                    [h2b.to_dev(p) for p in prods], [h2b.to_dev(p) for p in perms],
                                    [h2b.to_dev(c) for c in cols], beta, gamma, y, delta, delta_start, ext_omega,
                                    omega, chunk_len, last_rotation, rot_scale, n, n)
    assert_limbs_equal(h2b.to_host(d_vals), want, "permutation quotient")


def test_compress_expressions(h2b, orc, cuda):
    """Lookup compression (compress_expressions_in_place_device,
    halo2_proofs/src/plonk/evaluation.rs:1722-1856) runs through the same
    evaluator: value parts are the lookup expressions and the Horner factor is
    theta, giving sum_i theta^(m-1-i) expr_i per row.  Checked against a direct
    Python evaluation."""
    f = h2b.fields
    p = f.R_MOD
    nq = 1 << 9
    g = R.Graph()
    e0 = g.add("store", R.vs(R.ADVICE, 0, 0))
    e1 = g.add("mul", R.vs(R.FIXED, 0, 0), R.vs(R.ADVICE, 1, 1))
    e2 = g.add("add", R.vs(R.ADVICE, 2, -1), g.const(5))
    parts = [e0, e1, e2]
    fixed = columns(orc, 500, 1, nq)
    adv = columns(orc, 600, 3, nq)
    theta = 0xABCDEF0123456789
    consts = f.fr_mont_limbs(g.constants)
    d_out = h2b.dev_empty(32 * nq)
    h2b.quotient_device([h2b.to_dev(c) for c in fixed], [], [h2b.to_dev(c) for c in adv], np.zeros((0, 4), np.uint64),
                        consts, theta, np.array(g.rules, dtype=np.uint64), np.array(parts, dtype=np.uint64), nq, 1, 0,
                        nq, d_out, None)
    got = [f.from_mont(x) for x in f.limbs_to_ints(h2b.to_host(d_out))]
    F = [[f.from_mont(x) for x in f.limbs_to_ints(c)] for c in fixed]
    A = [[f.from_mont(x) for x in f.limbs_to_ints(c)] for c in adv]
    for r in range(nq):
        ex = [A[0][r], F[0][r] * A[1][(r + 1) % nq] % p, (A[2][(r - 1) % nq] + 5) % p]
        want = (ex[0] * theta * theta + ex[1] * theta + ex[2]) % p
        assert got[r] == want, r


def test_resident_program_matches_and_replays_in_a_graph(h2b, orc, cuda):
    """h2b_quotient_program_build / _run give the bytes of
    _halo2_quotient_device_columns_device_out, with and without a prev seed,
    on a row window, and the same again when replayed from a captured graph."""
    import torch
    f = h2b.fields
    g = R.Graph()
    parts = R.plonk_and_fibonacci(g)
    nq = 1 << 12
    fixed = [h2b.to_dev(c) for c in columns(orc, 1100, 3, nq)]
    inst = [h2b.to_dev(c) for c in columns(orc, 2100, 1, nq)]
    adv = [h2b.to_dev(c) for c in columns(orc, 3100, 4, nq)]
    chal = orc.chacha_fr(4100, 1)
    consts = f.fr_mont_limbs(g.constants)
    rules = np.array(g.rules, dtype=np.uint64)
    vp = np.array(parts, dtype=np.uint64)
    y = 0xFEEDF00D
    prev = h2b.to_dev(orc.chacha_fr(77, 1000))
    want = h2b.dev_empty(32 * nq)
    h2b.quotient_device(fixed, inst, adv, chal, consts, y, rules, vp, nq, 4, 0, nq, want)
    want_w = h2b.dev_empty(32 * 1000)
    h2b.quotient_device(fixed, inst, adv, chal, consts, y, rules, vp, nq, 4, 1500, 2500, want_w, prev)
    prog = h2b.ResidentQuotient(fixed, inst, adv, chal, consts, y, rules, vp, nq, 4)
    got, got_w = h2b.dev_empty(32 * nq), h2b.dev_empty(32 * 1000)
    prog.run(got)
    prog.run(got_w, prev, 1500, 2500)
    torch.cuda.synchronize()
    assert torch.equal(got, want) and torch.equal(got_w, want_w)
    st = torch.cuda.Stream()
    graph_out = h2b.dev_empty(32 * nq)
    graph_out.zero_()
    torch.cuda.synchronize()
    gr = h2b.Graph(st)
    gr.begin()
    prog.run(graph_out, stream=st)
    gr.end()
    try:
        gr.launch(st)
        st.synchronize()
    finally:
        gr.close()
    assert torch.equal(graph_out, want)
