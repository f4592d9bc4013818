"""End-to-end quotient identity over the whole device path of `create_proof`'s
phases 2-4 (halo2_proofs/src/plonk/prover.rs:56-482; evaluate_h,
halo2_proofs/src/plonk/evaluation.rs:1056-1417).

A config-3-shaped circuit (4 advice columns under a 2-set copy permutation,
a lookup column, an instance column; gates q_a a + q_b b + q_m a b - q_c c,
q_fib (d(w^2 X) - d(w X) - d(X)) and q_inst (a(w^-1 X) - inst(w^-1 X))) gets
a satisfying witness built on the host with blinding rows as the reference
lays them out.  Everything after that runs through this library: the lookup
permute-sort, the permutation and lookup products and their grand products,
lagrange_to_coeff, the four coset parts, the gate / permutation / lookup
quotients, the gather of the parts, the division by the vanishing polynomial
and extended_to_coeff.  When every constraint holds on the whole domain,
h = sum_i y^i C_i / Z_H is a polynomial of degree < 3n, so the top n of its
4n coefficients are exactly zero; a single wrong witness cell breaks that.
"""
import importlib
import random

import numpy as np
import pytest

B = 5            # blinding factors: rows u + 1 .. n - 1 are random, row u = n - B - 1 is l_last


def _gates(R):
    g = R.Graph()
    FX, AD, IN = R.FIXED, R.ADVICE, R.INSTANCE
    a, b, c = (g.add("store", R.vs(AD, i, 0)) for i in range(3))
    t1 = g.add("mul", a, R.vs(FX, 0))
    t2 = g.add("mul", b, R.vs(FX, 1))
    t3 = g.add("mul", g.add("mul", a, b), R.vs(FX, 2))
    t4 = g.add("mul", c, R.vs(FX, 3))
    g1 = g.add("sub", g.add("add", g.add("add", t1, t2), t3), t4)
    f = g.add("sub", g.add("sub", R.vs(AD, 3, 2), R.vs(AD, 3, 1)), R.vs(AD, 3, 0))
    g2 = g.add("mul", f, R.vs(FX, 4))
    g3 = g.add("mul", g.add("sub", R.vs(AD, 0, -1), R.vs(IN, 0, -1)), R.vs(FX, 5))
    return g, [g1, g2, g3]


def _witness(F, k, seed, break_cell=None):
    """Host witness and fixed columns (plain ints) for the circuit above."""
    p = F.R_MOD
    rng = random.Random(seed)
    n = 1 << k
    u = n - B - 1
    rnd = lambda: rng.randrange(p)  # noqa: E731
    qa, qb, qm, qc, qf, qi = ([0] * n for _ in range(6))
    a, b, c, d, e = ([rnd() for _ in range(n)] for _ in range(5))
    inst = [0] * n
    table = [rnd() for _ in range(256)]
    tcol = table + [table[0]] * (n - 256)
    # copy constraints: a quarter of the usable b cells equal some a cell
    parent = {}

    def find(x):
        while parent.get(x, x) != x:
            x = parent[x]
        return x

    for r in rng.sample(range(u), u // 4):
        j = rng.randrange(u)
        b[r] = a[j]
        ra, rb = find((0, j)), find((1, r))
        if ra != rb:
            parent[rb] = ra
    for r in range(u):
        qa[r], qb[r], qm[r], qc[r] = rnd(), rnd(), rnd(), 1
        c[r] = (qa[r] * a[r] + qb[r] * b[r] + qm[r] * a[r] * b[r]) % p
    d[0], d[1] = rnd(), rnd()
    for r in range(2, u):
        d[r] = (d[r - 1] + d[r - 2]) % p
    for r in range(u - 2):
        qf[r] = 1
    for r in range(u):
        inst[r] = a[r]
    for r in range(1, u + 1):
        qi[r] = 1
    for r in range(u):
        e[r] = table[rng.randrange(256)]
    if break_cell is not None:
        col, row = break_cell
        {"c": c, "d": d, "b": b}[col][row] = (({"c": c, "d": d, "b": b}[col][row]) + 1) % p
    # sigma: each cycle of equal cells maps a cell to the next one; the rest map to themselves
    dom = F.EvaluationDomain(4, k)
    w = dom.omega
    groups = {}
    for cell in list(parent.keys()) + list(parent.values()):
        groups.setdefault(find(cell), set()).add(cell)
    sigma = [[pow(F.DELTA, col, p) * pow(w, row, p) % p for row in range(n)] for col in range(4)]
    for cells in groups.values():
        cyc = sorted(cells)
        for i, (col, row) in enumerate(cyc):
            ncol, nrow = cyc[(i + 1) % len(cyc)]
            sigma[col][row] = pow(F.DELTA, ncol, p) * pow(w, nrow, p) % p
    l0 = [1] + [0] * (n - 1)
    llast = [0] * n
    llast[u] = 1
    lact = [1] * u + [0] * (n - u)
    return dict(n=n, u=u, fixed=[qa, qb, qm, qc, qf, qi], advice=[a, b, c, d, e], inst=inst, table=tcol,
                sigma=sigma, l=[l0, llast, lact], rng=rng, dom=dom)


def _run(h2b, k, seed, break_cell=None):
    import torch
    F = h2b.fields
    R = importlib.import_module(h2b.__name__ + ".rules")
    p = F.R_MOD
    W = _witness(F, k, seed, break_cell)
    n, u, rng, dom = W["n"], W["u"], W["rng"], W["dom"]
    up = lambda vals: h2b.to_dev(F.fr_mont_limbs([v % p for v in vals]))  # noqa: E731
    down = lambda t: F.fr_from_mont_limbs(h2b.to_host(t))  # noqa: E731
    blind = lambda t, start: t.__setitem__(slice(32 * start, 32 * n),  # noqa: E731
                                           up([rng.randrange(p) for _ in range(n - start)]))
    fixed = [up(c) for c in W["fixed"]]
    adv = [up(c) for c in W["advice"]]
    inst = up(W["inst"])
    sig = [up(c) for c in W["sigma"]]
    lag = [up(c) for c in W["l"]]
    tab = up(W["table"])
    beta, gamma, y = (rng.randrange(1, p) for _ in range(3))
    sc = lambda v: F.fr_mont_limbs([v % p])  # noqa: E731
    d_beta, d_gamma, d_y, d_one = (h2b.to_dev(sc(v)) for v in (beta, gamma, y, 1))
    # lookup: permute-sort of the usable rows, blinded tails
    pa, ps = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
    h2b.permute_expression_pair_device(adv[4], tab, pa, ps, n, u)
    blind(pa, u)
    blind(ps, u)
    # permutation grand products, 2 sets of 2 columns; z_s[0] = carry, z_s[u + 1 ..] blinds
    d_delta, d_om = h2b.to_dev(sc(F.DELTA)), h2b.to_dev(sc(dom.omega))
    d_dw = h2b.to_dev(sc(1))
    zs, carry = [], 1
    for s in range(2):
        mod = h2b.dev_empty(32 * n)
        h2b.call("_halo2_poly_fill_one", h2b.ptr(mod), n, h2b.stream_handle())
        h2b.permutation_product_device(mod, sig[2 * s: 2 * s + 2], adv[2 * s: 2 * s + 2], d_beta, d_gamma, d_delta,
                                       d_om, d_dw, u)
        z = h2b.dev_empty(32 * n)
        z[:32] = up([carry])
        z[32: 32 * (u + 1)] = mod[: 32 * u]
        h2b.grand_product_device(z, h2b.to_dev(sc(carry)), u, offset=1)
        carry = down(z[32 * u: 32 * (u + 1)])[0]
        blind(z, u + 1)
        zs.append(z)
    z_perm_end = carry
    # lookup grand product
    zl = h2b.dev_empty(32 * n)
    ratio = h2b.dev_empty(32 * n)
    h2b.lookup_product_device(ratio, pa, ps, adv[4], tab, d_beta, d_gamma, u)
    zl[:32] = up([1])
    zl[32: 32 * (u + 1)] = ratio[: 32 * u]
    h2b.grand_product_device(zl, d_one, u, offset=1)
    z_look_end = down(zl[32 * u: 32 * (u + 1)])[0]
    blind(zl, u + 1)
    # lagrange_to_coeff of every column
    cols = fixed + adv + [inst] + sig + lag + [tab, pa, ps] + zs + [zl]
    coef = [h2b.dev_empty(32 * n) for _ in cols]
    h2b.fft_many_to_device(2, k, k, cols, coef, dom.omega_inv, dom.ifft_divisor)
    NF, NA = 6, 5
    iF, iA, iI, iS, iL = 0, NF, NF + NA, NF + NA + 1, NF + NA + 5
    iT, iPA, iPS, iZ, iZL = iL + 3, iL + 4, iL + 5, iL + 6, iL + 8
    g, vp = _gates(R)
    rules, vp = np.array(g.rules, dtype=np.uint64), np.array(vp, dtype=np.uint64)
    consts = F.fr_mont_limbs(g.constants)
    parts_n = 1 << (dom.extended_k - k)
    hs = [h2b.dev_empty(32 * n) for _ in range(parts_n)]
    parts = [h2b.dev_empty(32 * n) for _ in coef]
    for j in range(parts_n):
        shift = pow(dom.extended_omega, j, p)
        h2b.fft_many_to_device(6, k, k, coef, parts, dom.omega, F.ZETA * shift % p)
        h2b.quotient_device(parts[iF:iF + NF], [parts[iI]], parts[iA:iA + NA], [], consts, y, rules, vp, n, 1, 0, n,
                            hs[j])
        h2b.quotient_permutation_device(hs[j], parts[iL], parts[iL + 1], parts[iL + 2], parts[iZ:iZ + 2],
                                        parts[iS:iS + 4], parts[iA:iA + 4], beta, gamma, y, sc(F.DELTA),
                                        sc(beta * F.ZETA), sc(shift), sc(dom.omega), 2, -(B + 1), 1, n, n)
        ev, tv = down(parts[iA + 4]), down(parts[iT])
        tvals = up([(x + beta) * (t + gamma) for x, t in zip(ev, tv)])
        h2b.quotient_lookups_device(hs[j], tvals, parts[iZL], parts[iPA], parts[iPS], parts[iL], parts[iL + 1],
                                    parts[iL + 2], d_beta, d_gamma, d_y, n)
    ext = h2b.dev_empty(32 * parts_n * n)
    ptab = h2b.to_dev(np.array([t.data_ptr() for t in hs], dtype=np.uint64))
    sh = h2b.stream_handle()
    h2b.call("_halo2_extended_from_lagrange_vec_device", h2b.ptr(ext), h2b.ptr(ptab), parts_n, n, sh)
    h2b.call("_halo2_divide_by_vanishing_poly", h2b.ptr(ext), h2b.ptr(up(dom.t_evaluations)),
             len(dom.t_evaluations), parts_n * n, sh)
    hc = h2b.dev_empty(32 * parts_n * n)
    h2b.fft_many_to_device(2, dom.extended_k, dom.extended_k, [ext], [hc], dom.extended_omega_inv,
                           dom.extended_ifft_divisor)
    h2b.call("_halo2_distribute_powers_zeta", h2b.ptr(hc), h2b.ptr(up([dom.g_coset_inv, dom.g_coset])), 2,
             parts_n * n, sh)
    torch.cuda.synchronize()
    return down(hc), z_perm_end, z_look_end, n


@pytest.mark.gpu
@pytest.mark.parametrize("k,seed", [(10, 1), (11, 2)])
def test_quotient_identity_holds(h2b, k, seed):
    h, z_perm, z_look, n = _run(h2b, k, seed)
    assert z_perm == 1 and z_look == 1, "grand products must telescope to 1 at row u"
    assert all(v == 0 for v in h[3 * n:]), "h must have degree < 3n when every constraint holds"
    assert any(v != 0 for v in h[:3 * n])


@pytest.mark.gpu
@pytest.mark.parametrize("cell", [("c", 7), ("d", 100), ("b", 3)])
def test_quotient_identity_detects_a_wrong_cell(h2b, cell):
    h, _, _, n = _run(h2b, 10, 1, break_cell=cell)
    assert any(v != 0 for v in h[3 * n:])


def test_witness_satisfies_gates_on_host(h2b):
    """The host witness itself: every gate vanishes on every row (checked with
    plain integers), so a failing GPU identity points at the device path."""
    F = h2b.fields
    p = F.R_MOD
    W = _witness(F, 9, 3)
    n = W["n"]
    qa, qb, qm, qc, qf, qi = W["fixed"]
    a, b, c, d, _ = W["advice"]
    inst = W["inst"]
    for r in range(n):
        assert (qa[r] * a[r] + qb[r] * b[r] + qm[r] * a[r] * b[r] - qc[r] * c[r]) % p == 0
        assert qf[r] * (d[(r + 2) % n] - d[(r + 1) % n] - d[r]) % p == 0
        assert qi[r] * (a[(r - 1) % n] - inst[(r - 1) % n]) % p == 0
