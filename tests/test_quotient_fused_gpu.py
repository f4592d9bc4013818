"""The fused extended-part quotient (h2b_quotient_fused) against the oracle's
composition of the reference's per-part launchers: the gate evaluator
(o_quotient, quotient.h:57-303), then the permutation constraints
(o_permutation_quotient, permutation_quotient.cu:23-93), then per lookup its
product expression (o_quotient) and its five constraints (o_quotient_lookups,
quotient_lookups.cu:16-53) -- the per-part sequence of
halo2_proofs/src/plonk/evaluation.rs:1107-1417.  Bit-exact, on the config-3
shape up to a full 2^20-row part, on random graphs with several sets and
lookups, on row windows, and with the interleaved, vanishing-divided output."""
import importlib
import random

import numpy as np
import pytest

from conftest import assert_limbs_equal
import rules as R

pytestmark = pytest.mark.gpu


def _circuit(h2b):
    return importlib.import_module(h2b.__name__ + ".circuit")


def make_case(h2b, orc, n, gates, lookups, nf, ni, na, ncols, chunk_len, seed):
    """Random columns and scalars for one part; `gates` is (challenges, consts,
    rules, parts), each lookup (challenges, consts, rules, parts)."""
    f = h2b.fields
    rng = random.Random(seed)
    p = f.R_MOD
    cols = {
        "fixed": [orc.chacha_fr(100 * seed + i, n) for i in range(nf)],
        "inst": [orc.chacha_fr(100 * seed + 20 + i, n) for i in range(ni)],
        "adv": [orc.chacha_fr(100 * seed + 40 + i, n) for i in range(na)],
    }
    nsets = (ncols + chunk_len - 1) // chunk_len if ncols else 0
    perm = None
    if nsets:
        dom = f.EvaluationDomain(4, 10)
        perm = {
            "prods": [orc.chacha_fr(100 * seed + 60 + i, n) for i in range(nsets)],
            "sigmas": [orc.chacha_fr(100 * seed + 70 + i, n) for i in range(ncols)],
            "beta": rng.randrange(p), "gamma": rng.randrange(p), "delta": f.DELTA,
            "delta_start": rng.randrange(p), "ext_omega": pow(dom.extended_omega, 3, p),
            "omega": dom.extended_omega, "chunk_len": chunk_len,
        }
    lk = []
    for i, graph in enumerate(lookups):
        lk.append({"rules": graph, "z": orc.chacha_fr(100 * seed + 80 + 3 * i, n),
                   "pin": orc.chacha_fr(100 * seed + 81 + 3 * i, n), "ptab": orc.chacha_fr(100 * seed + 82 + 3 * i, n),
                   "beta": rng.randrange(p), "gamma": rng.randrange(p)})
    lag = [orc.chacha_fr(100 * seed + 95 + i, n) for i in range(3)]
    return cols, perm, lk, lag, rng.randrange(p)


def oracle_chain(h2b, orc, n, cols, gates, perm, pcols, lk, lag, y, rot_scale, prot, last_rotation):
    f = h2b.fields
    m = lambda v: f.fr_mont_limbs([v])  # noqa: E731
    ec = f.fr_mont_limbs([0, 1, f.R_MOD - 1, 2, y])

    def run(graph):
        ch, cs, rules, parts = graph
        return orc.quotient(cols["fixed"], cols["inst"], cols["adv"], ch if len(ch) else np.zeros((1, 4), np.uint64),
                            cs, ec, rules, parts, n, rot_scale, 0, n, None)

    v = run(gates)
    if perm is not None:
        v = orc.permutation_quotient(v, 0, prot, n, last_rotation, perm["chunk_len"], pcols, perm["prods"],
                                     perm["sigmas"], *lag, m(y), m(perm["beta"]), m(perm["gamma"]), m(perm["delta"]),
                                     m(perm["delta_start"]), m(perm["ext_omega"]), m(perm["omega"]))
    for L in lk:
        tv = run(L["rules"])
        v = orc.quotient_lookups(v, tv, L["z"], L["pin"], L["ptab"], *lag, m(L["beta"]), m(L["gamma"]), m(y))
    return v


def fused(h2b, n, cols, gates, perm, pcol_idx, lk, lag, y, rot_scale, prot, last_rotation, row_start=0, row_end=None,
          out_stride=1, out_offset=0, scale=None, d_out=None, stream=None):
    """Uploads the case and runs h2b_quotient_fused; returns (d_out, device copies)."""
    row_end = n if row_end is None else row_end
    dv = {k: [h2b.to_dev(c) for c in v] for k, v in cols.items()}
    allc = dv["fixed"] + dv["inst"] + dv["adv"]
    d_perm = None
    if perm is not None:
        d_perm = dict(perm)
        d_perm["prods"] = [h2b.to_dev(c) for c in perm["prods"]]
        d_perm["sigmas"] = [h2b.to_dev(c) for c in perm["sigmas"]]
        d_perm["cols"] = [allc[i] for i in pcol_idx]
        d_perm.update(last_rotation=last_rotation, rot_scale=prot, isize=n)
    d_lk = [dict(L, z=h2b.to_dev(L["z"]), pin=h2b.to_dev(L["pin"]), ptab=h2b.to_dev(L["ptab"])) for L in lk]
    d_lag = [h2b.to_dev(c) for c in lag]
    if d_out is None:
        d_out = h2b.dev_empty(32 * (row_end - row_start) * out_stride)
    h2b.quotient_fused_device(dv["fixed"], dv["inst"], dv["adv"], gates, y, *d_lag, d_perm, d_lk, n, rot_scale,
                              row_start, row_end, d_out, out_stride, out_offset, scale, stream)
    return d_out, (dv, d_perm, d_lk, d_lag)


def config3(h2b, orc, n, seed):
    C = _circuit(h2b)
    g_rules, g_parts, g_consts = C.gate_graph()
    l_rules, l_parts, l_consts = C.lookup_product_graph()
    gates = (np.zeros((0, 4), np.uint64), g_consts, g_rules, g_parts)
    cols, perm, lk, lag, y = make_case(h2b, orc, n, gates, [None], 3, 1, 4, 4, C.CHUNK_LEN, seed)
    f = h2b.fields
    # the lookup expression takes beta and gamma as its challenges 0 and 1, as in the prover
    lk[0]["rules"] = (f.fr_mont_limbs([lk[0]["beta"], lk[0]["gamma"]]), l_consts, l_rules, l_parts)
    # permutation columns a, b, c, instance: column table order is fixed (3), instance (1), advice (4)
    pcol_idx = [4, 5, 6, 3]
    pcols = [cols["adv"][0], cols["adv"][1], cols["adv"][2], cols["inst"][0]]
    return gates, cols, perm, lk, lag, y, pcol_idx, pcols, -(C.BLINDING_FACTORS + 1)


@pytest.mark.parametrize("log_n", [12, 16, 20])
def test_config3_part_matches_the_launcher_chain(h2b, orc, cuda, log_n):
    """Gates, the 2-set copy permutation and the range lookup of the config-3
    circuit on one extended part (rotation scale 1), up to the full 2^20 rows."""
    n = 1 << log_n
    gates, cols, perm, lk, lag, y, pcol_idx, pcols, last = config3(h2b, orc, n, 7)
    want = oracle_chain(h2b, orc, n, cols, gates, perm, pcols, lk, lag, y, 1, 1, last)
    got, _ = fused(h2b, n, cols, gates, perm, pcol_idx, lk, lag, y, 1, 1, last)
    assert_limbs_equal(h2b.to_host(got), want, f"fused quotient 2^{log_n}")


def test_interleaved_divided_output_equals_gather_and_division(h2b, orc, cuda):
    """out_stride = 4 parts, out_offset = the part, scale = 1/t[part]: the
    part's slice of _halo2_extended_from_lagrange_vec_device followed by
    _halo2_divide_by_vanishing_poly."""
    f = h2b.fields
    p = f.R_MOD
    n, parts = 1 << 12, 4
    rng = random.Random(3)
    t_inv = [rng.randrange(1, p) for _ in range(parts)]
    ext = h2b.dev_empty(32 * n * parts)
    outs = []
    for j in range(parts):
        gates, cols, perm, lk, lag, y, pcol_idx, pcols, last = config3(h2b, orc, n, 20 + j)
        want = oracle_chain(h2b, orc, n, cols, gates, perm, pcols, lk, lag, y, 1, 1, last)
        outs.append(h2b.to_dev(want))
        fused(h2b, n, cols, gates, perm, pcol_idx, lk, lag, y, 1, 1, last, out_stride=parts, out_offset=j,
              scale=t_inv[j], d_out=ext)
    want_ext = h2b.dev_empty(32 * n * parts)
    tab = h2b.to_dev(np.array([t.data_ptr() for t in outs], dtype=np.uint64))
    h2b.call("_halo2_extended_from_lagrange_vec_device", h2b.ptr(want_ext), h2b.ptr(tab), parts, n, None)
    t_dev = h2b.to_dev(f.fr_mont_limbs(t_inv))
    h2b.call("_halo2_divide_by_vanishing_poly", h2b.ptr(want_ext), h2b.ptr(t_dev), parts, n * parts, None)
    cuda.cuda.synchronize()
    assert cuda.equal(ext, want_ext)


@pytest.mark.parametrize("seed", [1, 2])
def test_random_graphs_sets_lookups_and_windows(h2b, orc, cuda, seed):
    """A random gate graph with challenges, 5 permutation columns in 3 sets,
    two lookups with their own constants and challenges, rotation scale 4 and
    last rotation -5; the full range and two row windows (one wrapping)."""
    rng = random.Random(seed)
    f = h2b.fields
    n = 1 << 12
    g, parts = R.random_graph(rng, [40, 120][seed - 1], num_fixed=3, num_instance=1, num_advice=5, num_challenges=2)
    gates = (orc.chacha_fr(900 + seed, 2), f.fr_mont_limbs(g.constants), np.array(g.rules, np.uint64),
             np.array(parts, np.uint64))
    look = []
    for i in range(2):
        lg = R.Graph()
        x = lg.add("add", lg.add("mul", R.vs(R.ADVICE, i, 0), lg.const(3 + i)), R.vs(R.CHAL, 0))
        t = lg.add("add", R.vs(R.FIXED, i, 1), R.vs(R.CHAL, 1))
        prod = lg.add("mul", x, t)
        look.append((orc.chacha_fr(950 + 2 * seed + i, 2), f.fr_mont_limbs(lg.constants),
                     np.array(lg.rules, np.uint64), np.array([prod], np.uint64)))
    cols, perm, lk, lag, y = make_case(h2b, orc, n, gates, look, 3, 1, 5, 5, 2, 30 + seed)
    for L, gr in zip(lk, look):
        L["rules"] = gr
    pcol_idx = [4, 5, 0, 3, 8]
    allc = cols["fixed"] + cols["inst"] + cols["adv"]
    pcols = [allc[i] for i in pcol_idx]
    want = oracle_chain(h2b, orc, n, cols, gates, perm, pcols, lk, lag, y, 4, 4, -5)
    got, _ = fused(h2b, n, cols, gates, perm, pcol_idx, lk, lag, y, 4, 4, -5)
    assert_limbs_equal(h2b.to_host(got), want, "fused quotient")
    for a, b in ((1500, 2500), (n - 700, n)):
        got, _ = fused(h2b, n, cols, gates, perm, pcol_idx, lk, lag, y, 4, 4, -5, row_start=a, row_end=b)
        assert_limbs_equal(h2b.to_host(got), want[a:b], f"fused quotient rows [{a}, {b})")


def test_gates_only_and_no_lookups(h2b, orc, cuda):
    """Without a permutation and lookups it is the gate evaluator alone."""
    n = 1 << 11
    gates, cols, perm, lk, lag, y, pcol_idx, pcols, last = config3(h2b, orc, n, 5)
    want = oracle_chain(h2b, orc, n, cols, gates, None, [], [], lag, y, 1, 1, last)
    got, _ = fused(h2b, n, cols, gates, None, [], [], lag, y, 1, 1, last)
    assert_limbs_equal(h2b.to_host(got), want, "gates only")


def test_register_budgets_agree_and_graph_replay(h2b, orc, cuda):
    """3, 4 and 5 blocks per SM give the same bytes; a captured launch replays them."""
    torch = cuda
    L = h2b.lib()
    n = 1 << 14
    gates, cols, perm, lk, lag, y, pcol_idx, pcols, last = config3(h2b, orc, n, 9)
    prev = L.h2b_quotient_fused_get_blocks()
    try:
        L.h2b_quotient_fused_set_blocks(3)
        a, _ = fused(h2b, n, cols, gates, perm, pcol_idx, lk, lag, y, 1, 1, last)
        for blocks in (4, 5):
            L.h2b_quotient_fused_set_blocks(blocks)
            assert L.h2b_quotient_fused_get_blocks() == blocks
            b, _ = fused(h2b, n, cols, gates, perm, pcol_idx, lk, lag, y, 1, 1, last)
            torch.cuda.synchronize()
            assert torch.equal(a, b), blocks
    finally:
        L.h2b_quotient_fused_set_blocks(prev)
    st = torch.cuda.Stream()
    out = h2b.dev_empty(32 * n)
    with torch.cuda.stream(st):
        _, keep = fused(h2b, n, cols, gates, perm, pcol_idx, lk, lag, y, 1, 1, last, d_out=out, stream=st)
        st.synchronize()
        out.zero_()
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr, stream=st):
            dv, d_perm, d_lk, d_lag = keep
            h2b.quotient_fused_device(dv["fixed"], dv["inst"], dv["adv"], gates, y, *d_lag, d_perm, d_lk, n, 1, 0,
                                      n, out, 1, 0, None, st)
        gr.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, a)


def test_limits_and_bad_arguments(h2b, orc, cuda):
    n = 1 << 10
    gates, cols, perm, lk, lag, y, pcol_idx, pcols, last = config3(h2b, orc, n, 11)
    with pytest.raises(h2b.Halo2GpuError, match="more than 8 lookups"):
        fused(h2b, n, cols, gates, perm, pcol_idx, lk * 9, lag, y, 1, 1, last)
    rng = random.Random(5)
    g, parts = R.random_graph(rng, 400, num_fixed=3, num_instance=1, num_advice=4, num_challenges=0)
    big = (np.zeros((0, 4), np.uint64), h2b.fields.fr_mont_limbs(g.constants), np.array(g.rules, np.uint64),
           np.array(parts, np.uint64))
    with pytest.raises(h2b.Halo2GpuError, match="parameter block"):
        fused(h2b, n, cols, big, perm, pcol_idx, lk, lag, y, 1, 1, last)
    with pytest.raises(h2b.Halo2GpuError, match="row range"):
        fused(h2b, n, cols, gates, perm, pcol_idx, lk, lag, y, 1, 1, last, row_start=10, row_end=n + 1)
    bad = dict(perm, chunk_len=1)
    with pytest.raises(h2b.Halo2GpuError, match="permutation shape"):
        fused(h2b, n, cols, gates, bad, pcol_idx, lk, lag, y, 1, 1, last)
