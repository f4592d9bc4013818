"""The prover of the config-3 circuit (halo2_proofs/src/plonk/prover.rs:140-622
issues the same device work per proof) and the serving loop around it.

A proof of a satisfying witness verifies (verify.verify_proof: the
vanishing argument at x from the opened evaluations and the SHPLONK opening
ending in the reference's pairing check) at k = 10, 16 and 20; one wrong witness cell, one
changed commitment, one changed evaluation or a wrong public input makes it
fail.  The device-synthesised witness satisfies every gate, copy and lookup
on the host.  Proofs are the same bytes alone and in a concurrent mix."""
import importlib

import numpy as np
import pytest


def _prover(h2b):
    return importlib.import_module(h2b.__name__ + ".prover")


def _mods(h2b):
    imp = lambda m: importlib.import_module(h2b.__name__ + "." + m)  # noqa: E731
    return imp("prover"), imp("circuit"), imp("verify"), imp("transcript")


def test_request_trace_is_seeded(h2b):
    P = _prover(h2b)
    a, b = P.requests(200, 50.0, 7), P.requests(200, 50.0, 7)
    assert a == b
    arr = np.array([r[0] for r in a])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    ks = np.array([r[1] for r in a])
    assert set(ks.tolist()) <= {16, 18, 20, 22}
    assert (ks == 16).sum() > (ks == 22).sum()
    assert len({r[2] for r in a}) == 200
    burst = P.requests(5, 0, 1, ks=(10,), weights=(1,))
    assert [r[0] for r in burst] == [0.0] * 5


def test_summary_percentiles(h2b):
    P = _prover(h2b)
    reqs = [(0.0, 10, 1), (0.0, 12, 2), (0.1, 10, 3), (0.2, 12, 4)]
    res = {"latency_s": np.array([0.01, 0.05, 0.02, 0.04]), "makespan_s": 0.5}
    s = P.summary(reqs, res)
    assert s["proofs_per_s"] == 8.0
    assert s["per_k"]["10"]["count"] == 2 and s["per_k"]["12"]["count"] == 2
    assert s["p50_ms"] == 30.0


def test_query_and_transcript_orders(h2b):
    """The opening's 25 queries and the 24 written evaluations name the same
    (polynomial, point) pairs, apart from h, whose evaluation the verifier
    derives, and every evaluation the expressions read is written."""
    P, C, _, _ = _mods(h2b)
    dom = h2b.fields.EvaluationDomain(C.DEGREE, 10)
    _, labels = P.open_queries_for(dom, 12345, {k: None for k in
                                                ["adv0", "adv1", "adv2", "adv3", "z0", "z1", "zl", "pa", "ps",
                                                 "fixed0", "fixed1", "fixed2", "sigma0", "sigma1", "sigma2",
                                                 "sigma3", "h", "random"]})
    order = P.transcript_eval_order(dom, 12345)
    assert len(labels) == 25 and len(order) == P.NUM_EVALS == 24
    assert set(labels) - set(order) == {("h", 12345)} and set(order) <= set(labels)
    assert len(set(labels)) == len(labels)


def _bytes(outs):
    c, e = outs[0], outs[1]
    return b"".join(t.numpy().tobytes() for t in c), b"".join(t.numpy().tobytes() for t in e)


@pytest.mark.gpu
def test_fibonacci_generator(h2b):
    F = h2b.fields
    p = F.R_MOD
    for n, s0, s1 in ((1, 5, 7), (64, 3, p - 1), (1000, 2 ** 200 + 1, 99), (4099, 11, 13)):
        got = F.fr_from_mont_limbs(h2b.to_host(h2b.fibonacci_device(s0, s1, n)))
        want = [s0 % p, s1 % p]
        while len(want) < n:
            want.append((want[-1] + want[-2]) % p)
        assert got == want[:n]


@pytest.mark.gpu
def test_gather_rows(h2b):
    """h2b_gather_fr: out[i] = table[idx[i]] for 32-byte rows; indices outside
    the table (negative, equal to or past its length) give zero rows."""
    import torch
    rng = np.random.default_rng(5)
    table = rng.integers(0, 256, (300, 32), dtype=np.uint8)
    idx = rng.integers(0, 300, 100003).astype(np.int64)
    idx[[0, 7, 99]] = [-1, 300, 1 << 40]
    out = h2b.gather_fr_device(torch.from_numpy(table).cuda(), torch.from_numpy(idx).cuda())
    want = np.zeros((idx.size, 32), np.uint8)
    ok = (idx >= 0) & (idx < 300)
    want[ok] = table[idx[ok]]
    assert np.array_equal(out.cpu().numpy().reshape(-1, 32), want)
    with pytest.raises(TypeError):
        h2b.gather_fr_device(torch.from_numpy(table).cuda(), torch.zeros(4, dtype=torch.int32, device="cuda"))


@pytest.mark.gpu
def test_synthesised_witness_satisfies_the_circuit(h2b):
    """Gates on every row, copies on every wired cell, lookup inputs inside
    the table on the usable rows, the public inputs in the instance column:
    checked with Python integers on the downloaded columns."""
    import torch
    _, C, _, _ = _mods(h2b)
    F = h2b.fields
    p, k = F.R_MOD, 9
    pk = C.ProvingKey(h2b, k)
    n, u = pk.n, pk.u
    adv, inst, public = C.synthesize(h2b, pk, 77)
    torch.cuda.synchronize()
    a, b, c, d = (F.fr_from_mont_limbs(h2b.to_host(t)) for t in adv)
    q_ar, q_fib, tab = (F.fr_from_mont_limbs(h2b.to_host(t)) for t in pk.fixed_values)
    ins = F.fr_from_mont_limbs(h2b.to_host(inst))
    for r in range(n):
        assert q_ar[r] * (C.QA * a[r] + C.QB * b[r] + C.QM * a[r] * b[r] - c[r] + C.K) % p == 0
        assert q_fib[r] * (d[(r + 2) % n] - d[(r + 1) % n] - d[r]) % p == 0
    assert sum(q_ar) == u and sum(q_fib) == u - 2
    table = set(tab[:C.TABLE_SIZE])
    assert table == set(range(C.TABLE_SIZE))
    assert all(b[r] in table for r in range(u))
    nxt, b_rows, a_rows = C.wiring(n, 0xC0FFEE)
    cols = [a, b, c, ins]
    for cell in range(4 * n):
        assert cols[cell // n][cell % n] == cols[nxt[cell] // n][nxt[cell] % n]
    assert ins[:C.NUM_PUBLIC] == public and not any(ins[C.NUM_PUBLIC:])
    assert 4 * b_rows.size >= u - 4
    # the permutation polynomials map each cell to its successor's delta^c w^r
    sig = [F.fr_from_mont_limbs(h2b.to_host(t)) for t in pk.sigma_values]
    w = pk.dom.omega
    for cell in (0, 3, n + int(b_rows[0]), int(a_rows[0]), 3 * n + 1, 2 * n + 5):
        c2, r2 = divmod(int(nxt[cell]), n)
        assert sig[cell // n][cell % n] == pow(F.DELTA, c2, p) * pow(w, r2, p) % p


@pytest.mark.gpu
def test_served_outputs_match_alone(h2b):
    import torch
    P, C, V, _ = _mods(h2b)
    res = P.Resident(h2b, 12)
    reqs = [(0.0, 12, 11), (0.0, 10, 12), (0.0, 11, 13), (0.0, 10, 14), (0.0, 12, 15)]
    alone = []
    with P.Server(res, 1, 1 << 38, transcript=True) as one:
        for r in reqs:
            alone.append(one.serve([r], keep_outputs=True)["outputs"][0])
        need12 = one.bytes_for(12)
    with P.Server(res, 3, 1 << 38, transcript=True) as srv:
        mixed = srv.serve(reqs, keep_outputs=True)["outputs"]
        again = srv.serve(reqs, keep_outputs=True)["outputs"]   # workers persist across calls
    for a, m, g in zip(alone, mixed, again):
        assert _bytes(a) == _bytes(m) == _bytes(g) and a[2] == m[2] == g[2]
    # a budget that admits one request at a time gives the same bytes too
    with P.Server(res, 3, res.device_bytes() + need12, transcript=True) as tight_srv:
        tight = tight_srv.serve(reqs, keep_outputs=True)["outputs"]
    for a, m in zip(alone, tight):
        assert a[2] == m[2]
    # every proof verifies
    for (_, k, _), out in zip(reqs, alone):
        assert V.verify_proof(res.verifying_key(k), out[3], out[2], res.verifier_params())
    c, e = _bytes(alone[0])
    assert len(c) == 96 * 15 and len(e) == 32 * P.NUM_EVALS
    assert len(alone[0][2]) == 32 * (15 + P.NUM_EVALS)
    # the first commitment is the MSM of the first advice column's coefficients over the plain SRS
    n = 1 << 12
    pk = res.key(12)
    adv, _, _ = C.synthesize(h2b, pk, 11)
    adv0_c = h2b.dev_empty(32 * n)
    h2b.fft_normal_to_device(2, 12, adv[0], adv0_c, pk.dom.omega_inv, pk.dom.ifft_divisor)
    out = h2b.dev_empty(96)
    h2b.msm_device(adv0_c, res.srs, out, n, h2b.msm_workspace(n))
    torch.cuda.synchronize()
    assert out.cpu().numpy().tobytes() == c[:96]
    assert alone[1][2] != alone[3][2]


@pytest.mark.gpu
def test_server_rejects_oversize(h2b):
    P = _prover(h2b)
    res = P.Resident(h2b, 10)
    with P.Server(res, 2, 1 << 20) as srv, pytest.raises(ValueError):
        srv.serve([(0.0, 10, 1)])


@pytest.mark.gpu
def test_keygen_commitments(h2b):
    """The verifying-key commitments equal the plain MSM of each key polynomial."""
    import torch
    P = _prover(h2b)
    res = P.Resident(h2b, 11)
    k, n = 10, 1 << 10
    vk = res.keygen(k)
    torch.cuda.synchronize()
    pk = res.key(k)
    for poly, got in zip(pk.fixed + pk.sigma, vk):
        out = h2b.dev_empty(96)
        h2b.msm_device(poly, res.srs, out, n, h2b.msm_workspace(n))
        torch.cuda.synchronize()
        assert out.cpu().numpy().tobytes() == got.cpu().numpy().tobytes()


def _prove(h2b, res, k, seed, tamper=None, check_degree=False, fused_quotient=True, merged_msm=False):
    import torch
    P = _prover(h2b)
    st = torch.cuda.Stream()
    w = P.ProofWorkload(res, k, seed, transcript=True, tamper=tamper, check_degree=check_degree,
                        fused_quotient=fused_quotient, merged_msm=merged_msm)
    commits, evals = w.run(st)
    st.synchronize()
    return w, commits, evals


@pytest.mark.gpu
def test_proof_verifies_and_rejects_changes(h2b):
    """k = 10: the proof verifies; a changed evaluation, a changed commitment,
    a wrong public input, a truncated proof or one wrong witness cell (a gate
    output, a Fibonacci cell, a wired cell) each make it fail, and a lookup
    input outside the table makes the prover refuse.  The reader recovers every commitment the device
    computed and every challenge the prover drew."""
    P, C, V, T = _mods(h2b)
    F = h2b.fields
    res = P.Resident(h2b, 11)
    k = 10
    vk = res.verifying_key(k)
    w, commits, evals = _prove(h2b, res, k, 21, check_degree=True)
    assert w.h_degree_ok
    proof, public = w.proof, w.public
    assert V.verify_proof(vk, public, proof, res.verifier_params())
    pts = [T.commitment_to_affine(c.cpu().numpy().view(np.uint64)) for c in commits]
    assert [T.decompress(proof[32 * i: 32 * i + 32]) for i in range(10)] == pts[:10]
    assert pts[9] == F.G1_GENERATOR                                   # the constant random polynomial
    # a changed evaluation (the third advice evaluation) or commitment (advice 1 -> G)
    at = 32 * 13 + 32 * 2
    bad = bytearray(proof)
    bad[at] ^= 1
    assert not V.verify_proof(vk, public, bytes(bad), res.verifier_params())
    bad = bytearray(proof)
    bad[32: 64] = T.compress(F.G1_GENERATOR)
    assert not V.verify_proof(vk, public, bytes(bad), res.verifier_params())
    assert not V.verify_proof(vk, [public[0] + 1] + public[1:], proof, res.verifier_params())
    assert not V.verify_proof(vk, public, proof[:-32], res.verifier_params())
    assert not V.verify_proof(vk, public, proof + bytes(32), res.verifier_params())
    # one wrong witness cell: the quotient is no longer a polynomial
    n = 1 << k
    one = h2b.to_dev(F.fr_mont_limbs([1]))
    big = h2b.to_dev(F.fr_mont_limbs([1000]))

    def add_one(col, row):
        def tamper(adv, inst):
            h2b.call("_halo2_poly_multiply_add", h2b.ptr(adv[col][32 * row:32 * row + 32]), h2b.ptr(one),
                     h2b.ptr(one), 1, h2b.stream_handle())
        return tamper

    def set_big(col, row):
        def tamper(adv, inst):
            adv[col][32 * row:32 * row + 32] = big
        return tamper

    nxt, b_rows, a_rows = C.wiring(n, 0xC0FFEE)
    for tamper in (add_one(C.ADV_C, 7), add_one(C.ADV_D, 100), add_one(C.ADV_B, int(b_rows[3]))):
        wt, _, _ = _prove(h2b, res, k, 21, tamper, check_degree=True)
        assert wt.h_degree_ok is False
        assert not V.verify_proof(vk, wt.public, wt.proof, res.verifier_params())
    # a lookup input outside the table: the prover refuses at the permute-sort, as the
    # reference's permute_expression_pair does (lookup/prover.rs:788-880)
    with pytest.raises(h2b.Halo2GpuError, match="not found in the table"):
        _prove(h2b, res, k, 21, set_big(C.ADV_B, 40))
    # the same seed gives the same proof
    w2, _, _ = _prove(h2b, res, k, 21)
    assert w2.proof == proof and w2.challenges == w.challenges
    # the reference's per-part launcher sequence gives the same proof bytes as the fused quotient pass
    w3, _, _ = _prove(h2b, res, k, 21, fused_quotient=False)
    assert w3.proof == proof
    # and the merged phase commitments the same bytes as separate MSMs on forked streams
    w4, _, _ = _prove(h2b, res, k, 21, merged_msm=True)
    assert w4.proof == proof


@pytest.mark.gpu
@pytest.mark.parametrize("k", [16, 20])
def test_proof_verifies_at_config_sizes(h2b, k):
    """The circuit at k = 16 and at the config-3 size k = 20: the proof of a
    satisfying witness verifies, and the grand products close (z = 1 at the
    last usable row is what the l_last constraints enforce)."""
    P, C, V, _ = _mods(h2b)
    res = P.Resident(h2b, k)
    w, _, _ = _prove(h2b, res, k, 1000 + k, check_degree=True)
    assert w.h_degree_ok, "h must have degree < 3n when every constraint holds"
    assert V.verify_proof(res.verifying_key(k), w.public, w.proof, res.verifier_params())
    if k == 20:
        w2, _, _ = _prove(h2b, res, k, 1000 + k, fused_quotient=False, merged_msm=True)
        assert w2.proof == w.proof, "fused quotient and merged MSMs must not change the proof"
    bad = bytearray(w.proof)
    bad[-32 * 3] ^= 4                                 # inside the last evaluations
    assert not V.verify_proof(res.verifying_key(k), w.public, bytes(bad), res.verifier_params())
