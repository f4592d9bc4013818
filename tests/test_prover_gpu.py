"""Prover-shaped workload and the serving loop (halo2_proofs/src/plonk/prover.rs:56-482
issues the same device work per proof).  The workload's outputs are deterministic
GPU work, so a request served alone and in a mix of concurrent requests of other
sizes must give the same bytes; its first commitment must equal the plain MSM."""
import importlib

import numpy as np
import pytest


def _prover(h2b):
    return importlib.import_module(h2b.__name__ + ".prover")


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


def _bytes(outs):
    c, e = outs
    return b"".join(t.numpy().tobytes() for t in c), b"".join(t.numpy().tobytes() for t in e)


@pytest.mark.gpu
def test_served_outputs_match_alone(h2b):
    import torch
    P = _prover(h2b)
    res = P.Resident(h2b, 12)
    reqs = [(0.0, 12, 11), (0.0, 10, 12), (0.0, 11, 13), (0.0, 10, 14), (0.0, 12, 15)]
    alone = []
    with P.Server(res, 1, 1 << 36) as one:
        for r in reqs:
            alone.append(_bytes(one.serve([r], keep_outputs=True)["outputs"][0]))
        need12 = one.bytes_for(12)
    with P.Server(res, 3, 1 << 36) as srv:
        mixed = srv.serve(reqs, keep_outputs=True)["outputs"]
        again = srv.serve(reqs, keep_outputs=True)["outputs"]   # workers persist across calls
    for a, m, g in zip(alone, mixed, again):
        assert a == _bytes(m) == _bytes(g)
    # a budget that admits one request at a time gives the same bytes too
    with P.Server(res, 3, need12) as tight_srv:
        tight = tight_srv.serve(reqs, keep_outputs=True)["outputs"]
    for a, m in zip(alone, tight):
        assert a == _bytes(m)
    # each request's outputs: 4 advice + A' + S' + 2 z + lookup z + the vanishing argument's
    # random polynomial + 3 h pieces + the 2 SHPLONK commitments, and the 29 opened evaluations
    c, e = alone[0]
    assert len(c) == 96 * 15 and len(e) == 32 * 29
    # the first commitment is the MSM of the advice column's coefficient form over the plain SRS
    n = 1 << 12
    adv0 = h2b.random_fr_device(n, 11 * 64, 1)
    dom = h2b.fields.EvaluationDomain(4, 12)
    adv0_c = h2b.dev_empty(32 * n)
    h2b.fft_normal_to_device(2, 12, adv0, adv0_c, dom.omega_inv, dom.ifft_divisor)
    out = h2b.dev_empty(96)
    h2b.msm_device(adv0_c, res.srs, out, n, h2b.msm_workspace(n))
    torch.cuda.synchronize()
    assert out.cpu().numpy().tobytes() == c[:96]
    # distinct seeds give distinct outputs
    assert alone[1] != alone[3]


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
    for poly, got in zip(pk["fixed"] + pk["sigma"], vk):
        out = h2b.dev_empty(96)
        h2b.msm_device(poly, res.srs, out, n, h2b.msm_workspace(n))
        torch.cuda.synchronize()
        assert out.cpu().numpy().tobytes() == got.cpu().numpy().tobytes()


@pytest.mark.gpu
def test_transcript_proof_replays(h2b):
    """With the Fiat-Shamir transcript, the proof bytes are the same alone and
    in a concurrent mix, and a reader that replays them (verifying-key scalar,
    public rows, then the proof in the prover's order) recovers every
    commitment the device computed, every evaluation, and every challenge."""
    import torch
    P = _prover(h2b)
    T = importlib.import_module(h2b.__name__ + ".transcript")
    F = h2b.fields
    res = P.Resident(h2b, 11)
    reqs = [(0.0, 10, 21), (0.0, 11, 22), (0.0, 10, 23)]
    with P.Server(res, 1, 1 << 36, transcript=True) as one:
        alone = [one.serve([r], keep_outputs=True)["outputs"][0] for r in reqs]
    with P.Server(res, 3, 1 << 36, transcript=True) as srv:
        mixed = srv.serve(reqs, keep_outputs=True)["outputs"]
    for a, m in zip(alone, mixed):
        assert a[2] == m[2] and _bytes(a[:2]) == _bytes(m[:2])
    assert alone[0][2] != alone[2][2]

    st = torch.cuda.Stream()
    w = P.ProofWorkload(res, 10, 21, transcript=True)
    commits, evals = w.run(st)
    st.synchronize()
    proof = w.proof
    assert proof == alone[0][2] and len(proof) == 32 * (15 + 29)
    r = T.Blake2bRead(proof)
    r.common_scalar(res.vk_repr(10))
    inst = h2b.random_fr_device(1 << 10, 21 * 64 + 4, 0)
    for v in F.fr_from_mont_limbs(h2b.to_host(inst[: 32 * P.NUM_PUBLIC])):
        r.common_scalar(int(v))
    pts, ch = [], []

    def points(m):
        pts.extend(r.read_point() for _ in range(m))

    points(4)                                                # advice
    ch.append(r.squeeze_challenge())                         # theta
    points(2)                                                # A', S'
    ch += [r.squeeze_challenge(), r.squeeze_challenge()]     # beta, gamma
    points(4)                                                # 2 z, lookup z, random polynomial
    ch.append(r.squeeze_challenge())                         # y
    points(3)                                                # h pieces
    ch.append(r.squeeze_challenge())                         # x
    ev = [r.read_scalar() for _ in range(29)]
    ch += [r.squeeze_challenge(), r.squeeze_challenge()]     # SHPLONK y, v
    points(1)                                                # W
    ch.append(r.squeeze_challenge())                         # u
    points(1)                                                # W'
    assert r.remaining() == 0
    assert ch == w.challenges
    assert pts == [T.commitment_to_affine(c.cpu().numpy().view(np.uint64)) for c in commits]
    assert ev == F.fr_from_mont_limbs(evals[0].numpy().view(np.uint64).reshape(-1, 4))
    # the opening verifies: F == (tau - u) W' with the SRS trapdoor (the G1
    # form of SHPLONK's pairing check); a changed evaluation breaks it
    V = importlib.import_module(h2b.__name__ + ".verify")
    vk = res.keygen(10)
    torch.cuda.synchronize()
    cm = dict(zip(P.COMMIT_LABELS, pts))
    cm.update({f"vk{i}": T.commitment_to_affine(c.cpu().numpy().view(np.uint64)) for i, c in enumerate(vk)})
    x = ch[4]
    assert w.query_labels[0] == ("adv0", x) and len(w.query_labels) == 29
    sy, sv, su = ch[5], ch[6], ch[7]
    assert V.shplonk_check_trapdoor(cm, w.query_labels, ev, sy, sv, su, cm["W"], cm["W2"], res.tau)
    bad = list(ev)
    bad[3] = (bad[3] + 1) % F.R_MOD
    assert not V.shplonk_check_trapdoor(cm, w.query_labels, bad, sy, sv, su, cm["W"], cm["W2"], res.tau)
    assert not V.shplonk_check_trapdoor(cm, w.query_labels, ev, sy, sv, (su + 1) % F.R_MOD, cm["W"], cm["W2"],
                                        res.tau)
    # advice commitments do not depend on challenges; the grand products do
    c0, _ = P.ProofWorkload(res, 10, 21).run(st)
    st.synchronize()
    assert all(torch.equal(a.cpu(), b.cpu()) for a, b in zip(c0[:4], commits[:4]))
    assert not torch.equal(c0[6].cpu(), commits[6].cpu())
