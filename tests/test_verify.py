"""SHPLONK's final check (halo2-gpu_b200/verify.py), in the reference's
pairing form and in the G1 (trapdoor) form, against an opening made by a
pure-Python restatement of the SHPLONK prover, all on the host: a correct
opening passes both; a changed evaluation, challenge, commitment or W'
fails both."""
import importlib
import random

from test_shplonk_gpu import _restate


def _both(V, *args):
    """The pairing and trapdoor verdicts, which must agree."""
    tr = V.shplonk_check_trapdoor(*args)
    pr = V.shplonk_check_pairing(*args)
    assert tr == pr
    return pr


def test_final_check_accepts_opening_and_rejects_changes(h2b):
    F = h2b.fields
    S = importlib.import_module(h2b.__name__ + ".shplonk")
    V = importlib.import_module(h2b.__name__ + ".verify")
    p, rng = F.R_MOD, random.Random(5)
    n, tau = 8, rng.randrange(2, p)
    polys = [[rng.randrange(p) for _ in range(n)] for _ in range(4)]
    x, w = rng.randrange(p), pow(F.ROOT_OF_UNITY, 1 << (F.S - 3), p)
    queries = [(0, x), (0, x * w % p), (1, x), (2, x), (2, x * w % p), (2, x * w * w % p), (3, x)]
    y, v, u = (rng.randrange(p) for _ in range(3))
    h, q = _restate(polys, queries, y, v, u, p, S)

    def commit(c):
        return F.g1_mul(F.G1_GENERATOR, S._eval_host(c, tau))

    cm = {i: commit(c) for i, c in enumerate(polys)}
    W, W2 = commit(h), commit(q)
    evals = [S._eval_host(polys[k], pt) for k, pt in queries]
    assert _both(V, cm, queries, evals, y, v, u, W, W2, tau)
    bad = list(evals)
    bad[4] = (bad[4] + 1) % p
    assert not _both(V, cm, queries, bad, y, v, u, W, W2, tau)
    assert not _both(V, cm, queries, evals, y, (v + 1) % p, u, W, W2, tau)
    assert not _both(V, cm, queries, evals, y, v, u, W, F.g1_add(W2, F.G1_GENERATOR), tau)
    cm2 = dict(cm)
    cm2[3] = F.g1_add(cm[3], F.G1_GENERATOR)
    assert not _both(V, cm2, queries, evals, y, v, u, W, W2, tau)


def test_final_check_rejects_an_unnormalised_w2(h2b):
    """W' must be the commitment to L(X) / ((X - u) Z_{T\\S_0}(u)), as the
    reference's prover scales it (shplonk/prover.rs:423-430): the quotient
    without the factor fails the check whenever Z_{T\\S_0}(u) != 1."""
    F = h2b.fields
    S = importlib.import_module(h2b.__name__ + ".shplonk")
    V = importlib.import_module(h2b.__name__ + ".verify")
    p, rng = F.R_MOD, random.Random(9)
    n, tau = 8, rng.randrange(2, p)
    polys = [[rng.randrange(p) for _ in range(n)] for _ in range(3)]
    x, w = rng.randrange(p), pow(F.ROOT_OF_UNITY, 1 << (F.S - 3), p)
    queries = [(0, x), (1, x), (1, x * w % p), (2, x * w % p)]
    y, v, u = (rng.randrange(p) for _ in range(3))
    h, q = _restate(polys, queries, y, v, u, p, S)
    commit = lambda c: F.g1_mul(F.G1_GENERATOR, S._eval_host(c, tau))  # noqa: E731
    cm = {i: commit(c) for i, c in enumerate(polys)}
    evals = [S._eval_host(polys[k], pt) for k, pt in queries]
    assert _both(V, cm, queries, evals, y, v, u, commit(h), commit(q), tau)
    z0_diff = S._vanishing_at([x * w % p], u)          # T \ S_0 for S_0 = {x}
    assert z0_diff != 1
    raw = [c * z0_diff % p for c in q]
    assert not _both(V, cm, queries, evals, y, v, u, commit(h), commit(raw), tau)
