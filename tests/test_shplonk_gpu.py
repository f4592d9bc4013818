"""SHPLONK opening over the device entry points (halo2-gpu_b200/shplonk.py;
the flow of halo2_proofs/src/poly/kzg/multiopen/shplonk/prover.rs:97-466):
evaluations against Python integers, L(u) = 0, and both commitments against a
pure-Python restatement of the opening committed by the oracle's MSM."""
import importlib
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mod():
    return importlib.import_module("halo2_gpu_b200.shplonk")


def _synth_div(coeffs, s, p):
    """(a(X) - a(s)) / (X - s), low coefficients first."""
    n = len(coeffs)
    q = [0] * (n - 1)
    acc = 0
    for i in range(n - 1, 0, -1):
        acc = (acc * s + coeffs[i]) % p
        q[i - 1] = acc
    return q + [0]


def _restate(polys, queries, y, v, u, p, S):
    """Host SHPLONK: returns h and h' coefficient lists, h' normalised by
    1 / Z_{T\\S_0}(u) as the reference's prover does (prover.rs:423-430)."""
    pe = {}
    for k, x in queries:
        pe.setdefault(k, {})[x] = S._eval_host(polys[k], x)
    sets = {}
    for k, d in pe.items():
        sets.setdefault(tuple(sorted(d)), []).append(k)
    n = len(polys[0])
    sup = sorted({x for s in sets for x in s})
    first = list(sets)[0]
    z0_diff_inv = pow(S._vanishing_at([x for x in sup if x not in first], u), -1, p)
    h = [0] * n
    lx = [0] * n
    const = 0
    for i, (pts, ks) in enumerate(sets.items()):
        num = [0] * n
        r_u = 0
        for j, k in enumerate(ks):
            yj = pow(y, j, p)
            r = S._interpolate(list(pts), [pe[k][x] for x in pts])
            for t in range(n):
                num[t] = (num[t] + yj * polys[k][t]) % p
            for t in range(len(r)):
                num[t] = (num[t] - yj * r[t]) % p
            r_u = (r_u + yj * S._eval_host(r, u)) % p
        for s in pts:
            num = _synth_div(num, s, p)
        vi = pow(v, i, p)
        h = [(a + vi * b) % p for a, b in zip(h, num)]
        c = vi * S._vanishing_at([x for x in sup if x not in pts], u) * z0_diff_inv % p
        for j, k in enumerate(ks):
            cj = c * pow(y, j, p) % p
            lx = [(a + cj * b) % p for a, b in zip(lx, polys[k])]
        const = (const + c * r_u) % p
    lx[0] = (lx[0] - const) % p
    zt = S._vanishing_at(sup, u) * z0_diff_inv % p       # = Z_{S_0}(u)
    lx = [(a - zt * b) % p for a, b in zip(lx, h)]
    assert S._eval_host(lx, u) == 0
    return h, _synth_div(lx, u, p)


@pytest.mark.parametrize("seed", [1, 2])
def test_shplonk_open(h2b, orc, cuda, seed):
    import torch
    S = _mod()
    f = h2b.fields
    p = f.R_MOD
    k = 8
    n = 1 << k
    rng = random.Random(seed)
    polys = [[rng.randrange(p) for _ in range(n)] for _ in range(6)]
    d_polys = [h2b.to_dev(f.fr_mont_limbs(c)) for c in polys]
    w = f.EvaluationDomain(4, k).omega
    x = rng.randrange(p)
    xs = [x * pow(w, r % n, p) % p for r in (0, 1, 2, -1)]
    # rotation sets: {x}, {x, xw}, {x, xw, xw^2}, {x^-} style mixes
    qidx = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (3, 3), (4, 0), (4, 1), (5, 0)]
    queries = [(d_polys[a], xs[b]) for a, b in qidx]
    tau = f.fr_mont_limbs([0x5A11])
    srs = orc.srs(tau, n)
    d_srs = h2b.to_dev(srs)

    def commit(d):
        out = h2b.dev_empty(96)
        h2b.msm_device(d, d_srs, out, n, h2b.msm_workspace(n))
        return out

    ch = [rng.randrange(1, p) for _ in range(3)]
    evals, (cw, cw2), l_u = S.open_queries(h2b, queries, iter(ch), commit)
    torch.cuda.synchronize()
    assert l_u == 0
    for (a, b), e in zip(qidx, evals):
        assert e == S._eval_host(polys[a], xs[b])
    h, h2 = _restate(polys, [(a, xs[b]) for a, b in qidx], *ch, p, S)
    for coeffs, got in ((h, cw), (h2, cw2)):
        want = orc.msm(f.fr_mont_limbs(coeffs), srs)
        assert np.array_equal(h2b.to_host(got, (12,)), want)
