"""Verifier of the config-3 circuit's proofs (host side, Python integers).

`verify_proof` restates the reference's `verify_proof`
(halo2_proofs/src/plonk/verifier.rs:19-378) for the circuit in circuit.py
with SHPLONK as the multi-open scheme (QUERY_INSTANCE false: the instance
column is evaluated from the public inputs, verifier.rs:162-198):

1. the transcript replays the proof: the verifying key's scalar and the
   public inputs, the advice commitments, theta, A' and S', beta, gamma,
   the permutation and lookup product commitments, the random polynomial's
   commitment, y, the h pieces, x, then the evaluations in the order the
   prover wrote them (advice, fixed, random, sigma, permutation sets,
   lookup);
2. the vanishing argument (vanishing/verifier.rs:90-118): the gate
   polynomials, the permutation expressions (permutation/verifier.rs:
   112-214) and the lookup expressions (lookup/verifier.rs:96-166) at x,
   folded with y, give the expected h(x) = fold / (x^n - 1); the h
   commitment is sum_i x^(n i) H_i;
3. the SHPLONK opening of every query (shplonk/verifier.rs:60-135) against
   the commitments, with that h(x) as the claimed evaluation of h, ending in
   the reference's pairing product (poly/kzg/msm.rs:159-176)
       e(W', [s]_2) * e(F + u W', -[1]_2) == 1,
   F = sum_i v^i (Z_{T\\S_i}(u) / Z_{T\\S_0}(u)) (sum_j y^j C_ij - r_i(u) G)
       - Z_{S_0}(u) W,
   computed by pairing.py's optimal ate pairing.

The SRS here is synthetic ([tau^i] G with a seeded tau, never a ceremony),
so its G2 elements are [1]_2 = the standard generator and [s]_2 = tau [1]_2,
as the reference's setup makes them (poly/kzg/commitment.rs:188-189).
Because e is non-degenerate the pairing product is 1 exactly when
F + u W' = tau W' in G1; `shplonk_check_trapdoor` checks that G1 form
directly (no pairing), and the tests hold both checks to the same verdicts.
"""
from . import circuit as C
from . import fields as F
from . import pairing as E
from . import transcript as T
from .shplonk import _eval_host, _interpolate, _vanishing_at

P = F.R_MOD


class VerifyingKey:
    """What the verifier knows of the 2^k circuit: its commitments to the
    fixed columns and the permutation polynomials (affine points), and the
    scalar that stands for the key in the transcript."""

    def __init__(self, k, fixed_commitments, permutation_commitments, transcript_repr):
        self.k = k
        self.dom = F.EvaluationDomain(C.DEGREE, k)
        self.fixed_commitments = list(fixed_commitments)
        self.permutation_commitments = list(permutation_commitments)
        self.transcript_repr = transcript_repr


def _neg(pt):
    return None if pt is None else (pt[0], (F.Q_MOD - pt[1]) % F.Q_MOD)


def _mul(pt, s):
    s %= P
    if pt is None or s == 0:
        return None
    if s == 1:
        return pt
    return F.g1_mul(pt, s)


class KZGVerifierParams:
    """The SRS's G2 elements the final check needs: [1]_2 and [s]_2
    (ParamsKZG's g2 and s_g2, poly/kzg/commitment.rs:32-33)."""

    def __init__(self, g2, s_g2):
        if not (E.g2_on_curve(g2) and E.g2_on_curve(s_g2)):
            raise ValueError("G2 element off the twist")
        self.g2, self.s_g2 = g2, s_g2


_PARAMS = {}


def params_from_tau(tau):
    """[1]_2 = the standard G2 generator and [s]_2 = tau [1]_2 for the
    synthetic SRS with trapdoor tau (cached per tau)."""
    tau %= P
    if tau not in _PARAMS:
        _PARAMS[tau] = KZGVerifierParams(E.G2_GENERATOR, E.g2_mul(E.G2_GENERATOR, tau))
    return _PARAMS[tau]


def shplonk_dual_msm(commitments, queries, evals, y, v, u, w, w2):
    """The two G1 sums of the final check, (left, right) = (W', F + u W').

    commitments: {label: affine point or None}; queries: [(label, point)]
    in query order; evals: the claimed evaluations; y, v, u: the SHPLONK
    challenges; w, w2: W and W' (affine).  Mirrors shplonk/verifier.rs:60-131:
    rotation sets in the order of their first commitment, each set's
    coefficient Z_{T\\S_i}(u) normalised by the first set's (so set 0 enters
    with 1), r_outer = sum_i v^i z_i sum_j y^j r_ij(u), and
    F = outer - r_outer G - Z_{S_0}(u) W; left gets W' (msm_accumulator.left),
    right gets F + u W' (msm_accumulator.right)."""
    point_sets = {}
    for (lab, x), e in zip(queries, evals):
        point_sets.setdefault(lab, {})[x % P] = e % P
    sets = {}
    for lab, pe in point_sets.items():
        sets.setdefault(tuple(sorted(pe)), []).append(lab)
    super_points = sorted({x for s in sets for x in s})
    outer, r_outer, z_0, z0_diff_inv = None, 0, 0, 0
    for i, (pts, labs) in enumerate(sets.items()):
        z_diff = _vanishing_at([x for x in super_points if x not in pts], u)
        if i == 0:
            z_0 = _vanishing_at(list(pts), u)
            z0_diff_inv = pow(z_diff, -1, P)
            z_diff = 1
        else:
            z_diff = z_diff * z0_diff_inv % P
        inner, r_inner = None, 0
        for j, lab in enumerate(labs):
            yj = pow(y, j, P)
            r = _interpolate(list(pts), [point_sets[lab][x] for x in pts])
            r_inner = (r_inner + yj * _eval_host(r, u)) % P
            inner = F.g1_add(inner, _mul(commitments[lab], yj))
        vi = pow(v, i, P)
        outer = F.g1_add(outer, _mul(inner, vi * z_diff))
        r_outer = (r_outer + vi * r_inner * z_diff) % P
    outer = F.g1_add(outer, _mul(F.G1_GENERATOR, -r_outer))
    outer = F.g1_add(outer, _mul(w, -z_0))
    outer = F.g1_add(outer, _mul(w2, u))
    return w2, outer


def shplonk_check_pairing(commitments, queries, evals, y, v, u, w, w2, params):
    """The reference's final check (poly/kzg/msm.rs:159-176):
    e(left, [s]_2) * e(right, -[1]_2) == 1."""
    if isinstance(params, int):
        params = params_from_tau(params)
    left, right = shplonk_dual_msm(commitments, queries, evals, y, v, u, w, w2)
    return E.pairing_check([(left, params.s_g2), (right, E.g2_neg(params.g2))])


def shplonk_check_trapdoor(commitments, queries, evals, y, v, u, w, w2, tau):
    """The same check in G1 with the SRS trapdoor tau: right == tau left."""
    left, right = shplonk_dual_msm(commitments, queries, evals, y, v, u, w, w2)
    return right == _mul(left, tau)


def lagrange_at(dom, x, i):
    """L_i(x) = w^i (x^n - 1) / (n (x - w^i)) for a row i (negative rows count
    from the end), the domain's l_i_range evaluations."""
    wi = pow(dom.omega, i % dom.n, P)
    den = dom.n * (x - wi) % P
    if den == 0:
        raise ValueError("x lies in the domain")
    return wi * (pow(x, dom.n, P) - 1) * pow(den, -1, P) % P


def expressions(dom, ev, public_eval, theta, beta, gamma, x):
    """Every constraint at x, in the order the prover's quotient folds them:
    the gates, the permutation's, the lookup's.  `ev` maps (label, rotation)
    to the opened evaluations."""
    del theta                  # one input and one table expression: compression is the identity
    B = C.BLINDING_FACTORS
    l_last = lagrange_at(dom, x, -(B + 1))
    l_blind = sum(lagrange_at(dom, x, -i) for i in range(1, B + 1)) % P
    l_0 = lagrange_at(dom, x, 0)
    active = (1 - l_last - l_blind) % P
    advice = [ev[(f"adv{c}", r)] for c, r in C.ADVICE_QUERIES]
    fixed = [ev[(f"fixed{c}", r)] for c, r in C.FIXED_QUERIES]
    out = C.gate_values(advice, fixed)
    # permutation (permutation/verifier.rs:112-214)
    col_eval = [advice[C.advice_query_index(i, 0)] if kind == 0 else public_eval for kind, i in C.PERM_COLUMNS]
    sets = len(C.PERM_COLUMNS) // C.CHUNK_LEN
    z = [ev[(f"z{s}", 0)] for s in range(sets)]
    z_next = [ev[(f"z{s}", 1)] for s in range(sets)]
    z_last = [ev[(f"z{s}", -(B + 1))] for s in range(sets - 1)]
    out.append(l_0 * (1 - z[0]) % P)
    out.append((z[-1] * z[-1] - z[-1]) * l_last % P)
    for s in range(1, sets):
        out.append((z[s] - z_last[s - 1]) * l_0 % P)
    for s in range(sets):
        cols = range(C.CHUNK_LEN * s, C.CHUNK_LEN * (s + 1))
        left, right = z_next[s], z[s]
        cur = beta * x * pow(F.DELTA, C.CHUNK_LEN * s, P) % P
        for c in cols:
            left = left * (col_eval[c] + beta * ev[(f"sigma{c}", 0)] + gamma) % P
            right = right * (col_eval[c] + cur + gamma) % P
            cur = cur * F.DELTA % P
        out.append((left - right) * active % P)
    # lookup (lookup/verifier.rs:96-166): input b, table t
    zl, zl_next = ev[("zl", 0)], ev[("zl", 1)]
    a_, a_prev, s_ = ev[("pa", 0)], ev[("pa", -1)], ev[("ps", 0)]
    inp = advice[C.advice_query_index(C.ADV_B, 0)]
    tab = fixed[C.FIXED_QUERIES.index((C.FIX_TABLE, 0))]
    out.append(l_0 * (1 - zl) % P)
    out.append(l_last * (zl * zl - zl) % P)
    out.append((zl_next * (a_ + beta) * (s_ + gamma) - zl * (inp + beta) * (tab + gamma)) * active % P)
    out.append(l_0 * (a_ - s_) % P)
    out.append((a_ - s_) * (a_ - a_prev) * active % P)
    return out


def verify_proof(vk, public, proof, params):
    """True when `proof` (bytes) is a valid proof of the circuit with public
    inputs `public` (ints) under `vk`, its opening checked by the pairing
    product against `params` (KZGVerifierParams, or the synthetic SRS's
    trapdoor tau, from which they are made).  A malformed proof (a point off
    the curve, a non-canonical scalar, missing or extra bytes) is rejected."""
    from .prover import open_queries_for, transcript_eval_order
    dom, B = vk.dom, C.BLINDING_FACTORS
    try:
        r = T.Blake2bRead(proof)
        r.common_scalar(vk.transcript_repr)
        for v in public:
            r.common_scalar(v % P)
        cm = {f"adv{i}": r.read_point() for i in range(C.NUM_ADVICE)}
        theta = r.squeeze_challenge()
        cm["pa"], cm["ps"] = r.read_point(), r.read_point()
        beta, gamma = r.squeeze_challenge(), r.squeeze_challenge()
        sets = len(C.PERM_COLUMNS) // C.CHUNK_LEN
        for s in range(sets):
            cm[f"z{s}"] = r.read_point()
        cm["zl"] = r.read_point()
        cm["random"] = r.read_point()
        y = r.squeeze_challenge()
        hs = [r.read_point() for _ in range(dom.quotient_poly_degree)]
        x = r.squeeze_challenge()
        order = transcript_eval_order(dom, x)
        evals = {lab: r.read_scalar() for lab in order}
        sy, sv = r.squeeze_challenge(), r.squeeze_challenge()
        w = r.read_point()
        u = r.squeeze_challenge()
        w2 = r.read_point()
        if r.remaining() != 0:
            return False
    except T.TranscriptError:
        return False
    # evaluations keyed by (label, rotation)
    rot_of = {}
    for lab, r_ in [(f"adv{c}", rr) for c, rr in C.ADVICE_QUERIES] + [(f"fixed{c}", rr) for c, rr in C.FIXED_QUERIES] \
            + [("random", 0)] + [(f"sigma{i}", 0) for i in range(len(C.PERM_COLUMNS))] \
            + [(f"z{s}", rr) for s in range(sets) for rr in (0, 1, -(B + 1))] \
            + [("zl", 0), ("zl", 1), ("pa", 0), ("pa", -1), ("ps", 0)]:
        rot_of[(lab, x * pow(dom.omega, r_ % dom.n, P) % P)] = r_
    ev = {(lab, rot_of[(lab, pt)]): val for (lab, pt), val in evals.items()}
    public_eval = C.instance_eval(dom, public, x)
    xn = pow(x, dom.n, P)
    acc = 0
    for e in expressions(dom, ev, public_eval, theta, beta, gamma, x):
        acc = (acc * y + e) % P
    if xn == 1:
        return False
    expected_h = acc * pow(xn - 1, -1, P) % P
    h_commitment = None
    for H in reversed(hs):
        h_commitment = F.g1_add(_mul(h_commitment, xn), H)
    cm["h"] = h_commitment
    for i, pt in enumerate(vk.fixed_commitments):
        cm[f"fixed{i}"] = pt
    for i, pt in enumerate(vk.permutation_commitments):
        cm[f"sigma{i}"] = pt
    _, labels = open_queries_for(dom, x, {lab: None for lab in cm})
    values = dict(evals)
    values[("h", x)] = expected_h
    claimed = [values[lab] for lab in labels]
    return shplonk_check_pairing(cm, labels, claimed, sy, sv, u, w, w2, params)
