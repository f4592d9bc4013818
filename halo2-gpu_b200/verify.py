"""Host-side check of a proof's SHPLONK opening (the multi-open part of the
verifier, halo2's `VerifierSHPLONK` as called from the reference's
`verify_proof`; the reference's verifier lives in halo2-axiom, absent from
the reference tree).

The verifier's final check is the pairing equation
    e(F + u W', [1]_2) = e(W', [tau]_2),
with F = sum_i v^i Z_{T \\ S_i}(u) (sum_j y^j C_ij - r_i(u) G) - Z_T(u) W
over the rotation sets S_i (polynomials opened at the same point set, in
first-query order), T the union of all points, r_i the y-combined
interpolant of set i's claimed evaluations, W and W' the two opening
commitments.  Because e is non-degenerate, that equation holds exactly when
F = (tau - u) W' in G1.  For a synthetic SRS whose trapdoor tau is known
(here [tau^i] G with a seeded tau, never a ceremony), this module checks the
G1 form directly with Python integers, so no pairing is needed; with a real
SRS the pairing form is the only option.  It is a check of the opening
only: the vanishing argument (the gate, permutation and lookup constraints
at x from the opened evaluations) needs a satisfying witness, which the
prover-shaped workload does not have.
"""
from . import fields as F
from .shplonk import _eval_host, _interpolate, _vanishing_at

P = F.R_MOD


def _neg(pt):
    return None if pt is None else (pt[0], (F.Q_MOD - pt[1]) % F.Q_MOD)


def _mul(pt, s):
    s %= P
    if pt is None or s == 0:
        return None
    if s == 1:
        return pt
    return F.g1_mul(pt, s)


def shplonk_check_trapdoor(commitments, queries, evals, y, v, u, w, w2, tau):
    """commitments: {label: affine point or None}; queries: [(label, point)]
    in the order the evaluations were written; evals: the claimed
    evaluations; y, v, u: the SHPLONK challenges; w, w2: W and W' (affine);
    tau: the SRS trapdoor.  True when F == (tau - u) W'."""
    point_sets = {}
    for (lab, x), e in zip(queries, evals):
        point_sets.setdefault(lab, {})[x % P] = e % P
    sets = {}
    for lab, pe in point_sets.items():
        sets.setdefault(tuple(sorted(pe)), []).append(lab)
    super_points = sorted({x for s in sets for x in s})
    acc = None
    for i, (pts, labs) in enumerate(sets.items()):
        short = [0] * len(pts)
        comb = None
        for j, lab in enumerate(labs):
            yj = pow(y, j, P)
            r = _interpolate(list(pts), [point_sets[lab][x] for x in pts])
            short = [(a + yj * b) % P for a, b in zip(short, r)]
            comb = F.g1_add(comb, _mul(commitments[lab], yj))
        term = F.g1_add(comb, _neg(_mul(F.G1_GENERATOR, _eval_host(short, u))))
        diff = [x for x in super_points if x not in pts]
        acc = F.g1_add(acc, _mul(term, pow(v, i, P) * _vanishing_at(diff, u)))
    acc = F.g1_add(acc, _neg(_mul(w, _vanishing_at(super_points, u))))
    return acc == _mul(w2, tau - u)
