"""SHPLONK multi-point opening on the device (the flow of
halo2_proofs/src/poly/kzg/multiopen/shplonk/prover.rs:97-466, over this
library's entry points).

Queries are (device polynomial in coefficient form, length n; point).
Polynomials queried at the same SET of points form a rotation set.  With
challenges y, v, u (from a seeded generator here, not a transcript):

  q_i(X) = sum_j y^j (p_ij(X) - r_ij(X)) / Z_{S_i}(X)   r_ij interpolates p_ij on S_i
  h(X)   = sum_i v^i q_i(X)                             -> commitment W
  L(X)   = sum_i v^i Z_{T \\ S_i}(u) sum_j y^j (p_ij(X) - r_ij(u)) - Z_T(u) h(X)
  h'(X)  = L(X) / ((X - u) Z_{T \\ S_0}(u))              -> commitment W'

with T the union of all points.  L(u) = 0 whenever every evaluation is
right, so the division is exact; `open_queries` returns it for checking.
W' is normalised by the first set's coefficient 1 / Z_{T \\ S_0}(u), as the
reference's prover scales its final quotient (prover.rs:423-430) and its
verifier divides every set's coefficient by Z_{T \\ S_0}(u)
(verifier.rs:82-96).  The factor is folded into L's coefficients here:
set i enters with v^i Z_{T \\ S_i}(u) / Z_{T \\ S_0}(u) and h with
-Z_T(u) / Z_{T \\ S_0}(u) = -Z_{S_0}(u), so no extra pass scales the quotient.
Device
work: Horner evaluations (_halo2_eval_polynomial), linear combinations
(_halo2_poly_multiply_add), the interpolant subtraction
(_halo2_poly_sub_short_inplace, _halo2_poly_sub_scalar_at_zero), divisions by
(X - s) (_halo2_kate_division_device_padded) and the two MSMs (the caller's
`commit`).  Host work: the interpolants (at most a few points per set) and
the scalar bookkeeping.
"""
import ctypes

from . import fields as F

P = F.R_MOD


def _interpolate(points, values):
    """Coefficients (low first) of the polynomial of degree < len(points)
    through (points[k], values[k]), by Lagrange's formula mod r."""
    m = len(points)
    coeffs = [0] * m
    for k in range(m):
        basis = [1]                     # prod_{l != k} (X - x_l)
        denom = 1
        for l_ in range(m):
            if l_ == k:
                continue
            basis = [(a - points[l_] * b) % P for a, b in zip([0] + basis, basis + [0])]
            denom = denom * (points[k] - points[l_]) % P
        scale = values[k] * pow(denom, -1, P) % P
        for i in range(m):
            coeffs[i] = (coeffs[i] + scale * basis[i]) % P
    return coeffs


def _eval_host(coeffs, x):
    acc = 0
    for c in reversed(coeffs):
        acc = (acc * x + c) % P
    return acc


def _vanishing_at(points, u):
    acc = 1
    for s in points:
        acc = acc * (u - s) % P
    return acc


class Shplonk:
    """Device scratch and helpers for one opening of polynomials of length n."""

    def __init__(self, h2b, n, stream=None):
        self.h2b, self.n, self.stream = h2b, n, stream
        self.st = stream if stream is not None else __import__("torch").cuda.current_stream()
        self.sh = h2b.stream_handle(self.st)
        self.ews = h2b.dev_empty(h2b.lib()._halo2_eval_polynomial_workspace_size(n))
        self.kws = h2b.dev_empty(h2b.lib()._halo2_kate_division_workspace_size(n))

    def _scalar(self, v):
        return self.h2b.to_dev(F.fr_mont_limbs([v % P]), self.st)

    def eval_device(self, d_poly, x):
        """p(x) left on the device (a 32-byte view into fresh scratch)."""
        h2b = self.h2b
        ws = h2b.dev_empty(self.ews.numel())
        pt = F.fr_mont_limbs([x % P])
        res = ctypes.c_void_p()
        h2b.call("_halo2_eval_polynomial", h2b.ptr(d_poly), ctypes.byref(h2b.host_ffi(pt)), ctypes.byref(res),
                 self.n, h2b.ptr(ws), ws.numel(), self.sh)
        off = res.value - ws.data_ptr()
        return ws[off:off + 32]

    def eval_many(self, items):
        """[p(x) for (p, x) in items] as ints: up to 64 evaluations per
        h2b_eval_many_device call, one synchronisation."""
        if not items:
            return []
        torch = __import__("torch")
        outs = [self.h2b.eval_many_device([d for d, _ in items[i:i + 64]], [x for _, x in items[i:i + 64]], self.n,
                                          stream=self.st) for i in range(0, len(items), 64)]
        packed = torch.cat(outs).cpu().numpy().view("<u8").reshape(-1, 4)
        return F.fr_from_mont_limbs(packed)

    def eval(self, d_poly, x):
        """p(x) as an int (synchronises the stream)."""
        return self.eval_many([(d_poly, x)])[0]

    def madd(self, d_acc, d_in, c):
        """acc += c * in over n coefficients."""
        self.combine(d_acc, [d_in], [c])

    def combine(self, d_acc, d_polys, coeffs, accumulate=True):
        """acc = (acc if accumulate else 0) + sum_t coeffs[t] polys[t], one
        pass per 64 terms (h2b_poly_linear_combination)."""
        for i in range(0, max(len(d_polys), 1), 64):
            self.h2b.linear_combination_device(d_acc, d_polys[i:i + 64], coeffs[i:i + 64], self.n,
                                               accumulate=accumulate or i > 0, stream=self.st)

    def sub_short(self, d_acc, coeffs):
        d = self.h2b.to_dev(F.fr_mont_limbs([c % P for c in coeffs]), self.st)
        self.h2b.call("_halo2_poly_sub_short_inplace", self.h2b.ptr(d_acc), self.h2b.ptr(d), len(coeffs), self.sh)

    def div_linear(self, d_a, d_q, s):
        """q = (a - a(s)) / (X - s), written with zeros up to n."""
        self.h2b.call("_halo2_kate_division_device_padded", self.h2b.ptr(d_a), self.h2b.ptr(d_q),
                      self.h2b.ptr(self._scalar(s)), self.n, self.n, self.h2b.ptr(self.kws), self.kws.numel(),
                      self.sh)

    def zeros(self):
        t = self.h2b.dev_empty(32 * self.n)
        t.zero_()
        return t


def open_queries(h2b, queries, challenges, commit, stream=None, on_evals=None):
    """SHPLONK opening of `queries` = [(device poly, point)] (all of length n).
    `challenges` yields three ints, drawn in the transcript order of the
    reference's SHPLONK prover: y and v after the evaluations, u after the
    first commitment W (so a lazy generator over a Fiat-Shamir transcript
    sees W before it squeezes u); `commit(d_poly)` returns the 96-byte device
    commitment of a length-n polynomial; `on_evals(evals)` (optional) gets
    the evaluations before y is drawn.  Returns (evaluations in query order,
    [W, W'], L(u)) with L(u) == 0 for a sound opening."""
    n = queries[0][0].numel() // 32
    sp = Shplonk(h2b, n, stream)
    # evaluations, and the point set of every polynomial (by identity)
    evals, point_sets, polys = sp.eval_many(queries), {}, {}
    if on_evals is not None:
        on_evals(evals)
    for (d, x), e in zip(queries, evals):
        key = d.data_ptr()
        polys[key] = d
        point_sets.setdefault(key, {})[x % P] = e
    # rotation sets: polynomials with the same point set, in first-query order
    sets = {}
    for key, pe in point_sets.items():
        sets.setdefault(tuple(sorted(pe)), []).append(key)
    y, v = (next(challenges) % P for _ in range(2))
    super_points = sorted({x for s in sets for x in s})
    # h = sum_i v^i (sum_j y^j (p_ij - r_ij)) / Z_{S_i}
    h = sp.zeros()
    bufs = [sp.zeros(), sp.zeros()]
    lin_terms = []
    for i, (pts, keys) in enumerate(sets.items()):
        num = bufs[0]
        short = [0] * len(pts)
        for j, key in enumerate(keys):
            yj = pow(y, j, P)
            r = _interpolate(list(pts), [point_sets[key][x] for x in pts])
            short = [(a + yj * b) % P for a, b in zip(short, r)]
        sp.combine(num, [polys[key] for key in keys], [pow(y, j, P) for j in range(len(keys))], accumulate=False)
        sp.sub_short(num, short)
        cur, other = bufs
        for pt in pts:                   # divide by (X - s) for every point of the set
            sp.div_linear(cur, other, pt)
            cur, other = other, cur
        vi = pow(v, i, P)
        sp.madd(h, cur, vi)
        diff = [x for x in super_points if x not in pts]
        lin_terms.append((keys, vi, diff, short))
    w = commit(h)
    u = next(challenges) % P
    # per rotation set: v^i Z_{T\S_i}(u) / Z_{T\S_0}(u) and the combined interpolant at u
    z0_diff_inv = pow(_vanishing_at(lin_terms[0][2], u), -1, P)
    lin_terms = [(keys, vi * _vanishing_at(diff, u) * z0_diff_inv % P, _eval_host(short, u))
                 for keys, vi, diff, short in lin_terms]
    # L / Z_{T\S_0}(u) = sum_i v^i Z_{T\S_i}(u) / Z_{T\S_0}(u) sum_j y^j (p_ij - r_ij(u)) - Z_{S_0}(u) h
    lx = h2b.dev_empty(32 * n)
    const = 0
    terms, coeffs = [], []
    for keys, c_i, r_at_u in lin_terms:
        for j, key in enumerate(keys):
            terms.append(polys[key])
            coeffs.append(c_i * pow(y, j, P))
        const = (const + c_i * r_at_u) % P
    terms.append(h)
    coeffs.append(-_vanishing_at(list(sets)[0], u))
    sp.combine(lx, terms, coeffs, accumulate=False)
    h2b.call("_halo2_poly_sub_scalar_at_zero", h2b.ptr(lx), h2b.ptr(sp._scalar(const)), sp.sh)
    l_at_u = sp.eval(lx, u)
    q = sp.zeros()
    sp.div_linear(lx, q, u)
    w2 = commit(q)
    return evals, [w, w2], l_at_u
