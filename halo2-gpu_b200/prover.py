"""Prover for the config-3 circuit family and a serving loop around it.

`ProofWorkload.run` proves one instance of the circuit in `circuit.py` (4
advice, 3 fixed, 1 instance column; a standard-PLONK gate and a Fibonacci
rotation gate; a 4-column copy permutation; one lookup into a 2^8-entry
table) with a satisfying witness synthesised on the device, issuing on one
stream the device work of `create_proof`
(halo2_proofs/src/plonk/prover.rs:140-622) through this library's entry
points, in the reference's phase order:

  phase 1  the verifying key and the public inputs into the transcript;
           advice commitments (commit_lagrange over the Lagrange bases);
           theta
  phase 2  lookup: permute-sort of the compressed input against the
           compressed table over the usable rows, blinding rows, A' and S'
           commitments; beta, gamma
  phase 3  permutation grand products (2 sets of 2 columns, the carry of one
           set seeding the next) and the lookup grand product, blinding rows,
           their commitments; the vanishing argument's random polynomial
           (the constant 1 with zero knowledge off, committed as g[0]:
           halo2_proofs/src/plonk/vanishing/prover.rs:64-99); y
  phase 4  lagrange_to_coeff of the per-proof polynomials; per extended part
           the coset parts, the gate quotient, the permutation quotient, the
           lookup product coset (the lookup's graph through the same
           evaluator) and the lookup quotient; h gathered, divided by the
           vanishing polynomial, brought to coefficients, its 3 pieces
           committed; x
  phase 5  evaluations in the transcript's order (advice, fixed, the random
           polynomial's 1, sigma, permutation products, lookup), then the
           SHPLONK opening (shplonk.py) of the queries in the reference's
           order, with h folded to sum_i x^(n i) h_i (vanishing/prover.rs:
           190-240).

Challenges come from the Fiat-Shamir transcript (transcript.py) when
`transcript=True`, and from a seeded generator otherwise (same device work,
no proof bytes).  `verify.verify_proof` checks a proof from its bytes, the
public inputs, the verifying key and the SRS's G2 elements
(`Resident.verifier_params`), ending in the reference's pairing check.  Blinding values come from this
library's seeded device generator, not the reference's ChaCha RNG, so proof
bytes are this build's own; parity of the bytes is unpinned.

`Server` runs such requests with `slots` worker threads, each on its own
stream (the GPU overlaps them), admitting a request when a slot is free and
the HBM budget allows; `plain` runs them one at a time.
"""
import hashlib
import queue
import threading
import time

import numpy as np

from . import circuit as C
from . import fields as F
from . import shplonk
from . import transcript as T

NUM_PUBLIC = C.NUM_PUBLIC
# the proof's commitments in the order they are written
COMMIT_LABELS = ("adv0", "adv1", "adv2", "adv3", "pa", "ps", "z0", "z1", "zl", "random", "h0", "h1", "h2", "W", "W2")
NUM_EVALS = len(C.ADVICE_QUERIES) + len(C.FIXED_QUERIES) + 1 + 4 + 5 + 5

_torch = None


def _t():
    global _torch
    if _torch is None:
        import torch
        _torch = torch
    return _torch


def _bytes_per_proof(k):
    """Device memory one in-flight proof of size 2^k holds besides its MSM
    scratch (upper bound): 10 Lagrange and 10 coefficient polynomials, 10
    coset parts, the extended-domain vectors, the unfused quotient's 4 parts
    and lookup product coset, the opening's buffers and small tensors."""
    n = 1 << k
    return 64 * 32 * n + (64 << 20)


class Resident:
    """State kept on the device across requests: the SRS and its window
    table, the Lagrange-basis window table per k, and per k the circuit's
    proving key (circuit.ProvingKey) with the extended coset parts of its
    key polynomials."""

    def __init__(self, h2b, kmax, seed=0x5EED):
        self.h2b = h2b
        self.kmax = kmax
        self.tau = seed % F.R_MOD   # the synthetic SRS's trapdoor: [tau^i] G, never a ceremony
        self.srs = h2b.srs_device(seed, 1 << kmax)
        self.table = h2b.msm_table_precompute(self.srs, 1 << kmax)
        self.pk = {}
        self._lock = threading.Lock()
        self._lag_tables = {}
        self._cosets = {}
        self._vk = {}

    def key(self, k):
        with self._lock:
            if k not in self.pk:
                self.pk[k] = C.ProvingKey(self.h2b, k)
        return self.pk[k]

    def lagrange_table(self, k):
        """Window table of the 2^k Lagrange bases [L_i(tau)] G of the same
        SRS (ParamsKZG's g_lagrange, halo2_proofs/src/poly/kzg/commitment.rs:
        158-186), so commit_lagrange commits a column's values directly.  The
        scalars L_i(tau) = (1/n) sum_j tau^j w^(-ij) are the inverse NTT of the
        powers of tau; the points come from the SRS kernel.  Built once per k,
        with the monomial table's geometry (2^kmax points, the Lagrange bases
        first, SRS points after them that an MSM of 2^k scalars never reads),
        so its window width is the one measured for the monomial table: a table
        of only 2^k points takes narrower windows, whose single bucket set
        holds longer buckets (k = 16 proof 17.3 -> 21.0 ms)."""
        with self._lock:
            if k not in self._lag_tables:
                torch, h2b, n, tn = _t(), self.h2b, 1 << k, 1 << self.kmax
                dom = F.EvaluationDomain(C.DEGREE, k)
                lam = h2b.dev_empty(32 * n)
                h2b.fft_normal_to_device(2, k, h2b.powers_device(self.tau, n), lam, dom.omega_inv,
                                         dom.ifft_divisor)
                bases = self.srs.clone()
                h2b.call("h2b_srs_from_powers", h2b.ptr(bases), h2b.ptr(lam), n,
                         h2b.ptr(h2b.to_dev(F.g1_pow2_table(256))), h2b.stream_handle())
                self._lag_tables[k] = h2b.msm_table_precompute(bases, tn)
                torch.cuda.synchronize()
        return self._lag_tables[k]

    def key_cosets(self, k, stream=None):
        """The 4 extended coset parts of the 2^k key polynomials (3 fixed, 4
        permutation, l_0, l_last, l_active), computed once and kept
        resident, as halo2's ProvingKey keeps `fixed_cosets` and the
        permutation cosets from keygen on: a proof then transforms only its
        own 10 polynomials per part.  [part][polynomial] device vectors."""
        pk = self.key(k)
        with self._lock:
            if k not in self._cosets:
                torch, h2b, n, dom = _t(), self.h2b, 1 << k, pk.dom
                keyp = pk.fixed + pk.sigma + pk.lag
                st = stream if stream is not None else torch.cuda.current_stream()
                cos = []
                with torch.cuda.stream(st):
                    for j in range(1 << (dom.extended_k - k)):
                        outs = [h2b.dev_empty(32 * n) for _ in keyp]
                        shift = pow(dom.extended_omega, j, F.R_MOD)
                        h2b.fft_many_to_device(6, k, k, keyp, outs, dom.omega, F.ZETA * shift % F.R_MOD, stream=st)
                        cos.append(outs)
                st.synchronize()
                self._cosets[k] = cos
        return self._cosets[k]

    def keygen(self, k, stream=None):
        """Verifying-key commitments of the 2^k key (keygen_vk's GPU part,
        halo2_proofs/src/plonk/keygen.rs:265-290): the 3 fixed and 4
        permutation polynomials, committed in one MSM batch over the resident
        SRS table (coefficient form with monomial bases: the same points as
        the Lagrange form with Lagrange bases).  Returns 96-byte device images."""
        torch, h2b = _t(), self.h2b
        pk, n, tn = self.key(k), 1 << k, 1 << self.kmax
        polys = pk.fixed + pk.sigma
        st = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(st):
            outs = [h2b.dev_empty(96) for _ in polys]
            jobs = h2b.msm_batch_jobs(polys, [self.table] * len(polys), outs, [n] * len(polys), table_n=tn)
            ws = h2b.msm_batch_workspace(jobs, len(polys), len(polys))
            h2b.msm_batch(jobs, len(polys), len(polys), ws, stream=st)
        return outs

    def verifying_key(self, k, stream=None):
        """The host verifying key of the 2^k circuit (verify.VerifyingKey):
        its fixed and permutation commitments as affine points, and the
        transcript scalar standing for it."""
        if k not in self._vk:
            from . import verify as V
            outs = self.keygen(k, stream)
            (stream if stream is not None else _t().cuda.current_stream()).synchronize()
            pts = [T.commitment_to_affine(o.cpu().numpy().view(np.uint64)) for o in outs]
            h = hashlib.blake2b(digest_size=64, person=b"Halo2-Verify-Key")
            for pt in pts:
                h.update(T.compress(pt))
            rep = int.from_bytes(h.digest(), "little") % F.R_MOD
            self._vk[k] = V.VerifyingKey(k, pts[:3], pts[3:], rep)
        return self._vk[k]

    def verifier_params(self):
        """The SRS's G2 elements for the verifier's pairing check
        (verify.KZGVerifierParams: [1]_2 and [s]_2 = tau [1]_2)."""
        from . import verify as V
        return V.params_from_tau(self.tau)

    def vk_repr(self, k, stream=None):
        """One Fr scalar standing for the 2^k verifying key in the transcript:
        BLAKE2b of its compressed fixed and permutation commitments, mod r
        (halo2's `vk.hash_into` absorbs `vk.transcript_repr`, a BLAKE2b digest
        of the pinned verifying key; this key has no pinned form, so its
        commitments stand in).  Computed once per k."""
        return self.verifying_key(k, stream).transcript_repr

    def device_bytes(self):
        """Device memory held resident: SRS and its window table, Lagrange
        window tables, proving keys and their coset parts."""
        total = self.srs.numel() + self.table.numel() + sum(t.numel() for t in self._lag_tables.values())
        for k, pk in self.pk.items():
            total += pk.device_bytes()
        for cos in self._cosets.values():
            total += sum(t.numel() for part in cos for t in part)
        return total


def _slice(t, i, n):
    """Elements [i n, (i + 1) n) of a device field vector."""
    return t[32 * n * i: 32 * n * (i + 1)]


_G_JAC = None


def _generator_image():
    """The 96-byte Jacobian image of G = g[0] (Montgomery Fq {1, 2, 1})."""
    global _G_JAC
    if _G_JAC is None:
        _G_JAC = F.fq_mont_limbs([1, 2, 1]).reshape(-1)
    return _G_JAC


class ProofWorkload:
    """One proof of the 2^k circuit (see the module docstring)."""

    def __init__(self, res, k, seed, transcript=False, tamper=None, check_degree=False, fused_quotient=True,
                 merged_msm=False):
        """transcript=False draws the challenges from a generator seeded with
        `seed`; transcript=True runs the Fiat-Shamir transcript
        (transcript.Blake2bWrite): every commitment is read back and absorbed
        before the next challenge is squeezed, and `self.proof` holds the
        proof bytes.  `tamper(advice, instance)`, if given, may change the
        synthesised witness before anything is committed (tests use it to
        break one cell).  check_degree=True reads back whether the top n of
        h's 4n coefficients are zero (`self.h_degree_ok`): they are exactly
        when every constraint holds on the whole domain, the quotient
        identity h = sum_i y^i C_i / (X^n - 1) with deg h < 3n.
        fused_quotient=True evaluates each extended part with one
        h2b_quotient_fused launch that writes the part interleaved into the
        extended array, already divided by X^n - 1; False runs the
        reference's per-part launcher sequence (gates, permutation, lookup
        expression, lookup constraints) and then gathers and divides.  The
        proofs are the same bytes.  merged_msm=True commits each phase's
        polynomials over one window table as one merged MSM (h2b_msm_merged);
        False (the default) runs them as separate MSMs on forked streams
        (h2b_msm_batch), which measured faster here (k = 16 / 20 / 22 proofs
        17.8 / 79 / 280 ms against 18.6 / 81 / 286 ms merged): one MSM's sort
        overlaps another's accumulation.  Same bytes."""
        self.res, self.k, self.seed, self.transcript, self.tamper = res, k, seed, transcript, tamper
        self.fused_quotient = fused_quotient
        self.merged_msm = merged_msm
        self.check_degree = check_degree
        self.h_degree_ok = None
        self.proof = None
        self.public = None

    def run(self, stream):
        """Issues everything on `stream` (the calling thread blocks only where
        an entry point synchronises: the permute-sort's error check and the
        opening's evaluations); returns the commitments (96 B each, in
        COMMIT_LABELS order) and the evaluations (32 B each, transcript order)
        as device tensors, complete once `stream` is."""
        torch, h2b, res = _t(), self.res.h2b, self.res
        k, n, seed = self.k, 1 << self.k, self.seed
        p = F.R_MOD
        pk = res.key(k)
        dom, u = pk.dom, pk.u
        tn = 1 << res.kmax
        tr = T.Blake2bWrite() if self.transcript else None
        if tr is None:
            rng = np.random.default_rng(seed)
            _draw = lambda: int(rng.integers(1, 1 << 62))  # noqa: E731
        else:
            _draw = tr.squeeze_challenge
        drawn = []
        self.challenges = drawn

        def chal():
            drawn.append(_draw())
            return drawn[-1]
        sc = lambda v: F.fr_mont_limbs([v % p])  # noqa: E731
        sh = h2b.stream_handle(stream)

        def absorb(outs):
            """Reads the phase's commitments back (waits for `stream`) and
            writes them to the transcript."""
            if tr is not None:
                for o in outs:
                    tr.write_point(T.commitment_to_affine(o.cpu().numpy().view(np.uint64)))

        with torch.cuda.stream(stream):
            commits, pending = [], []
            probe = h2b.dev_empty(32)
            lag_tab = res.lagrange_table(k)
            slots = h2b.msm_batch_jobs([probe] * 4, [res.table] * 4, [probe] * 4, [n] * 4, table_n=tn)
            msm_ws = h2b.msm_batch_workspace(slots, 4, 4)   # both tables have 2^kmax points

            def commit(d, lagrange=False):
                """Queues the commitment of a length-n vector: Lagrange values
                over the Lagrange bases (commit_lagrange), coefficients over
                the monomial SRS (commit)."""
                out = h2b.dev_empty(96)
                pending.append((d, out, lagrange))
                commits.append(out)

            def flush():
                """The commitments of one phase: those over the same window table
                as one merged MSM (one sort, accumulation and reduction for
                all), or each MSM on its own forked stream."""
                if self.merged_msm:
                    for lagr in (True, False):
                        group = [q for q in pending if q[2] == lagr]
                        if not group:
                            continue
                        jobs = h2b.msm_batch_jobs([q[0] for q in group], [lag_tab if lagr else res.table] * len(group),
                                                  [q[1] for q in group], [n] * len(group), table_n=tn)
                        ws = h2b.dev_empty(h2b.msm_merged_workspace_bytes(jobs, len(group)))
                        h2b.msm_merged(jobs, len(group), ws, stream=stream)
                else:
                    jobs = (h2b.MsmJob * len(pending))()
                    for i, (d, out, lagr) in enumerate(pending):
                        jobs[i].d_scalars, jobs[i].d_out, jobs[i].n = d.data_ptr(), out.data_ptr(), n
                        jobs[i].d_bases = (lag_tab if lagr else res.table).data_ptr()
                        jobs[i].table_n = tn
                    h2b.msm_batch(jobs, len(pending), len(pending), msm_ws, stream=stream)
                outs = [q[1] for q in pending]
                pending.clear()
                absorb(outs)

            def blind(t, start, tag):
                """Rows [start, n) of a column from the seeded device generator."""
                t[32 * start:] = h2b.random_fr_device(n - start, ((seed << 4) + tag) & (2 ** 64 - 1), 0, stream)

            # phase 1: witness, verifying key and public inputs, advice commitments
            adv, inst, public = C.synthesize(h2b, pk, seed, stream)
            if self.tamper is not None:
                self.tamper(adv, inst)
            self.public = public
            if tr is not None:
                tr.common_scalar(res.vk_repr(k, stream))
                for v in public:
                    tr.common_scalar(v)
            for a in adv:
                commit(a, lagrange=True)
            flush()
            chal()                                   # theta (one input and one table expression: no compression)
            # phase 2: lookup permute over the usable rows, blinding rows, A' and S'
            b_col, t_col = adv[C.ADV_B], pk.fixed_values[C.FIX_TABLE]
            pa, ps = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
            h2b.permute_expression_pair_device(b_col, t_col, pa, ps, n, u, stream=stream)
            blind(pa, u, 8)
            blind(ps, u, 9)
            commit(pa, lagrange=True)
            commit(ps, lagrange=True)
            flush()
            beta, gamma = chal(), chal()
            # phase 3: permutation products (2 sets of 2 columns), lookup product, random polynomial
            d_beta, d_gamma = h2b.to_dev(sc(beta), stream), h2b.to_dev(sc(gamma), stream)
            d_delta = h2b.to_dev(sc(F.DELTA), stream)
            d_om = h2b.to_dev(sc(dom.omega), stream)
            d_one = h2b.to_dev(sc(1), stream)
            cols = [adv[C.ADV_A], adv[C.ADV_B], adv[C.ADV_C], inst]
            zs, prefix = [], d_one
            for s in range(len(cols) // C.CHUNK_LEN):
                mod = h2b.dev_empty(32 * n)
                h2b.call("_halo2_poly_fill_one", h2b.ptr(mod), n, sh)
                d_dw = h2b.to_dev(sc(pow(F.DELTA, C.CHUNK_LEN * s, p)), stream)
                sl = slice(C.CHUNK_LEN * s, C.CHUNK_LEN * (s + 1))
                h2b.permutation_product_device(mod, pk.sigma_values[sl], cols[sl], d_beta, d_gamma, d_delta, d_om,
                                               d_dw, u, stream=stream)
                z = h2b.dev_empty(32 * n)
                z[:32] = prefix
                z[32: 32 * (u + 1)] = mod[: 32 * u]
                h2b.grand_product_device(z, prefix, u, offset=1, stream=stream)
                prefix = z[32 * u: 32 * (u + 1)]     # the carry: this set's last value seeds the next set
                blind(z, u + 1, 10 + s)
                zs.append(z)
            zl, ratio = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
            h2b.lookup_product_device(ratio, pa, ps, b_col, t_col, d_beta, d_gamma, u, stream=stream)
            zl[:32] = d_one
            zl[32: 32 * (u + 1)] = ratio[: 32 * u]
            h2b.grand_product_device(zl, d_one, u, offset=1, stream=stream)
            blind(zl, u + 1, 12)
            del ratio
            for z in zs + [zl]:
                commit(z, lagrange=True)
            flush()
            g_img = h2b.to_dev(_generator_image(), stream)       # the random polynomial's commitment, g[0]
            commits.append(g_img)
            if tr is not None:
                tr.write_point(F.G1_GENERATOR)
            y = chal()
            # phase 4: coefficients, the quotient per extended part, h
            lag = adv + [inst] + zs + [zl, pa, ps]
            coef = [h2b.dev_empty(32 * n) for _ in lag]
            h2b.fft_many_to_device(2, k, k, lag, coef, dom.omega_inv, dom.ifft_divisor, stream=stream)
            del lag
            ca, ci, cz, czl, cpa, cps = coef[0:4], coef[4], coef[5:7], coef[7], coef[8], coef[9]
            d_y = h2b.to_dev(sc(y), stream)
            kcos = res.key_cosets(k, stream)
            own = [h2b.dev_empty(32 * n) for _ in coef]
            n_parts = 1 << (dom.extended_k - k)
            en = n_parts * n
            ext = h2b.dev_empty(32 * en)
            fused = self.fused_quotient
            tv = None if fused else h2b.dev_empty(32 * n)
            hs = [] if fused else [h2b.dev_empty(32 * n) for _ in range(n_parts)]
            nws = h2b.dev_empty(h2b.lib()._halo2_fft_many_to_device_workspace_size(6, k, k))
            g_rules, g_parts, g_consts = pk.gates
            l_rules, l_parts, l_consts = pk.lookup_graph
            bg = np.concatenate([sc(beta), sc(gamma)])
            no_chal = np.zeros((0, 4), np.uint64)
            for j in range(n_parts):
                shift = pow(dom.extended_omega, j, p)
                h2b.fft_many_to_device(6, k, k, coef, own, dom.omega, F.ZETA * shift % p, ws=nws, stream=stream)
                fx, sg, (l0, llast, lact) = kcos[j][0:3], kcos[j][3:7], kcos[j][7:10]
                a_p, i_p, z_p, zl_p, pa_p, ps_p = own[0:4], own[4], own[5:7], own[7], own[8], own[9]
                perm_cols = [a_p[0], a_p[1], a_p[2], i_p]
                if fused:
                    perm = dict(prods=z_p, sigmas=sg, cols=perm_cols, beta=beta, gamma=gamma, delta=F.DELTA,
                                delta_start=beta * F.ZETA % p, ext_omega=shift, omega=dom.omega,
                                chunk_len=C.CHUNK_LEN, last_rotation=-(C.BLINDING_FACTORS + 1), rot_scale=1, isize=n)
                    look = dict(rules=(bg, l_consts, l_rules, l_parts), z=zl_p, pin=pa_p, ptab=ps_p, beta=beta,
                                gamma=gamma)
                    h2b.quotient_fused_device(fx, [i_p], a_p, (no_chal, g_consts, g_rules, g_parts), y, l0, llast,
                                              lact, perm, [look], n, 1, 0, n, ext, n_parts, j,
                                              dom.t_evaluations[j], stream=stream)
                    continue
                hj = hs[j]
                h2b.quotient_device(fx, [i_p], a_p, [], g_consts, y, g_rules, g_parts, n, 1, 0, n, hj,
                                    stream=stream)
                h2b.quotient_permutation_device(hj, l0, llast, lact, z_p, sg, perm_cols, beta,
                                                gamma, sc(y), sc(F.DELTA), sc(beta * F.ZETA), sc(shift),
                                                sc(dom.omega), C.CHUNK_LEN, -(C.BLINDING_FACTORS + 1), 1, n, n,
                                                stream=stream)
                h2b.quotient_device(fx, [i_p], a_p, bg, l_consts, y, l_rules, l_parts, n, 1, 0, n, tv,
                                    stream=stream)
                h2b.quotient_lookups_device(hj, tv, zl_p, pa_p, ps_p, l0, llast, lact, d_beta, d_gamma, d_y, n,
                                            stream=stream)
            del own, tv
            if not fused:
                tab = h2b.to_dev(np.array([t.data_ptr() for t in hs], dtype=np.uint64), stream)
                h2b.call("_halo2_extended_from_lagrange_vec_device", h2b.ptr(ext), h2b.ptr(tab), n_parts, n, sh)
                h2b.call("_halo2_divide_by_vanishing_poly", h2b.ptr(ext), h2b.ptr(pk.t_evals),
                         len(dom.t_evaluations), en, sh)
            hc = h2b.dev_empty(32 * en)
            h2b.fft_many_to_device(2, dom.extended_k, dom.extended_k, [ext], [hc], dom.extended_omega_inv,
                                   dom.extended_ifft_divisor, stream=stream)
            del ext, hs
            zp = h2b.to_dev(F.fr_mont_limbs([dom.g_coset_inv, dom.g_coset]), stream)
            h2b.call("_halo2_distribute_powers_zeta", h2b.ptr(hc), h2b.ptr(zp), 2, en, sh)
            if self.check_degree:
                self.h_degree_ok = not bool(hc[32 * n * dom.quotient_poly_degree:].any().item())
            pieces = [_slice(hc, i, n) for i in range(dom.quotient_poly_degree)]
            for piece in pieces:
                commit(piece)
            flush()
            x = chal()
            # phase 5: h folded at x, the queries in the reference's order, the evaluations
            xn = pow(x, n, p)
            h_x = h2b.dev_empty(32 * n)
            h_x.zero_()
            for i, piece in enumerate(pieces):
                h2b.call("_halo2_poly_multiply_add", h2b.ptr(h_x), h2b.ptr(piece),
                         h2b.ptr(h2b.to_dev(sc(pow(xn, i, p)), stream)), n, sh)
            queries, labels = open_queries_for(dom, x, {
                **{f"adv{i}": c for i, c in enumerate(ca)}, "z0": cz[0], "z1": cz[1], "zl": czl, "pa": cpa,
                "ps": cps, **{f"fixed{i}": c for i, c in enumerate(pk.fixed)},
                **{f"sigma{i}": c for i, c in enumerate(pk.sigma)}, "h": h_x, "random": pk.random_poly})
            self.query_labels = labels
            order = transcript_eval_order(dom, x)
            cws = h2b.dev_empty(h2b.lib().h2b_msm_table_workspace_size(n, tn))
            written = []

            def commit_now(d):
                out = h2b.dev_empty(96)
                h2b.msm_device_table(d, res.table, tn, out, n, ws=cws, stream=stream)
                commits.append(out)
                absorb([out])
                return out

            def write_evals(values):
                at = dict(zip(labels, values))
                for lab in order:
                    written.append(at[lab])
                    if tr is not None:
                        tr.write_scalar(at[lab] % p)

            _, _, l_at_u = shplonk.open_queries(h2b, queries, iter(chal, None), commit_now, stream=stream,
                                                on_evals=write_evals)
            if l_at_u != 0:
                raise RuntimeError("SHPLONK linearisation does not vanish at u")
            evals = [torch.from_numpy(np.ascontiguousarray(F.fr_mont_limbs(written)).view(np.uint8).reshape(-1))]
        self.proof = tr.finalize() if tr is not None else None
        return commits, evals


def _rot(dom, x, r):
    return x * pow(dom.omega, r % dom.n, F.R_MOD) % F.R_MOD


def open_queries_for(dom, x, polys):
    """The opening's queries in the order create_proof builds them
    (halo2_proofs/src/plonk/prover.rs:569-614): advice queries, then each
    permutation set at x and w x and every set but the last at w^last x
    (permutation/prover.rs:339-379), the lookup's five (lookup/verifier.rs:
    175-210 order), fixed queries, the permutation polynomials at x, then
    h folded and the random polynomial at x.  `polys` maps labels to
    whatever stands for each polynomial (device vectors for the prover,
    commitments for the verifier).  Returns ([(poly, point)], [(label, point)])."""
    q = [(f"adv{c}", r) for c, r in C.ADVICE_QUERIES]
    sets = len(C.PERM_COLUMNS) // C.CHUNK_LEN
    for s in range(sets):
        q += [(f"z{s}", 0), (f"z{s}", 1)]
    for s in reversed(range(sets - 1)):
        q.append((f"z{s}", -(C.BLINDING_FACTORS + 1)))
    q += [("zl", 0), ("pa", 0), ("ps", 0), ("pa", -1), ("zl", 1)]
    q += [(f"fixed{c}", r) for c, r in C.FIXED_QUERIES]
    q += [(f"sigma{i}", 0) for i in range(len(C.PERM_COLUMNS))]
    q += [("h", 0), ("random", 0)]
    labels = [(lab, _rot(dom, x, r)) for lab, r in q]
    return [(polys[lab], pt) for lab, pt in labels], labels


def transcript_eval_order(dom, x):
    """The (label, point) of each evaluation in the order the prover writes
    them (prover.rs:386-560 and the verifier's reads, verifier.rs:200-225):
    advice, fixed, the random polynomial, the permutation polynomials, each
    permutation set's z(x), z(w x) and (all but the last set) z(w^last x),
    then the lookup's z(x), z(w x), A'(x), A'(w^-1 x), S'(x)."""
    o = [(f"adv{c}", r) for c, r in C.ADVICE_QUERIES]
    o += [(f"fixed{c}", r) for c, r in C.FIXED_QUERIES]
    o += [("random", 0)]
    o += [(f"sigma{i}", 0) for i in range(len(C.PERM_COLUMNS))]
    sets = len(C.PERM_COLUMNS) // C.CHUNK_LEN
    for s in range(sets):
        o += [(f"z{s}", 0), (f"z{s}", 1)]
        if s + 1 < sets:
            o.append((f"z{s}", -(C.BLINDING_FACTORS + 1)))
    o += [("zl", 0), ("zl", 1), ("pa", 0), ("pa", -1), ("ps", 0)]
    return [(lab, _rot(dom, x, r)) for lab, r in o]


def requests(count, rate, seed, ks=(16, 18, 20, 22), weights=(0.4, 0.3, 0.2, 0.1)):
    """A seeded open-loop request trace: Poisson arrivals at `rate` per second,
    k drawn from `ks` with `weights`.  Returns [(arrival_s, k, seed)]."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count) if rate > 0 else np.zeros(count)
    arrivals = np.cumsum(gaps) - gaps[0]
    kk = rng.choice(np.asarray(ks), size=count, p=np.asarray(weights) / np.sum(weights))
    return [(float(a), int(k), 1 + seed * 1000 + i) for i, (a, k) in enumerate(zip(arrivals, kk))]


class Server:
    """Runs proof requests with `slots` worker threads, each issuing on its
    own CUDA stream, so that the GPU overlaps one request's kernels with
    another's (and a small request is not stuck behind a large one).  A
    request is admitted when a slot is free and the device memory it will
    hold fits in `hbm_budget` bytes beside those in flight; `slots=1` is the
    plain one-at-a-time prover.  The workers (and their streams, forked
    streams and memory pools) persist across `serve` calls until `close`.
    Latency is arrival to completion of the request's stream, measured on the
    host clock."""

    def __init__(self, res, slots, hbm_budget, transcript=False):
        """hbm_budget counts every device byte the prover holds: the resident
        state (the SRS and its window tables, proving keys and their coset
        parts, Resident.device_bytes) and the requests in flight.
        transcript=True proves with the Fiat-Shamir transcript; each
        request's outputs then carry its proof bytes third and its public
        inputs fourth."""
        self.res, self.slots, self.budget, self.transcript = res, slots, hbm_budget, transcript
        self.in_use = 0
        self.avail = hbm_budget
        self.cv = threading.Condition()
        self.streams = [_t().cuda.Stream() for _ in range(slots)]
        self.q = queue.Queue()
        self.threads = [threading.Thread(target=self._worker, args=(s,), daemon=True) for s in range(slots)]
        for th in self.threads:
            th.start()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def close(self):
        for _ in self.threads:
            self.q.put(None)
        for th in self.threads:
            th.join()
        self.threads = []

    def bytes_for(self, k):
        """Device bytes a 2^k request holds while in flight (its polynomials
        and the scratch of 4 concurrent MSMs)."""
        n = 1 << k
        return _bytes_per_proof(k) + 4 * int(self.res.h2b.lib().h2b_msm_table_workspace_size(n, 1 << self.res.kmax))

    def _worker(self, slot):
        st = self.streams[slot]
        while True:
            job = self.q.get()
            if job is None:
                return
            k, seed, finish = job
            need = self.bytes_for(k)
            with self.cv:
                while self.in_use + need > self.avail and self.in_use > 0:
                    self.cv.wait()
                self.in_use += need
            try:
                w = ProofWorkload(self.res, k, seed, self.transcript)
                out = w.run(st)
                st.synchronize()
                if self.transcript:
                    out = (out[0], out[1], w.proof, w.public)
                finish(time.perf_counter(), out, None)
            except Exception as e:  # handed to serve(), which raises it
                finish(time.perf_counter(), None, e)
            finally:
                with self.cv:
                    self.in_use -= need
                    self.cv.notify_all()

    def serve(self, reqs, keep_outputs=False):
        """Serves `reqs` (from `requests`) in arrival order; returns a dict of
        latencies (s), the makespan and, if asked, each request's outputs."""
        torch = _t()
        for _, k, _ in reqs:
            self.res.key_cosets(k)
            self.res.lagrange_table(k)
            if self.transcript:
                self.res.verifying_key(k)
        torch.cuda.synchronize()
        self.avail = self.budget - self.res.device_bytes()
        for _, k, _ in reqs:
            if self.bytes_for(k) > self.avail:
                raise ValueError(f"a 2^{k} proof needs {self.bytes_for(k)} bytes beside the resident "
                                 f"{self.res.device_bytes()}, more than the {self.budget}-byte budget")
        done = [None] * len(reqs)
        outs = [None] * len(reqs)
        errors = []
        left = [len(reqs)]
        lock = threading.Lock()
        finished = threading.Event()
        if not reqs:
            finished.set()
        t0 = time.perf_counter()

        def finisher(i):
            def finish(t, out, err):
                done[i] = t - t0
                if err is not None:
                    errors.append(err)
                elif keep_outputs:
                    outs[i] = ([c.cpu() for c in out[0]], [e.cpu() for e in out[1]]) + tuple(out[2:])
                with lock:
                    left[0] -= 1
                    if left[0] == 0:
                        finished.set()
            return finish

        for i, (arr, k, seed) in enumerate(reqs):
            wait = arr - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            self.q.put((k, seed, finisher(i)))
        finished.wait()
        if errors:
            raise errors[0]
        lat = np.array([d - r[0] for d, r in zip(done, reqs)])
        return {"latency_s": lat, "makespan_s": float(max(done)) if done else 0.0,
                "outputs": outs if keep_outputs else None}


def summary(reqs, result):
    """proofs/s over the makespan and latency percentiles, overall and per k."""
    lat = result["latency_s"]
    ks = np.array([k for _, k, _ in reqs])
    out = {"requests": len(reqs), "proofs_per_s": round(len(reqs) / result["makespan_s"], 3),
           "makespan_s": round(result["makespan_s"], 4),
           "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 2),
           "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 2), "per_k": {}}
    for k in sorted(set(ks.tolist())):
        lk = lat[ks == k]
        out["per_k"][str(k)] = {"count": int(lk.size), "p50_ms": round(float(np.percentile(lk, 50)) * 1e3, 2),
                                "p99_ms": round(float(np.percentile(lk, 99)) * 1e3, 2)}
    return out
