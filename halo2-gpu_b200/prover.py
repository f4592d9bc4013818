"""Prover-shaped GPU workload and a serving loop around it.

`ProofWorkload.run` issues, on one stream, the device work that `create_proof`
(halo2_proofs/src/plonk/prover.rs:56-482) sends to the GPU for the config-3
circuit family (4 advice, 3 fixed, 1 instance column; a standard-PLONK gate
and a Fibonacci rotation gate; a 4-column copy permutation; one lookup into a
2^8-entry table), through this library's entry points in the reference's
order:

  1. witness columns (seeded, generated on the device: synthesis stands in);
  2. advice commitments (MSMs over the resident SRS window table);
  3. lookup: permute-sort of the input against the table, A' and S' commits;
  4. permutation grand products (2 sets of 2 columns) and lookup grand
     product, and their commits;
  5. lagrange_to_coeff of the per-proof polynomials (iNTT);
  6. per extended part (4): coset-part NTTs of every polynomial, the gate
     quotient (evaluate_h), the permutation and the lookup quotients;
  7. h: the parts gathered and brought to coefficients on the extended
     coset, and its 3 pieces committed;
  8. opening: SHPLONK over the committed polynomials at x and their
     rotations (shplonk.py), 2 commits.

The vanishing argument's random polynomial is committed with the grand
products and opened at x.  Challenges come from a seeded generator, or, with
`transcript=True`, from the Fiat-Shamir transcript (transcript.py: BLAKE2b,
Challenge255) in the reference's order: the verifying key and the public
instance rows, the advice commitments, theta, A' and S', beta and gamma, the
grand products and the random polynomial, y, the h pieces, x, the
evaluations, then SHPLONK's y, v, W, u, W'.  The witness is seeded random
data that does not satisfy the circuit, so the outputs are deterministic GPU
work, not a valid proof, and whole-proof parity needs the Rust crates.  What
this measures is the served prover's device side: proofs/s and latency when
requests of uneven k share one GPU.

`Server` runs such requests with `slots` worker threads, each on its own
stream (the GPU overlaps them), admitting a request when a slot is free and
the HBM budget allows; `plain` runs them one at a time.
"""
import hashlib
import queue
import threading
import time

import numpy as np

from . import fields as F
from . import rules as R
from . import shplonk
from . import transcript as T

NUM_PUBLIC = 8   # rows of the instance column that are public inputs (absorbed into the transcript)
# the proof's commitments in the order they are written
COMMIT_LABELS = ("adv0", "adv1", "adv2", "adv3", "pa", "ps", "z0", "z1", "zl", "hr", "h0", "h1", "h2", "W", "W2")

_torch = None


def _t():
    global _torch
    if _torch is None:
        import torch
        _torch = torch
    return _torch


def _bytes_per_proof(k):
    """Device memory one in-flight proof of size 2^k holds besides its MSM
    scratch (upper bound): 11 Lagrange and 11 coefficient polynomials, 21
    coset parts, 4 quotient parts, 8 extended-domain vectors, 2 Kate
    quotients, evaluation scratch and small tensors."""
    n = 1 << k
    return 64 * 32 * n + (64 << 20)


class Resident:
    """State kept on the device across requests: the SRS window table and,
    per k, the proving-key polynomials (fixed, sigma, Lagrange selectors) in
    coefficient form and their extended coset parts (key_cosets), the lookup
    table column and the domain constants."""

    def __init__(self, h2b, kmax, seed=0x5EED):
        self.h2b = h2b
        self.kmax = kmax
        self.tau = seed % F.R_MOD   # the synthetic SRS's trapdoor: [tau^i] G, never a ceremony
        self.srs = h2b.srs_device(seed, 1 << kmax)
        self.table = h2b.msm_table_precompute(self.srs, 1 << kmax)
        self.pk = {}
        self._lock = threading.Lock()
        self._lag_tables = {}
        g = R.Graph()
        self.parts = np.array(R.plonk_and_fibonacci(g), dtype=np.uint64)
        self.rules = np.array(g.rules, dtype=np.uint64)
        self.consts = F.fr_mont_limbs(g.constants)

    def key(self, k):
        if k not in self.pk:
            h2b, n = self.h2b, 1 << k
            dom = F.EvaluationDomain(4, k)
            rnd = lambda s: h2b.random_fr_device(n, s, 0)  # noqa: E731
            pk = {"dom": dom,
                  "fixed": [rnd(1000 * k + i) for i in range(3)],
                  "sigma": [rnd(1000 * k + 10 + i) for i in range(4)],
                  "lag": [rnd(1000 * k + 20 + i) for i in range(3)],  # l0, l_last, l_active
                  "table": h2b.random_fr_device(256, 1000 * k + 30, 0),
                  "t_evals": h2b.to_dev(F.fr_mont_limbs(dom.t_evaluations))}
            tab_col = _t().zeros(32 * n, dtype=_t().uint8, device="cuda")
            tab_col[: 32 * 256] = pk["table"]
            pk["table_col"] = tab_col
            self.pk[k] = pk
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
                dom = F.EvaluationDomain(4, k)
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
        permutation, 3 Lagrange selectors), computed once and kept resident,
        as halo2's ProvingKey keeps `fixed_cosets` and the permutation cosets
        from keygen on: a proof then transforms only its own 11 polynomials
        per part.  [part][polynomial] device vectors."""
        pk = self.key(k)
        with self._lock:
            if "cosets" not in pk:
                torch, h2b, n, dom = _t(), self.h2b, 1 << k, pk["dom"]
                keyp = pk["fixed"] + pk["sigma"] + pk["lag"]
                st = stream if stream is not None else torch.cuda.current_stream()
                cos = []
                with torch.cuda.stream(st):
                    for j in range(1 << (dom.extended_k - k)):
                        outs = [h2b.dev_empty(32 * n) for _ in keyp]
                        shift = pow(dom.extended_omega, j, F.R_MOD)
                        h2b.fft_many_to_device(6, k, k, keyp, outs, dom.omega, F.ZETA * shift % F.R_MOD, stream=st)
                        cos.append(outs)
                st.synchronize()
                pk["cosets"] = cos
        return pk["cosets"]

    def keygen(self, k, stream=None):
        """Verifying-key commitments of the 2^k key (keygen_vk's GPU part,
        halo2_proofs/src/plonk/keygen.rs:265-290): the 3 fixed and 4
        permutation polynomials, committed in one MSM batch over the resident
        SRS table (coefficient form with monomial bases: the same points as
        the Lagrange form with Lagrange bases).  Returns 96-byte device images."""
        torch, h2b = _t(), self.h2b
        pk, n, tn = self.key(k), 1 << k, 1 << self.kmax
        polys = pk["fixed"] + pk["sigma"]
        st = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(st):
            outs = [h2b.dev_empty(96) for _ in polys]
            jobs = h2b.msm_batch_jobs(polys, [self.table] * len(polys), outs, [n] * len(polys), table_n=tn)
            ws = h2b.msm_batch_workspace(jobs, len(polys), len(polys))
            h2b.msm_batch(jobs, len(polys), len(polys), ws, stream=st)
        return outs


    def vk_repr(self, k, stream=None):
        """One Fr scalar standing for the 2^k verifying key in the transcript:
        BLAKE2b of its compressed fixed and permutation commitments, mod r
        (halo2's `vk.hash_into` absorbs `vk.transcript_repr`, a BLAKE2b digest
        of the pinned verifying key; this key has no pinned form, so its
        commitments stand in).  Computed once per k."""
        if not hasattr(self, "_vk_repr"):
            self._vk_repr = {}
        if k not in self._vk_repr:
            outs = self.keygen(k, stream)
            (stream if stream is not None else _t().cuda.current_stream()).synchronize()
            h = hashlib.blake2b(digest_size=64, person=b"Halo2-Verify-Key")
            for o in outs:
                h.update(T.compress(T.commitment_to_affine(o.cpu().numpy().view(np.uint64))))
            self._vk_repr[k] = int.from_bytes(h.digest(), "little") % F.R_MOD
        return self._vk_repr[k]


def _slice(t, i, n):
    """Elements [i n, (i + 1) n) of a device field vector."""
    return t[32 * n * i: 32 * n * (i + 1)]


class ProofWorkload:
    """The device work of one proof of size 2^k (see the module docstring)."""

    def __init__(self, res, k, seed, transcript=False):
        """transcript=False draws the challenges from a generator seeded with
        `seed`; transcript=True runs the Fiat-Shamir transcript
        (transcript.Blake2bWrite): every commitment is read back and absorbed
        before the next challenge is squeezed, and `self.proof` holds the
        proof bytes (commitments and evaluations in the order written)."""
        self.res, self.k, self.seed, self.transcript = res, k, seed, transcript
        self.proof = None

    def run(self, stream):
        """Issues everything on `stream` (the calling thread blocks only where
        an entry point synchronises: the permute-sort and the permutation
        quotient); returns the commitments (96 B each) and evaluations (32 B
        each) as device tensors, complete once `stream` is."""
        torch, h2b, res = _t(), self.res.h2b, self.res
        k, n, seed = self.k, 1 << self.k, self.seed
        pk = res.key(k)
        dom = pk["dom"]
        tn = 1 << res.kmax
        tr = T.Blake2bWrite() if self.transcript else None
        if tr is None:
            rng = np.random.default_rng(seed)
            chal = lambda: int(rng.integers(1, 1 << 62))  # noqa: E731
        else:
            chal = tr.squeeze_challenge
        drawn = []
        self.challenges = drawn
        _draw = chal

        def chal():
            drawn.append(_draw())
            return drawn[-1]
        sc = lambda v: F.fr_mont_limbs([v % F.R_MOD])  # noqa: E731

        def absorb(outs):
            """Reads the phase's commitments back (waits for `stream`) and
            writes them to the transcript."""
            if tr is not None:
                for o in outs:
                    tr.write_point(T.commitment_to_affine(o.cpu().numpy().view(np.uint64)))
        with torch.cuda.stream(stream):
            commits, evals, pending = [], [], []
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
                """The commitments of one phase as one batch: each MSM on its own
                forked stream, so their serial tails overlap."""
                jobs = h2b.MsmJob * len(pending)
                jobs = jobs()
                for i, (d, out, lagr) in enumerate(pending):
                    jobs[i].d_scalars, jobs[i].d_out, jobs[i].n = d.data_ptr(), out.data_ptr(), n
                    jobs[i].d_bases = (lag_tab if lagr else res.table).data_ptr()
                    jobs[i].table_n = tn
                h2b.msm_batch(jobs, len(pending), len(pending), msm_ws, stream=stream)
                outs = [p[1] for p in pending]
                pending.clear()
                absorb(outs)

            # 1-2. witness and advice commitments
            adv = [h2b.random_fr_device(n, seed * 64 + i, 1, stream) for i in range(4)]
            inst = h2b.random_fr_device(n, seed * 64 + 4, 0, stream)
            if tr is not None:
                # the verifying key (its commitments, as one scalar) and the public inputs
                tr.common_scalar(res.vk_repr(k, stream))
                for v in F.fr_from_mont_limbs(h2b.to_host(inst[: 32 * NUM_PUBLIC])):
                    tr.common_scalar(int(v))
            for a in adv:
                commit(a, lagrange=True)
            flush()
            theta = chal()
            # 3. lookup: the input takes values of the table; permute-sort, commit A', S'
            gen = torch.Generator(device="cuda")
            gen.manual_seed(seed)
            idx = torch.randint(0, 256, (n,), device="cuda", generator=gen)
            lin = pk["table"].view(256, 32)[idx].reshape(-1)
            pa, ps = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
            h2b.permute_expression_pair_device(lin, pk["table_col"], pa, ps, n, n - 10, stream=stream)
            commit(pa, lagrange=True)
            commit(ps, lagrange=True)
            flush()
            # 4. permutation grand products (2 sets of 2 columns), lookup grand product,
            #    and the vanishing argument's random polynomial
            beta, gamma = sc(chal()), sc(chal())
            d_beta, d_gamma = h2b.to_dev(beta, stream), h2b.to_dev(gamma, stream)
            d_delta = h2b.to_dev(F.fr_mont_limbs([F.DELTA]), stream)
            d_om = h2b.to_dev(F.fr_mont_limbs([dom.omega]), stream)
            d_one = h2b.to_dev(sc(1), stream)
            zs = []
            for s in range(2):
                z = h2b.dev_empty(32 * n)
                h2b.call("_halo2_poly_fill_one", h2b.ptr(z), n, h2b.stream_handle(stream))
                d_dw = h2b.to_dev(sc(pow(F.DELTA, 2 * s, F.R_MOD)), stream)
                h2b.permutation_product_device(z, pk["sigma"][2 * s: 2 * s + 2], adv[2 * s: 2 * s + 2], d_beta,
                                               d_gamma, d_delta, d_om, d_dw, n, stream=stream)
                h2b.grand_product_device(z, d_one, n, stream=stream)
                zs.append(z)
            zl = h2b.dev_empty(32 * n)
            h2b.lookup_product_device(zl, pa, ps, lin, pk["table_col"], d_beta, d_gamma, n, stream=stream)
            h2b.grand_product_device(zl, d_one, n, stream=stream)
            for z in zs + [zl]:
                commit(z, lagrange=True)
            h_rand = h2b.random_fr_device(n, seed * 64 + 5, 0, stream)
            commit(h_rand)
            flush()
            y = chal()
            # 5. lagrange_to_coeff of the per-proof polynomials
            lag = adv + [inst] + zs + [zl, pa, ps, lin]
            coef = [h2b.dev_empty(32 * n) for _ in lag]
            h2b.fft_many_to_device(2, k, k, lag, coef, dom.omega_inv, dom.ifft_divisor, stream=stream)
            del lag
            # 6. per extended part: coset-part NTTs, gate / permutation / lookup quotients.
            #    Columns: advice 0-3, instance 4, z 5-6, lookup z 7, A' 8, S' 9,
            #    compressed input 10, fixed 11-13, sigma 14-17, l0 18, l_last 19, l_active 20.
            d_y = h2b.to_dev(sc(y), stream)
            kcos = res.key_cosets(k, stream)
            own = [h2b.dev_empty(32 * n) for _ in coef]
            hs = [h2b.dev_empty(32 * n) for _ in range(1 << (dom.extended_k - k))]
            ext_w = dom.extended_omega
            nws = h2b.dev_empty(h2b.lib()._halo2_fft_many_to_device_workspace_size(6, k, k))
            beta_v = F.fr_from_mont_limbs(beta)[0]
            for j, hj in enumerate(hs):
                shift = pow(ext_w, j, F.R_MOD)
                h2b.fft_many_to_device(6, k, k, coef, own, dom.omega, F.ZETA * shift % F.R_MOD, ws=nws,
                                       stream=stream)
                parts = own + kcos[j]
                h2b.quotient_device(parts[11:14], [parts[4]], parts[0:4], sc(theta), res.consts, y, res.rules,
                                    res.parts, n, 1, 0, n, hj, None, stream=stream)
                h2b.quotient_permutation_device(hj, parts[18], parts[19], parts[20], parts[5:7], parts[14:18],
                                                parts[0:4], beta, gamma, sc(y), F.fr_mont_limbs([F.DELTA]),
                                                sc(beta_v * F.ZETA), sc(shift), sc(dom.omega), 2, -3, 1, n, n,
                                                stream=stream)
                h2b.quotient_lookups_device(hj, parts[10], parts[7], parts[8], parts[9], parts[18], parts[19],
                                            parts[20], d_beta, d_gamma, d_y, n, stream=stream)
            del parts, own
            # 7. h on the extended coset: gather the parts, divide by the vanishing
            #    polynomial, back to coefficients (extended_to_coeff), commit its pieces
            en = len(hs) * n
            ext, hc = h2b.dev_empty(32 * en), h2b.dev_empty(32 * en)
            tab = h2b.to_dev(np.array([t.data_ptr() for t in hs], dtype=np.uint64), stream)
            h2b.call("_halo2_extended_from_lagrange_vec_device", h2b.ptr(ext), h2b.ptr(tab), len(hs), n,
                     h2b.stream_handle(stream))
            h2b.call("_halo2_divide_by_vanishing_poly", h2b.ptr(ext), h2b.ptr(pk["t_evals"]),
                     len(dom.t_evaluations), en, h2b.stream_handle(stream))
            h2b.fft_many_to_device(2, dom.extended_k, dom.extended_k, [ext], [hc], dom.extended_omega_inv,
                                   dom.extended_ifft_divisor, stream=stream)
            del ext, hs
            zp = h2b.to_dev(F.fr_mont_limbs([dom.g_coset_inv, dom.g_coset]), stream)
            h2b.call("_halo2_distribute_powers_zeta", h2b.ptr(hc), h2b.ptr(zp), 2, en, h2b.stream_handle(stream))
            for i in range(dom.quotient_poly_degree):
                commit(_slice(hc, i, n))
            flush()
            # 8. opening (SHPLONK): the committed polynomials at x and their
            #    rotations -- advice 0 at x, x w^-1; advice 3 (Fibonacci) at x, x w,
            #    x w^2; the permutation products at x, x w, x w^last; the lookup
            #    product at x, x w; A' at x, x w^-1; the rest at x
            x = chal()
            w = dom.omega
            at = lambda r: x * pow(w, r % n, F.R_MOD) % F.R_MOD  # noqa: E731
            rots = {0: (0, -1), 3: (0, 1, 2), 5: (0, 1, -3), 6: (0, 1, -3), 7: (0, 1), 8: (0, -1)}
            queries, labels = [], []
            names = {0: "adv0", 1: "adv1", 2: "adv2", 3: "adv3", 5: "z0", 6: "z1", 7: "zl", 8: "pa", 9: "ps"}
            for idx in (0, 1, 2, 3, 5, 6, 7, 8, 9):
                queries += [(coef[idx], at(r)) for r in rots.get(idx, (0,))]
                labels += [(names[idx], at(r)) for r in rots.get(idx, (0,))]
            queries += [(c, at(0)) for c in pk["fixed"] + pk["sigma"]]
            labels += [(f"vk{i}", at(0)) for i in range(len(pk["fixed"]) + len(pk["sigma"]))]
            queries += [(_slice(hc, i, n), at(0)) for i in range(dom.quotient_poly_degree)]
            labels += [(f"h{i}", at(0)) for i in range(dom.quotient_poly_degree)]
            queries += [(h_rand, at(0))]
            labels += [("hr", at(0))]
            # what a verifier needs besides the proof: each query's polynomial
            # (a label) and point, in the order the evaluations were written;
            # labels name the proof's commitments in order (COMMIT_LABELS) or
            # the verifying key's commitments ("vk0".., fixed then sigma)
            self.query_labels = labels
            cws = h2b.dev_empty(h2b.lib().h2b_msm_table_workspace_size(n, tn))

            def commit_now(d):
                out = h2b.dev_empty(96)
                h2b.msm_device_table(d, res.table, tn, out, n, ws=cws, stream=stream)
                commits.append(out)
                absorb([out])
                return out

            def write_evals(values):
                if tr is not None:
                    for e in values:
                        tr.write_scalar(e % F.R_MOD)

            opened, _, l_at_u = shplonk.open_queries(h2b, queries, iter(chal, None), commit_now, stream=stream,
                                                     on_evals=write_evals)
            if l_at_u != 0:
                raise RuntimeError("SHPLONK linearisation does not vanish at u")
            evals.append(torch.from_numpy(np.ascontiguousarray(F.fr_mont_limbs(opened)).view(np.uint8).reshape(-1)))
        self.proof = tr.finalize() if tr is not None else None
        return commits, evals


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
        """transcript=True proves with the Fiat-Shamir transcript; each
        request's outputs then carry its proof bytes third."""
        self.res, self.slots, self.budget, self.transcript = res, slots, hbm_budget, transcript
        self.in_use = 0
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
                while self.in_use + need > self.budget and self.in_use > 0:
                    self.cv.wait()
                self.in_use += need
            try:
                w = ProofWorkload(self.res, k, seed, self.transcript)
                out = w.run(st)
                st.synchronize()
                if self.transcript:
                    out = (out[0], out[1], w.proof)
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
            if self.bytes_for(k) > self.budget:
                raise ValueError(f"a 2^{k} proof needs more than the {self.budget}-byte budget")
            self.res.key_cosets(k)
            self.res.lagrange_table(k)
        torch.cuda.synchronize()
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
