"""The config-3 circuit family: its constraint system, keygen and witness
synthesis, all on the device except the host bookkeeping.

Columns: 4 advice (a, b, c, d), 3 fixed (q_arith, q_fib, the range table t)
and 1 instance column.  Constraints, written the way halo2's
`ConstraintSystem` would hold them after `configure`:

* gate 0, standard PLONK under a selector (degree 3):
      q_arith * (QA a + QB b + QM a b - c + K) = 0
* gate 1, Fibonacci rotation gate (degree 2):
      q_fib * (d(w^2 X) - d(w X) - d(X)) = 0
* one copy-constraint permutation over the columns [a, b, c, instance]
  (`enable_equality` order): a quarter of the usable rows wire b[r] to
  a[s(r)] for a seeded injection s, and the public inputs wire
  instance[i] to a[i] for i < NUM_PUBLIC;
* one lookup of the input expression b into the table expression t, a fixed
  column holding 0..255 (unassigned rows 0).

Derived like halo2's ConstraintSystem (halo2-axiom, the crate the reference
builds on): advice queries a, b, c, d at rotation 0 and d at rotations 1 and
2 (so blinding_factors = max(3, 3) + 2 = 5); degree max(gates 3, permutation
3, lookup max(4, 2 + 1 + 1)) = 4, so the extended domain is 4n, the
quotient has 3 pieces and each permutation set holds degree - 2 = 2 columns
(halo2_proofs/src/plonk/permutation/verifier.rs:47, the chunk_len
`vk.cs_degree - 2`).  Usable rows are [0, u) with u = n - blinding_factors - 1;
rows [u, n) of every advice column are random (witness.rs:669-702 of the
reference draws them for `n - unusable_rows_start` rows).

Keygen (`ProvingKey`) builds the fixed columns, the permutation polynomials
sigma_c(w^r) = delta^c' w^r' of the next cell (c', r') in each copy cycle, and
l_0, l_last, l_active, in Lagrange and coefficient form on the device.
`synthesize` draws a satisfying witness on the device from a seed: a and b
are small values (< 256) gathered from a table of their Montgomery images,
b copies a on the wired rows, c = QA a + QB b + QM a b + K is gathered from a
2^16-entry table indexed by (a, b), d runs the Fibonacci recurrence from two
random seeds (h2b_fibonacci_fr), and the blinding rows are random.
"""
import hashlib

import numpy as np

from . import fields as F
from . import rules as R

NUM_PUBLIC = 8
BLINDING_FACTORS = 5
DEGREE = 4
CHUNK_LEN = DEGREE - 2
TABLE_SIZE = 256

ADV_A, ADV_B, ADV_C, ADV_D = range(4)
FIX_ARITH, FIX_FIB, FIX_TABLE = range(3)
NUM_ADVICE, NUM_FIXED, NUM_INSTANCE = 4, 3, 1
# cs.advice_queries / fixed_queries / instance_queries as (column, rotation), in the order configure creates them
ADVICE_QUERIES = [(ADV_A, 0), (ADV_B, 0), (ADV_C, 0), (ADV_D, 0), (ADV_D, 1), (ADV_D, 2)]
FIXED_QUERIES = [(FIX_ARITH, 0), (FIX_FIB, 0), (FIX_TABLE, 0)]
INSTANCE_QUERIES = [(0, 0)]
# permutation columns in enable_equality order: (kind, index), kind 0 advice, 1 instance
PERM_COLUMNS = [(0, ADV_A), (0, ADV_B), (0, ADV_C), (1, 0)]


def _constant(tag):
    h = hashlib.blake2b(tag.encode(), digest_size=64).digest()
    return int.from_bytes(h, "little") % F.R_MOD


# the standard-PLONK gate's coefficients (circuit constants, q_c = -1)
QA, QB, QM, K = (_constant(f"config-3 gate {t}") for t in ("qa", "qb", "qm", "const"))


def usable_rows(n):
    return n - BLINDING_FACTORS - 1


def advice_query_index(col, rot):
    return ADVICE_QUERIES.index((col, rot))


# --- the constraint system as device rule graphs ------------------------------

def gate_graph():
    """Both gates in the reference's quotient-rule encoding: (rules, value
    parts, constants).  The value parts are the gate polynomials in order,
    folded by the evaluator as values = values * y + part."""
    g = R.Graph()
    AD, FX = R.ADVICE, R.FIXED
    a, b, c = (g.add("store", R.vs(AD, i, 0)) for i in (ADV_A, ADV_B, ADV_C))
    t = g.add("add", g.add("mul", a, g.const(QA)), g.add("mul", b, g.const(QB)))
    t = g.add("add", t, g.add("mul", g.add("mul", a, b), g.const(QM)))
    t = g.add("add", g.add("sub", t, c), g.const(K))
    gate0 = g.add("mul", t, R.vs(FX, FIX_ARITH, 0))
    f = g.add("sub", g.add("sub", R.vs(AD, ADV_D, 2), R.vs(AD, ADV_D, 1)), R.vs(AD, ADV_D, 0))
    gate1 = g.add("mul", f, R.vs(FX, FIX_FIB, 0))
    return (np.array(g.rules, dtype=np.uint64), np.array([gate0, gate1], dtype=np.uint64),
            F.fr_mont_limbs(g.constants))


def lookup_product_graph():
    """(compressed input + beta) * (compressed table + gamma) with beta and
    gamma as challenges 0 and 1: the lookup's graph that the reference's
    evaluate_h runs through compress_expressions_with_runtime_constants_device
    (halo2_proofs/src/plonk/evaluation.rs:1320-1334) to give the lookup
    quotient its product coset.  One input and one table expression, so the
    theta compression is the expression itself."""
    g = R.Graph()
    x = g.add("add", R.vs(R.ADVICE, ADV_B, 0), R.vs(R.CHAL, 0))
    t = g.add("add", R.vs(R.FIXED, FIX_TABLE, 0), R.vs(R.CHAL, 1))
    prod = g.add("mul", x, t)
    return (np.array(g.rules, dtype=np.uint64), np.array([prod], dtype=np.uint64), F.fr_mont_limbs(g.constants))


# --- the constraint system on evaluations (the verifier's side) -------------------

def gate_values(advice_evals, fixed_evals):
    """The gate polynomials at x from the opened evaluations, in the order of
    `gate_graph`'s value parts (halo2_proofs/src/plonk/verifier.rs:271-287)."""
    p = F.R_MOD
    ev = lambda c, r: advice_evals[advice_query_index(c, r)]  # noqa: E731
    a, b, c = ev(ADV_A, 0), ev(ADV_B, 0), ev(ADV_C, 0)
    g0 = fixed_evals[FIX_ARITH] * (QA * a + QB * b + QM * a * b - c + K) % p
    g1 = fixed_evals[FIX_FIB] * (ev(ADV_D, 2) - ev(ADV_D, 1) - ev(ADV_D, 0)) % p
    return [g0, g1]


# --- keygen -------------------------------------------------------------------

def wiring(n, seed):
    """The copy cycles as a map `nxt` over cells c * n + r of the permutation
    columns (order PERM_COLUMNS): every cycle here has two cells.  Returns
    (nxt, b_rows, a_rows) with b[b_rows[i]] wired to a[a_rows[i]]."""
    u = usable_rows(n)
    rng = np.random.default_rng(seed)
    b_rows = np.sort(rng.choice(u, u // 4, replace=False))
    a_rows = rng.choice(np.arange(NUM_PUBLIC, u), b_rows.size, replace=False)
    nxt = np.arange(4 * n, dtype=np.int64)
    nxt[1 * n + b_rows] = 0 * n + a_rows
    nxt[0 * n + a_rows] = 1 * n + b_rows
    pub = np.arange(NUM_PUBLIC)
    nxt[0 * n + pub] = 3 * n + pub
    nxt[3 * n + pub] = 0 * n + pub
    return nxt, b_rows, a_rows


def _torch():
    import torch
    return torch


_C_TABLE = None


def _c_table_host():
    """c = QA a + QB b + QM a b + K for every pair of small values, row 256 a + b,
    as Montgomery bytes (2^16 x 32); built once per process."""
    global _C_TABLE
    if _C_TABLE is None:
        av = np.repeat(np.arange(TABLE_SIZE), TABLE_SIZE)
        bv = np.tile(np.arange(TABLE_SIZE), TABLE_SIZE)
        cv = [(QA * int(x) + QB * int(y) + QM * int(x) * int(y) + K) % F.R_MOD for x, y in zip(av, bv)]
        _C_TABLE = np.ascontiguousarray(F.fr_mont_limbs(cv).view(np.uint8).reshape(-1, 32))
    return _C_TABLE


class ProvingKey:
    """Device state of the circuit at size 2^k: domain constants, the fixed
    and permutation columns (`fixed_values` / `sigma_values` Lagrange,
    `fixed` / `sigma` coefficients), l_0, l_last, l_active in coefficient
    form (`lag`), the wiring rows and the witness tables."""

    def __init__(self, h2b, k, seed=0xC0FFEE, stream=None):
        torch = _torch()
        self.h2b, self.k = h2b, k
        n = self.n = 1 << k
        u = self.u = usable_rows(n)
        if u - 2 < TABLE_SIZE:
            raise ValueError(f"2^{k} rows leave {u} usable rows, fewer than the {TABLE_SIZE}-entry table needs")
        self.dom = dom = F.EvaluationDomain(DEGREE, k)
        st = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(st):
            one = torch.from_numpy(F.fr_mont_limbs([1]).view(np.uint8).reshape(32)).cuda()
            small = torch.from_numpy(F.fr_mont_limbs(range(TABLE_SIZE)).view(np.uint8).reshape(TABLE_SIZE, 32)).cuda()
            self.small = small
            col = lambda: torch.zeros((n, 32), dtype=torch.uint8, device="cuda")  # noqa: E731
            q_arith, q_fib, table = col(), col(), col()
            q_arith[:u] = one
            q_fib[:u - 2] = one
            table[:TABLE_SIZE] = small
            l0, l_last = col(), col()
            l0[0] = one
            l_last[u] = one
            self.fixed_values = [t.reshape(-1) for t in (q_arith, q_fib, table)]
            lag_values = [l0.reshape(-1), l_last.reshape(-1), q_arith.reshape(-1)]    # l_active = q_arith
            # permutation: identity delta^c w^r, then each cell takes its successor's value
            pw = h2b.powers_device(dom.omega, n, st)
            ident = torch.empty((4 * n, 32), dtype=torch.uint8, device="cuda")
            ident.zero_()
            for c in range(4):
                d_dc = h2b.to_dev(F.fr_mont_limbs([pow(F.DELTA, c, F.R_MOD)]), st)
                h2b.call("_halo2_poly_multiply_add", h2b.ptr(ident[c * n:(c + 1) * n]), h2b.ptr(pw), h2b.ptr(d_dc),
                         n, h2b.stream_handle(st))
            nxt, b_rows, a_rows = wiring(n, seed)
            perm = ident[torch.from_numpy(nxt).cuda()]
            self.sigma_values = [perm[c * n:(c + 1) * n].reshape(-1) for c in range(4)]
            self.b_rows = torch.from_numpy(b_rows).cuda()
            self.a_rows = torch.from_numpy(a_rows).cuda()
            self.c_table = torch.from_numpy(_c_table_host()).cuda()
            keyv = self.fixed_values + self.sigma_values + lag_values
            coef = [h2b.dev_empty(32 * n) for _ in keyv]
            h2b.fft_many_to_device(2, k, k, keyv, coef, dom.omega_inv, dom.ifft_divisor, stream=st)
            self.fixed, self.sigma, self.lag = coef[:3], coef[3:7], coef[7:]
            self.t_evals = h2b.to_dev(F.fr_mont_limbs(dom.t_evaluations), st)
            # the constant polynomial 1: the vanishing argument's random polynomial with zk off
            rp = col()
            rp[0] = one
            self.random_poly = rp.reshape(-1)
        st.synchronize()
        self.gates = gate_graph()
        self.lookup_graph = lookup_product_graph()

    def device_bytes(self):
        """Device memory the key holds (columns, tables, coset parts excluded)."""
        return 32 * self.n * (3 + 4 + 3 + 3 + 4 + 1) + 32 * 4 * self.n + 32 * (TABLE_SIZE + TABLE_SIZE ** 2)


def synthesize(h2b, pk, seed, stream=None):
    """A satisfying witness of the 2^k circuit drawn from `seed`, on the device
    (queued on `stream`).  Returns (advice Lagrange columns [a, b, c, d] with
    random blinding rows, the instance column, the public inputs as ints)."""
    torch = _torch()
    n, u = pk.n, pk.u
    st = stream if stream is not None else torch.cuda.current_stream()
    rng = np.random.default_rng(seed)
    public = rng.integers(0, TABLE_SIZE, NUM_PUBLIC)
    fib_seeds = F.fr_mont_limbs([int(v) for v in rng.integers(1, 1 << 62, 2)])
    with torch.cuda.stream(st):
        gen = torch.Generator(device="cuda")
        gen.manual_seed(int(seed) & 0x7FFFFFFFFFFFFFFF)
        ai = torch.randint(0, TABLE_SIZE, (n,), device="cuda", generator=gen)
        bi = torch.randint(0, TABLE_SIZE, (n,), device="cuda", generator=gen)
        ai[:NUM_PUBLIC] = torch.from_numpy(public).cuda()
        bi[pk.b_rows] = ai[pk.a_rows]
        # the small values and c = QA a + QB b + QM a b + K come from tables of
        # their Montgomery images by the library's row gather
        a = h2b.gather_fr_device(pk.small, ai, st)
        b = h2b.gather_fr_device(pk.small, bi, st)
        c = h2b.gather_fr_device(pk.c_table, ai * TABLE_SIZE + bi, st)
        d = h2b.dev_empty(32 * n)
        h2b.call("h2b_fibonacci_fr", h2b.ptr(d), n, h2b.ptr(h2b.to_dev(fib_seeds, st)), h2b.stream_handle(st))
        adv = [a, b, c, d]
        for i, col in enumerate(adv):
            col[32 * u:] = h2b.random_fr_device(n - u, (seed << 3) + i, 0, st)
        inst = torch.zeros(32 * n, dtype=torch.uint8, device="cuda")
        inst[:32 * NUM_PUBLIC] = adv[ADV_A][:32 * NUM_PUBLIC]
    return adv, inst, [int(v) for v in public]


def instance_eval(dom, public, x):
    """The instance column at x from the public inputs (the verifier's
    instance_evals without instance commitments, halo2_proofs/src/plonk/
    verifier.rs:162-198): sum_i public[i] L_i(x)."""
    p, n = F.R_MOD, dom.n
    xn1 = (pow(x, n, p) - 1) % p
    ninv = pow(n, -1, p)
    acc, wi = 0, 1
    for v in public:
        acc = (acc + v * wi * xn1 * ninv * pow((x - wi) % p, -1, p)) % p
        wi = wi * dom.omega % p
    return acc
