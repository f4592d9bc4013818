"""Host-side encoder of quotient rule bytecode in the reference's wire format
(the role of ValueSource::encode / Calculation::encode,
halo2_proofs/src/plonk/evaluation.rs:107-352), used to build expression
graphs for the quotient evaluator (tests and the benchmark).

ValueSource (40 bits): src(4) | idx(20) << 4 | |rot|(15) << 24 | sign << 39,
with src Fixed=0, Instance=1, Advice=2, Intermediate=3, Constant=4,
Challenge=5, dummy=6.  Calculation (128 bits): low = a | c1 << 40 | d << 44,
high = b | c2 << 40, CombineType index Zero=0/One=1/NegOne=2/Two=3,
CalcDegree One=0/Two=1.
"""
import random

FIXED, INSTANCE, ADVICE, INTER, CONST, CHAL, DUMMY = range(7)


def vs(src, idx=0, rot=0):
    return src | (idx << 4) | (abs(rot) << 24) | ((1 if rot < 0 else 0) << 39)


def calc(kind, a, b=None):
    d = vs(DUMMY)
    table = {
        "add": (a, b, 1, 1, 0), "sub": (a, b, 1, 2, 0), "mul": (a, b, 1, 0, 1),
        "neg": (a, d, 2, 0, 0), "store": (a, d, 1, 0, 0), "double": (a, d, 3, 0, 0), "square": (a, a, 1, 0, 1),
    }
    A, B, c1, c2, deg = table[kind]
    return [A | (c1 << 40) | (deg << 44), B | (c2 << 40)]


class Graph:
    def __init__(self):
        self.rules = []          # flat list of u64 pairs
        self.constants = [0, 1, 2]

    def add(self, kind, a, b=None):
        self.rules += calc(kind, a, b)
        return vs(INTER, len(self.rules) // 2 - 1)

    def const(self, value):
        if value not in self.constants:
            self.constants.append(value)
        return vs(CONST, self.constants.index(value))


def plonk_and_fibonacci(g):
    """Config-3 gates: q_a*a + q_b*b + q_m*a*b + q_c*c + const and
    a(w^2 X) - a(w X) - a(X), with fixed q_a, q_b, q_m as columns 0..2 and the
    constant folded into q_c = const column via a Constant."""
    a = g.add("store", vs(ADVICE, 0, 0))
    b = g.add("store", vs(ADVICE, 1, 0))
    c = g.add("store", vs(ADVICE, 2, 0))
    qa = g.add("store", vs(FIXED, 0, 0))
    qb = g.add("store", vs(FIXED, 1, 0))
    qm = g.add("store", vs(FIXED, 2, 0))
    t1 = g.add("mul", a, qa)
    t2 = g.add("mul", b, qb)
    ab = g.add("mul", a, b)
    t3 = g.add("mul", ab, qm)
    t4 = g.add("mul", c, g.const(7))
    s = g.add("add", t1, t2)
    s = g.add("add", s, t3)
    s = g.add("add", s, t4)
    gate1 = g.add("add", s, g.const(12345))
    a1 = g.add("store", vs(ADVICE, 3, 1))
    a2 = g.add("store", vs(ADVICE, 3, 2))
    a0 = g.add("store", vs(ADVICE, 3, 0))
    f = g.add("sub", a2, a1)
    gate2 = g.add("sub", f, a0)
    inst = g.add("store", vs(INSTANCE, 0, -1))
    gate3 = g.add("mul", inst, vs(CHAL, 0))
    return [gate1, gate2, gate3]


def random_graph(rng, n_ops, num_fixed, num_instance, num_advice, num_challenges, rots=(0, 1, -1, 2, -3)):
    g = Graph()
    vals = []
    for _ in range(6):
        src = rng.choice([FIXED, ADVICE, INSTANCE] if num_instance else [FIXED, ADVICE])
        n = {FIXED: num_fixed, ADVICE: num_advice, INSTANCE: num_instance}[src]
        vals.append(g.add("store", vs(src, rng.randrange(n), rng.choice(rots))))
    for _ in range(n_ops):
        kind = rng.choice(["add", "sub", "mul", "mul", "neg", "double", "square", "store"])
        a = rng.choice(vals + [g.const(rng.randrange(1, 1 << 60))])
        b = rng.choice(vals + [vs(CHAL, rng.randrange(num_challenges))] if num_challenges else vals)
        if kind == "store":
            src = rng.choice([FIXED, ADVICE])
            n = num_fixed if src == FIXED else num_advice
            a = vs(src, rng.randrange(n), rng.choice(rots))
        vals.append(g.add(kind, a, b))
    parts = rng.sample(vals, min(5, len(vals))) + [g.const(rng.randrange(1, 1 << 60))]
    return g, parts


def vp_rules(parts):
    return list(parts)
