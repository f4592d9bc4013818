"""Generates tests/golden/golden.json with an independent pure-Python
big-integer restatement of the hot-path functions (no numpy, no C).

Pins used: the BN254 moduli and Montgomery radix, and zeta in the Montgomery
image stored by the reference (halo2_proofs/cuda/include/field/alt_bn128.hpp,
halo2_proofs/cuda/include/kernel/zeta.h); the fixed MSM test scalar of
halo2_proofs/tests/multiexp_dense_bucket_edge_equivalence.rs:48-55 is read from
that file when the reference tree is present and recorded here.

Run:  python tests/golden/make_golden.py  [reference_root]
"""
import json
import os
import random
import re
import sys

R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
Q = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
RAD = 1 << 256
ZETA_MONT = [244305545194690131, 8351807910065594880, 14266533074055306532, 404339206190769364]


def limbs(x):
    return [(x >> (64 * k)) & (2**64 - 1) for k in range(4)]


def unlimbs(ls):
    return sum(v << (64 * k) for k, v in enumerate(ls))


def mont(x, m=R):
    return x * RAD % m


def hexl(x, m=R):
    """Montgomery image of plain x as a hex string of 4 little-endian u64 limbs."""
    return [f"{v:016x}" for v in limbs(mont(x, m))]


ZETA = unlimbs(ZETA_MONT) * pow(RAD, -1, R) % R
ROOT = pow(7, (R - 1) >> 28, R)


def omega(k):
    return pow(ROOT, 1 << (28 - k), R)


def dft(a, w):
    n = len(a)
    return [sum(a[i] * pow(w, i * j, R) for i in range(n)) % R for j in range(n)]


def g_add(P, Qp):
    if P is None:
        return Qp
    if Qp is None:
        return P
    (x1, y1), (x2, y2) = P, Qp
    if x1 == x2:
        if (y1 + y2) % Q == 0:
            return None
        lam = 3 * x1 * x1 * pow(2 * y1, -1, Q) % Q
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, Q) % Q
    x3 = (lam * lam - x1 - x2) % Q
    return (x3, (lam * (x1 - x3) - y1) % Q)


def g_mul(P, s):
    acc, A = None, P
    while s:
        if s & 1:
            acc = g_add(acc, A)
        A = g_add(A, A)
        s >>= 1
    return acc


def jac_image(P):
    if P is None:
        return [[f"{0:016x}"] * 4, hexl(1, Q), [f"{0:016x}"] * 4]
    return [hexl(P[0], Q), hexl(P[1], Q), hexl(1, Q)]


def aff_image(P):
    if P is None:
        return [[f"{0:016x}"] * 4, [f"{0:016x}"] * 4]
    return [hexl(P[0], Q), hexl(P[1], Q)]


def reference_fixed_scalar(ref_root):
    path = os.path.join(ref_root, "halo2_proofs/tests/multiexp_dense_bucket_edge_equivalence.rs")
    if not os.path.exists(path):
        return None
    text = open(path).read()
    m = re.search(r"from_raw\(\[\s*([^\]]+)\]\)", text)
    if not m:
        return None
    words = [int(w.strip().rstrip(","), 0) for w in m.group(1).split(",") if w.strip()]
    return unlimbs(words[:4])


def main():
    rng = random.Random(20240601)
    out = {"meta": {"generator": "tests/golden/make_golden.py", "format": "hex u64 limbs, Montgomery form"}}
    # field products
    fm = []
    for _ in range(8):
        a, b = rng.randrange(R), rng.randrange(R)
        fm.append({"a": hexl(a), "b": hexl(b), "ab": hexl(a * b % R), "a_plus_b": hexl((a + b) % R),
                   "a_minus_b": hexl((a - b) % R), "inv_a": hexl(pow(a, -1, R))})
    out["fr_ops"] = fm
    qm = []
    for _ in range(4):
        a, b = rng.randrange(Q), rng.randrange(Q)
        qm.append({"a": hexl(a, Q), "b": hexl(b, Q), "ab": hexl(a * b % Q, Q), "inv_a": hexl(pow(a, -1, Q), Q)})
    out["fq_ops"] = qm
    # NTTs
    ntts = []
    for k in (1, 2, 3, 4):
        n = 1 << k
        a = [rng.randrange(R) for _ in range(n)]
        w = omega(k)
        winv = pow(w, -1, R)
        ninv = pow(n, -1, R)
        c = rng.randrange(1, R)
        fwd = dft(a, w)
        inv = [x * ninv % R for x in dft(a, winv)]
        part = dft([a[i] * pow(c, i, R) % R for i in range(n)], w)
        ntts.append({"k": k, "input": [hexl(x) for x in a], "omega": hexl(w), "omega_inv": hexl(winv),
                     "divisor": hexl(ninv), "coset_factor": hexl(c), "fft": [hexl(x) for x in fwd],
                     "ifft": [hexl(x) for x in inv], "coset_part": [hexl(x) for x in part]})
    out["ntt"] = ntts
    # coset extension k=2 -> ext 4 (factor 4)
    k, ek = 2, 4
    a = [rng.randrange(R) for _ in range(1 << k)]
    pad = a + [0] * ((1 << ek) - (1 << k))
    tw = [pad[i] * pow(ZETA, i % 3, R) % R for i in range(1 << ek)]
    we = omega(ek)
    out["coset_ext"] = {"k": k, "ek": ek, "input": [hexl(x) for x in a], "omega_ext": hexl(we),
                        "output": [hexl(x) for x in dft(tw, we)]}
    # MSM over a tiny SRS [tau^i] G plus special bases
    G = (1, 2)
    tau = rng.randrange(R)
    n = 6
    bases = [g_mul(G, pow(tau, i, R)) for i in range(n)]
    scal = [rng.randrange(R) for _ in range(n)]
    scal[2] = 0
    scal[4] = 1
    acc = None
    for s, P in zip(scal, bases):
        acc = g_add(acc, g_mul(P, s))
    out["msm"] = {"scalars": [hexl(s) for s in scal], "bases": [aff_image(P) for P in bases],
                  "result": jac_image(acc)}
    # all bases = G: (sum s) G
    scal2 = [rng.randrange(R) for _ in range(5)]
    out["msm_all_g"] = {"scalars": [hexl(s) for s in scal2], "result": jac_image(g_mul(G, sum(scal2) % R))}
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    fixed = reference_fixed_scalar(ref_root)
    if fixed is not None:
        out["reference_fixed_scalar"] = {"raw_limbs": [f"{v:016x}" for v in limbs(fixed)],
                                         "times_g": jac_image(g_mul(G, fixed % R))}
    # batch invert with zeros
    xs = [rng.randrange(1, R) for _ in range(9)]
    xs[3] = 0
    xs[7] = 0
    out["batch_invert"] = {"input": [hexl(x) for x in xs],
                           "output": [hexl(pow(x, -1, R) if x else 0) for x in xs]}
    # grand product
    ys = [rng.randrange(R) for _ in range(10)]
    pre = rng.randrange(R)
    gp, accv = [], pre
    for y in ys:
        accv = accv * y % R
        gp.append(accv)
    out["grand_product"] = {"input": [hexl(y) for y in ys], "prefix": hexl(pre), "output": [hexl(v) for v in gp]}
    # lookup permute: table of 4 values, input drawn from it, n = 8, usable 6
    table_vals = [rng.randrange(R) for _ in range(4)]
    n, usable = 8, 6
    table = [table_vals[i % 4] for i in range(usable)] + [0, 0]
    inp = [table_vals[rng.randrange(4)] for _ in range(usable)] + [0, 0]
    pin = sorted(inp[:usable])
    left = {}
    for t in table[:usable]:
        left[t] = left.get(t, 0) + 1
    ptab = [0] * usable
    rep = []
    for r, v in enumerate(pin):
        if r == 0 or v != pin[r - 1]:
            ptab[r] = v
            left[v] -= 1
        else:
            rep.append(r)
    for v in sorted(left):
        for _ in range(left[v]):
            ptab[rep.pop()] = v
    out["permute_pair"] = {"n": n, "usable": usable, "input": [hexl(x) for x in inp],
                           "table": [hexl(x) for x in table], "permuted_input": [hexl(x) for x in pin + [0, 0]],
                           "permuted_table": [hexl(x) for x in ptab + [0, 0]]}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
