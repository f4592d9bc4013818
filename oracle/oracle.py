"""ctypes loader for the CPU oracle (oracle.c) -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, by __graft_entry__.smoke() as the checker and by
bench.py's cpu_baseline leg.  Never used on the product path.  Arrays follow
the product's conventions: Fr/Fq elements (n, 4) uint64 Montgomery limbs,
affine points (n, 8), MSM results (12,) Jacobian images.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build():
    src = os.path.join(HERE, "oracle.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
        _lib.o_chacha_fr.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_void_p]
        _lib.o_ntt.restype = ctypes.c_int
        _lib.o_ntt.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32] + [ctypes.c_void_p] * 4
        _lib.o_msm.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p]
        _lib.o_msm_naive.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        _lib.o_batch_invert.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        _lib.o_batch_invert_par.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int]
        _lib.o_grand_product.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        _lib.o_srs.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        _lib.o_permute_pair.restype = ctypes.c_int
        _lib.o_permute_pair.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t,
                                        ctypes.c_void_p, ctypes.c_void_p]
        _lib.o_quotient.argtypes = [ctypes.c_void_p] * 7 + [ctypes.c_uint64, ctypes.c_void_p] + \
            [ctypes.c_uint64] * 5 + [ctypes.c_void_p, ctypes.c_void_p]
        _lib.o_quotient_lookups.argtypes = [ctypes.c_void_p] * 11 + [ctypes.c_size_t]
        _lib.o_permutation_quotient.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                                ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t] + \
            [ctypes.c_void_p] * 11
        _lib.o_permutation_product.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                               ctypes.c_size_t] + [ctypes.c_void_p] * 5
        _lib.o_lookup_product.argtypes = [ctypes.c_void_p] * 7 + [ctypes.c_size_t]
        _lib.o_num_threads.restype = ctypes.c_int
        _lib.o_to_mont.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
        _lib.o_from_mont.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
        _lib.o_fr_pow.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        _lib.o_fr_eval.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
        _lib.o_fr_eval_many.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.c_void_p]
        for n in ("o_field_mul", "o_field_add", "o_field_sub"):
            getattr(_lib, n).argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib.o_field_inv.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        _lib.o_g1_mul.argtypes = [ctypes.c_void_p] * 3
        _lib.o_g1_add.argtypes = [ctypes.c_void_p] * 3
        _lib.o_g1_generator.argtypes = [ctypes.c_void_p]
        _lib.o_g1_on_curve.restype = ctypes.c_int
        _lib.o_g1_on_curve.argtypes = [ctypes.c_void_p]
    return _lib


def _p(a):
    return a.ctypes.data if a is not None else None


def _fe(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint64).reshape(-1, 4))


def chacha_fr(seed, n, first=0):
    out = np.zeros((n, 4), dtype=np.uint64)
    lib().o_chacha_fr(seed, first, n, _p(out))
    return out


def ntt(ntt_type, log_n, log_ext, values, omega, divisor):
    size = 1 << (log_ext if ntt_type in (3, 4) else log_n)
    out = np.zeros((size, 4), dtype=np.uint64)
    inp, om, dv = _fe(values), _fe(omega), _fe(divisor)
    rc = lib().o_ntt(ntt_type, log_n, log_ext, _p(inp), _p(out), _p(om), _p(dv))
    if rc != 0:
        raise ValueError(f"unsupported ntt type {ntt_type}")
    return out


def msm(scalars, bases, threads=None):
    out = np.zeros(12, dtype=np.uint64)
    sc = _fe(scalars)
    bs = np.ascontiguousarray(bases, dtype=np.uint64)
    lib().o_msm(_p(sc), _p(bs), sc.shape[0], threads or lib().o_num_threads(), _p(out))
    return out


def msm_naive(scalars, bases):
    out = np.zeros(12, dtype=np.uint64)
    sc = _fe(scalars)
    bs = np.ascontiguousarray(bases, dtype=np.uint64)
    lib().o_msm_naive(_p(sc), _p(bs), sc.shape[0], _p(out))
    return out


def g1_mul(scalar, point):
    out = np.zeros(12, dtype=np.uint64)
    s = _fe(scalar)
    p = np.ascontiguousarray(point, dtype=np.uint64).reshape(8)
    lib().o_g1_mul(_p(s), _p(p), _p(out))
    return out


def g1_generator():
    g = np.zeros(8, dtype=np.uint64)
    lib().o_g1_generator(_p(g))
    return g


def g1_on_curve(point):
    p = np.ascontiguousarray(point, dtype=np.uint64).reshape(8)
    return bool(lib().o_g1_on_curve(_p(p)))


def srs(tau, n):
    out = np.zeros((n, 8), dtype=np.uint64)
    t = _fe(tau)
    lib().o_srs(_p(t), n, _p(out))
    return out


def batch_invert(values, field_type=0):
    d = _fe(values).copy()
    lib().o_batch_invert(_p(d), d.shape[0], field_type)
    return d


def batch_invert_par(values, field_type=0, threads=None):
    d = _fe(values).copy()
    lib().o_batch_invert_par(_p(d), d.shape[0], field_type, threads or lib().o_num_threads())
    return d


def grand_product(values, prefix):
    inp = _fe(values)
    out = np.zeros_like(inp)
    pf = _fe(prefix)
    lib().o_grand_product(_p(inp), _p(out), inp.shape[0], _p(pf))
    return out


def lookup_product(pin, ptab, cin, ctab, beta, gamma):
    arrs = [_fe(x) for x in (pin, ptab, cin, ctab)]
    out = np.zeros_like(arrs[0])
    b, g = _fe(beta), _fe(gamma)
    lib().o_lookup_product(_p(out), *[_p(a) for a in arrs], _p(b), _p(g), out.shape[0])
    return out


def permutation_product(modified, values, perms, omega, beta, gamma, delta, deltaomega):
    mod = _fe(modified).copy()
    vals = [_fe(v) for v in values]
    prm = [_fe(p) for p in perms]
    vp = (ctypes.c_void_p * max(len(vals), 1))(*[v.ctypes.data for v in vals])
    pp = (ctypes.c_void_p * max(len(prm), 1))(*[p.ctypes.data for p in prm])
    sc = [_fe(x) for x in (omega, beta, gamma, delta)]
    dw = _fe(deltaomega).copy()
    lib().o_permutation_product(_p(mod), vp, pp, len(vals), mod.shape[0], *[_p(s) for s in sc], _p(dw))
    return mod, dw[0]


def permute_pair(inp, table, n, usable):
    a, t = _fe(inp), _fe(table)
    pin = np.zeros((n, 4), dtype=np.uint64)
    ptab = np.zeros((n, 4), dtype=np.uint64)
    rc = lib().o_permute_pair(_p(a), _p(t), n, usable, _p(pin), _p(ptab))
    if rc != 0:
        raise ValueError("input value missing from the lookup table")
    return pin, ptab


def _ptr_array(arrs):
    return (ctypes.c_void_p * max(len(arrs), 1))(*[a.ctypes.data for a in arrs])


def quotient(fixed, instance, advice, challenges, constants, expr_constants, rules, vp_rules, num_quotient,
             rot_scale, row_start, row_end, prev=None):
    fx = [_fe(c) for c in fixed]
    ins = [_fe(c) for c in instance]
    adv = [_fe(c) for c in advice]
    ch, cs, ec = _fe(challenges) if len(challenges) else np.zeros((1, 4), np.uint64), _fe(constants), _fe(
        expr_constants)
    r = np.ascontiguousarray(rules, dtype=np.uint64)
    vp = np.ascontiguousarray(vp_rules, dtype=np.uint64)
    out = np.zeros((row_end - row_start, 4), dtype=np.uint64)
    pv = _fe(prev) if prev is not None else None
    lib().o_quotient(_ptr_array(fx), _ptr_array(ins), _ptr_array(adv), _p(ch), _p(cs), _p(ec), _p(r),
                     len(r) // 2, _p(vp), len(vp), num_quotient, rot_scale, row_start, row_end, _p(pv), _p(out))
    return out


def quotient_lookups(values, table_values, product, pin, ptab, l0, l_last, l_active, beta, gamma, y):
    v = _fe(values).copy()
    arrs = [_fe(x) for x in (table_values, product, pin, ptab, l0, l_last, l_active)]
    sc = [_fe(x) for x in (beta, gamma, y)]
    lib().o_quotient_lookups(_p(v), *[_p(a) for a in arrs], *[_p(s) for s in sc], v.shape[0])
    return v


def permutation_quotient(values, start, rot_scale, isize, last_rotation, chunk_len, cols, prods, perms, l0, l_last,
                         l_active, y, beta, gamma, delta, delta_start, cur_ext_omega, omega):
    v = _fe(values).copy()
    c = [_fe(x) for x in cols]
    pr = [_fe(x) for x in prods]
    pm = [_fe(x) for x in perms]
    ls = [_fe(x) for x in (l0, l_last, l_active)]
    sc = [_fe(x) for x in (y, beta, gamma, delta, delta_start, cur_ext_omega, omega)]
    lib().o_permutation_quotient(_p(v), start, v.shape[0], rot_scale, isize, last_rotation, chunk_len,
                                 _ptr_array(c), len(c), _ptr_array(pr), len(pr), _ptr_array(pm),
                                 *[_p(x) for x in ls], *[_p(s) for s in sc])
    return v


def fr_eval(coeffs, x):
    """sum_i c_i x^i (Montgomery limbs in and out)."""
    c = _fe(coeffs)
    xx = _fe(x)
    out = np.zeros((1, 4), dtype=np.uint64)
    lib().o_fr_eval(_p(c), c.shape[0], _p(xx), _p(out))
    return out


def fr_eval_many(coeffs, xs):
    """[sum_i c_i x^i for x in xs] (Montgomery limbs in and out), threads over the points."""
    c = _fe(coeffs)
    pts = _fe(xs)
    out = np.zeros((pts.shape[0], 4), dtype=np.uint64)
    lib().o_fr_eval_many(_p(c), c.shape[0], _p(pts), pts.shape[0], _p(out))
    return out


def num_threads():
    return lib().o_num_threads()
