// BN254 G1 (y^2 = x^3 + 3 over Fq) point arithmetic for the MSM.
//
// Affine points are 64 bytes {x, y} in Montgomery form with the point at
// infinity encoded as (0, 0) -- the halo2curves `G1Affine` memory image the
// reference passes to its MSM (halo2_proofs/cuda/include/curve/xyzz_t.hpp:49-50).
// Bucket accumulators use XYZZ coordinates (x = X/ZZ, y = Y/ZZZ, ZZ^3 = ZZZ^2,
// infinity <=> ZZ == 0) with the EFD formulas madd-2008-s (8M+2S),
// add-2008-s (12M+2S), mdbl-2008-s-1 and dbl-2008-s-1, written from the
// published formulas.  The MSM result leaves the device as the reference's
// 96-byte Jacobian image {X, Y, Z}: affine coordinates with Z = 1, or
// (0, 1, 0) for infinity (halo2_proofs/cuda/include/kernel/pippenger.h:659-668,
// halo2_proofs/cuda/include/curve/jacobian_t.hpp:64-83).
#pragma once
#include "field.cuh"
#include "inverse.cuh"
#include "lazy.cuh"
#include "lazy64.cuh"

namespace h2b {

struct G1Affine {
    Fq x, y;
};

struct G1Xyzz {
    Fq X, Y, ZZ, ZZZ;
};

struct G1Jac {
    Fq X, Y, Z;
};

H2B_DEV bool is_inf(const G1Affine& p) { return p.x.is_zero() && p.y.is_zero(); }
H2B_DEV bool is_inf(const G1Xyzz& p) { return p.ZZ.is_zero(); }

H2B_DEV G1Xyzz xyzz_inf()
{
    G1Xyzz r;
    r.X = Fq::zero(); r.Y = Fq::zero(); r.ZZ = Fq::zero(); r.ZZZ = Fq::zero();
    return r;
}

H2B_DEV G1Xyzz xyzz_from_affine(const G1Affine& p)
{
    if (is_inf(p)) return xyzz_inf();
    G1Xyzz r;
    r.X = p.x; r.Y = p.y; r.ZZ = Fq::one(); r.ZZZ = Fq::one();
    return r;
}

H2B_DEV G1Affine ld_affine(const G1Affine* p)
{
    G1Affine r;
    r.x = ldg(&p->x);
    r.y = ldg(&p->y);
    return r;
}

H2B_DEV G1Xyzz ld_xyzz(const G1Xyzz* p)
{
    G1Xyzz r;
    r.X = ld(&p->X); r.Y = ld(&p->Y); r.ZZ = ld(&p->ZZ); r.ZZZ = ld(&p->ZZZ);
    return r;
}
H2B_DEV void st_xyzz(G1Xyzz* p, const G1Xyzz& a)
{
    st(&p->X, a.X); st(&p->Y, a.Y); st(&p->ZZ, a.ZZ); st(&p->ZZZ, a.ZZZ);
}

// mdbl-2008-s-1: double an affine point into XYZZ.
H2B_DEV G1Xyzz xyzz_dbl_affine(const G1Affine& p)
{
    if (is_inf(p) || p.y.is_zero()) return xyzz_inf();
    Fq U = fdbl(p.y);
    Fq V = fsqr(U);
    Fq W = U * V;
    Fq S = p.x * V;
    Fq xx = fsqr(p.x);
    Fq M = fdbl(xx) + xx;
    G1Xyzz r;
    r.X = fsqr(M) - fdbl(S);
    r.Y = M * (S - r.X) - W * p.y;
    r.ZZ = V;
    r.ZZZ = W;
    return r;
}

// dbl-2008-s-1 (a = 0).
H2B_DEV G1Xyzz xyzz_dbl(const G1Xyzz& p)
{
    if (is_inf(p) || p.Y.is_zero()) return xyzz_inf();
    Fq U = fdbl(p.Y);
    Fq V = fsqr(U);
    Fq W = U * V;
    Fq S = p.X * V;
    Fq xx = fsqr(p.X);
    Fq M = fdbl(xx) + xx;
    G1Xyzz r;
    r.X = fsqr(M) - fdbl(S);
    r.Y = M * (S - r.X) - W * p.Y;
    r.ZZ = V * p.ZZ;
    r.ZZZ = W * p.ZZZ;
    return r;
}

// madd-2008-s: acc += q (q affine), with the exceptional cases handled.
H2B_DEV void xyzz_madd(G1Xyzz& acc, const G1Affine& q)
{
    if (is_inf(q)) return;
    if (is_inf(acc)) {
        acc.X = q.x; acc.Y = q.y; acc.ZZ = Fq::one(); acc.ZZZ = Fq::one();
        return;
    }
    Fq U2 = q.x * acc.ZZ;
    Fq S2 = q.y * acc.ZZZ;
    Fq P = U2 - acc.X;
    Fq R = S2 - acc.Y;
    if (P.is_zero()) {
        if (R.is_zero()) acc = xyzz_dbl_affine(q);
        else acc = xyzz_inf();
        return;
    }
    Fq PP = fsqr(P);
    Fq PPP = P * PP;
    Fq Q = acc.X * PP;
    Fq X3 = fsqr(R) - PPP - fdbl(Q);
    acc.Y = R * (Q - X3) - acc.Y * PPP;
    acc.X = X3;
    acc.ZZ = acc.ZZ * PP;
    acc.ZZZ = acc.ZZZ * PPP;
}

// add-2008-s: acc += q (both XYZZ).
H2B_DEV void xyzz_add(G1Xyzz& acc, const G1Xyzz& q)
{
    if (is_inf(q)) return;
    if (is_inf(acc)) { acc = q; return; }
    Fq U1 = acc.X * q.ZZ;
    Fq U2 = q.X * acc.ZZ;
    Fq S1 = acc.Y * q.ZZZ;
    Fq S2 = q.Y * acc.ZZZ;
    Fq P = U2 - U1;
    Fq R = S2 - S1;
    if (P.is_zero()) {
        if (R.is_zero()) acc = xyzz_dbl(acc);
        else acc = xyzz_inf();
        return;
    }
    Fq PP = fsqr(P);
    Fq PPP = P * PP;
    Fq Q = U1 * PP;
    Fq X3 = fsqr(R) - PPP - fdbl(Q);
    acc.Y = R * (Q - X3) - S1 * PPP;
    acc.X = X3;
    acc.ZZ = acc.ZZ * q.ZZ * PP;
    acc.ZZZ = acc.ZZZ * q.ZZZ * PPP;
}

// ---- XYZZ in 29-bit limb form (MSM bucket accumulation) -------------------
// Same madd-2008-s formula over Fl<FqCfg>: coordinates stay below 2p in limb
// form between products, so a bucket addition converts only the loaded point
// (and the accumulator when it is stored).

typedef Fl<FqCfg> FqL;

struct G1XyzzL {
    FqL X, Y, ZZ, ZZZ;
};

H2B_DEV G1XyzzL xyzzl_inf()
{
    G1XyzzL r;
    r.X = fl_zero<FqCfg>(); r.Y = fl_zero<FqCfg>(); r.ZZ = fl_zero<FqCfg>(); r.ZZZ = fl_zero<FqCfg>();
    return r;
}

H2B_DEV bool is_inf(const G1XyzzL& p) { return fl_is_zero(p.ZZ); }

H2B_DEV G1XyzzL xyzzl_from(const G1Xyzz& p)
{
    G1XyzzL r;
    r.X = to_l(p.X); r.Y = to_l(p.Y); r.ZZ = to_l(p.ZZ); r.ZZZ = to_l(p.ZZZ);
    return r;
}

// Canonical XYZZ (infinity keeps ZZ = 0).
H2B_DEV G1Xyzz xyzzl_to(const G1XyzzL& p)
{
    G1Xyzz r;
    r.X = from_l(p.X); r.Y = from_l(p.Y); r.ZZ = from_l(p.ZZ); r.ZZZ = from_l(p.ZZZ);
    return r;
}

// Product helpers by call structure: MODE 0 pairs two independent products
// per out-of-line call, MODE 1 inlines every product, MODE 2 makes one
// out-of-line call per product.
template <int MODE>
H2B_DEV Fl2<FqCfg> xl_mul2(const FqL& a0, const FqL& b0, const FqL& a1, const FqL& b1)
{
    if (MODE == 0) return fl_mul2(a0, b0, a1, b1);
    Fl2<FqCfg> r;
    if (MODE == 1) { r.a = mul29(a0, b0); r.b = mul29(a1, b1); }
    else { r.a = fl_mul(a0, b0); r.b = fl_mul(a1, b1); }
    return r;
}

template <int MODE>
H2B_DEV Fl2<FqCfg> xl_sqr2(const FqL& a0, const FqL& a1)
{
    if (MODE == 0) return fl_sqr2(a0, a1);
    Fl2<FqCfg> r;
    if (MODE == 1) { r.a = sqr29(a0); r.b = sqr29(a1); }
    else { r.a = fl_sqr(a0); r.b = fl_sqr(a1); }
    return r;
}

// madd-2008-s: acc += (qx, qy), an affine point that is not infinity.
template <int MODE = 0>
H2B_DEV void xyzzl_madd(G1XyzzL& acc, const FqL& qx, const FqL& qy)
{
    if (is_inf(acc)) {
        acc.X = qx; acc.Y = qy; acc.ZZ = to_l(Fq::one()); acc.ZZZ = acc.ZZ;
        return;
    }
    // products grouped in independent pairs: 8M + 2S in five pairs
    const Fl2<FqCfg> us = xl_mul2<MODE>(qx, acc.ZZ, qy, acc.ZZZ);     // U2, S2
    const FqL P = fl_sub(us.a, acc.X);
    const FqL R = fl_sub(us.b, acc.Y);
    if (fl_is_zero_mod(P)) {
        G1Affine q;
        q.x = from_l(qx); q.y = from_l(qy);
        acc = fl_is_zero_mod(R) ? xyzzl_from(xyzz_dbl_affine(q)) : xyzzl_inf();
        return;
    }
    const Fl2<FqCfg> sq = xl_sqr2<MODE>(P, R);                        // PP, R^2
    const Fl2<FqCfg> pq = xl_mul2<MODE>(P, sq.a, acc.X, sq.a);        // PPP, Q
    const FqL X3 = fl_sub(fl_sub(sq.b, pq.a), fl_add(pq.b, pq.b));
    const Fl2<FqCfg> yy = xl_mul2<MODE>(R, fl_sub(pq.b, X3), acc.Y, pq.a);
    const Fl2<FqCfg> zz = xl_mul2<MODE>(acc.ZZ, sq.a, acc.ZZZ, pq.a); // ZZ*PP, ZZZ*PPP
    acc.Y = fl_sub(yy.a, yy.b);
    acc.X = X3;
    acc.ZZ = zz.a;
    acc.ZZZ = zz.b;
}

// dbl-2008-s-1 and add-2008-s in limb form with out-of-line latency-oriented
// products, for the single-thread tails of the MSM (window combination, final
// doubling chain): one warp runs them, so latency sets the time; each
// product's own critical path is short and the formula's code stays small
// (fully inlined formulas measured twice as slow there).
H2B_DEV G1XyzzL xyzzl_dbl(const G1XyzzL& p)
{
    if (is_inf(p) || fl_is_zero_mod(p.Y)) return xyzzl_inf();
    const FqL U = fl_add(p.Y, p.Y);
    const FqL V = fl_sqr_ilp(U);
    const FqL xx = fl_sqr_ilp(p.X);
    const FqL W = fl_mul_ilp(U, V);
    const FqL S = fl_mul_ilp(p.X, V);
    const FqL M = fl_add(fl_add(xx, xx), xx);
    G1XyzzL r;
    r.ZZ = fl_mul_ilp(V, p.ZZ);
    r.ZZZ = fl_mul_ilp(W, p.ZZZ);
    r.X = fl_sub(fl_sqr_ilp(M), fl_add(S, S));
    r.Y = fl_sub(fl_mul_ilp(M, fl_sub(S, r.X)), fl_mul_ilp(W, p.Y));
    return r;
}

H2B_DEV void xyzzl_add(G1XyzzL& acc, const G1XyzzL& q)
{
    if (is_inf(q)) return;
    if (is_inf(acc)) { acc = q; return; }
    const FqL U1 = fl_mul_ilp(acc.X, q.ZZ);
    const FqL U2 = fl_mul_ilp(q.X, acc.ZZ);
    const FqL S1 = fl_mul_ilp(acc.Y, q.ZZZ);
    const FqL S2 = fl_mul_ilp(q.Y, acc.ZZZ);
    const FqL P = fl_sub(U2, U1);
    const FqL R = fl_sub(S2, S1);
    if (fl_is_zero_mod(P)) {
        acc = fl_is_zero_mod(R) ? xyzzl_dbl(acc) : xyzzl_inf();
        return;
    }
    const FqL PP = fl_sqr_ilp(P);
    const FqL RR = fl_sqr_ilp(R);
    const FqL zz = fl_mul_ilp(acc.ZZ, q.ZZ);
    const FqL zzz = fl_mul_ilp(acc.ZZZ, q.ZZZ);
    const FqL PPP = fl_mul_ilp(P, PP);
    const FqL Q = fl_mul_ilp(U1, PP);
    const FqL X3 = fl_sub(fl_sub(RR, PPP), fl_add(Q, Q));
    acc.Y = fl_sub(fl_mul_ilp(R, fl_sub(Q, X3)), fl_mul_ilp(S1, PPP));
    acc.X = X3;
    acc.ZZ = fl_mul_ilp(zz, PP);
    acc.ZZZ = fl_mul_ilp(zzz, PPP);
}

// ---- XYZZ in the lazy form (R = 2^261), for the bucket accumulation -------
// Bounds (multiples of p) that every step relies on are written beside it;
// products follow (1 + 0.0059 a b) p (lazy.cuh).  The accumulator keeps
// X < 5.39p, Y < 3.34p, ZZ and ZZZ < 2p from one addition to the next;
// affine inputs are qx < 1.01p (canonical, or times beta) and qy < 2p
// (canonical, or negated as 2p - y).

typedef Fz<FqCfg> FqZ;

struct G1XyzzZ {
    FqZ X, Y, ZZ, ZZZ;
};

H2B_DEV G1XyzzZ xyzzz_inf()
{
    G1XyzzZ r;
    r.X = fz_zero<FqCfg>(); r.Y = fz_zero<FqCfg>(); r.ZZ = fz_zero<FqCfg>(); r.ZZZ = fz_zero<FqCfg>();
    return r;
}

// infinity is the explicit all-zero ZZ (no other path makes ZZ vanish)
H2B_DEV bool is_inf(const G1XyzzZ& p) { return fz_is_zero(p.ZZ); }

// 2 q for an affine q (qx < 1.01p, qy < 2p, qy != 0): dbl-2008-s-1 with Z = 1.
H2B_DEV G1XyzzZ xyzzz_dbl_affine(const FqZ& qx, const FqZ& qy)
{
    const FqZ U = fz_add(qy, qy);                              // < 4p
    const Fz2<FqCfg> vx = fz_sqr2(U, qx);                      // V < 1.094p, xx < 1.006p
    const Fz2<FqCfg> ws = fz_mul2(U, vx.a, qx, vx.a);          // W < 1.026p, S < 1.0065p
    const FqZ M = fz_add(fz_add(vx.b, vx.b), vx.b);            // < 3.02p
    const Fz2<FqCfg> mm = fz_mul2(M, M, ws.a, qy);             // MM < 1.054p, W y < 1.012p
    G1XyzzZ r;
    r.X = fz_sub<FqCfg, 3>(mm.a, fz_add(ws.b, ws.b));          // 2S < 2.013p; X3 < 4.054p
    const FqZ t1 = fz_mul_call(M, fz_sub<FqCfg, 5>(ws.b, r.X)); // S - X3 + 5p < 6.007p; t1 < 1.107p
    r.Y = fz_sub<FqCfg, 2>(t1, mm.b);                          // < 3.107p
    r.ZZ = vx.a;                                               // < 1.094p
    r.ZZZ = ws.a;                                              // < 1.026p
    return r;
}

// madd-2008-s: acc += (qx, qy), q affine and not infinity.  PP and R^2 are
// formed before the equal-x test (PP == 0 mod p exactly when P is).
H2B_DEV void xyzzz_madd(G1XyzzZ& acc, const FqZ& qx, const FqZ& qy, const FqZ& one)
{
    if (is_inf(acc)) {
        acc.X = qx; acc.Y = qy; acc.ZZ = one; acc.ZZZ = one;
        return;
    }
    const Fz2<FqCfg> us = fz_mul2(qx, acc.ZZ, qy, acc.ZZZ);   // U2 < 1.012p, S2 < 1.024p
    const FqZ P = fz_sub<FqCfg, 6>(us.a, acc.X);               // X1 < 5.39p; P < 7.01p
    const FqZ R = fz_sub<FqCfg, 4>(us.b, acc.Y);               // Y1 < 3.34p; R < 5.02p
    const Fz2<FqCfg> sq = fz_sqr2(P, R);                       // PP < 1.29p, RR < 1.149p
    if (fz_is_zero_mod(sq.a)) {
        acc = fz_is_zero_mod(sq.b) ? xyzzz_dbl_affine(qx, qy) : xyzzz_inf();
        return;
    }
    const Fz2<FqCfg> pq = fz_mul2(P, sq.a, acc.X, sq.a);       // PPP < 1.053p, Q < 1.041p
    const FqZ X3 = fz_sub<FqCfg, 4>(sq.b, fz_add(pq.a, fz_add(pq.b, pq.b)));  // PPP + 2Q < 3.135p; X3 < 5.149p
    const Fz2<FqCfg> yy = fz_mul2(R, fz_sub<FqCfg, 6>(pq.b, X3), acc.Y, pq.a); // Q - X3 + 6p < 7.041p;
                                                                              // < 1.209p, < 1.021p
    const Fz2<FqCfg> zz = fz_mul2(acc.ZZ, sq.a, acc.ZZZ, pq.a); // < 1.015p, < 1.012p
    acc.Y = fz_sub<FqCfg, 2>(yy.a, yy.b);                     // < 3.209p
    acc.X = X3;
    acc.ZZ = zz.a;
    acc.ZZZ = zz.b;
}

// Stores the canonical memory image of the accumulator (infinity stays
// ZZ = 0): four products by 2^256 mod p through the shared out-of-line
// product bodies, then the conditional subtractions.  Out of line itself, so
// the rarely taken store path does not crowd the addition loop's code.
static __device__ __noinline__ void st_xyzzz(G1Xyzz* dst, const G1XyzzZ p, const FqZ r256)
{
    const Fz2<FqCfg> a = fz_mul2(p.X, r256, p.Y, r256);    // X < 5.39p, Y < 3.34p: both < 1.032p
    const Fz2<FqCfg> b = fz_mul2(p.ZZ, r256, p.ZZZ, r256);  // < 1.012p
    G1Xyzz r;
    r.X = fz_canonical(a.a); r.Y = fz_canonical(a.b);
    r.ZZ = fz_canonical(b.a); r.ZZZ = fz_canonical(b.b);
    st_xyzz(dst, r);
}

// ---- XYZZ in the FP64 lazy form (R' = 2^260), accumulate variant 6 -------
// The same formulas as the R = 2^261 form above; products follow
// (1 + 0.0118 a b) p, so the accumulator bounds are X < 5.4p, Y < 3.45p,
// ZZ and ZZZ < 1.2p (stable from one addition to the next); affine inputs
// are qx < p and qy < 2p.

typedef Fd<FqCfg> FqD;

struct G1XyzzD {
    FqD X, Y, ZZ, ZZZ;
};

H2B_DEV G1XyzzD xyzzd_inf()
{
    G1XyzzD r;
    r.X = fd_zero<FqCfg>(); r.Y = fd_zero<FqCfg>(); r.ZZ = fd_zero<FqCfg>(); r.ZZZ = fd_zero<FqCfg>();
    return r;
}

H2B_DEV bool is_inf(const G1XyzzD& p) { return fd_is_zero(p.ZZ); }

// 2 q for an affine q (qx < p, qy < 2p, qy != 0): dbl-2008-s-1 with Z = 1.
H2B_DEV G1XyzzD xyzzd_dbl_affine(const FqD& qx, const FqD& qy)
{
    const FqD U = fd_add(qy, qy);                              // < 4p
    const Fd2<FqCfg> vx = fd_mul2(U, U, qx, qx);               // V < 1.19p, xx < 1.012p
    const Fd2<FqCfg> ws = fd_mul2(U, vx.a, qx, vx.a);          // W < 1.057p, S < 1.015p
    const FqD M = fd_add(fd_add(vx.b, vx.b), vx.b);            // < 3.04p
    const Fd2<FqCfg> mm = fd_mul2(M, M, ws.a, qy);             // MM < 1.11p, W y < 1.025p
    G1XyzzD r;
    r.X = fd_sub<FqCfg, 3>(mm.a, fd_add(ws.b, ws.b));          // 2S < 2.03p; X3 < 4.11p
    const FqD t1 = fd_mul_call(M, fd_sub<FqCfg, 5>(ws.b, r.X)); // S - X3 + 5p < 6.02p; t1 < 1.22p
    r.Y = fd_sub<FqCfg, 2>(t1, mm.b);                          // < 3.22p
    r.ZZ = vx.a;                                               // < 1.19p
    r.ZZZ = ws.a;                                              // < 1.057p
    return r;
}

// madd-2008-s: acc += (qx, qy), q affine and not infinity.  PP == 0 mod p
// exactly when P is, so the equal-x test reads the square.
H2B_DEV void xyzzd_madd(G1XyzzD& acc, const FqD& qx, const FqD& qy)
{
    if (is_inf(acc)) {
        acc.X = qx; acc.Y = qy; acc.ZZ = fd_one<FqCfg>(); acc.ZZZ = fd_one<FqCfg>();
        return;
    }
    const Fd2<FqCfg> us = fd_mul2(qx, acc.ZZ, qy, acc.ZZZ);   // U2 < 1.015p, S2 < 1.03p
    const FqD P = fd_sub<FqCfg, 6>(us.a, acc.X);               // X1 < 5.4p; P < 7.02p
    const FqD R = fd_sub<FqCfg, 4>(us.b, acc.Y);               // Y1 < 3.45p; R < 5.03p
    const Fd2<FqCfg> sq = fd_mul2(P, P, R, R);                 // PP < 1.59p, RR < 1.3p
    if (fd_is_zero_mod(sq.a)) {
        acc = fd_is_zero_mod(sq.b) ? xyzzd_dbl_affine(qx, qy) : xyzzd_inf();
        return;
    }
    const Fd2<FqCfg> pq = fd_mul2(P, sq.a, acc.X, sq.a);       // PPP < 1.14p, Q < 1.11p
    const FqD X3 = fd_sub<FqCfg, 4>(sq.b, fd_add(pq.a, fd_add(pq.b, pq.b)));  // PPP + 2Q < 3.36p; X3 < 5.3p
    const Fd2<FqCfg> yy = fd_mul2(R, fd_sub<FqCfg, 6>(pq.b, X3), acc.Y, pq.a); // Q - X3 + 6p < 7.11p;
                                                                              // < 1.43p, < 1.05p
    const Fd2<FqCfg> zz = fd_mul2(acc.ZZ, sq.a, acc.ZZZ, pq.a); // < 1.03p, < 1.02p
    acc.Y = fd_sub<FqCfg, 2>(yy.a, yy.b);                     // < 3.43p
    acc.X = X3;
    acc.ZZ = zz.a;
    acc.ZZZ = zz.b;
}

// Two independent madd-2008-s additions, a0 += q0 and a1 += q1, whose
// products share out-of-line calls four at a time (the latency of one chain
// hides behind the other).  When an accumulator is at infinity or a
// square reads zero (equal x: a doubling or P + (-P)) the two additions run
// one after the other through xyzzd_madd instead; no accumulator has been
// written when that is decided.  Bounds as in xyzzd_madd.
H2B_DEV void xyzzd_madd_x2(G1XyzzD& a0, const FqD& q0x, const FqD& q0y, G1XyzzD& a1, const FqD& q1x,
                           const FqD& q1y)
{
    if (is_inf(a0) || is_inf(a1)) {
        xyzzd_madd(a0, q0x, q0y);
        xyzzd_madd(a1, q1x, q1y);
        return;
    }
    const Fd4<FqCfg> us = fd_mul4(q0x, a0.ZZ, q0y, a0.ZZZ, q1x, a1.ZZ, q1y, a1.ZZZ);
    const FqD P0 = fd_sub<FqCfg, 6>(us.a, a0.X), R0 = fd_sub<FqCfg, 4>(us.b, a0.Y);
    const FqD P1 = fd_sub<FqCfg, 6>(us.c, a1.X), R1 = fd_sub<FqCfg, 4>(us.d, a1.Y);
    const Fd4<FqCfg> sq = fd_mul4(P0, P0, R0, R0, P1, P1, R1, R1);
    if (fd_is_zero_mod(sq.a) || fd_is_zero_mod(sq.c)) {
        xyzzd_madd(a0, q0x, q0y);
        xyzzd_madd(a1, q1x, q1y);
        return;
    }
    const Fd4<FqCfg> pq = fd_mul4(P0, sq.a, a0.X, sq.a, P1, sq.c, a1.X, sq.c);
    const FqD X30 = fd_sub<FqCfg, 4>(sq.b, fd_add(pq.a, fd_add(pq.b, pq.b)));
    const FqD X31 = fd_sub<FqCfg, 4>(sq.d, fd_add(pq.c, fd_add(pq.d, pq.d)));
    const Fd4<FqCfg> yy = fd_mul4(R0, fd_sub<FqCfg, 6>(pq.b, X30), a0.Y, pq.a, R1, fd_sub<FqCfg, 6>(pq.d, X31), a1.Y,
                                  pq.c);
    const Fd4<FqCfg> zz = fd_mul4(a0.ZZ, sq.a, a0.ZZZ, pq.a, a1.ZZ, sq.c, a1.ZZZ, pq.c);
    a0.Y = fd_sub<FqCfg, 2>(yy.a, yy.b);
    a0.X = X30;
    a0.ZZ = zz.a;
    a0.ZZZ = zz.b;
    a1.Y = fd_sub<FqCfg, 2>(yy.c, yy.d);
    a1.X = X31;
    a1.ZZ = zz.c;
    a1.ZZZ = zz.d;
}

// Canonical memory image of the accumulator (infinity stays ZZ = 0): four
// products by 2^256 mod p (each below 1.07p), then conditional subtractions.
static __device__ __noinline__ G1Xyzz xyzzd_canonical(const G1XyzzD p)
{
    const FqD r256 = fd_r256<FqCfg>();
    const Fd4<FqCfg> a = fd_mul4(p.X, r256, p.Y, r256, p.ZZ, r256, p.ZZZ, r256);
    G1Xyzz r;
    r.X = fd_canonical(a.a); r.Y = fd_canonical(a.b);
    r.ZZ = fd_canonical(a.c); r.ZZZ = fd_canonical(a.d);
    return r;
}

// The sum of two accumulators, stored in the canonical memory image.
static __device__ __noinline__ void st_xyzzd_pair(G1Xyzz* dst, const G1XyzzD p0, const G1XyzzD p1)
{
    G1Xyzz r = xyzzd_canonical(p0);
    if (!is_inf(p1)) xyzz_add(r, xyzzd_canonical(p1));
    st_xyzz(dst, r);
}

static __device__ __noinline__ void st_xyzzd(G1Xyzz* dst, const G1XyzzD p)
{
    const FqD r256 = fd_r256<FqCfg>();
    const Fd2<FqCfg> a = fd_mul2(p.X, r256, p.Y, r256);
    const Fd2<FqCfg> b = fd_mul2(p.ZZ, r256, p.ZZZ, r256);
    G1Xyzz r;
    r.X = fd_canonical(a.a); r.Y = fd_canonical(a.b);
    r.ZZ = fd_canonical(b.a); r.ZZZ = fd_canonical(b.b);
    st_xyzz(dst, r);
}

// ---- lane-parallel XYZZ formulas for one warp ------------------------------
// A serial tail (the window doubling chain, the Horner combination of bit
// sums, the sum of window results) runs one point formula after another, and
// one thread needs about 1200 cycles per dependent product.  Here the whole
// warp holds the same operands and its lanes compute the independent products
// of one formula level at once (lane i mod 8 takes product i of the level),
// then every lane reads the results back by shuffle.  A doubling becomes 3
// product latencies instead of 9, an addition 4 instead of 14.  All 32 lanes
// must call these with identical arguments; every lane ends with the result.

H2B_DEV FqL lane_bcast(const FqL& v, int src)
{
    FqL r;
#pragma unroll
    for (int i = 0; i < 9; i++) r.l[i] = __shfl_sync(0xffffffffu, v.l[i], src);
    return r;
}

// operand k of a level for lane slot s = lane mod 8 (slots past the last operand repeat it)
H2B_DEV FqL lane_pick(int s, const FqL& a0, const FqL& a1, const FqL& a2, const FqL& a3, const FqL& a4,
                      const FqL& a5)
{
    FqL r;
#pragma unroll
    for (int i = 0; i < 9; i++)
        r.l[i] = s == 0 ? a0.l[i] : s == 1 ? a1.l[i] : s == 2 ? a2.l[i] : s == 3 ? a3.l[i] : s == 4 ? a4.l[i]
                                                                                                    : a5.l[i];
    return r;
}

H2B_DEV int lane_slot() { return (int)(threadIdx.x & 7); }

// dbl-2008-s-1 in three levels: {U^2, X^2}, {U V, X V, V ZZ, M^2}, {W ZZZ, M (S - X3), W Y}.
H2B_DEV G1XyzzL xyzzw_dbl(const G1XyzzL& p)
{
    if (is_inf(p) || fl_is_zero_mod(p.Y)) return xyzzl_inf();
    const int s = lane_slot();
    const FqL U = fl_add(p.Y, p.Y);
    FqL a = (s & 1) ? p.X : U;
    FqL r = fl_mul_ilp(a, a);
    const FqL V = lane_bcast(r, 0), xx = lane_bcast(r, 1);
    const FqL M = fl_add(fl_add(xx, xx), xx);
    r = fl_mul_ilp(lane_pick(s, U, p.X, V, M, M, M), lane_pick(s, V, V, p.ZZ, M, M, M));
    const FqL W = lane_bcast(r, 0), S = lane_bcast(r, 1);
    G1XyzzL o;
    o.ZZ = lane_bcast(r, 2);
    o.X = fl_sub(lane_bcast(r, 3), fl_add(S, S));
    const FqL sx = fl_sub(S, o.X);
    r = fl_mul_ilp(lane_pick(s, W, M, W, W, W, W), lane_pick(s, p.ZZZ, sx, p.Y, p.Y, p.Y, p.Y));
    o.ZZZ = lane_bcast(r, 0);
    o.Y = fl_sub(lane_bcast(r, 1), lane_bcast(r, 2));
    return o;
}

// add-2008-s in four levels: {U1, U2, S1, S2, ZZ1 ZZ2, ZZZ1 ZZZ2}, {P^2, R^2},
// {P PP, U1 PP, zz PP}, {R (Q - X3), S1 PPP, zzz PPP}.
H2B_DEV void xyzzw_add(G1XyzzL& acc, const G1XyzzL& q)
{
    if (is_inf(q)) return;
    if (is_inf(acc)) { acc = q; return; }
    const int s = lane_slot();
    FqL r = fl_mul_ilp(lane_pick(s, acc.X, q.X, acc.Y, q.Y, acc.ZZ, acc.ZZZ),
                       lane_pick(s, q.ZZ, acc.ZZ, q.ZZZ, acc.ZZZ, q.ZZ, q.ZZZ));
    const FqL U1 = lane_bcast(r, 0), S1 = lane_bcast(r, 2);
    const FqL zz = lane_bcast(r, 4), zzz = lane_bcast(r, 5);
    const FqL P = fl_sub(lane_bcast(r, 1), U1);
    const FqL R = fl_sub(lane_bcast(r, 3), S1);
    if (fl_is_zero_mod(P)) {
        acc = fl_is_zero_mod(R) ? xyzzw_dbl(acc) : xyzzl_inf();
        return;
    }
    FqL a = (s & 1) ? R : P;
    r = fl_mul_ilp(a, a);
    const FqL PP = lane_bcast(r, 0), RR = lane_bcast(r, 1);
    r = fl_mul_ilp(lane_pick(s, P, U1, zz, zz, zz, zz), PP);
    const FqL PPP = lane_bcast(r, 0), Q = lane_bcast(r, 1);
    acc.ZZ = lane_bcast(r, 2);
    const FqL X3 = fl_sub(fl_sub(RR, PPP), fl_add(Q, Q));
    r = fl_mul_ilp(lane_pick(s, R, S1, zzz, zzz, zzz, zzz), lane_pick(s, fl_sub(Q, X3), PPP, PPP, PPP, PPP, PPP));
    acc.Y = fl_sub(lane_bcast(r, 0), lane_bcast(r, 1));
    acc.ZZZ = lane_bcast(r, 2);
    acc.X = X3;
}

H2B_DEV G1Affine affine_neg(const G1Affine& p)
{
    G1Affine r;
    r.x = p.x;
    r.y = p.y.is_zero() ? p.y : fneg(p.y);
    return r;
}

H2B_DEV G1Xyzz xyzz_neg(const G1Xyzz& p)
{
    G1Xyzz r = p;
    if (!is_inf(p)) r.Y = fneg(p.Y);
    return r;
}

// XYZZ -> reference Jacobian image (affine with Z = 1; infinity = (0, 1, 0)).
H2B_DEV G1Jac xyzz_to_jac_affine(const G1Xyzz& p)
{
    G1Jac r;
    if (is_inf(p)) {
        r.X = Fq::zero(); r.Y = Fq::one(); r.Z = Fq::zero();
        return r;
    }
    Fq inv = finv_fast(p.ZZ * p.ZZZ); // 1 / (ZZ * ZZZ)
    Fq izz = inv * p.ZZZ;             // 1 / ZZ
    Fq izzz = inv * p.ZZ;             // 1 / ZZZ
    r.X = p.X * izz;
    r.Y = p.Y * izzz;
    r.Z = Fq::one();
    return r;
}

// Scalar multiplication by a small non-negative integer (double-and-add).
H2B_DEV G1Xyzz xyzz_mul_u32(const G1Xyzz& p, uint32_t k)
{
    G1Xyzz r = xyzz_inf();
    if (k == 0 || is_inf(p)) return r;
    int top = 31 - __clz(k);
#pragma unroll 1
    for (int i = top; i >= 0; i--) {
        r = xyzz_dbl(r);
        if ((k >> i) & 1u) xyzz_add(r, p);
    }
    return r;
}

} // namespace h2b
