// Lazy 29-bit limb arithmetic for the MSM bucket accumulation.
//
// The accumulation runs one mixed XYZZ addition per sorted entry; in the
// normalised limb form (field.cuh, R = 2^256) each of its seven additions and
// subtractions needs two serial carry chains and a conditional correction,
// which made the addition cost about 1.8x its ten products.  Here:
//
//  * R = 2^261 (nine full 29-bit reduction steps): p/R is 0.0059 for BN254
//    Fq, so a product of two values below a*p and b*p is below
//    (1 + 0.0059 a b) p.  Values may therefore sit well above p between
//    products ("lazy"): every bound used by the formulas below is written
//    next to the operation that relies on it.
//  * a + b and a - b + K p are limb-wise, followed by ONE parallel carry step
//    (each limb keeps its low 29 bits and adds the carry of the limb below),
//    no conditional subtraction.  Limbs then stay below 2^29 + 8 ("almost
//    normalised"), which the product's 64-bit column sums absorb: 18 terms
//    below 2^58.01 each.
//  * K p is added in a borrow-adjusted limb form (every limb below the top
//    one raised by 2^30, the next one lowered by 2) so that a_i + L_i - b_i
//    is never negative for an almost-normalised b below (K - 0.001) p.
//
// Values in this form are x * 2^261 mod p (plus multiples of p).  Affine
// bases enter as canonical x * 2^261 mod p (converted once per MSM by a shift
// and a reduction, to_r261, or stored that way in window tables); the
// results leave through one product by 2^256 mod p, which yields the memory
// image x * 2^256 mod p, then a final conditional subtraction.
#pragma once
#include "field.cuh"

namespace h2b {

template <class C>
struct Fz {
    uint32_t l[9];
};

// limb i (29-bit grid, normalised) of K * p
template <class C>
__host__ __device__ constexpr uint32_t kp29(int K, int i)
{
    uint64_t carry = 0, t = 0;
    for (int j = 0; j <= i; j++) {
        t = (uint64_t)K * p29<C>(j) + carry;
        carry = t >> 29;
        if (j < i) t &= M29;
    }
    return (uint32_t)(i < 8 ? (t & M29) : t);
}

// borrow-adjusted limb i of K * p: the same value, every limb below the top
// one at least 2^30 - 2
template <class C>
__host__ __device__ constexpr uint32_t kp29_adj(int K, int i)
{
    return kp29<C>(K, i) + (i < 8 ? (1u << 30) : 0u) - (i > 0 ? 2u : 0u);
}

// One parallel carry step: limb i keeps its low 29 bits plus the carry of
// limb i - 1; the top limb keeps everything.
template <class C>
H2B_DEV Fz<C> fz_carry(const uint32_t (&d)[9])
{
    Fz<C> r;
    r.l[0] = d[0] & M29;
#pragma unroll
    for (int i = 1; i < 8; i++) r.l[i] = (d[i] & M29) + (d[i - 1] >> 29);
    r.l[8] = d[8] + (d[7] >> 29);
    return r;
}

template <class C>
H2B_DEV Fz<C> fz_add(const Fz<C>& a, const Fz<C>& b)
{
    uint32_t d[9];
#pragma unroll
    for (int i = 0; i < 9; i++) d[i] = a.l[i] + b.l[i];
    return fz_carry<C>(d);
}

// a - b + K p.  Every limb below the top one is non-negative for any
// almost-normalised b; the top one is when b <= K p - 3 * 2^232 in value
// (kp29(K, 8) >= K p / 2^232 - 1 and b's top limb <= b / 2^232), which holds
// for every b below (K - 0.001) p.
// the borrow-adjusted limbs as compile-time constants (constexpr variables,
// so the loop in kp29 is never evaluated on the device)
template <class C, int K>
struct KP29 {
    static constexpr uint32_t l0 = kp29_adj<C>(K, 0), l1 = kp29_adj<C>(K, 1), l2 = kp29_adj<C>(K, 2),
                              l3 = kp29_adj<C>(K, 3), l4 = kp29_adj<C>(K, 4), l5 = kp29_adj<C>(K, 5),
                              l6 = kp29_adj<C>(K, 6), l7 = kp29_adj<C>(K, 7), l8 = kp29_adj<C>(K, 8);
};

template <class C, int K>
H2B_DEV Fz<C> fz_sub(const Fz<C>& a, const Fz<C>& b)
{
    using L = KP29<C, K>;
    const uint32_t kp[9] = {L::l0, L::l1, L::l2, L::l3, L::l4, L::l5, L::l6, L::l7, L::l8};
    uint32_t d[9];
#pragma unroll
    for (int i = 0; i < 9; i++) d[i] = a.l[i] + kp[i] - b.l[i];
    return fz_carry<C>(d);
}

// Montgomery product with R = 2^261: (a b + M p) / 2^261, M < 2^261 chosen
// limb by limb.  Output limbs are normalised (the top one holds the rest).
template <class C>
H2B_DEV Fz<C> fz_mul(const Fz<C>& a, const Fz<C>& b)
{
    const uint32_t np = C::N0 & M29;
    uint32_t m[9];
    uint64_t acc = 0;
#if H2B_MUL_KARATSUBA
    uint64_t T[17];
    kcols29(a.l, b.l, T);
#endif
#pragma unroll
    for (int k = 0; k < 9; k++) {
#if H2B_MUL_KARATSUBA
        acc += T[k];
#else
#pragma unroll
        for (int i = 0; i <= k; i++) acc = madw(a.l[i], b.l[k - i], acc);
#endif
#pragma unroll
        for (int i = 0; i < k; i++) acc = madw(m[i], p29<C>(k - i), acc);
        const uint32_t mk = ((uint32_t)acc * np) & M29;
        m[k] = mk;
        acc = madw(mk, p29<C>(0), acc);
        acc >>= 29;
    }
    Fz<C> r;
#pragma unroll
    for (int k = 9; k < 17; k++) {
#if H2B_MUL_KARATSUBA
        acc += T[k];
#else
#pragma unroll
        for (int i = k - 8; i <= 8; i++) acc = madw(a.l[i], b.l[k - i], acc);
#endif
#pragma unroll
        for (int i = k - 8; i <= 8; i++) acc = madw(m[i], p29<C>(k - i), acc);
        r.l[k - 9] = (uint32_t)acc & M29;
        acc >>= 29;
    }
    r.l[8] = (uint32_t)acc;
    return r;
}

// a^2: each cross product once, against the doubled limb (2 a_j < 2^30.1,
// so a doubled term stays below 2^59.1 and a column below 2^62.4).
template <class C>
H2B_DEV Fz<C> fz_sqr(const Fz<C>& a)
{
    const uint32_t np = C::N0 & M29;
    uint32_t d[9], m[9];
#pragma unroll
    for (int i = 0; i < 9; i++) d[i] = a.l[i] << 1;
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
#pragma unroll
        for (int i = 0; 2 * i < k; i++) acc = madw(a.l[i], d[k - i], acc);
        if ((k & 1) == 0) acc = madw(a.l[k / 2], a.l[k / 2], acc);
#pragma unroll
        for (int i = 0; i < k; i++) acc = madw(m[i], p29<C>(k - i), acc);
        const uint32_t mk = ((uint32_t)acc * np) & M29;
        m[k] = mk;
        acc = madw(mk, p29<C>(0), acc);
        acc >>= 29;
    }
    Fz<C> r;
#pragma unroll
    for (int k = 9; k < 17; k++) {
#pragma unroll
        for (int i = k - 8; 2 * i < k; i++) acc = madw(a.l[i], d[k - i], acc);
        if ((k & 1) == 0) acc = madw(a.l[k / 2], a.l[k / 2], acc);
#pragma unroll
        for (int i = k - 8; i <= 8; i++) acc = madw(m[i], p29<C>(k - i), acc);
        r.l[k - 9] = (uint32_t)acc & M29;
        acc >>= 29;
    }
    r.l[8] = (uint32_t)acc;
    return r;
}

template <class C>
__device__ __noinline__ Fz<C> fz_mul_call(const Fz<C> a, const Fz<C> b)
{
    return fz_mul<C>(a, b);
}

template <class C>
struct Fz2 {
    Fz<C> a, b;
};

// two independent products per out-of-line call (two dependency chains for
// the scheduler, one call overhead)
template <class C>
__device__ __noinline__ Fz2<C> fz_mul2(const Fz<C> a0, const Fz<C> b0, const Fz<C> a1, const Fz<C> b1)
{
    Fz2<C> r;
    r.a = fz_mul<C>(a0, b0);
    r.b = fz_mul<C>(a1, b1);
    return r;
}

template <class C>
__device__ __noinline__ Fz2<C> fz_sqr2(const Fz<C> a0, const Fz<C> a1)
{
    Fz2<C> r;
    r.a = fz_sqr<C>(a0);
    r.b = fz_sqr<C>(a1);
    return r;
}

template <class C>
H2B_DEV Fz<C> fz_zero()
{
    Fz<C> r;
#pragma unroll
    for (int i = 0; i < 9; i++) r.l[i] = 0;
    return r;
}

template <class C>
H2B_DEV bool fz_is_zero(const Fz<C>& a)
{
    uint32_t z = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) z |= a.l[i];
    return z == 0;
}

// a == 0 (mod p) for a product output (normalised limbs, value < 2p): a is 0 or p
template <class C>
H2B_DEV bool fz_is_zero_mod(const Fz<C>& a)
{
    uint32_t z = 0, e = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        z |= a.l[i];
        e |= a.l[i] ^ p29<C>(i);
    }
    return z == 0 || e == 0;
}

// bit-sliced view of a 256-bit word image (value < 2^256, normalised limbs)
template <class C>
H2B_DEV Fz<C> fz_from_words(const Fp<C>& a)
{
    Fl<C> t = to_l(a);
    Fz<C> r;
#pragma unroll
    for (int i = 0; i < 9; i++) r.l[i] = t.l[i];
    return r;
}

// memory image X = x 2^256 mod p -> canonical x 2^261 mod p = 32 X mod p:
// a 5-bit shift and one subtraction of q p, with q = floor(32 X / p) taken
// from the top 64 bits (q_est <= q <= q_est + 1 since p's top word M7 is
// above 2^29), then one conditional subtraction.  No product.
template <class C>
H2B_DEV Fp<C> to_r261(const Fp<C>& x)
{
    uint32_t y[9];
    y[0] = x.v[0] << 5;
#pragma unroll
    for (int i = 1; i < 8; i++) y[i] = (x.v[i] << 5) | (x.v[i - 1] >> 27);
    y[8] = x.v[7] >> 27;
    const uint64_t top = ((uint64_t)y[8] << 32) | y[7];
    const uint32_t q = (uint32_t)(top / ((uint64_t)C::M7 + 1));
    uint32_t r[8];
    uint64_t carry = 0;
    uint32_t borrow = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint64_t qp = (uint64_t)q * mword<C>(i) + carry;
        carry = qp >> 32;
        const uint64_t d = (uint64_t)y[i] - (uint32_t)qp - borrow;
        r[i] = (uint32_t)d;
        borrow = (uint32_t)(d >> 63);
    }
    Fp<C> out;
    cond_sub<C>(out.v, r);
    return out;
}

// A product output (normalised limbs, value < 2p) packed to 8 x 32 and
// reduced below p.  With a product by 2^256 mod p before it, a lazy
// x 2^261 value (below 8p) becomes the memory image x 2^256 mod p.
template <class C>
H2B_DEV Fp<C> fz_canonical(const Fz<C>& t)
{
    Fl<C> u;
#pragma unroll
    for (int i = 0; i < 9; i++) u.l[i] = t.l[i];
    return from_l(u);
}

} // namespace h2b
