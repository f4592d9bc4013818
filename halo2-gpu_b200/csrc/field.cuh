// BN254 prime-field arithmetic for sm_100a: 8 x 32-bit limbs, Montgomery form
// with R = 2^256, little-endian limb order.  Memory layout is byte-identical to
// halo2curves' `Fr` / `Fq` (4 x u64 little-endian, Montgomery form), which is
// what the reference's device type `fr_t` / `fp_t` stores
// (halo2_proofs/cuda/include/field/alt_bn128.hpp:15-43 pins the moduli,
// R^2 mod m, R mod m and n0' = -m^-1 mod 2^64).
//
// Four Montgomery products are provided: word-serial CIOS with
// `mad.lo.cc` / `madc.hi.cc` chains (mont_mul_inline), the same recurrence
// with mad.wide products (mont_mul_wide), product scanning over 29-bit limbs
// with 64-bit column sums (mul29 / mont_mul_29), and product scanning over
// 52-bit limbs on the FP64 pipe (mont_mul_f64), which is the one operator*
// uses.
// Every value handed out of this header through Fp is fully
// reduced (canonical Montgomery residue), so outputs are bit-exact with any
// other correct implementation; Fl values (29-bit limbs) are below 2p until
// from_l() reduces them.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace h2b {

#define H2B_DEV __device__ __forceinline__

// Scalar field r (halo2curves bn256::Fr); constants from alt_bn128.hpp:30-43.
struct FrCfg {
    static constexpr uint32_t M0 = 0xf0000001u, M1 = 0x43e1f593u, M2 = 0x79b97091u, M3 = 0x2833e848u,
                              M4 = 0x8181585du, M5 = 0xb85045b6u, M6 = 0xe131a029u, M7 = 0x30644e72u;
    static constexpr uint32_t N0 = 0xefffffffu;  // low word of 0xc2e1f593efffffff
    static constexpr uint64_t NP52 = 0x1f593efffffffull;  // low 52 bits of the same n'
    static constexpr uint32_t O0 = 0x4ffffffbu, O1 = 0xac96341cu, O2 = 0x9f60cd29u, O3 = 0x36fc7695u,
                              O4 = 0x7879462eu, O5 = 0x666ea36fu, O6 = 0x9a07df2fu, O7 = 0x0e0a77c1u;
    static constexpr uint32_t Q0 = 0xae216da7u, Q1 = 0x1bb8e645u, Q2 = 0xe35c59e3u, Q3 = 0x53fe3ab1u,
                              Q4 = 0x53bb8085u, Q5 = 0x8c49833du, Q6 = 0x7f4e44a5u, Q7 = 0x0216d0b1u;
};

// Base field p (halo2curves bn256::Fq); constants from alt_bn128.hpp:15-29.
struct FqCfg {
    static constexpr uint32_t M0 = 0xd87cfd47u, M1 = 0x3c208c16u, M2 = 0x6871ca8du, M3 = 0x97816a91u,
                              M4 = 0x8181585du, M5 = 0xb85045b6u, M6 = 0xe131a029u, M7 = 0x30644e72u;
    static constexpr uint32_t N0 = 0xe4866389u;  // low word of 0x87d20782e4866389
    static constexpr uint64_t NP52 = 0x20782e4866389ull;  // low 52 bits of the same n'
    static constexpr uint32_t O0 = 0xc58f0d9du, O1 = 0xd35d438du, O2 = 0xf5c70b3du, O3 = 0x0a78eb28u,
                              O4 = 0x7879462cu, O5 = 0x666ea36fu, O6 = 0x9a07df2fu, O7 = 0x0e0a77c1u;
    static constexpr uint32_t Q0 = 0x538afa89u, Q1 = 0xf32cfc5bu, Q2 = 0xd44501fbu, Q3 = 0xb5e71911u,
                              Q4 = 0x0a417ff6u, Q5 = 0x47ab1effu, Q6 = 0xcab8351fu, Q7 = 0x06d89f71u;
};

template <class C>
struct Fp {
    uint32_t v[8];

    H2B_DEV static Fp zero()
    {
        Fp r;
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = 0;
        return r;
    }
    H2B_DEV static Fp one()
    {
        Fp r;
        r.v[0] = C::O0; r.v[1] = C::O1; r.v[2] = C::O2; r.v[3] = C::O3;
        r.v[4] = C::O4; r.v[5] = C::O5; r.v[6] = C::O6; r.v[7] = C::O7;
        return r;
    }
    H2B_DEV static Fp r2()
    {
        Fp r;
        r.v[0] = C::Q0; r.v[1] = C::Q1; r.v[2] = C::Q2; r.v[3] = C::Q3;
        r.v[4] = C::Q4; r.v[5] = C::Q5; r.v[6] = C::Q6; r.v[7] = C::Q7;
        return r;
    }
    H2B_DEV bool is_zero() const
    {
        uint32_t acc = v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7];
        return acc == 0;
    }
    H2B_DEV bool operator==(const Fp& o) const
    {
        uint32_t acc = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) acc |= v[i] ^ o.v[i];
        return acc == 0;
    }
    H2B_DEV bool operator!=(const Fp& o) const { return !(*this == o); }
};

using Fr = Fp<FrCfg>;
using Fq = Fp<FqCfg>;

// One Montgomery word step: t (9 words, t < 2p on entry, t8 == 0) becomes
// (t + a*b + m*p) / 2^32 with m chosen so the low word vanishes.
template <class C>
H2B_DEV void mont_step(uint32_t (&t)[9], const uint32_t (&a)[8], uint32_t b)
{
    asm("{\n\t"
        ".reg .u32 m;\n\t"
        "mad.lo.cc.u32  %0, %9, %17, %0;\n\t"
        "madc.lo.cc.u32 %1, %10, %17, %1;\n\t"
        "madc.lo.cc.u32 %2, %11, %17, %2;\n\t"
        "madc.lo.cc.u32 %3, %12, %17, %3;\n\t"
        "madc.lo.cc.u32 %4, %13, %17, %4;\n\t"
        "madc.lo.cc.u32 %5, %14, %17, %5;\n\t"
        "madc.lo.cc.u32 %6, %15, %17, %6;\n\t"
        "madc.lo.cc.u32 %7, %16, %17, %7;\n\t"
        "addc.u32       %8, %8, 0;\n\t"
        "mad.hi.cc.u32  %1, %9, %17, %1;\n\t"
        "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"
        "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"
        "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"
        "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"
        "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"
        "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"
        "madc.hi.u32    %8, %16, %17, %8;\n\t"
        "mul.lo.u32     m, %0, %26;\n\t"
        "mad.lo.cc.u32  %0, m, %18, %0;\n\t"
        "madc.lo.cc.u32 %1, m, %19, %1;\n\t"
        "madc.lo.cc.u32 %2, m, %20, %2;\n\t"
        "madc.lo.cc.u32 %3, m, %21, %3;\n\t"
        "madc.lo.cc.u32 %4, m, %22, %4;\n\t"
        "madc.lo.cc.u32 %5, m, %23, %5;\n\t"
        "madc.lo.cc.u32 %6, m, %24, %6;\n\t"
        "madc.lo.cc.u32 %7, m, %25, %7;\n\t"
        "addc.u32       %8, %8, 0;\n\t"
        "mad.hi.cc.u32  %1, m, %18, %1;\n\t"
        "madc.hi.cc.u32 %2, m, %19, %2;\n\t"
        "madc.hi.cc.u32 %3, m, %20, %3;\n\t"
        "madc.hi.cc.u32 %4, m, %21, %4;\n\t"
        "madc.hi.cc.u32 %5, m, %22, %5;\n\t"
        "madc.hi.cc.u32 %6, m, %23, %6;\n\t"
        "madc.hi.cc.u32 %7, m, %24, %7;\n\t"
        "madc.hi.u32    %8, m, %25, %8;\n\t"
        "}"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]),
          "+r"(t[8])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b),
          "n"(C::M0), "n"(C::M1), "n"(C::M2), "n"(C::M3), "n"(C::M4), "n"(C::M5), "n"(C::M6), "n"(C::M7),
          "n"(C::N0));
    // t0 is now zero; shift one word down.
#pragma unroll
    for (int i = 0; i < 8; i++) t[i] = t[i + 1];
    t[8] = 0;
}

// r = t - m if t >= m else t  (t < 2m).
template <class C>
H2B_DEV void cond_sub(uint32_t (&r)[8], const uint32_t (&t)[8])
{
    uint32_t s[8], bw;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7]),
          "=r"(bw)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
          "n"(C::M0), "n"(C::M1), "n"(C::M2), "n"(C::M3), "n"(C::M4), "n"(C::M5), "n"(C::M6), "n"(C::M7));
#pragma unroll
    for (int i = 0; i < 8; i++) r[i] = bw ? t[i] : s[i];
}

template <class C>
H2B_DEV Fp<C> mont_mul_inline(const Fp<C>& a, const Fp<C>& b)
{
    uint32_t t[9];
#pragma unroll
    for (int i = 0; i < 9; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) mont_step<C>(t, a.v, b.v[i]);
    Fp<C> r;
    uint32_t lo[8];
#pragma unroll
    for (int i = 0; i < 8; i++) lo[i] = t[i];
    cond_sub<C>(r.v, lo);
    return r;
}

// Same CIOS recurrence with each limb product formed by one 32x32->64
// multiply-add (mad.wide.u32) and the 32-bit carry folded in with integer
// adds: on sm_100a mad.hi issues at half the rate of mad.lo, so a lo/hi pair
// costs three issue slots of the multiply pipe where one mad.wide costs about
// 1.5, and the adds go to the ALU pipe.  Every intermediate fits its word:
// a_j*b_i + t_j + c <= (2^32-1)^2 + 2(2^32-1) = 2^64 - 1.
template <class C>
H2B_DEV Fp<C> mont_mul_wide(const Fp<C>& a, const Fp<C>& b)
{
    const uint32_t P[8] = {C::M0, C::M1, C::M2, C::M3, C::M4, C::M5, C::M6, C::M7};
    uint32_t t[9];
#pragma unroll
    for (int i = 0; i < 9; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint32_t bi = b.v[i];
        uint32_t c = 0;
        uint64_t w;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            w = (uint64_t)a.v[j] * bi + t[j] + c;
            t[j] = (uint32_t)w;
            c = (uint32_t)(w >> 32);
        }
        t[8] += c;                         // t < 2p + p 2^32 < 2^287: no carry out
        const uint32_t m = t[0] * C::N0;
        w = (uint64_t)m * P[0] + t[0];     // low word becomes zero
        c = (uint32_t)(w >> 32);
#pragma unroll
        for (int j = 1; j < 8; j++) {
            w = (uint64_t)m * P[j] + t[j] + c;
            t[j - 1] = (uint32_t)w;
            c = (uint32_t)(w >> 32);
        }
        w = (uint64_t)t[8] + c;
        t[7] = (uint32_t)w;
        t[8] = (uint32_t)(w >> 32);        // zero: t < 2p after the shift
    }
    Fp<C> r;
    uint32_t lo[8];
#pragma unroll
    for (int i = 0; i < 8; i++) lo[i] = t[i];
    cond_sub<C>(r.v, lo);
    return r;
}

// Montgomery multiplication over 29-bit limbs with 64-bit column sums.
//
// A residue x R mod m (R = 2^256, the same Montgomery form as field.cuh) is
// re-sliced into nine limbs of 29 bits (the top limb holds bits 232..255).
// Each limb product is one 32x32->64 multiply-add (mad.wide.u32) into a
// 64-bit column sum; a column holds at most 18 products below 2^58 plus a
// carry below 2^35, so it never overflows and no per-product carry handling
// is needed.  On sm_100a mad.wide issues about twice as many full products per
// clock as a mad.lo/mad.hi pair, so the 162 products here (81 for a*b, 81 for
// m*p) cost fewer multiply-pipe cycles than the 264 lo/hi operations of 32-bit
// CIOS.
//
// Reduction is product-scanning Montgomery with eight 29-bit steps and a final
// 24-bit step (8*29 + 24 = 256), so R stays 2^256: m_k = (column_k * n') mod
// 2^w zeroes the low w bits of the running column.  The quotient then starts
// 5 bits into the 29-bit column grid (bit 261 - 256), and the result limbs are
// re-aligned with two shifts each.
//
// Bounds: inputs < 2p (limbs < 2^29) give a*b + M*p < 4p^2 + 2^256 p, so the
// result is < (4p/2^256 + 1) p < 2p; from_l() makes it canonical.

constexpr uint32_t M29 = (1u << 29) - 1;

template <class C>
__host__ __device__ constexpr uint32_t mword(int w)
{
    return w == 0 ? C::M0 : w == 1 ? C::M1 : w == 2 ? C::M2 : w == 3 ? C::M3 : w == 4 ? C::M4
         : w == 5 ? C::M5 : w == 6 ? C::M6 : w == 7 ? C::M7 : 0u;
}

// limb i of the modulus in the 29-bit grid
template <class C>
__host__ __device__ constexpr uint32_t p29(int i)
{
    return (uint32_t)((((uint64_t)mword<C>((29 * i) / 32)) | ((uint64_t)mword<C>((29 * i) / 32 + 1) << 32)) >>
                      ((29 * i) % 32)) & M29;
}

template <class C>
struct Fl {
    uint32_t l[9];
};

H2B_DEV uint64_t madw(uint32_t a, uint32_t b, uint64_t c) { return (uint64_t)a * b + c; }

template <class C>
H2B_DEV Fl<C> to_l(const Fp<C>& a)
{
    Fl<C> r;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        const int w = (29 * i) / 32, o = (29 * i) % 32;
        const uint32_t lo = a.v[w], hi = w + 1 < 8 ? a.v[w + 1] : 0u;
        r.l[i] = __funnelshift_r(lo, hi, o) & (i < 8 ? M29 : 0xffffffu);
    }
    return r;
}

// Packs normalised limbs (value < 2p) back to 8 x 32 and reduces below p.
template <class C>
H2B_DEV Fp<C> from_l(const Fl<C>& a)
{
    uint32_t w[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        // word j covers bits [32j, 32j + 32): limbs i0 = floor(32j/29) and i0 + 1 (and i0 + 2 for some j)
        const int i0 = (32 * j) / 29, o = 32 * j - 29 * i0;
        uint64_t x = (uint64_t)a.l[i0] >> o;
        x |= (uint64_t)(i0 + 1 < 9 ? a.l[i0 + 1] : 0u) << (29 - o);
        if (i0 + 2 < 9 && 58 - o < 32) x |= (uint64_t)a.l[i0 + 2] << (58 - o);
        w[j] = (uint32_t)x;
    }
    Fp<C> r;
    cond_sub<C>(r.v, w);
    return r;
}

// Column sums T_k = sum_{i+j=k} a_i b_j (k < 17) of two 9-limb operands by
// one Karatsuba step (5 + 4 limbs): z0 = a0 b0 and z2 = a1 b1 schoolbook,
// the middle term as (a0 + a1)(b0 + b1) - z0 - z2 with 30-bit limb sums, so 66
// limb products instead of 81.  Every column is the exact integer sum
// (no carries between columns), so the reduction that consumes them is
// unchanged.  Bounds: limbs below 2^29 + 8 give sums below 2^30.1, middle
// products below 2^60.1, five of them below 2^62.5.
// Off by default: measured on B200 it is slower despite the fewer multiplies
// (MSM at 2^22 13.59 -> 13.92 ms, 8 coset parts at 2^22 12.98 -> 13.28 ms, 8
// inverse NTTs 14.31 -> 15.80 ms): the limb sums, the 64-bit column
// subtractions and the extra live registers cost more than the 15 products,
// and the interleaved product-scanning form overlaps better.
#ifndef H2B_MUL_KARATSUBA
#define H2B_MUL_KARATSUBA 0
#endif
H2B_DEV void kcols29(const uint32_t (&a)[9], const uint32_t (&b)[9], uint64_t (&T)[17])
{
    uint32_t sa[5], sb[5];
#pragma unroll
    for (int i = 0; i < 5; i++) {
        sa[i] = a[i] + (i < 4 ? a[5 + i] : 0u);
        sb[i] = b[i] + (i < 4 ? b[5 + i] : 0u);
    }
#pragma unroll
    for (int k = 0; k < 17; k++) T[k] = 0;
    uint64_t z0[9], z2[7];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        uint64_t acc = 0;
#pragma unroll
        for (int i = 0; i < 5; i++)
            if (k - i >= 0 && k - i < 5) acc = madw(a[i], b[k - i], acc);
        z0[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < 7; k++) {
        uint64_t acc = 0;
#pragma unroll
        for (int i = 0; i < 4; i++)
            if (k - i >= 0 && k - i < 4) acc = madw(a[5 + i], b[5 + k - i], acc);
        z2[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < 9; k++) {
        uint64_t acc = 0;
#pragma unroll
        for (int i = 0; i < 5; i++)
            if (k - i >= 0 && k - i < 5) acc = madw(sa[i], sb[k - i], acc);
        acc -= z0[k];
        if (k < 7) acc -= z2[k];
        T[k] += z0[k];
        T[k + 5] += acc;
        if (k < 7) T[k + 10] += z2[k];
    }
}

template <class C>
H2B_DEV Fl<C> mul29(const Fl<C>& a, const Fl<C>& b)
{
#if H2B_MUL_KARATSUBA
    uint64_t T[17];
    kcols29(a.l, b.l, T);
#endif
    const uint32_t np = C::N0 & M29;
    uint32_t m[9];
    uint64_t acc = 0;
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
        const uint32_t mk = ((uint32_t)acc * np) & (k < 8 ? M29 : 0xffffffu);
        m[k] = mk;
        acc = madw(mk, p29<C>(0), acc);
        if (k < 8) acc >>= 29;
    }
    // acc: column 8 with its low 24 bits zero; bit 24 of it is result bit 0
    const uint32_t low5 = (uint32_t)(acc >> 24) & 31u;
    acc >>= 29;
    uint32_t h[9];
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
        h[k - 9] = (uint32_t)acc & M29;
        acc >>= 29;
    }
    h[8] = (uint32_t)acc;
    Fl<C> r;
    r.l[0] = (low5 | (h[0] << 5)) & M29;
#pragma unroll
    for (int j = 1; j < 9; j++) r.l[j] = ((h[j] << 5) | (h[j - 1] >> 24)) & M29;
    return r;
}

// Fp in, Fp out through the 29-bit product.
template <class C>
H2B_DEV Fp<C> mont_mul_29(const Fp<C>& a, const Fp<C>& b)
{
    return from_l(mul29(to_l(a), to_l(b)));
}

// Square through the same column grid: the cross products a_i a_j (i < j)
// appear twice, so they are formed once against d_i = 2 a_i (limbs < 2^30,
// products < 2^59, column sums still below 2^62): 45 products instead of 81.
template <class C>
H2B_DEV Fl<C> sqr29(const Fl<C>& a)
{
    const uint32_t np = C::N0 & M29;
    uint32_t d[9], m[9];
#pragma unroll
    for (int i = 0; i < 9; i++) d[i] = a.l[i] << 1;
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
#pragma unroll
        for (int i = 0; 2 * i < k; i++) acc = madw(d[i], a.l[k - i], acc);
        if ((k & 1) == 0) acc = madw(a.l[k / 2], a.l[k / 2], acc);
#pragma unroll
        for (int i = 0; i < k; i++) acc = madw(m[i], p29<C>(k - i), acc);
        const uint32_t mk = ((uint32_t)acc * np) & (k < 8 ? M29 : 0xffffffu);
        m[k] = mk;
        acc = madw(mk, p29<C>(0), acc);
        if (k < 8) acc >>= 29;
    }
    const uint32_t low5 = (uint32_t)(acc >> 24) & 31u;
    acc >>= 29;
    uint32_t h[9];
#pragma unroll
    for (int k = 9; k < 17; k++) {
#pragma unroll
        for (int i = k - 8; 2 * i < k; i++) acc = madw(d[i], a.l[k - i], acc);
        if ((k & 1) == 0) acc = madw(a.l[k / 2], a.l[k / 2], acc);
#pragma unroll
        for (int i = k - 8; i <= 8; i++) acc = madw(m[i], p29<C>(k - i), acc);
        h[k - 9] = (uint32_t)acc & M29;
        acc >>= 29;
    }
    h[8] = (uint32_t)acc;
    Fl<C> r;
    r.l[0] = (low5 | (h[0] << 5)) & M29;
#pragma unroll
    for (int j = 1; j < 9; j++) r.l[j] = ((h[j] << 5) | (h[j - 1] >> 24)) & M29;
    return r;
}

// Latency-oriented forms of mul29 / sqr29 (same results), for single-thread
// chains such as the MSM's final doubling chain, where nothing hides the
// latency of one product.  All limb products first go into 17 independent
// column sums; reduction step i then takes m_i from column i and adds m_i * p
// into columns i..i+8 -- nine independent multiply-adds -- so the serial
// part of a step is only m_i, m_i * p_0 and the carry into column i+1
// (mul29 chains every multiply-add of a column through one accumulator).
// Column sums stay below 2^63 as in mul29.  At full occupancy the extra
// registers make these slower than mul29 (measured 62 against 68 G/s).
template <class C>
H2B_DEV Fl<C> mont_reduce29_ilp(uint64_t (&t)[17])
{
    const uint32_t np = C::N0 & M29;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        const uint32_t mi = ((uint32_t)t[i] * np) & (i < 8 ? M29 : 0xffffffu);
#pragma unroll
        for (int j = 0; j < 9; j++) t[i + j] = madw(mi, p29<C>(j), t[i + j]);
        if (i < 8) t[i + 1] += t[i] >> 29;  // the low 29 bits of t[i] are zero now
    }
    // t[8] has its low 24 bits zero; its bit 24 is result bit 0
    const uint32_t low5 = (uint32_t)(t[8] >> 24) & 31u;
    uint64_t acc = t[8] >> 29;
    uint32_t h[9];
#pragma unroll
    for (int k = 9; k < 17; k++) {
        acc += t[k];
        h[k - 9] = (uint32_t)acc & M29;
        acc >>= 29;
    }
    h[8] = (uint32_t)acc;
    Fl<C> r;
    r.l[0] = (low5 | (h[0] << 5)) & M29;
#pragma unroll
    for (int j = 1; j < 9; j++) r.l[j] = ((h[j] << 5) | (h[j - 1] >> 24)) & M29;
    return r;
}

template <class C>
H2B_DEV Fl<C> mul29_ilp(const Fl<C>& a, const Fl<C>& b)
{
    uint64_t t[17];
#pragma unroll
    for (int k = 0; k < 17; k++) t[k] = 0;
#pragma unroll
    for (int i = 0; i < 9; i++)
#pragma unroll
        for (int j = 0; j < 9; j++) t[i + j] = madw(a.l[i], b.l[j], t[i + j]);
    return mont_reduce29_ilp<C>(t);
}

template <class C>
H2B_DEV Fl<C> sqr29_ilp(const Fl<C>& a)
{
    uint64_t t[17];
#pragma unroll
    for (int k = 0; k < 17; k++) t[k] = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        const uint32_t d = a.l[i] << 1;
        t[2 * i] = madw(a.l[i], a.l[i], t[2 * i]);
#pragma unroll
        for (int j = i + 1; j < 9; j++) t[i + j] = madw(d, a.l[j], t[i + j]);
    }
    return mont_reduce29_ilp<C>(t);
}

template <class C>
H2B_DEV Fp<C> mont_sqr_29(const Fp<C>& a)
{
    return from_l(sqr29(to_l(a)));
}

// ---- Montgomery product on the FP64 pipe ---------------------------------
//
// Five 52-bit limbs held exactly in doubles.  A limb product a b < 2^104 is
// split into its high and low 52-bit halves by two FMAs and one subtraction
// (the exact-split technique of Emmart, Zheng and Weems, "Faster modular
// exponentiation using double precision floating point arithmetic on the
// GPU", ARITH 2018):
//   h = fma_rz(a, b, 2^104)            in [2^104, 2^105): ulp 2^52, so
//                                      h = 2^104 + floor(ab / 2^52) 2^52 exactly
//   l = fma(a, b, (2^104 + 2^52) - h)  = 2^52 + (ab mod 2^52), exact
// The bit patterns of h and l are then 0x467.. + hi and 0x433.. + lo, so
// column sums are plain 64-bit integer additions of the patterns; the
// exponent fields of every term that lands in a column are subtracted once,
// through the column's initial value.
//
// Montgomery reduction runs five 52-bit digit steps (R' = 2^260): q_i =
// (t_i mod 2^52) n' mod 2^52 on the integer multiply pipe, then q_i p added
// with the same splits.  The low half of q_i p_0 cancels t_i mod 2^52 by
// construction, so only its carry (1 unless t_i mod 2^52 is 0) is added.
// One operand enters as 16 a (still below 2^260), so the result is
// a b 2^-256 like the 29-bit product.  Bounds: 16 a b + Q p < 16 p^2 + 2^260 p,
// so the result is below (p / 2^256 + 1) p < 1.19 p; one conditional
// subtraction makes it canonical.  Column values stay below 2^57.
//
// Throughput measured on B200 (two independent product chains per thread):
// 53-54 G products/s against 41-42 G for mont_mul_29.  The products use the
// FP64 pipe and the column sums the integer ALU, leaving the multiply pipe
// (which the 29-bit form saturates) almost idle.

namespace f64 {
constexpr uint64_t M52 = (1ull << 52) - 1;
constexpr uint64_t EXP_LO = 0x4330000000000000ull;  // pattern of 2^52
constexpr uint64_t EXP_HI = 0x4670000000000000ull;  // pattern of 2^104
constexpr double C52 = 4503599627370496.0;
constexpr double C104 = 20282409603651670423947251286016.0;
constexpr double C104_52 = 20282409603651670423947251286016.0 + 4503599627370496.0;

// an integer below 2^52 as a double: the pattern of 2^52 + x, minus 2^52
H2B_DEV double u52d(uint64_t x) { return __dsub_rn(__longlong_as_double((long long)(x | EXP_LO)), C52); }
H2B_DEV uint64_t dbits(double x) { return (uint64_t)__double_as_longlong(x); }

// bits [S, S + 52) of the 256-bit value v (S < 0: zeros below bit 0)
template <int S>
H2B_DEV uint64_t bits52(const uint32_t (&v)[8])
{
    uint64_t r = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        const int off = 32 * w - S;
        if (off >= 0 && off < 52) r |= (uint64_t)v[w] << off;
        else if (off < 0 && off > -32) r |= (uint64_t)(v[w] >> (-off));
    }
    return r & M52;
}

// limb i of the modulus in the 52-bit grid
template <class C>
__host__ __device__ constexpr uint64_t p52(int i)
{
    uint64_t r = 0;
    for (int w = 0; w < 8; w++) {
        const int off = 32 * w - 52 * i;
        if (off >= 0 && off < 52) r |= (uint64_t)mword<C>(w) << off;
        else if (off < 0 && off > -32) r |= (uint64_t)(mword<C>(w) >> (-off));
    }
    return r & M52;
}

// how many low and high halves land in column k (product and reduction)
__host__ __device__ constexpr uint64_t bias(int k)
{
    uint64_t nl = 0, nh = 0;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            nl += (i + j == k);
            nh += (i + j + 1 == k) * 2;     // product hi, reduction hi (j = 0 included)
            nl += (j > 0 && i + j == k);    // reduction lo (j = 0 cancels)
        }
    return nl * EXP_LO + nh * EXP_HI;
}
}  // namespace f64

// The Montgomery core over 52-bit limbs: l = A B / 2^260 + (multiple of p
// absorbed), limbs normalised below 2^52 except the top one, which holds the
// rest.  A and B are limbs below 2^52 held exactly in doubles (any value
// below 2^260); the result is below A B / 2^260 + p.
namespace f64 {
template <class C>
H2B_DEV void mont52(const double (&A)[5], const double (&B)[5], uint64_t (&l)[5])
{
    // every constant below is a constexpr variable, so it is folded at
    // compile time (a constexpr call in a plain expression may be evaluated
    // on the device)
    constexpr uint64_t B0 = bias(0), B1 = bias(1), B2 = bias(2), B3 = bias(3), B4 = bias(4);
    constexpr uint64_t B5 = bias(5), B6 = bias(6), B7 = bias(7), B8 = bias(8), B9 = bias(9);
    constexpr double P0 = (double)p52<C>(0), P1 = (double)p52<C>(1), P2 = (double)p52<C>(2);
    constexpr double P3 = (double)p52<C>(3), P4 = (double)p52<C>(4);
    constexpr uint64_t NP = C::NP52;
    const double PD[5] = {P0, P1, P2, P3, P4};
    uint64_t col[10] = {0 - B0, 0 - B1, 0 - B2, 0 - B3, 0 - B4, 0 - B5, 0 - B6, 0 - B7, 0 - B8, 0 - B9};
#pragma unroll
    for (int i = 0; i < 5; i++) {
        uint64_t hp = 0;
#pragma unroll
        for (int j = 0; j < 5; j++) {
            const double h = __fma_rz(A[i], B[j], C104);
            const double lo = __fma_rn(A[i], B[j], __dsub_rn(C104_52, h));
            col[i + j] = j == 0 ? col[i + j] + dbits(lo) : col[i + j] + (dbits(lo) + hp);
            hp = dbits(h);
        }
        col[i + 5] += hp;
    }
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const uint64_t t = col[i];
        const uint64_t tl = t & M52;
        const double qd = u52d((tl * NP) & M52);
        uint64_t hp = dbits(__fma_rz(qd, PD[0], C104)) + (t >> 52) + (tl != 0 ? 1u : 0u);
#pragma unroll
        for (int j = 1; j < 5; j++) {
            const double pj = PD[j];
            const double h = __fma_rz(qd, pj, C104);
            const double lo = __fma_rn(qd, pj, __dsub_rn(C104_52, h));
            col[i + j] = col[i + j] + (dbits(lo) + hp);
            hp = dbits(h);
        }
        col[i + 5] += hp;
    }
    uint64_t c = 0;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const uint64_t x = col[5 + k] + c;
        l[k] = k < 4 ? (x & M52) : x;
        c = x >> 52;
    }
}
}  // namespace f64

template <class C>
H2B_DEV Fp<C> mont_mul_f64(const Fp<C>& a, const Fp<C>& b)
{
    using namespace f64;
    double A[5], B[5];
    A[0] = u52d(bits52<-4>(a.v)); A[1] = u52d(bits52<48>(a.v)); A[2] = u52d(bits52<100>(a.v));
    A[3] = u52d(bits52<152>(a.v)); A[4] = u52d(bits52<204>(a.v));
    B[0] = u52d(bits52<0>(b.v)); B[1] = u52d(bits52<52>(b.v)); B[2] = u52d(bits52<104>(b.v));
    B[3] = u52d(bits52<156>(b.v)); B[4] = u52d(bits52<208>(b.v));
    uint64_t l[5];
    mont52<C>(A, B, l);
    // 52-bit limbs -> 8 x 32 words
    uint32_t w[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int i0 = (32 * j) / 52, o = 32 * j - 52 * i0;
        uint64_t x = l[i0] >> o;
        if (i0 + 1 < 5) x |= l[i0 + 1] << (52 - o);
        w[j] = (uint32_t)x;
    }
    Fp<C> r;
    cond_sub<C>(r.v, w);
    return r;
}

// ---- residues in [0, 2p) ----------------------------------------------------
// A chain of products and sums (an NTT pass) can keep its values in [0, 2p)
// and make them canonical once at the end.  The FP64 product's bound with
// a, b < 2p: 16 a b + Q p < 64 p^2 + 2^260 p, so the result is below
// (64 p / 2^260 + 1) p < 1.76 p for both BN254 moduli (p < 2^253.6), and its closing
// subtraction can be left out; a sum below 4p (< 2^256) or a difference in
// (-2p, 2p) takes one correction by 2p.  Column bounds of the product do not
// depend on the operands' size (every limb is below 2^52 and 16 a < 2^260).

// word w of 2m (8 x 32 grid)
template <class C>
__host__ __device__ constexpr uint32_t m2word(int w)
{
    return (mword<C>(w) << 1) | (w > 0 ? mword<C>(w - 1) >> 31 : 0u);
}

// a b 2^-256 mod p in [0, 2p) for a, b < 2p
template <class C>
H2B_DEV Fp<C> mont_mul_f64_lazy(const Fp<C>& a, const Fp<C>& b)
{
    using namespace f64;
    double A[5], B[5];
    A[0] = u52d(bits52<-4>(a.v)); A[1] = u52d(bits52<48>(a.v)); A[2] = u52d(bits52<100>(a.v));
    A[3] = u52d(bits52<152>(a.v)); A[4] = u52d(bits52<204>(a.v));
    B[0] = u52d(bits52<0>(b.v)); B[1] = u52d(bits52<52>(b.v)); B[2] = u52d(bits52<104>(b.v));
    B[3] = u52d(bits52<156>(b.v)); B[4] = u52d(bits52<208>(b.v));
    uint64_t l[5];
    mont52<C>(A, B, l);
    Fp<C> r;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int i0 = (32 * j) / 52, o = 32 * j - 52 * i0;
        uint64_t x = l[i0] >> o;
        if (i0 + 1 < 5) x |= l[i0 + 1] << (52 - o);
        r.v[j] = (uint32_t)x;
    }
    return r;
}

// (a + b) mod 2p in [0, 2p) for a, b < 2p
template <class C>
H2B_DEV Fp<C> add2p(const Fp<C>& a, const Fp<C>& b)
{
    uint32_t t[8], s[8], bw;
    asm("add.cc.u32  %0, %8, %16;\n\t"
        "addc.cc.u32 %1, %9, %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.u32    %7, %15, %23;"
        : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7]),
          "=r"(bw)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
          "n"(m2word<C>(0)), "n"(m2word<C>(1)), "n"(m2word<C>(2)), "n"(m2word<C>(3)), "n"(m2word<C>(4)),
          "n"(m2word<C>(5)), "n"(m2word<C>(6)), "n"(m2word<C>(7)));
    Fp<C> r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = bw ? t[i] : s[i];
    return r;
}

// (a - b) mod 2p in [0, 2p) for a, b < 2p
template <class C>
H2B_DEV Fp<C> sub2p(const Fp<C>& a, const Fp<C>& b)
{
    Fp<C> r;
    uint32_t bw;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
          "=r"(r.v[7]), "=r"(bw)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    const uint32_t q0 = bw & m2word<C>(0), q1 = bw & m2word<C>(1), q2 = bw & m2word<C>(2), q3 = bw & m2word<C>(3);
    const uint32_t q4 = bw & m2word<C>(4), q5 = bw & m2word<C>(5), q6 = bw & m2word<C>(6), q7 = bw & m2word<C>(7);
    asm("add.cc.u32  %0, %0, %8;\n\t"
        "addc.cc.u32 %1, %1, %9;\n\t"
        "addc.cc.u32 %2, %2, %10;\n\t"
        "addc.cc.u32 %3, %3, %11;\n\t"
        "addc.cc.u32 %4, %4, %12;\n\t"
        "addc.cc.u32 %5, %5, %13;\n\t"
        "addc.cc.u32 %6, %6, %14;\n\t"
        "addc.u32    %7, %7, %15;"
        : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]), "+r"(r.v[6]),
          "+r"(r.v[7])
        : "r"(q0), "r"(q1), "r"(q2), "r"(q3), "r"(q4), "r"(q5), "r"(q6), "r"(q7));
    return r;
}

// the canonical residue of a < 2p
template <class C>
H2B_DEV Fp<C> canon2p(const Fp<C>& a)
{
    Fp<C> r;
    cond_sub<C>(r.v, a.v);
    return r;
}

// The 29-bit limb form (Fl: value below 2p, R = 2^256) through the FP64
// core: the limbs are re-sliced into 52-bit limbs (one operand as 16 a, still
// below 2^260), and the result, below (1 + 64 p / 2^260) p < 1.76 p, is
// sliced back, so it keeps the Fl invariant.  Its dependent chain is five
// reduction digits instead of nine, which is what the single-warp tails
// (window doubling chain, bucket-reduction Horner steps) wait on.
namespace f64 {
// bits [S, S + 52) of sum l[k] 2^(29 k) (S < 0: zeros below bit 0)
template <int S>
H2B_DEV uint64_t bits52_of29(const uint32_t (&l)[9])
{
    uint64_t r = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const int off = 29 * k - S;
        if (off >= 0 && off < 52) r |= (uint64_t)l[k] << off;
        else if (off < 0 && off > -29) r |= (uint64_t)(l[k] >> (-off));
    }
    return r & M52;
}

// bits [S, S + 29) of sum l[i] 2^(52 i)
template <int S>
H2B_DEV uint32_t bits29_of52(const uint64_t (&l)[5])
{
    uint64_t r = 0;
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const int off = 52 * i - S;
        if (off >= 0 && off < 29) r |= l[i] << off;
        else if (off < 0 && off > -52) r |= l[i] >> (-off);
    }
    return (uint32_t)r & M29;
}
}  // namespace f64

template <class C>
H2B_DEV Fl<C> mul_f64_l(const Fl<C>& a, const Fl<C>& b)
{
    using namespace f64;
    double A[5], B[5];
    A[0] = u52d(bits52_of29<-4>(a.l)); A[1] = u52d(bits52_of29<48>(a.l)); A[2] = u52d(bits52_of29<100>(a.l));
    A[3] = u52d(bits52_of29<152>(a.l)); A[4] = u52d(bits52_of29<204>(a.l));
    B[0] = u52d(bits52_of29<0>(b.l)); B[1] = u52d(bits52_of29<52>(b.l)); B[2] = u52d(bits52_of29<104>(b.l));
    B[3] = u52d(bits52_of29<156>(b.l)); B[4] = u52d(bits52_of29<208>(b.l));
    uint64_t l[5];
    mont52<C>(A, B, l);
    Fl<C> r;
    r.l[0] = bits29_of52<0>(l); r.l[1] = bits29_of52<29>(l); r.l[2] = bits29_of52<58>(l);
    r.l[3] = bits29_of52<87>(l); r.l[4] = bits29_of52<116>(l); r.l[5] = bits29_of52<145>(l);
    r.l[6] = bits29_of52<174>(l); r.l[7] = bits29_of52<203>(l); r.l[8] = bits29_of52<232>(l);
    return r;
}

// ---- Fl arithmetic kept in limb form (values < 2p, limbs < 2^29) ---------

// limb i of 2m (m2word above) in the 29-bit grid
template <class C>
__host__ __device__ constexpr uint32_t p2_29(int i)
{
    return (uint32_t)((((uint64_t)m2word<C>((29 * i) / 32)) | ((uint64_t)m2word<C>((29 * i) / 32 + 1) << 32)) >>
                      ((29 * i) % 32)) & M29;
}

// Signed limbs -> normalised limbs, carries/borrows moved up (top limb keeps the sign).
H2B_DEV void fl_normalise(int32_t (&d)[9])
{
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int32_t c = d[i] >> 29;
        d[i] &= (int32_t)M29;
        d[i + 1] += c;
    }
}

// a - b (+ 2m when negative); inputs and output < 2m.
template <class C>
H2B_DEV Fl<C> fl_sub(const Fl<C>& a, const Fl<C>& b)
{
    int32_t d[9];
#pragma unroll
    for (int i = 0; i < 9; i++) d[i] = (int32_t)a.l[i] - (int32_t)b.l[i];
    fl_normalise(d);
    const int32_t neg = d[8] >> 31;
#pragma unroll
    for (int i = 0; i < 9; i++) d[i] += (int32_t)(p2_29<C>(i) & (uint32_t)neg);
    fl_normalise(d);
    Fl<C> r;
#pragma unroll
    for (int i = 0; i < 9; i++) r.l[i] = (uint32_t)d[i];
    return r;
}

// a + b (- 2m when >= 2m); inputs and output < 2m.
template <class C>
H2B_DEV Fl<C> fl_add(const Fl<C>& a, const Fl<C>& b)
{
    int32_t s[9], t[9];
#pragma unroll
    for (int i = 0; i < 9; i++) s[i] = (int32_t)(a.l[i] + b.l[i]);
    fl_normalise(s);
#pragma unroll
    for (int i = 0; i < 9; i++) t[i] = s[i] - (int32_t)p2_29<C>(i);
    fl_normalise(t);
    const bool keep = t[8] < 0;
    Fl<C> r;
#pragma unroll
    for (int i = 0; i < 9; i++) r.l[i] = (uint32_t)(keep ? s[i] : t[i]);
    return r;
}

// a == 0 (mod m) for a < 2m: a is 0 or m.
template <class C>
H2B_DEV bool fl_is_zero_mod(const Fl<C>& a)
{
    uint32_t z = 0, e = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        z |= a.l[i];
        e |= a.l[i] ^ p29<C>(i);
    }
    return z == 0 || e == 0;
}

template <class C>
H2B_DEV bool fl_is_zero(const Fl<C>& a)
{
    uint32_t z = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) z |= a.l[i];
    return z == 0;
}

template <class C>
H2B_DEV Fl<C> fl_zero()
{
    Fl<C> r;
#pragma unroll
    for (int i = 0; i < 9; i++) r.l[i] = 0;
    return r;
}

// Out-of-line products for kernels that chain many of them.  A call costs
// about a fifth of a product (measured: 42 G/s out of line against 54.7 G/s
// inline), so the paired forms compute two independent products per call,
// which also gives the scheduler two dependency chains to interleave.
// H2B_FL_F64 selects the FP64 core for the latency-oriented forms used by
// the single-warp tails (fl_mul_ilp / fl_sqr_ilp).
#ifndef H2B_FL_F64
#define H2B_FL_F64 1
#endif
template <class C>
__device__ __noinline__ Fl<C> fl_mul(const Fl<C> a, const Fl<C> b)
{
    return mul29<C>(a, b);
}

template <class C>
__device__ __noinline__ Fl<C> fl_sqr(const Fl<C> a)
{
    return sqr29<C>(a);
}

// Out-of-line latency-oriented products (one code copy for single-warp chains).
template <class C>
__device__ __noinline__ Fl<C> fl_mul_ilp(const Fl<C> a, const Fl<C> b)
{
#if H2B_FL_F64
    return mul_f64_l<C>(a, b);
#else
    return mul29_ilp<C>(a, b);
#endif
}

template <class C>
__device__ __noinline__ Fl<C> fl_sqr_ilp(const Fl<C> a)
{
#if H2B_FL_F64
    return mul_f64_l<C>(a, a);
#else
    return sqr29_ilp<C>(a);
#endif
}

template <class C>
struct Fl2 {
    Fl<C> a, b;
};

template <class C>
__device__ __noinline__ Fl2<C> fl_mul2(const Fl<C> a0, const Fl<C> b0, const Fl<C> a1, const Fl<C> b1)
{
    Fl2<C> r;
    r.a = mul29<C>(a0, b0);
    r.b = mul29<C>(a1, b1);
    return r;
}

template <class C>
__device__ __noinline__ Fl2<C> fl_sqr2(const Fl<C> a0, const Fl<C> a1)
{
    Fl2<C> r;
    r.a = sqr29<C>(a0);
    r.b = sqr29<C>(a1);
    return r;
}

// The product behind operator* is the FP64 form (mont_mul_f64; the 29-bit
// column form measured 54.7 G products/s with the 8 x 32 conversions in a
// four-chain probe, against 41.5 G for the mad.lo/mad.hi CIOS above and
// 46.9 G for its mad.wide variant).  One out-of-line body per field: kernels that chain many products (curve
// formulas, the quotient interpreter) otherwise inline hundreds of
// instructions per product and starve on instruction fetch.  H2B_INLINE_MUL=1
// restores full inlining for kernels that want it.
#ifndef H2B_INLINE_MUL
#define H2B_INLINE_MUL 0
#endif
// operator* and fsqr use the FP64 product (mont_mul_f64) unless
// H2B_MUL_F64=0 selects the 29-bit one.  Measured on B200, FP64 against
// 29-bit: batch inversion of 2^24 elements 2.11 -> 1.62 ms, permutation
// quotient (4 columns, 2^20 rows) 1.04 -> 0.80 ms, 8 coset parts at 2^22
// 12.52 -> 11.47 ms, 8 inverse NTTs at 2^22 14.09 -> 12.90 ms.
#ifndef H2B_MUL_F64
#define H2B_MUL_F64 1
#endif

template <class C>
H2B_DEV Fp<C> mont_mul_sel(const Fp<C>& a, const Fp<C>& b)
{
#if H2B_MUL_F64
    return mont_mul_f64<C>(a, b);
#else
    return mont_mul_29<C>(a, b);
#endif
}

template <class C>
H2B_DEV Fp<C> mont_sqr_sel(const Fp<C>& a)
{
#if H2B_MUL_F64
    return mont_mul_f64<C>(a, a);
#else
    return mont_sqr_29<C>(a);
#endif
}

template <class C>
__device__ __noinline__ Fp<C> mont_mul_outline(const Fp<C> a, const Fp<C> b)
{
    return mont_mul_sel<C>(a, b);
}

template <class C>
__device__ __noinline__ Fp<C> mont_sqr_outline(const Fp<C> a)
{
    return mont_sqr_sel<C>(a);
}

// a b 2^-256 mod p in [0, 2p) for a, b < 2p, out of line (residues in [0, 2p)
// above; the 29-bit build returns the canonical product, which is below 2p too)
template <class C>
__device__ __noinline__ Fp<C> mont_mul_lazy_outline(const Fp<C> a, const Fp<C> b)
{
#if H2B_MUL_F64
    return mont_mul_f64_lazy<C>(a, b);
#else
    return mont_mul_sel<C>(a, b);
#endif
}

template <class C>
H2B_DEV Fp<C> operator*(const Fp<C>& a, const Fp<C>& b)
{
#if H2B_INLINE_MUL
    return mont_mul_sel<C>(a, b);
#else
    return mont_mul_outline<C>(a, b);
#endif
}

template <class C>
H2B_DEV Fp<C> operator+(const Fp<C>& a, const Fp<C>& b)
{
    uint32_t t[8];
    asm("add.cc.u32  %0, %8, %16;\n\t"
        "addc.cc.u32 %1, %9, %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.u32    %7, %15, %23;"
        : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    Fp<C> r;
    cond_sub<C>(r.v, t);
    return r;
}

template <class C>
H2B_DEV Fp<C> operator-(const Fp<C>& a, const Fp<C>& b)
{
    Fp<C> r;
    uint32_t bw;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
          "=r"(r.v[7]), "=r"(bw)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    // On borrow add the modulus back (bw is 0 or all-ones).
    const uint32_t q0 = bw & C::M0, q1 = bw & C::M1, q2 = bw & C::M2, q3 = bw & C::M3;
    const uint32_t q4 = bw & C::M4, q5 = bw & C::M5, q6 = bw & C::M6, q7 = bw & C::M7;
    asm("add.cc.u32  %0, %0, %8;\n\t"
        "addc.cc.u32 %1, %1, %9;\n\t"
        "addc.cc.u32 %2, %2, %10;\n\t"
        "addc.cc.u32 %3, %3, %11;\n\t"
        "addc.cc.u32 %4, %4, %12;\n\t"
        "addc.cc.u32 %5, %5, %13;\n\t"
        "addc.cc.u32 %6, %6, %14;\n\t"
        "addc.u32    %7, %7, %15;"
        : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]), "+r"(r.v[6]),
          "+r"(r.v[7])
        : "r"(q0), "r"(q1), "r"(q2), "r"(q3), "r"(q4), "r"(q5), "r"(q6), "r"(q7));
    return r;
}

template <class C>
H2B_DEV Fp<C>& operator*=(Fp<C>& a, const Fp<C>& b) { a = a * b; return a; }
template <class C>
H2B_DEV Fp<C>& operator+=(Fp<C>& a, const Fp<C>& b) { a = a + b; return a; }
template <class C>
H2B_DEV Fp<C>& operator-=(Fp<C>& a, const Fp<C>& b) { a = a - b; return a; }

template <class C>
H2B_DEV Fp<C> fneg(const Fp<C>& a) { return Fp<C>::zero() - a; }
template <class C>
H2B_DEV Fp<C> fdbl(const Fp<C>& a) { return a + a; }
template <class C>
H2B_DEV Fp<C> fsqr(const Fp<C>& a)
{
#if H2B_INLINE_MUL
    return mont_sqr_sel<C>(a);
#else
    return mont_sqr_outline<C>(a);
#endif
}

// Montgomery residue -> canonical integer (multiply by 1).
template <class C>
H2B_DEV Fp<C> from_mont(const Fp<C>& a)
{
    Fp<C> one_int = Fp<C>::zero();
    one_int.v[0] = 1;
    return a * one_int;
}
template <class C>
H2B_DEV Fp<C> to_mont(const Fp<C>& a) { return a * Fp<C>::r2(); }

// a^e for a 256-bit exponent given as 8 little-endian words; 4-bit fixed window.
template <class C>
H2B_DEV Fp<C> fpow(const Fp<C>& a, const uint32_t (&e)[8])
{
    Fp<C> tbl[16];
    tbl[0] = Fp<C>::one();
    tbl[1] = a;
#pragma unroll 1
    for (int i = 2; i < 16; i++) tbl[i] = tbl[i - 1] * a;
    Fp<C> r = Fp<C>::one();
#pragma unroll 1
    for (int w = 63; w >= 0; w--) {
        r = r * r; r = r * r; r = r * r; r = r * r;
        uint32_t d = (e[w >> 3] >> ((w & 7) * 4)) & 15u;
        if (d) r = r * tbl[d];
    }
    return r;
}

// Fermat inverse a^(m-2); inverse of zero is zero.
template <class C>
H2B_DEV Fp<C> finv(const Fp<C>& a)
{
    const uint32_t e[8] = {C::M0 - 2u, C::M1, C::M2, C::M3, C::M4, C::M5, C::M6, C::M7};
    return fpow<C>(a, e);
}

template <class C>
H2B_DEV Fp<C> ldg(const Fp<C>* p)
{
    Fp<C> r;
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4 x = __ldg(q), y = __ldg(q + 1);
    r.v[0] = x.x; r.v[1] = x.y; r.v[2] = x.z; r.v[3] = x.w;
    r.v[4] = y.x; r.v[5] = y.y; r.v[6] = y.z; r.v[7] = y.w;
    return r;
}
template <class C>
H2B_DEV Fp<C> ld(const Fp<C>* p)
{
    Fp<C> r;
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4 x = q[0], y = q[1];
    r.v[0] = x.x; r.v[1] = x.y; r.v[2] = x.z; r.v[3] = x.w;
    r.v[4] = y.x; r.v[5] = y.y; r.v[6] = y.z; r.v[7] = y.w;
    return r;
}
template <class C>
H2B_DEV void st(Fp<C>* p, const Fp<C>& a)
{
    uint4* q = reinterpret_cast<uint4*>(p);
    q[0] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
    q[1] = make_uint4(a.v[4], a.v[5], a.v[6], a.v[7]);
}

} // namespace h2b
