// Lazy 52-bit limb arithmetic on the FP64 pipe, for the MSM bucket
// accumulation (accumulate variant 6).
//
// Same idea as the 29-bit lazy form (lazy.cuh), on the FP64 Montgomery core
// of field.cuh (f64::mont52):
//
//  * Values are x * 2^260 mod p plus multiples of p, as five limbs below
//    2^52 (the top one holds the rest; every value stays below 2^257).
//    R' = 2^260 gives p / R' = 0.0118 for BN254 Fq, so a product of values
//    below a*p and b*p is below (1 + 0.0118 a b) p.
//  * a + b and a - b + K p are limb-wise in 64-bit integers followed by a
//    serial carry over the five limbs (the FP64 split needs every limb
//    below 2^52 exactly), never a conditional subtraction.
//  * Bases are stored as canonical x * 2^261 mod p (the table and split
//    kernels' form, shared with the 29-bit variant); one halving modulo p
//    per coordinate turns them into x * 2^260.  Results leave through one
//    product by 2^256 mod p (giving x * 2^256 mod p) and a conditional
//    subtraction.
//
// Bounds of the accumulator from one addition to the next: X < 5.4p,
// Y < 3.45p, ZZ and ZZZ < 1.2p; affine inputs qx < p, qy < 2p.
#pragma once
#include "field.cuh"

namespace h2b {

template <class C>
struct Fd {
    uint64_t l[5];
};

// limb i of K p in the 52-bit grid, normalised (the top limb holds the rest)
template <class C>
__host__ __device__ constexpr uint64_t kp52(int K, int i)
{
    uint64_t carry = 0, t = 0;
    for (int j = 0; j <= i; j++) {
        t = (uint64_t)K * f64::p52<C>(j) + carry;
        carry = t >> 52;
        if (j < i) t &= f64::M52;
    }
    return i < 4 ? (t & f64::M52) : t;
}

// word w of R mod p = 2^256 mod p (the Montgomery one)
template <class C>
__host__ __device__ constexpr uint32_t oword(int w)
{
    return w == 0 ? C::O0 : w == 1 ? C::O1 : w == 2 ? C::O2 : w == 3 ? C::O3 : w == 4 ? C::O4
         : w == 5 ? C::O5 : w == 6 ? C::O6 : C::O7;
}

// limb i of 2^(256 + s) mod p in the 52-bit grid, s in 0..4 (compile-time:
// 2^s (2^256 mod p) reduced by repeated subtraction of p)
template <class C>
__host__ __device__ constexpr uint64_t r2x52(int s, int i)
{
    uint64_t x[5] = {0, 0, 0, 0, 0};
    for (int k = 0; k < 5; k++) {
        uint64_t r = 0;
        for (int w = 0; w < 8; w++) {
            const int off = 32 * w + s - 52 * k;
            if (off >= 0 && off < 52) r |= (uint64_t)oword<C>(w) << off;
            else if (off < 0 && off > -32) r |= (uint64_t)(oword<C>(w) >> (-off));
        }
        x[k] = k < 4 ? (r & f64::M52) : r;
    }
    for (int it = 0; it < 32; it++) {
        bool ge = true;
        for (int k = 4; k >= 0; k--) {
            if (x[k] != f64::p52<C>(k)) {
                ge = x[k] > f64::p52<C>(k);
                break;
            }
        }
        if (!ge) break;
        int64_t borrow = 0;
        for (int k = 0; k < 5; k++) {
            int64_t d = (int64_t)x[k] - (int64_t)f64::p52<C>(k) - borrow;
            borrow = d < 0 ? 1 : 0;
            x[k] = (uint64_t)(d + (borrow && k < 4 ? (int64_t)1 << 52 : 0));
        }
    }
    return x[i];
}

// constants of the form as immediates: 1 (= 2^260 mod p) and the store
// factor 2^256 mod p
template <class C>
H2B_DEV Fd<C> fd_one()
{
    constexpr uint64_t a0 = r2x52<C>(4, 0), a1 = r2x52<C>(4, 1), a2 = r2x52<C>(4, 2), a3 = r2x52<C>(4, 3),
                       a4 = r2x52<C>(4, 4);
    return Fd<C>{{a0, a1, a2, a3, a4}};
}

template <class C>
H2B_DEV Fd<C> fd_r256()
{
    constexpr uint64_t a0 = r2x52<C>(0, 0), a1 = r2x52<C>(0, 1), a2 = r2x52<C>(0, 2), a3 = r2x52<C>(0, 3),
                       a4 = r2x52<C>(0, 4);
    return Fd<C>{{a0, a1, a2, a3, a4}};
}

// the limbs of p and of K p as compile-time constants
template <class C>
struct P52 {
    static constexpr uint64_t l0 = f64::p52<C>(0), l1 = f64::p52<C>(1), l2 = f64::p52<C>(2),
                              l3 = f64::p52<C>(3), l4 = f64::p52<C>(4);
};
template <class C, int K>
struct KP52 {
    static constexpr int64_t l0 = (int64_t)kp52<C>(K, 0), l1 = (int64_t)kp52<C>(K, 1),
                             l2 = (int64_t)kp52<C>(K, 2), l3 = (int64_t)kp52<C>(K, 3),
                             l4 = (int64_t)kp52<C>(K, 4);
};

// signed limb sums -> normalised limbs (serial carry; the value is >= 0)
template <class C>
H2B_DEV Fd<C> fd_norm(const int64_t (&d)[5])
{
    Fd<C> r;
    int64_t c = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int64_t x = d[i] + c;
        r.l[i] = (uint64_t)x & f64::M52;
        c = x >> 52;
    }
    r.l[4] = (uint64_t)(d[4] + c);
    return r;
}

template <class C>
H2B_DEV Fd<C> fd_add(const Fd<C>& a, const Fd<C>& b)
{
    int64_t d[5];
#pragma unroll
    for (int i = 0; i < 5; i++) d[i] = (int64_t)(a.l[i] + b.l[i]);
    return fd_norm<C>(d);
}

// a - b + K p, for b below K p
template <class C, int K>
H2B_DEV Fd<C> fd_sub(const Fd<C>& a, const Fd<C>& b)
{
    using L = KP52<C, K>;
    const int64_t kp[5] = {L::l0, L::l1, L::l2, L::l3, L::l4};
    int64_t d[5];
#pragma unroll
    for (int i = 0; i < 5; i++) d[i] = (int64_t)a.l[i] - (int64_t)b.l[i] + kp[i];
    return fd_norm<C>(d);
}

template <class C>
H2B_DEV Fd<C> fd_mul(const Fd<C>& a, const Fd<C>& b)
{
    double A[5], B[5];
#pragma unroll
    for (int i = 0; i < 5; i++) {
        A[i] = f64::u52d(a.l[i]);
        B[i] = f64::u52d(b.l[i]);
    }
    Fd<C> r;
    f64::mont52<C>(A, B, r.l);
    return r;
}

template <class C>
struct Fd2 {
    Fd<C> a, b;
};

// two independent products per out-of-line call
template <class C>
__device__ __noinline__ Fd2<C> fd_mul2(const Fd<C> a0, const Fd<C> b0, const Fd<C> a1, const Fd<C> b1)
{
    Fd2<C> r;
    r.a = fd_mul<C>(a0, b0);
    r.b = fd_mul<C>(a1, b1);
    return r;
}

template <class C>
struct Fd4 {
    Fd<C> a, b, c, d;
};

// four independent products per out-of-line call (two accumulation chains)
template <class C>
__device__ __noinline__ Fd4<C> fd_mul4(const Fd<C> a0, const Fd<C> b0, const Fd<C> a1, const Fd<C> b1,
                                      const Fd<C> a2, const Fd<C> b2, const Fd<C> a3, const Fd<C> b3)
{
    Fd4<C> r;
    r.a = fd_mul<C>(a0, b0);
    r.b = fd_mul<C>(a1, b1);
    r.c = fd_mul<C>(a2, b2);
    r.d = fd_mul<C>(a3, b3);
    return r;
}

template <class C>
__device__ __noinline__ Fd<C> fd_mul_call(const Fd<C> a, const Fd<C> b)
{
    return fd_mul<C>(a, b);
}

template <class C>
H2B_DEV Fd<C> fd_zero()
{
    Fd<C> r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.l[i] = 0;
    return r;
}

template <class C>
H2B_DEV bool fd_is_zero(const Fd<C>& a)
{
    uint64_t z = 0;
#pragma unroll
    for (int i = 0; i < 5; i++) z |= a.l[i];
    return z == 0;
}

// a == 0 (mod p) for a product output (normalised limbs, value < 2p): a is 0 or p
template <class C>
H2B_DEV bool fd_is_zero_mod(const Fd<C>& a)
{
    using L = P52<C>;
    const uint64_t pl[5] = {L::l0, L::l1, L::l2, L::l3, L::l4};
    uint64_t z = 0, e = 0;
#pragma unroll
    for (int i = 0; i < 5; i++) {
        z |= a.l[i];
        e |= a.l[i] ^ pl[i];
    }
    return z == 0 || e == 0;
}

// the 52-bit limbs of a 256-bit word image (no conversion)
template <class C>
H2B_DEV Fd<C> fd_from_words(const Fp<C>& a)
{
    Fd<C> r;
    r.l[0] = f64::bits52<0>(a.v);
    r.l[1] = f64::bits52<52>(a.v);
    r.l[2] = f64::bits52<104>(a.v);
    r.l[3] = f64::bits52<156>(a.v);
    r.l[4] = f64::bits52<208>(a.v);
    return r;
}

// canonical v = x 2^261 mod p -> x 2^260 mod p = v / 2 mod p
// ((v + p) / 2 when v is odd; canonical in, canonical out)
template <class C>
H2B_DEV Fd<C> fd_from_r261(const Fp<C>& v)
{
    using L = P52<C>;
    const uint64_t pl[5] = {L::l0, L::l1, L::l2, L::l3, L::l4};
    Fd<C> t = fd_from_words<C>(v);
    const uint64_t m = 0 - (t.l[0] & 1u);
    int64_t d[5];
#pragma unroll
    for (int i = 0; i < 5; i++) d[i] = (int64_t)(t.l[i] + (pl[i] & m));
    t = fd_norm<C>(d);
    Fd<C> r;
#pragma unroll
    for (int i = 0; i < 4; i++) r.l[i] = (t.l[i] >> 1) | ((t.l[i + 1] & 1u) << 51);
    r.l[4] = t.l[4] >> 1;
    return r;
}

// normalised limbs of a value below 2p -> canonical 8 x 32 words
template <class C>
H2B_DEV Fp<C> fd_canonical(const Fd<C>& t)
{
    uint32_t w[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int i0 = (32 * j) / 52, o = 32 * j - 52 * i0;
        uint64_t x = t.l[i0] >> o;
        if (i0 + 1 < 5) x |= t.l[i0 + 1] << (52 - o);
        w[j] = (uint32_t)x;
    }
    Fp<C> r;
    cond_sub<C>(r.v, w);
    return r;
}

} // namespace h2b
