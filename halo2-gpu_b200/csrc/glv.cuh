// GLV endomorphism of BN254 G1 for the MSM.
//
// phi(x, y) = (beta * x, y) equals [lambda] P, where lambda is the cube root
// of unity in Fr that the reference also uses as its coset generator zeta
// (halo2_proofs/cuda/include/kernel/zeta.h:19-22) and beta a cube root of
// unity in Fq.  A scalar k < r is split as k = k1 + k2 * lambda (mod r) with
// |k1|, |k2| < 2^127 by rounding against the short lattice basis
//   (a1, b1) = (0x6f4d8248eeb859fc8211bbeb7d4f1128, -0x89d3256894d213e3)
//   (a2, b2) = (0x89d3256894d213e3, 0x6f4d8248eeb859fd0be4e1541221250b),
// a1*b2 - a2*b1 = r:  c1 = floor(k * g1 / 2^256), c2 = floor(k * g2 / 2^256)
// with g1 = floor(2^256 b2 / r), g2 = floor(2^256 (-b1) / r), then
// k1 = k - c1 a1 - c2 a2 and k2 = c1 (-b1) - c2 b2 (mod 2^256, signed).
// The constants and the 127-bit bound were derived with exact integer
// arithmetic (extended Euclid on (r, lambda)) and are re-checked by
// tests/test_glv.py.  The MSM result does not depend on the split.
#pragma once
#include <cstdint>
#include "field.cuh"

namespace h2b {
namespace glv {

__device__ __constant__ static const uint64_t G1c[3] = {0x5398fd0300ff6565ull, 0x4ccef014a773d2d2ull, 0x2ull};
__device__ __constant__ static const uint64_t G2c[2] = {0xd91d232ec7e0b3d7ull, 0x2ull};
__device__ __constant__ static const uint64_t A1c[2] = {0x8211bbeb7d4f1128ull, 0x6f4d8248eeb859fcull};
__device__ __constant__ static const uint64_t B2c[2] = {0x0be4e1541221250bull, 0x6f4d8248eeb859fdull};
static constexpr uint64_t A2 = 0x89d3256894d213e3ull;   // = -b1

// beta in Montgomery form over Fq
H2B_DEV Fq beta()
{
    Fq b;
    b.v[0] = 0x13e80b9cu; b.v[1] = 0x3350c88eu; b.v[2] = 0xdb5e56b9u; b.v[3] = 0x7dce557cu;
    b.v[4] = 0xb615564au; b.v[5] = 0x6001b4b8u; b.v[6] = 0x020217e0u; b.v[7] = 0x2682e617u;
    return b;
}

// out[0..na+nb) = a * b (little-endian 64-bit limbs)
H2B_DEV void mp_mul(const uint64_t* a, int na, const uint64_t* b, int nb, uint64_t* out)
{
    for (int i = 0; i < na + nb; i++) out[i] = 0;
    for (int i = 0; i < na; i++) {
        unsigned __int128 carry = 0;
        for (int j = 0; j < nb; j++) {
            unsigned __int128 t = (unsigned __int128)a[i] * b[j] + out[i + j] + carry;
            out[i + j] = (uint64_t)t;
            carry = t >> 64;
        }
        out[i + nb] = (uint64_t)carry;
    }
}

// r -= x (4 limbs, mod 2^256); x has nx <= 4 limbs
H2B_DEV void mp_sub4(uint64_t* r, const uint64_t* x, int nx)
{
    unsigned __int128 borrow = 0;
    for (int i = 0; i < 4; i++) {
        uint64_t xi = i < nx ? x[i] : 0;
        unsigned __int128 d = (unsigned __int128)r[i] - xi - (uint64_t)borrow;
        r[i] = (uint64_t)d;
        borrow = (d >> 64) & 1;
    }
}

// |v| of a 256-bit two's-complement value known to satisfy |v| < 2^127;
// returns the sign (1 = negative).
H2B_DEV uint32_t mp_abs128(const uint64_t* v, uint64_t& lo, uint64_t& hi)
{
    uint32_t neg = (uint32_t)(v[3] >> 63);
    if (neg) {
        unsigned __int128 x = ~(((unsigned __int128)v[1] << 64) | v[0]);
        x += 1;
        lo = (uint64_t)x;
        hi = (uint64_t)(x >> 64);
    } else {
        lo = v[0];
        hi = v[1];
    }
    return neg;
}

// Canonical k (8 x u32) -> two 128-bit magnitudes with the sign in bit 127.
H2B_DEV void decompose(const Fr& kc, uint4& out1, uint4& out2)
{
    uint64_t k[4];
    for (int i = 0; i < 4; i++) k[i] = (uint64_t)kc.v[2 * i] | ((uint64_t)kc.v[2 * i + 1] << 32);
    uint64_t p1[7], p2[6];
    uint64_t g1[3] = {G1c[0], G1c[1], G1c[2]}, g2[2] = {G2c[0], G2c[1]};
    mp_mul(k, 4, g1, 3, p1);
    mp_mul(k, 4, g2, 2, p2);
    uint64_t c1[2] = {p1[4], p1[5]};   // < 2^128
    uint64_t c2[1] = {p2[4]};          // < 2^64
    uint64_t a1[2] = {A1c[0], A1c[1]}, b2[2] = {B2c[0], B2c[1]}, a2[1] = {A2};
    uint64_t t[4];
    // k1 = k - c1*a1 - c2*a2
    uint64_t k1[4] = {k[0], k[1], k[2], k[3]};
    mp_mul(c1, 2, a1, 2, t);
    mp_sub4(k1, t, 4);
    uint64_t u[3];
    mp_mul(c2, 1, a2, 1, u);
    mp_sub4(k1, u, 2);
    // k2 = c1*(-b1) - c2*b2
    uint64_t k2[4] = {0, 0, 0, 0};
    mp_mul(c1, 2, a2, 1, u);          // -b1 == a2
    k2[0] = u[0]; k2[1] = u[1]; k2[2] = u[2];
    mp_mul(c2, 1, b2, 2, u);
    mp_sub4(k2, u, 3);
    uint64_t lo, hi;
    uint32_t s1 = mp_abs128(k1, lo, hi);
    out1 = make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32) | (s1 << 31));
    uint32_t s2 = mp_abs128(k2, lo, hi);
    out2 = make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32) | (s2 << 31));
}

} // namespace glv
} // namespace h2b
