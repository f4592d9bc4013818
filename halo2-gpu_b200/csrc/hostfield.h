// Host-side BN254 Fr arithmetic for launch-time constants only (coset-factor
// power tables, zeta factors).  4 x 64-bit Montgomery CIOS with __int128; the
// same constants as the device header.  Nothing here runs per element.
#pragma once
#include <cstdint>
#include <cstring>

namespace h2b {
namespace host {

struct Fr64 {
    uint64_t v[4];
};

static const uint64_t FR_M[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull,
                                 0x30644e72e131a029ull};
static const uint64_t FR_N0 = 0xc2e1f593efffffffull;
static const uint64_t FR_ONE[4] = {0xac96341c4ffffffbull, 0x36fc76959f60cd29ull, 0x666ea36f7879462eull,
                                   0x0e0a77c19a07df2full};
// zeta (Montgomery form), the cube root of unity used by the coset twist
// (halo2_proofs/cuda/include/kernel/zeta.h:19-28) and its square = zeta^-1.
static const uint64_t FR_ZETA[4] = {244305545194690131ull, 8351807910065594880ull, 14266533074055306532ull,
                                    404339206190769364ull};
static const uint64_t FR_ZETA2[4] = {10657714497315350963ull, 9029678389775483239ull, 10080386412464207114ull,
                                     2070906320917503013ull};

inline Fr64 fr_mul(const Fr64& a, const Fr64& b)
{
    typedef unsigned __int128 u128;
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; j < 4; j++) {
            c += (u128)a.v[j] * b.v[i] + t[j];
            t[j] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[4] = (uint64_t)c;
        t[5] = (uint64_t)(c >> 64);
        uint64_t m = t[0] * FR_N0;
        c = (u128)m * FR_M[0] + t[0];
        c >>= 64;
        for (int j = 1; j < 4; j++) {
            c += (u128)m * FR_M[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    Fr64 r;
    // conditional subtract
    uint64_t s[4];
    unsigned __int128 bw = 0;
    for (int j = 0; j < 4; j++) {
        unsigned __int128 d = (unsigned __int128)t[j] - FR_M[j] - (uint64_t)bw;
        s[j] = (uint64_t)d;
        bw = (d >> 64) ? 1 : 0;
    }
    bool keep = (t[4] == 0) && bw;
    for (int j = 0; j < 4; j++) r.v[j] = keep ? t[j] : s[j];
    return r;
}

inline Fr64 fr_from(const void* p)
{
    Fr64 r;
    memcpy(r.v, p, 32);
    return r;
}
inline Fr64 fr_const(const uint64_t (&c)[4])
{
    Fr64 r;
    memcpy(r.v, c, 32);
    return r;
}

// lut[i] = base^(2^i), i < k
inline void fr_pow2_lut(const Fr64& base, int k, Fr64* lut)
{
    Fr64 cur = base;
    for (int i = 0; i < k; i++) {
        lut[i] = cur;
        cur = fr_mul(cur, cur);
    }
}

} // namespace host
} // namespace h2b
