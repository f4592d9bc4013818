/*
 * CPU oracle for the BN254 Halo2/KZG prover hot path -- TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of the reference's algorithms, used only by tests/,
 * by __graft_entry__.smoke() as the checker, and as bench.py's CPU baseline.
 * Nothing on the product path links or calls this file.
 *
 * What each function restates (paths relative to axiom-crypto/halo2-gpu):
 *   field constants         halo2_proofs/cuda/include/field/alt_bn128.hpp:15-43
 *   zeta, zeta^2            halo2_proofs/cuda/include/kernel/zeta.h:19-28
 *   o_msm                   multiexp_serial / best_multiexp_cpu,
 *                           halo2_proofs/src/cpu/arithmetic.rs:14-156
 *   o_ntt                   run_fft semantics, halo2_proofs/cuda/src/ntt.cu:202-375;
 *                           coset part = coeff_to_extended_part_cpu,
 *                           halo2_proofs/src/cpu/evaluator.rs:26-47
 *   o_batch_invert          zero-preserving Montgomery trick,
 *                           halo2_proofs/cuda/include/kernel/inverse.h:10-63
 *   o_grand_product         halo2_proofs/src/cuda/culib.rs:202-230 semantics
 *   o_fr_eval, o_fr_eval_many  Horner evaluation, eval_polynomial,
 *                           halo2_proofs/src/arithmetic.rs (coefficients low first)
 *   o_lookup_product        lookup_product_cpu, halo2_proofs/src/cpu/arithmetic.rs:158-197
 *   o_permutation_product   permutation_product_cpu, halo2_proofs/src/cpu/arithmetic.rs:287-327
 *   o_permute_pair          permute_expression_pair_seq,
 *                           halo2_proofs/src/plonk/lookup/prover.rs:787-880
 *   o_quotient              rule interpreter, halo2_proofs/cuda/include/kernel/quotient.h:57-303
 *                           (encoding: halo2_proofs/src/plonk/evaluation.rs:107-352)
 *   o_quotient_lookups      quotient_lookups_cpu, halo2_proofs/src/cpu/arithmetic.rs:223-280
 *   o_permutation_quotient  permutation_quotient_cpu_chunk,
 *                           halo2_proofs/src/cpu/evaluator.rs:63-148
 *
 * Parity pins: the moduli, Montgomery constants and zeta come from the
 * reference sources above; tests/golden holds vectors produced by an
 * independent pure-Python big-integer restatement.  The reference's Rust
 * crates (halo2curves-axiom 0.7.3, halo2-axiom @5e4f0e5) are not present, so
 * outputs are not pinned against the reference binary itself.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;
typedef struct { uint64_t v[4]; } fe;

typedef struct {
    uint64_t m[4];
    uint64_t n0;
    uint64_t one[4];
    uint64_t r2[4];
} field_t;

static const field_t FR = {
    {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull, 0x30644e72e131a029ull},
    0xc2e1f593efffffffull,
    {0xac96341c4ffffffbull, 0x36fc76959f60cd29ull, 0x666ea36f7879462eull, 0x0e0a77c19a07df2full},
    {0x1bb8e645ae216da7ull, 0x53fe3ab1e35c59e3ull, 0x8c49833d53bb8085ull, 0x0216d0b17f4e44a5ull}};
static const field_t FQ = {
    {0x3c208c16d87cfd47ull, 0x97816a916871ca8dull, 0xb85045b68181585dull, 0x30644e72e131a029ull},
    0x87d20782e4866389ull,
    {0xd35d438dc58f0d9dull, 0x0a78eb28f5c70b3dull, 0x666ea36f7879462cull, 0x0e0a77c19a07df2full},
    {0xf32cfc5b538afa89ull, 0xb5e71911d44501fbull, 0x47ab1eff0a417ff6ull, 0x06d89f71cab8351full}};

static const fe ZETA = {{244305545194690131ull, 8351807910065594880ull, 14266533074055306532ull, 404339206190769364ull}};
static const fe ZETA2 = {{10657714497315350963ull, 9029678389775483239ull, 10080386412464207114ull, 2070906320917503013ull}};

/* ---------------------------------------------------------------- field -- */

static inline int geq_m(const uint64_t* t, const uint64_t* m)
{
    for (int i = 3; i >= 0; i--) {
        if (t[i] > m[i]) return 1;
        if (t[i] < m[i]) return 0;
    }
    return 1;
}

static inline void sub_m(uint64_t* t, const uint64_t* m)
{
    uint64_t b = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)t[i] - m[i] - b;
        t[i] = (uint64_t)d;
        b = (uint64_t)(d >> 64) & 1;
    }
}

static inline fe f_mul(const field_t* F, fe a, fe b)
{
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
        uint64_t m = t[0] * F->n0;
        c = (u128)m * F->m[0] + t[0];
        c >>= 64;
        for (int j = 1; j < 4; j++) {
            c += (u128)m * F->m[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    fe r;
    if (t[4] || geq_m(t, F->m)) sub_m(t, F->m);
    memcpy(r.v, t, 32);
    return r;
}

static inline fe f_add(const field_t* F, fe a, fe b)
{
    fe r;
    u128 c = 0;
    for (int i = 0; i < 4; i++) {
        c += (u128)a.v[i] + b.v[i];
        r.v[i] = (uint64_t)c;
        c >>= 64;
    }
    if (geq_m(r.v, F->m)) sub_m(r.v, F->m);
    return r;
}

static inline fe f_sub(const field_t* F, fe a, fe b)
{
    fe r;
    uint64_t bw = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a.v[i] - b.v[i] - bw;
        r.v[i] = (uint64_t)d;
        bw = (uint64_t)(d >> 64) & 1;
    }
    if (bw) {
        u128 c = 0;
        for (int i = 0; i < 4; i++) {
            c += (u128)r.v[i] + F->m[i];
            r.v[i] = (uint64_t)c;
            c >>= 64;
        }
    }
    return r;
}

static inline int f_is_zero(fe a) { return (a.v[0] | a.v[1] | a.v[2] | a.v[3]) == 0; }
static inline int f_eq(fe a, fe b) { return memcmp(a.v, b.v, 32) == 0; }
static inline fe f_zero(void) { fe r = {{0, 0, 0, 0}}; return r; }
static inline fe f_one(const field_t* F) { fe r; memcpy(r.v, F->one, 32); return r; }
static inline fe f_neg(const field_t* F, fe a) { return f_sub(F, f_zero(), a); }
static inline fe f_dbl(const field_t* F, fe a) { return f_add(F, a, a); }

static fe f_pow(const field_t* F, fe a, const uint64_t* e, int words)
{
    fe r = f_one(F);
    for (int w = words - 1; w >= 0; w--)
        for (int b = 63; b >= 0; b--) {
            r = f_mul(F, r, r);
            if ((e[w] >> b) & 1) r = f_mul(F, r, a);
        }
    return r;
}

static fe f_pow_u64(const field_t* F, fe a, uint64_t e)
{
    uint64_t ee[1] = {e};
    return f_pow(F, a, ee, 1);
}

static fe f_inv(const field_t* F, fe a)
{
    uint64_t e[4];
    memcpy(e, F->m, 32);
    e[0] -= 2; /* m - 2, no borrow: m0 is odd and > 2 */
    return f_pow(F, a, e, 4);
}

static fe f_to_mont(const field_t* F, fe a) { fe r2; memcpy(r2.v, F->r2, 32); return f_mul(F, a, r2); }
static fe f_from_mont(const field_t* F, fe a) { fe one = {{1, 0, 0, 0}}; return f_mul(F, a, one); }

/* exported scalar helpers (tests) */
void o_field_mul(int fq, const fe* a, const fe* b, fe* r) { *r = f_mul(fq ? &FQ : &FR, *a, *b); }
void o_field_add(int fq, const fe* a, const fe* b, fe* r) { *r = f_add(fq ? &FQ : &FR, *a, *b); }
void o_field_sub(int fq, const fe* a, const fe* b, fe* r) { *r = f_sub(fq ? &FQ : &FR, *a, *b); }
void o_field_inv(int fq, const fe* a, fe* r) { *r = f_is_zero(*a) ? f_zero() : f_inv(fq ? &FQ : &FR, *a); }
void o_to_mont(int fq, const fe* a, fe* r, size_t n)
{
    const field_t* F = fq ? &FQ : &FR;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) r[i] = f_to_mont(F, a[i]);
}
void o_from_mont(int fq, const fe* a, fe* r, size_t n)
{
    const field_t* F = fq ? &FQ : &FR;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) r[i] = f_from_mont(F, a[i]);
}
void o_fr_pow(const fe* a, uint64_t e, fe* r) { *r = f_pow_u64(&FR, *a, e); }

/* ------------------------------------------------------------ ChaCha RNG -- */
/* ChaCha20 keystream (RFC 7539 block function, 64-bit counter, zero nonce)
 * seeded the way rand_core's seed_from_u64 expands a u64 (PCG32 output per
 * 4-byte word); Fr::random reduces eight next_u64 words as d0*R^2 + d1*R^3. */

static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
#define QR(a, b, c, d) a += b; d ^= a; d = rotl32(d, 16); c += d; b ^= c; b = rotl32(b, 12); \
                       a += b; d ^= a; d = rotl32(d, 8);  c += d; b ^= c; b = rotl32(b, 7);

static void chacha_block(const uint32_t key[8], uint64_t counter, uint32_t out[16])
{
    uint32_t s[16] = {0x61707865, 0x3320646e, 0x79622d32, 0x6b206574, key[0], key[1], key[2], key[3], key[4],
                      key[5], key[6], key[7], (uint32_t)counter, (uint32_t)(counter >> 32), 0, 0};
    uint32_t x[16];
    memcpy(x, s, sizeof(x));
    for (int i = 0; i < 10; i++) {
        QR(x[0], x[4], x[8], x[12]) QR(x[1], x[5], x[9], x[13]) QR(x[2], x[6], x[10], x[14]) QR(x[3], x[7], x[11], x[15])
        QR(x[0], x[5], x[10], x[15]) QR(x[1], x[6], x[11], x[12]) QR(x[2], x[7], x[8], x[13]) QR(x[3], x[4], x[9], x[14])
    }
    for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

static void seed_key(uint64_t state, uint32_t key[8])
{
    const uint64_t MUL = 6364136223846793005ull, INC = 11634580027462260723ull;
    for (int i = 0; i < 8; i++) {
        state = state * MUL + INC;
        uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
        uint32_t rot = (uint32_t)(state >> 59);
        key[i] = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
    }
}

/* n Fr elements (Montgomery form) from ChaCha20(seed); element i uses words
 * [16 i, 16 i + 16) of the stream, i.e. exactly one 64-byte block. */
void o_chacha_fr(uint64_t seed, uint64_t first, size_t n, fe* out)
{
    uint32_t key[8];
    seed_key(seed, key);
    fe r2, r3;
    memcpy(r2.v, FR.r2, 32);
    r3 = f_mul(&FR, r2, r2); /* R^2 * R^2 / R = R^3 mod r, raw */
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
        uint32_t w[16];
        chacha_block(key, first + (uint64_t)i, w);
        fe d0, d1;
        for (int k = 0; k < 4; k++) {
            d0.v[k] = (uint64_t)w[2 * k] | ((uint64_t)w[2 * k + 1] << 32);
            d1.v[k] = (uint64_t)w[8 + 2 * k] | ((uint64_t)w[8 + 2 * k + 1] << 32);
        }
        out[i] = f_add(&FR, f_mul(&FR, d0, r2), f_mul(&FR, d1, r3));
    }
}

/* ----------------------------------------------------------------- NTT --- */

static inline uint64_t bitrev64(uint64_t x, int k)
{
    uint64_t r = 0;
    for (int i = 0; i < k; i++) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

/* In-place radix-2 DIT with natural-order input/output: A_j = sum a_i w^(ij).
 * Each stage is one parallel loop over its n/2 butterflies (so the last
 * stages, with few blocks, still use every thread), as best_fft splits its
 * work over the host threads. */
static void fft_inplace(fe* a, int k, fe w)
{
    uint64_t n = 1ull << k;
#pragma omp parallel for schedule(static) if (n >= (1u << 14))
    for (long i = 0; i < (long)n; i++) {
        uint64_t j = bitrev64((uint64_t)i, k);
        if ((uint64_t)i < j) { fe t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    /* twiddle table w^e, e < n/2, in chunks that start from w^(chunk start) */
    uint64_t half = n / 2;
    fe* tw = (fe*)malloc(sizeof(fe) * (half ? half : 1));
    const uint64_t TC = 4096;
#pragma omp parallel for schedule(static) if (half >= (1u << 14))
    for (long c = 0; c < (long)((half + TC - 1) / TC); c++) {
        uint64_t e0 = (uint64_t)c * TC, e1 = e0 + TC < half ? e0 + TC : half;
        fe p = f_pow_u64(&FR, w, e0);
        for (uint64_t e = e0; e < e1; e++) { tw[e] = p; p = f_mul(&FR, p, w); }
    }
    for (int s = 0; s < k; s++) {
        uint64_t m = 1ull << s, step = n >> (s + 1);
#pragma omp parallel for schedule(static) if (n >= (1u << 14))
        for (long t = 0; t < (long)half; t++) {
            uint64_t j = (uint64_t)t & (m - 1);
            uint64_t base = ((uint64_t)t >> s) << (s + 1);
            fe x = a[base + j];
            fe y = f_mul(&FR, a[base + j + m], tw[j * step]);
            a[base + j] = f_add(&FR, x, y);
            a[base + j + m] = f_sub(&FR, x, y);
        }
    }
    free(tw);
}

/* type 1 FFT, 2 iFFT, 3 cosetFFT, 4 icosetFFT, 6 CosetFFT_Part; out has
 * 2^log_ext entries for types 3/4, else 2^log_n. Returns 0 or -1. */
int o_ntt(uint32_t type, uint32_t log_n, uint32_t log_ext, const fe* in, fe* out, const fe* omega, const fe* divisor)
{
    uint64_t n = 1ull << log_n;
    if (type == 1 || type == 2 || type == 6) {
        memcpy(out, in, n * sizeof(fe));
        if (type == 6) {
            fe p = f_one(&FR);
            for (uint64_t i = 0; i < n; i++) { out[i] = f_mul(&FR, out[i], p); p = f_mul(&FR, p, *divisor); }
        }
        fft_inplace(out, (int)log_n, *omega);
        if (type == 2)
            for (uint64_t i = 0; i < n; i++) out[i] = f_mul(&FR, out[i], *divisor);
        return 0;
    }
    if (type == 3 || type == 4) {
        uint64_t N = 1ull << log_ext;
        memset(out, 0, N * sizeof(fe));
        memcpy(out, in, n * sizeof(fe));
        fe z[3] = {f_one(&FR), ZETA, ZETA2};
        if (type == 3) {
#pragma omp parallel for schedule(static) if (n >= (1u << 14))
            for (long i = 0; i < (long)n; i++) out[i] = f_mul(&FR, out[i], z[i % 3]);
            fft_inplace(out, (int)log_ext, *omega);
        } else {
            fft_inplace(out, (int)log_ext, *omega);
            fe zi[3] = {f_one(&FR), ZETA2, ZETA};
#pragma omp parallel for schedule(static) if (N >= (1u << 14))
            for (long i = 0; i < (long)N; i++) out[i] = f_mul(&FR, f_mul(&FR, out[i], *divisor), zi[i % 3]);
        }
        return 0;
    }
    return -1;
}

/* --------------------------------------------------------------- G1 ------ */
/* Jacobian (X, Y, Z), x = X/Z^2, y = Y/Z^3, infinity Z = 0; y^2 = x^3 + 3. */
typedef struct { fe X, Y, Z; } jac;
typedef struct { fe x, y; } aff;

static jac j_inf(void) { jac r; r.X = f_zero(); r.Y = f_one(&FQ); r.Z = f_zero(); return r; }
static int j_is_inf(const jac* p) { return f_is_zero(p->Z); }
static int a_is_inf(const aff* p) { return f_is_zero(p->x) && f_is_zero(p->y); }

static jac j_dbl(jac p)
{
    if (j_is_inf(&p)) return p;
    const field_t* F = &FQ;
    fe A = f_mul(F, p.X, p.X), B = f_mul(F, p.Y, p.Y), C = f_mul(F, B, B);
    fe t = f_add(F, p.X, B);
    fe D = f_dbl(F, f_sub(F, f_sub(F, f_mul(F, t, t), A), C));
    fe E = f_add(F, f_dbl(F, A), A);
    fe G = f_mul(F, E, E);
    jac r;
    r.X = f_sub(F, G, f_dbl(F, D));
    fe C8 = f_dbl(F, f_dbl(F, f_dbl(F, C)));
    r.Y = f_sub(F, f_mul(F, E, f_sub(F, D, r.X)), C8);
    r.Z = f_dbl(F, f_mul(F, p.Y, p.Z));
    return r;
}

static jac j_add(jac p, jac q)
{
    if (j_is_inf(&p)) return q;
    if (j_is_inf(&q)) return p;
    const field_t* F = &FQ;
    fe Z1Z1 = f_mul(F, p.Z, p.Z), Z2Z2 = f_mul(F, q.Z, q.Z);
    fe U1 = f_mul(F, p.X, Z2Z2), U2 = f_mul(F, q.X, Z1Z1);
    fe S1 = f_mul(F, f_mul(F, p.Y, q.Z), Z2Z2), S2 = f_mul(F, f_mul(F, q.Y, p.Z), Z1Z1);
    fe H = f_sub(F, U2, U1), R = f_sub(F, S2, S1);
    if (f_is_zero(H)) {
        if (f_is_zero(R)) return j_dbl(p);
        return j_inf();
    }
    fe HH = f_mul(F, H, H), HHH = f_mul(F, H, HH), V = f_mul(F, U1, HH);
    jac r;
    r.X = f_sub(F, f_sub(F, f_mul(F, R, R), HHH), f_dbl(F, V));
    r.Y = f_sub(F, f_mul(F, R, f_sub(F, V, r.X)), f_mul(F, S1, HHH));
    r.Z = f_mul(F, f_mul(F, p.Z, q.Z), H);
    return r;
}

static jac j_from_aff(aff a)
{
    if (a_is_inf(&a)) return j_inf();
    jac r; r.X = a.x; r.Y = a.y; r.Z = f_one(&FQ);
    return r;
}

/* Mixed addition p + a with a affine (Z2 = 1): the formulas of j_add with
 * U1 = X1 and S1 = Y1, 8M + 3S -- the bucket addition of halo2curves'
 * multiexp (affine bases added into projective buckets). */
static jac j_madd(jac p, aff a)
{
    if (a_is_inf(&a)) return p;
    if (j_is_inf(&p)) return j_from_aff(a);
    const field_t* F = &FQ;
    fe Z1Z1 = f_mul(F, p.Z, p.Z);
    fe U2 = f_mul(F, a.x, Z1Z1);
    fe S2 = f_mul(F, f_mul(F, a.y, p.Z), Z1Z1);
    fe H = f_sub(F, U2, p.X), R = f_sub(F, S2, p.Y);
    if (f_is_zero(H)) {
        if (f_is_zero(R)) return j_dbl(p);
        return j_inf();
    }
    fe HH = f_mul(F, H, H), HHH = f_mul(F, H, HH), V = f_mul(F, p.X, HH);
    jac r;
    r.X = f_sub(F, f_sub(F, f_mul(F, R, R), HHH), f_dbl(F, V));
    r.Y = f_sub(F, f_mul(F, R, f_sub(F, V, r.X)), f_mul(F, p.Y, HHH));
    r.Z = f_mul(F, p.Z, H);
    return r;
}

/* The reference's 96-byte result image: affine with Z = 1, or (0, 1, 0). */
static jac j_normalize(jac p)
{
    if (j_is_inf(&p)) return j_inf();
    const field_t* F = &FQ;
    fe zi = f_inv(F, p.Z), zi2 = f_mul(F, zi, zi), zi3 = f_mul(F, zi2, zi);
    jac r;
    r.X = f_mul(F, p.X, zi2);
    r.Y = f_mul(F, p.Y, zi3);
    r.Z = f_one(F);
    return r;
}

static jac j_mul(jac p, fe s_canon)
{
    jac r = j_inf();
    for (int w = 3; w >= 0; w--)
        for (int b = 63; b >= 0; b--) {
            r = j_dbl(r);
            if ((s_canon.v[w] >> b) & 1) r = j_add(r, p);
        }
    return r;
}

/* out = s * P, s Montgomery Fr, P affine Montgomery Fq; out = 96-byte image. */
void o_g1_mul(const fe* s, const aff* P, jac* out)
{
    *out = j_normalize(j_mul(j_from_aff(*P), f_from_mont(&FR, *s)));
}

void o_g1_add(const jac* a, const jac* b, jac* out) { *out = j_normalize(j_add(*a, *b)); }

void o_g1_generator(aff* g)
{
    fe one = {{1, 0, 0, 0}}, two = {{2, 0, 0, 0}};
    g->x = f_to_mont(&FQ, one);
    g->y = f_to_mont(&FQ, two);
}

int o_g1_on_curve(const aff* p)
{
    if (a_is_inf(p)) return 1;
    const field_t* F = &FQ;
    fe three = f_to_mont(F, (fe){{3, 0, 0, 0}});
    fe lhs = f_mul(F, p->y, p->y);
    fe rhs = f_add(F, f_mul(F, f_mul(F, p->x, p->x), p->x), three);
    return f_eq(lhs, rhs);
}

/* [tau^i] G for i < n: fixed-base multiplication over byte windows, with a
 * table T[w][d] = [d 256^w] G (32 x 255 affine points, built once per call),
 * so each point costs 32 mixed additions and one inversion. */
void o_srs(const fe* tau, size_t n, aff* out)
{
    aff g;
    o_g1_generator(&g);
    fe* pw = (fe*)malloc(sizeof(fe) * (n ? n : 1));
    fe p = f_one(&FR);
    for (size_t i = 0; i < n; i++) { pw[i] = p; p = f_mul(&FR, p, *tau); }
    aff* T = (aff*)malloc(sizeof(aff) * 32 * 255);
    jac base = j_from_aff(g);
    for (int w = 0; w < 32; w++) {
        jac acc = base;
        for (int d = 1; d <= 255; d++) {
            jac q = j_normalize(acc);
            T[w * 255 + d - 1].x = q.X;
            T[w * 255 + d - 1].y = q.Y;
            acc = j_add(acc, base);
        }
        for (int b = 0; b < 8; b++) base = j_dbl(base);
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (long i = 0; i < (long)n; i++) {
        fe s = f_from_mont(&FR, pw[i]);
        jac r = j_inf();
        for (int w = 0; w < 32; w++) {
            unsigned d = (unsigned)((s.v[w >> 3] >> (8 * (w & 7))) & 0xFF);
            if (d) r = j_madd(r, T[w * 255 + d - 1]);
        }
        r = j_normalize(r);
        if (j_is_inf(&r)) { out[i].x = f_zero(); out[i].y = f_zero(); }
        else { out[i].x = r.X; out[i].y = r.Y; }
    }
    free(T);
    free(pw);
}

/* ---------------------------------------------------------------- MSM ---- */

static uint64_t get_window(const fe* s, size_t seg, int c)
{
    size_t skip = seg * (size_t)c;
    size_t word = skip / 64, bit = skip % 64;
    if (word >= 4) return 0;
    u128 v = s->v[word];
    if (word + 1 < 4) v |= (u128)s->v[word + 1] << 64;
    return (uint64_t)(v >> bit) & ((1ull << c) - 1);
}

/* multiexp_serial: unsigned c-bit windows, c = ceil(ln n) (n >= 32),
 * buckets summed by parts, windows combined top-down with c doublings. */
static jac msm_serial(const fe* canon, const aff* bases, size_t n)
{
    int c = n < 4 ? 1 : (n < 32 ? 3 : (int)ceil(log((double)n)));
    size_t segments = (254 + c - 1) / c;
    jac acc = j_inf();
    jac* buckets = (jac*)malloc(sizeof(jac) * ((1ull << c) - 1));
    for (long seg = (long)segments - 1; seg >= 0; seg--) {
        for (int d = 0; d < c; d++) acc = j_dbl(acc);
        for (size_t b = 0; b < (1ull << c) - 1; b++) buckets[b] = j_inf();
        for (size_t i = 0; i < n; i++) {
            uint64_t w = get_window(&canon[i], (size_t)seg, c);
            if (w) buckets[w - 1] = j_madd(buckets[w - 1], bases[i]);
        }
        jac run = j_inf();
        for (long b = (long)(1ull << c) - 2; b >= 0; b--) {
            run = j_add(run, buckets[b]);
            acc = j_add(acc, run);
        }
    }
    free(buckets);
    return acc;
}

/* best_multiexp_cpu: contiguous chunks, one per thread, summed. */
void o_msm(const fe* scalars, const aff* bases, size_t n, int threads, jac* out)
{
    fe* canon = (fe*)malloc(sizeof(fe) * (n ? n : 1));
    for (size_t i = 0; i < n; i++) canon[i] = f_from_mont(&FR, scalars[i]);
    if (threads < 1) threads = 1;
    jac total = j_inf();
    if ((size_t)threads < n) {
        size_t chunk = n / (size_t)threads;
        size_t nch = (n + chunk - 1) / chunk;
        jac* res = (jac*)malloc(sizeof(jac) * nch);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
        for (long k = 0; k < (long)nch; k++) {
            size_t s = (size_t)k * chunk, e = s + chunk < n ? s + chunk : n;
            res[k] = msm_serial(canon + s, bases + s, e - s);
        }
        for (size_t k = 0; k < nch; k++) total = j_add(total, res[k]);
        free(res);
    } else {
        total = msm_serial(canon, bases, n);
    }
    free(canon);
    *out = j_normalize(total);
}

/* Straight double-and-add sum, for cross-checking o_msm on small inputs. */
void o_msm_naive(const fe* scalars, const aff* bases, size_t n, jac* out)
{
    jac acc = j_inf();
    for (size_t i = 0; i < n; i++) acc = j_add(acc, j_mul(j_from_aff(bases[i]), f_from_mont(&FR, scalars[i])));
    *out = j_normalize(acc);
}

/* ------------------------------------------------------ batch inversion -- */

void o_batch_invert(fe* d, size_t n, int fq)
{
    const field_t* F = fq ? &FQ : &FR;
    fe* pre = (fe*)malloc(sizeof(fe) * (n ? n : 1));
    fe acc = f_one(F);
    for (size_t i = 0; i < n; i++) {
        if (!f_is_zero(d[i])) acc = f_mul(F, acc, d[i]);
        pre[i] = acc;
    }
    fe inv = f_inv(F, acc);
    for (long i = (long)n - 1; i >= 0; i--) {
        if (f_is_zero(d[i])) continue;
        fe prev = i > 0 ? pre[i - 1] : f_one(F);
        fe out = f_mul(F, inv, prev);
        inv = f_mul(F, inv, d[i]);
        d[i] = out;
    }
    free(pre);
}

/* Chunked (one Montgomery trick per thread) for the timed CPU baseline. */
void o_batch_invert_par(fe* d, size_t n, int fq, int threads)
{
    if (threads < 1) threads = 1;
    size_t chunk = (n + (size_t)threads - 1) / (size_t)threads;
#pragma omp parallel for num_threads(threads) schedule(static, 1)
    for (long k = 0; k < threads; k++) {
        size_t s = (size_t)k * chunk;
        if (s >= n) continue;
        size_t e = s + chunk < n ? s + chunk : n;
        o_batch_invert(d + s, e - s, fq);
    }
}

/* ---------------------------------------------------- products and scans -- */

void o_grand_product(const fe* in, fe* out, size_t n, const fe* prefix)
{
    fe acc = *prefix;
    for (size_t i = 0; i < n; i++) { acc = f_mul(&FR, acc, in[i]); out[i] = acc; }
}

void o_lookup_product(fe* out, const fe* pin, const fe* ptab, const fe* cin, const fe* ctab, const fe* beta,
                      const fe* gamma, size_t n)
{
    for (size_t i = 0; i < n; i++) out[i] = f_mul(&FR, f_add(&FR, *beta, pin[i]), f_add(&FR, *gamma, ptab[i]));
    o_batch_invert(out, n, 0);
    for (size_t i = 0; i < n; i++) {
        out[i] = f_mul(&FR, out[i], f_add(&FR, cin[i], *beta));
        out[i] = f_mul(&FR, out[i], f_add(&FR, ctab[i], *gamma));
    }
}

/* values[c], perms[c] point at the chunk (already offset); deltaomega is advanced by delta^batch. */
void o_permutation_product(fe* mod, const fe* const* values, const fe* const* perms, size_t batch, size_t n,
                           const fe* omega, const fe* beta, const fe* gamma, const fe* delta, fe* deltaomega)
{
    for (size_t c = 0; c < batch; c++)
        for (size_t i = 0; i < n; i++)
            mod[i] = f_mul(&FR, mod[i], f_add(&FR, f_add(&FR, f_mul(&FR, *beta, perms[c][i]), *gamma), values[c][i]));
    o_batch_invert(mod, n, 0);
    fe dw = *deltaomega;
    for (size_t c = 0; c < batch; c++) {
        fe cur = dw;
        for (size_t i = 0; i < n; i++) {
            mod[i] = f_mul(&FR, mod[i], f_add(&FR, f_add(&FR, f_mul(&FR, cur, *beta), *gamma), values[c][i]));
            cur = f_mul(&FR, cur, *omega);
        }
        dw = f_mul(&FR, dw, *delta);
    }
    *deltaomega = dw;
}

/* ----------------------------------------------------- lookup permute ---- */

static int cmp_canon(const void* a, const void* b)
{
    const fe* x = (const fe*)a;
    const fe* y = (const fe*)b;
    for (int i = 3; i >= 0; i--) {
        if (x->v[i] < y->v[i]) return -1;
        if (x->v[i] > y->v[i]) return 1;
    }
    return 0;
}

typedef struct { fe canon; fe mont; } keyed;
static int cmp_keyed(const void* a, const void* b) { return cmp_canon(&((const keyed*)a)->canon, &((const keyed*)b)->canon); }

/* Returns 0, or -1 when an input value is absent from the table (the reference panics). */
int o_permute_pair(const fe* input, const fe* table, size_t n, size_t usable, fe* pin, fe* ptab)
{
    keyed* a = (keyed*)malloc(sizeof(keyed) * (usable ? usable : 1));
    keyed* t = (keyed*)malloc(sizeof(keyed) * (usable ? usable : 1));
    for (size_t i = 0; i < usable; i++) {
        a[i].mont = input[i]; a[i].canon = f_from_mont(&FR, input[i]);
        t[i].mont = table[i]; t[i].canon = f_from_mont(&FR, table[i]);
    }
    qsort(a, usable, sizeof(keyed), cmp_keyed);
    qsort(t, usable, sizeof(keyed), cmp_keyed);
    /* distinct table values with counts, ascending */
    size_t nu = 0;
    keyed* uv = (keyed*)malloc(sizeof(keyed) * (usable ? usable : 1));
    uint32_t* cnt = (uint32_t*)malloc(sizeof(uint32_t) * (usable ? usable : 1));
    for (size_t i = 0; i < usable; i++) {
        if (nu == 0 || cmp_canon(&uv[nu - 1].canon, &t[i].canon) != 0) { uv[nu] = t[i]; cnt[nu] = 0; nu++; }
        cnt[nu - 1]++;
    }
    size_t* rep = (size_t*)malloc(sizeof(size_t) * (usable ? usable : 1));
    size_t nrep = 0;
    int rc = 0;
    size_t tp = 0; /* pointer into uv: inputs are sorted, so lookups are monotone */
    for (size_t r = 0; r < usable; r++) {
        pin[r] = a[r].mont;
        if (r == 0 || cmp_canon(&a[r].canon, &a[r - 1].canon) != 0) {
            ptab[r] = a[r].mont;
            while (tp < nu && cmp_canon(&uv[tp].canon, &a[r].canon) < 0) tp++;
            if (tp < nu && cmp_canon(&uv[tp].canon, &a[r].canon) == 0 && cnt[tp] > 0) cnt[tp]--;
            else { rc = -1; }
        } else {
            rep[nrep++] = r;
        }
    }
    for (size_t u = 0; u < nu && rc == 0; u++)
        for (uint32_t k = 0; k < cnt[u]; k++) {
            if (nrep == 0) { rc = -1; break; }
            ptab[rep[--nrep]] = uv[u].mont;
        }
    for (size_t r = usable; r < n; r++) { pin[r] = f_zero(); ptab[r] = f_zero(); }
    free(a); free(t); free(uv); free(cnt); free(rep);
    return rc;
}

/* ------------------------------------------------------------ quotient --- */

static inline int vs_rot(uint64_t r)
{
    int sign = (int)((r >> 15) & 1);
    int abs = (int)(r & 0x7fff);
    return sign ? -abs : abs;
}

/* Columns are full-length (num_quotient rows) arrays; rows [row_start,
 * row_end) are written to out[row - row_start].  prev may be NULL. */
void o_quotient(const fe* const* fixed, const fe* const* instance, const fe* const* advice, const fe* challenges,
                const fe* constants, const fe* expr_constants, const uint64_t* rules, uint64_t num_rules,
                const uint64_t* vp_rules, uint64_t num_vp, uint64_t num_quotient, uint64_t rot_scale,
                uint64_t row_start, uint64_t row_end, const fe* prev, fe* out)
{
    const fe y = expr_constants[4];
#pragma omp parallel
    {
        fe* inter = (fe*)malloc(sizeof(fe) * (num_rules ? num_rules : 1));
#pragma omp for schedule(static)
        for (long rr = (long)row_start; rr < (long)row_end; rr++) {
            for (uint64_t i = 0; i < num_rules; i++) {
                uint64_t lo = rules[2 * i], hi = rules[2 * i + 1];
                fe ab[2];
                for (int k = 0; k < 2; k++) {
                    uint64_t vs = k == 0 ? lo : hi;
                    int src = (int)(vs & 0xf);
                    uint64_t idx = (vs >> 4) & 0xfffff;
                    int rot = vs_rot(vs >> 24);
                    int64_t row = ((int64_t)rr + (int64_t)rot * (int64_t)rot_scale) % (int64_t)num_quotient;
                    if (row < 0) row += (int64_t)num_quotient;
                    fe v = f_zero();
                    switch (src) {
                    case 0: v = fixed[idx][row]; break;
                    case 1: v = instance[idx][row]; break;
                    case 2: v = advice[idx][row]; break;
                    case 3: v = inter[idx]; break;
                    case 4: v = constants[idx]; break;
                    case 5: v = challenges[idx]; break;
                    default: v = f_zero();
                    }
                    ab[k] = v;
                }
                int c1 = (int)((lo >> 40) & 0xf), d = (int)((lo >> 44) & 0xf), c2 = (int)((hi >> 40) & 0xf);
                fe r = f_zero();
                if (c1 == 1) {
                    if (c2 == 0) r = d == 1 ? f_mul(&FR, ab[0], ab[1]) : ab[0];
                    else if (c2 == 1) r = f_add(&FR, ab[0], ab[1]);
                    else if (c2 == 2) r = f_sub(&FR, ab[0], ab[1]);
                } else if (c1 == 2) {
                    r = f_neg(&FR, ab[0]);
                } else if (c1 == 3) {
                    r = f_add(&FR, ab[0], ab[0]);
                }
                inter[i] = r;
            }
            fe val = prev ? prev[rr - (long)row_start] : f_zero();
            for (uint64_t i = 0; i < num_vp; i++) {
                uint64_t vs = vp_rules[i];
                int src = (int)(vs & 0xf);
                uint64_t idx = (vs >> 4) & 0xfffff;
                fe part = src == 4 ? constants[idx] : inter[idx];
                val = f_add(&FR, f_mul(&FR, val, y), part);
            }
            out[rr - (long)row_start] = val;
        }
        free(inter);
    }
}

static inline size_t rot_idx(size_t idx, int rot, int scale, int isize)
{
    long r = ((long)idx + (long)rot * scale) % isize;
    if (r < 0) r += isize;
    return (size_t)r;
}

void o_quotient_lookups(fe* values, const fe* table_values, const fe* product, const fe* pin, const fe* ptab,
                        const fe* l0, const fe* l_last, const fe* l_active, const fe* beta, const fe* gamma,
                        const fe* y, size_t n)
{
    const field_t* F = &FR;
    fe one = f_one(F);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
        size_t nx = rot_idx((size_t)i, 1, 1, (int)n), pv = rot_idx((size_t)i, -1, 1, (int)n);
        fe v = values[i];
        fe ams = f_sub(F, pin[i], ptab[i]);
        v = f_add(F, f_mul(F, v, *y), f_mul(F, f_sub(F, one, product[i]), l0[i]));
        v = f_add(F, f_mul(F, v, *y), f_mul(F, f_sub(F, f_mul(F, product[i], product[i]), product[i]), l_last[i]));
        fe lhs = f_mul(F, f_mul(F, product[nx], f_add(F, pin[i], *beta)), f_add(F, ptab[i], *gamma));
        fe t = f_mul(F, f_sub(F, lhs, f_mul(F, product[i], table_values[i])), l_active[i]);
        v = f_add(F, f_mul(F, v, *y), t);
        v = f_add(F, f_mul(F, v, *y), f_mul(F, ams, l0[i]));
        v = f_add(F, f_mul(F, v, *y), f_mul(F, f_mul(F, ams, f_sub(F, pin[i], pin[pv])), l_active[i]));
        values[i] = v;
    }
}

void o_permutation_quotient(fe* values, size_t start, size_t len, int rot_scale, int isize, int last_rotation,
                            size_t chunk_len, const fe* const* cols, size_t ncols, const fe* const* prods,
                            size_t nsets, const fe* const* perms, const fe* l0, const fe* l_last, const fe* l_active,
                            const fe* y, const fe* beta, const fe* gamma, const fe* delta, const fe* delta_start,
                            const fe* cur_ext_omega, const fe* omega)
{
    const field_t* F = &FR;
    fe one = f_one(F);
    const fe* first = prods[0];
    const fe* last = prods[nsets - 1];
    fe beta_term = f_mul(F, *cur_ext_omega, f_pow_u64(F, *omega, start));
    for (size_t i = 0; i < len; i++) {
        size_t idx = start + i;
        size_t r_next = rot_idx(idx, 1, rot_scale, isize), r_last = rot_idx(idx, last_rotation, rot_scale, isize);
        fe v = values[i];
        v = f_add(F, f_mul(F, v, *y), f_mul(F, f_sub(F, one, first[idx]), l0[idx]));
        v = f_add(F, f_mul(F, v, *y), f_mul(F, f_sub(F, f_mul(F, last[idx], last[idx]), last[idx]), l_last[idx]));
        for (size_t s = 1; s < nsets; s++)
            v = f_add(F, f_mul(F, v, *y), f_mul(F, f_sub(F, prods[s][idx], prods[s - 1][r_last]), l0[idx]));
        fe cur_delta = f_mul(F, *delta_start, beta_term);
        for (size_t s = 0; s < nsets; s++) {
            size_t c0 = s * chunk_len, c1 = c0 + chunk_len < ncols ? c0 + chunk_len : ncols;
            fe left = prods[s][r_next];
            for (size_t c = c0; c < c1; c++)
                left = f_mul(F, left, f_add(F, f_add(F, cols[c][idx], f_mul(F, *beta, perms[c][idx])), *gamma));
            fe right = prods[s][idx];
            for (size_t c = c0; c < c1; c++) {
                right = f_mul(F, right, f_add(F, f_add(F, cols[c][idx], cur_delta), *gamma));
                cur_delta = f_mul(F, cur_delta, *delta);
            }
            v = f_add(F, f_mul(F, v, *y), f_mul(F, f_sub(F, left, right), l_active[idx]));
        }
        values[i] = v;
        beta_term = f_mul(F, beta_term, *omega);
    }
}

int o_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* f(x_j) for m points at once: each thread runs Horner for its share of the
 * points in one pass over the coefficients (Montgomery in, Montgomery out). */
void o_fr_eval_many(const fe* coeffs, size_t n, const fe* xs, size_t m, fe* out)
{
    const long B = 8;
#pragma omp parallel for schedule(dynamic, 1)
    for (long j0 = 0; j0 < (long)m; j0 += B) {
        long cnt = (long)m - j0 < B ? (long)m - j0 : B;
        fe acc[8];
        for (long t = 0; t < cnt; t++) acc[t] = f_zero();
        for (long i = (long)n - 1; i >= 0; i--)
            for (long t = 0; t < cnt; t++) acc[t] = f_add(&FR, f_mul(&FR, acc[t], xs[j0 + t]), coeffs[i]);
        for (long t = 0; t < cnt; t++) out[j0 + t] = acc[t];
    }
}

/* f(x) = sum_i c_i x^i by Horner (Montgomery in, Montgomery out). */
void o_fr_eval(const fe* coeffs, size_t n, const fe* x, fe* out)
{
    fe acc = f_zero();
    for (long i = (long)n - 1; i >= 0; i--) acc = f_add(&FR, f_mul(&FR, acc, *x), coeffs[i]);
    *out = acc;
}
