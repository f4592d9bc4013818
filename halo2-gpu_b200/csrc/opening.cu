// Opening-phase polynomial kernels (the KZG multi-open step after the
// quotient) and the witness decode before phase 1:
//
//  * _halo2_eval_polynomial{,_workspace_size} (halo2_proofs/cuda/src/polynomial/
//    polynomial.cu:15-110): sum_i a_i z^i of a device polynomial, result left
//    in device scratch.
//  * _halo2_eval_polynomial_batch{,_workspace_size}, _halo2_eval_poly_batch_max_len
//    (polynomial.cu:112-245): the same over chunks [offset, offset + len) of host
//    polynomials with local exponents (z^0 at `offset`), host results.
//  * _halo2_kate_division_device{,_padded,_workspace_size}
//    (halo2_proofs/cuda/src/polynomial/kate_division.cu:27-250):
//    q(X) = (a(X) - a(u)) / (X - u), i.e. q_{n-2} = a_{n-1} and
//    q_{j-1} = a_j + u q_j.
//  * _halo2_multiopen_poly_calculation{,_workspace_size}, _halo2_multiopen_poly_max_len
//    (halo2_proofs/cuda/src/multiopen.cu:30-175): per pair (poly_i chunk, z_i)
//    the chunk's evaluation, and acc = sum_i c_i poly_i over the chunk.
//  * _halo2_decode_assigned (halo2_proofs/cuda/src/polynomial/decode_assigned.cu:28-60):
//    Assigned<F> records -> numerators and denominators.
//
// Evaluation: CTA b owns a tile of EV_T * EV_E coefficients; thread c takes
// coefficients base + c + EV_T j (coalesced), runs Horner in z^EV_T over j
// and scales by z^(base + c) from a squaring chain; CTA partial sums are added
// by a second kernel.
//
// Kate division is the linear recurrence Y_t = r_t + u Y_{t-1} over the
// reversed coefficients r_t = a_{n-1-t} (q_{n-2-t} = Y_t).  With a constant
// multiplier it scans like a prefix sum over tiles of T = KD_T * KD_E = 2048
// values.  The coefficients' own level (level 0) is a weighted prefix sum:
// in tile k with local index j, the solution with zero carry-in is
// u^j P_j, P_j = sum_{s <= j} r_{kT+s} u^-s (one product per value, then
// additions only), and with the true value C before the tile
// Y_t = u^j (P_j + u C) (one product per value); u^j and u^-j for j < T are
// tables built once per division (one inversion of u).  The tile totals
// u^(T-1) P_{T-1} form the same recurrence one level up with multiplier
// u^T, solved by thread-sequential tiles and a Hillis-Steele scan of the
// thread totals with multipliers v^(8 * 2^d), whose down pass adds
// v^(position + 1) * carry.  Scratch is the two tables and a few small
// per-level arrays instead of n-length state arrays.
#define H2B_INLINE_MUL 1
#include <algorithm>
#include "abi.cuh"
#include "field.cuh"
#include "inverse.cuh"

namespace h2b {

namespace {
constexpr int EV_T = 256;
constexpr int EV_E = 16;
constexpr int EV_LOGT = 8;
constexpr uint64_t EV_TILE = (uint64_t)EV_T * EV_E;
constexpr int CHAIN = 48;      // z^(2^i), i < 48: exponents below 2^48

constexpr int KD_T = 256;
constexpr int KD_E = 8;
constexpr uint64_t KD_TILE = (uint64_t)KD_T * KD_E;  // 2048
constexpr int KD_TAB = 17;     // v^1..v^8, v^(8*2^d) for d = 0..8 (the last = v^2048)
constexpr int KD_MAX_LEVELS = 4;
}

// chain[i] = z^(2^i), i < CHAIN (one thread)
static __global__ void k_op_chain(const Fr* __restrict__ z, Fr* __restrict__ chain)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    Fr c = ld(z);
    for (int i = 0; i < CHAIN; i++) {
        st(&chain[i], c);
        c = c * c;
    }
}

static __device__ __forceinline__ Fr op_pow(const Fr* __restrict__ chain, uint64_t e)
{
    Fr r = Fr::one();
    for (int j = 0; e; j++, e >>= 1)
        if (e & 1) r = r * ldg(&chain[j]);
    return r;
}

// partial[b] = sum over the tile of a_i z^i (global exponents).
static __device__ __forceinline__ void eval_partial_tile(const Fr* __restrict__ a, uint64_t n,
                                                         const Fr* __restrict__ chain, Fr* __restrict__ partial);
static __global__ void __launch_bounds__(EV_T) k_eval_partial(const Fr* __restrict__ a, uint64_t n,
                                                               const Fr* __restrict__ chain, Fr* __restrict__ partial)
{
    eval_partial_tile(a, n, chain, partial);
}

static __device__ __forceinline__ void eval_partial_tile(const Fr* __restrict__ a, uint64_t n,
                                                         const Fr* __restrict__ chain, Fr* __restrict__ partial)
{
    __shared__ Fr red[EV_T];
    const uint64_t base = blockIdx.x * EV_TILE;
    const int c = threadIdx.x;
    const Fr zt = ldg(&chain[EV_LOGT]);  // z^EV_T
    Fr h = Fr::zero();
#pragma unroll 1
    for (int j = EV_E - 1; j >= 0; j--) {
        const uint64_t i = base + c + (uint64_t)EV_T * j;
        h = h * zt;
        if (i < n) h = h + ld(&a[i]);
    }
    h = h * op_pow(chain, base + c);
    red[c] = h;
    __syncthreads();
    for (int w = EV_T / 2; w >= 1; w >>= 1) {
        if (c < w) red[c] = red[c] + red[c + w];
        __syncthreads();
    }
    if (c == 0) st(&partial[blockIdx.x], red[0]);
}

static __device__ __forceinline__ void eval_sum_block(const Fr* __restrict__ partial, uint64_t nb, Fr* __restrict__ out);
static __global__ void __launch_bounds__(EV_T) k_eval_sum(const Fr* __restrict__ partial, uint64_t nb,
                                                           Fr* __restrict__ out)
{
    eval_sum_block(partial, nb, out);
}

static __device__ __forceinline__ void eval_sum_block(const Fr* __restrict__ partial, uint64_t nb, Fr* __restrict__ out)
{
    __shared__ Fr red[EV_T];
    const int c = threadIdx.x;
    Fr s = Fr::zero();
    for (uint64_t i = c; i < nb; i += EV_T) s = s + ld(&partial[i]);
    red[c] = s;
    __syncthreads();
    for (int w = EV_T / 2; w >= 1; w >>= 1) {
        if (c < w) red[c] = red[c] + red[c + w];
        __syncthreads();
    }
    if (c == 0) st(out, red[0]);
}

// acc[i] += c * p[i]
static __global__ void k_op_madd(Fr* __restrict__ acc, const Fr* __restrict__ p, const Fr* __restrict__ c, uint64_t n)
{
    const Fr cc = ldg(c);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        st(&acc[i], ld(&acc[i]) + cc * ld(&p[i]));
}

// ---- many polynomials per launch (device polynomials of one length) --------

constexpr int MANY_MAX = 64;
struct EvMany {
    const Fr* p[MANY_MAX];
    Fr z[MANY_MAX];
};
struct LinTerms {
    const Fr* p[MANY_MAX];
    Fr c[MANY_MAX];
};

// chain[y CHAIN + i] = z_y^(2^i) (one thread per polynomial)
static __global__ void k_op_chain_many(const __grid_constant__ EvMany E, Fr* __restrict__ chains)
{
    if (threadIdx.x != 0) return;
    Fr c = E.z[blockIdx.x];
    Fr* chain = chains + (uint64_t)blockIdx.x * CHAIN;
    for (int i = 0; i < CHAIN; i++) {
        st(&chain[i], c);
        c = c * c;
    }
}

// grid (tiles, polynomials): the tile partials of polynomial y
static __global__ void __launch_bounds__(EV_T) k_eval_partial_many(const __grid_constant__ EvMany E, uint64_t n,
                                                                    const Fr* __restrict__ chains,
                                                                    Fr* __restrict__ partial, uint64_t nb)
{
    const uint32_t y = blockIdx.y;
    eval_partial_tile(E.p[y], n, chains + (uint64_t)y * CHAIN, partial + (uint64_t)y * nb);
}

// block y: polynomial y's partials summed into out[y]
static __global__ void __launch_bounds__(EV_T) k_eval_sum_many(const Fr* __restrict__ partial, uint64_t nb,
                                                                Fr* __restrict__ out)
{
    eval_sum_block(partial + (uint64_t)blockIdx.x * nb, nb, out + blockIdx.x);
}

// acc[i] = (accumulate ? acc[i] : 0) + sum_t c_t p_t[i]: every polynomial
// read once, the accumulator read and written once
static __global__ void k_lin_comb(Fr* __restrict__ acc, const __grid_constant__ LinTerms L, uint32_t count,
                                  uint64_t n, int accumulate)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        Fr s = accumulate ? ld(&acc[i]) : Fr::zero();
        for (uint32_t t = 0; t < count; t++) s = s + L.c[t] * ld(&L.p[t][i]);
        st(&acc[i], s);
    }
}

// ---- Kate division ---------------------------------------------------------

// tab[0..7] = v^1..v^8, tab[8 + d] = v^(8 * 2^d) (d = 0..8), from v (one thread).
static __global__ void k_kd_table(const Fr* __restrict__ v_in, Fr* __restrict__ tab)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const Fr v = ld(v_in);
    Fr p = v;
    for (int k = 0; k < 8; k++) {
        st(&tab[k], p);
        if (k < 7) p = p * v;
    }
    for (int d = 0; d <= 8; d++) {
        st(&tab[8 + d], p);
        p = p * p;
    }
}

// Level L value t lives at: level 0 -> q[n-2-t] (reversed, written only below
// qlim), level >= 1 -> arr[t].
struct KdLevel {
    Fr* arr;
    uint64_t m;          // values on this level
    bool rev;            // level 0
    uint64_t n;          // level 0: polynomial length
    uint64_t qlim;       // level 0: q indices written are < qlim
};

static __device__ __forceinline__ uint64_t kd_qidx(const KdLevel& L, uint64_t t) { return L.n - 2 - t; }

// Up pass: solve each tile with zero carry-in; write the values and the tile
// total (the value at the tile's last position) to tot[tile].
static __global__ void __launch_bounds__(KD_T) k_kd_up(KdLevel L, const Fr* __restrict__ a, const Fr* __restrict__ tab,
                                                        Fr* __restrict__ tot)
{
    __shared__ Fr sm[2][KD_T];
    const int c = threadIdx.x;
    const uint64_t t0 = blockIdx.x * KD_TILE + (uint64_t)c * KD_E;
    const Fr v = ldg(&tab[0]);
    Fr y[KD_E];
#pragma unroll
    for (int k = 0; k < KD_E; k++) {
        const uint64_t t = t0 + k;
        Fr r = Fr::zero();
        if (t < L.m) r = L.rev ? ld(&a[L.n - 1 - t]) : ld(&L.arr[t]);
        y[k] = k == 0 ? r : r + v * y[k - 1];
    }
    // inclusive scan of thread totals: S_c = Z_c + V S_{c-1}, V = v^8
    Fr s = y[KD_E - 1];
    int buf = 0;
    sm[buf][c] = s;
    __syncthreads();
    for (int d = 0; (1 << d) < KD_T; d++) {
        if (c >= (1 << d)) s = s + ldg(&tab[8 + d]) * sm[buf][c - (1 << d)];
        buf ^= 1;
        sm[buf][c] = s;
        __syncthreads();
    }
    if (c > 0) {
        const Fr C = sm[buf][c - 1];  // exclusive carry
        Fr p = v;
#pragma unroll
        for (int k = 0; k < KD_E; k++) {
            y[k] = y[k] + p * C;
            p = p * v;
        }
    }
#pragma unroll
    for (int k = 0; k < KD_E; k++) {
        const uint64_t t = t0 + k;
        if (t >= L.m) break;
        if (L.rev) {
            const uint64_t q = kd_qidx(L, t);
            if (q < L.qlim) st(&L.arr[q], y[k]);
        } else {
            st(&L.arr[t], y[k]);
        }
    }
    if (c == KD_T - 1) st(&tot[blockIdx.x], s);
}

// Down pass: tile b >= 1 adds v^(pos + 1) * Y_end(b - 1), pos = t - tile start.
static __global__ void __launch_bounds__(KD_T) k_kd_down(KdLevel L, const Fr* __restrict__ tab,
                                                          const Fr* __restrict__ tot)
{
    const uint64_t b = blockIdx.x + 1;
    const int c = threadIdx.x;
    const uint64_t t0 = b * KD_TILE + (uint64_t)c * KD_E;
    if (t0 >= L.m) return;
    const Fr C = ld(&tot[b - 1]);
    const Fr v = ldg(&tab[0]);
    Fr p = v;  // v^(8c + 1)
    for (int d = 0; d < 8; d++)
        if ((c >> d) & 1) p = p * ldg(&tab[8 + d]);
#pragma unroll
    for (int k = 0; k < KD_E; k++) {
        const uint64_t t = t0 + k;
        if (t >= L.m) break;
        if (L.rev) {
            const uint64_t q = kd_qidx(L, t);
            if (q < L.qlim) st(&L.arr[q], ld(&L.arr[q]) + p * C);
        } else {
            st(&L.arr[t], ld(&L.arr[t]) + p * C);
        }
        p = p * v;
    }
}

// u^j and u^-j for j < KD_TILE (U and W), one CTA: thread 0 inverts u (0
// stays 0) and forms u^(8 * 2^d), u^-(8 * 2^d); thread c then builds
// entries 8c .. 8c + 7 from u^(8c) and u^-(8c).
static __global__ void __launch_bounds__(KD_T) k_kd_pow(const Fr* __restrict__ u_in, Fr* __restrict__ U,
                                                         Fr* __restrict__ W)
{
    __shared__ Fr base[2][9];  // [0]: u, u^8, u^16, ...; [1]: the same for u^-1
    const int c = threadIdx.x;
    if (c == 0) {
        Fr x[2];
        x[0] = ld(u_in);
        x[1] = finv_fast(x[0]);
        for (int s = 0; s < 2; s++) {
            base[s][0] = x[s];
            Fr p = x[s] * x[s];
            p = p * p;
            p = p * p;  // x^8
            for (int d = 0; d < 8; d++) {
                base[s][1 + d] = p;
                p = p * p;
            }
        }
    }
    __syncthreads();
    for (int s = 0; s < 2; s++) {
        Fr p = Fr::one();
        for (int d = 0; d < 8; d++)
            if ((c >> d) & 1) p = p * base[s][1 + d];
        Fr* out = s ? W : U;
        const Fr x = base[s][0];
#pragma unroll 1
        for (int k = 0; k < KD_E; k++) {
            st(&out[c * KD_E + k], p);
            if (k + 1 < KD_E) p = p * x;
        }
    }
}

// Level 0 up: P_j = sum_{s <= j} r_{kT+s} u^-s within the tile, written to q
// (below qlim); the tile's zero-carry end value u^(T-1) P_{T-1} to tot.
static __global__ void __launch_bounds__(KD_T, 2) k_kd0_up(KdLevel L, const Fr* __restrict__ a,
                                                            const Fr* __restrict__ U, const Fr* __restrict__ W,
                                                            Fr* __restrict__ tot)
{
    __shared__ Fr sm[2][KD_T];
    const int c = threadIdx.x;
    const uint64_t t0 = blockIdx.x * KD_TILE + (uint64_t)c * KD_E;
    Fr y[KD_E];
#pragma unroll
    for (int k = 0; k < KD_E; k++) {
        const uint64_t t = t0 + k;
        y[k] = t < L.m ? ld(&a[L.n - 1 - t]) * ldg(&W[c * KD_E + k]) : Fr::zero();
    }
#pragma unroll
    for (int k = 1; k < KD_E; k++) y[k] = y[k] + y[k - 1];
    // inclusive scan of the thread totals (additions)
    Fr s = y[KD_E - 1];
    int buf = 0;
    sm[buf][c] = s;
    __syncthreads();
    for (int d = 0; (1 << d) < KD_T; d++) {
        if (c >= (1 << d)) s = s + sm[buf][c - (1 << d)];
        buf ^= 1;
        sm[buf][c] = s;
        __syncthreads();
    }
    if (c > 0) {
        const Fr ex = sm[buf][c - 1];
#pragma unroll
        for (int k = 0; k < KD_E; k++) y[k] = y[k] + ex;
    }
#pragma unroll
    for (int k = 0; k < KD_E; k++) {
        const uint64_t t = t0 + k;
        if (t >= L.m) break;
        const uint64_t q = kd_qidx(L, t);
        if (q < L.qlim) st(&L.arr[q], y[k]);
    }
    if (c == KD_T - 1) st(&tot[blockIdx.x], ldg(&U[KD_TILE - 1]) * s);
}

// Level 0 down: Y_t = u^j (P_j + u C), C = tot[k - 1] (the solved value
// before tile k; 0 for tile 0).  With u = 0, Y_t = r_t.
static __global__ void __launch_bounds__(KD_T) k_kd0_down(KdLevel L, const Fr* __restrict__ a,
                                                           const Fr* __restrict__ U, const Fr* __restrict__ tot)
{
    const uint64_t b = blockIdx.x;
    const int c = threadIdx.x;
    const uint64_t t0 = b * KD_TILE + (uint64_t)c * KD_E;
    if (t0 >= L.m) return;
    const Fr u = ldg(&U[1]);
    const bool u_zero = u.is_zero();
    const Fr uc = b > 0 ? u * ld(&tot[b - 1]) : Fr::zero();
#pragma unroll
    for (int k = 0; k < KD_E; k++) {
        const uint64_t t = t0 + k;
        if (t >= L.m) break;
        const uint64_t q = kd_qidx(L, t);
        if (q >= L.qlim) continue;
        st(&L.arr[q], u_zero ? ld(&a[L.n - 1 - t]) : ldg(&U[c * KD_E + k]) * (ld(&L.arr[q]) + uc));
    }
}

struct KdPlan {
    int levels = 0;          // levels above 0
    uint64_t m[KD_MAX_LEVELS + 1];
};

static KdPlan kd_plan(uint64_t length)
{
    KdPlan P;
    P.m[0] = length;
    while (P.m[P.levels] > KD_TILE && P.levels < KD_MAX_LEVELS) {
        P.m[P.levels + 1] = (P.m[P.levels] + KD_TILE - 1) / KD_TILE;
        P.levels++;
    }
    return P;
}

static void kd_plan_scratch(ScratchPlan& sp, uint64_t n)
{
    if (n < 2) return;
    const KdPlan P = kd_plan(n - 1);
    sp.add_n<Fr>((uint64_t)KD_TAB * (P.levels + 1));          // power tables
    for (int l = 1; l <= P.levels; l++) sp.add_n<Fr>(P.m[l]);  // level values
    sp.add_n<Fr>(1);                                            // top-level total (unused)
    sp.add_n<Fr>(2 * KD_TILE);                                  // u^j, u^-j for level 0
}

static RustError kd_run(const Fr* a, Fr* q, const Fr* u, uint64_t n, uint64_t qlim, void* scratch, uint64_t bytes,
                        cudaStream_t st, const char* who)
{
    const uint64_t length = n - 1;
    const KdPlan P = kd_plan(length);
    if (P.m[P.levels] > KD_TILE)
        return err((int)cudaErrorInvalidValue, "kate division: length too large");
    ScratchArena ar(scratch, bytes);
    Fr* tabs = ar.take_n<Fr>((uint64_t)KD_TAB * (P.levels + 1));
    Fr* lv[KD_MAX_LEVELS + 2] = {nullptr};
    for (int l = 1; l <= P.levels; l++) lv[l] = ar.take_n<Fr>(P.m[l]);
    Fr* top = ar.take_n<Fr>(1);
    Fr* upow = ar.take_n<Fr>(KD_TILE);
    Fr* wpow = ar.take_n<Fr>(KD_TILE);
    if (!ar.good()) {
        ScratchPlan sp;
        kd_plan_scratch(sp, n);
        return scratch_too_small(who, bytes, sp.used);
    }
    lv[P.levels + 1] = top;
    // power tables: level 0 from u, level l from table l-1's v^2048
    k_kd_table<<<1, 32, 0, st>>>(u, tabs);
    H2B_LAUNCHED("k_kd_table");
    for (int l = 1; l <= P.levels; l++) {
        k_kd_table<<<1, 32, 0, st>>>(tabs + (uint64_t)KD_TAB * (l - 1) + 16, tabs + (uint64_t)KD_TAB * l);
        H2B_LAUNCHED("k_kd_table");
    }
    auto level = [&](int l) {
        KdLevel L;
        L.arr = l == 0 ? q : lv[l];
        L.m = P.m[l];
        L.rev = l == 0;
        L.n = n;
        L.qlim = qlim;
        return L;
    };
    k_kd_pow<<<1, KD_T, 0, st>>>(u, upow, wpow);
    H2B_LAUNCHED("k_kd_pow");
    const unsigned tiles0 = (unsigned)((P.m[0] + KD_TILE - 1) / KD_TILE);
    k_kd0_up<<<tiles0, KD_T, 0, st>>>(level(0), a, upow, wpow, lv[1]);
    H2B_LAUNCHED("k_kd0_up");
    for (int l = 1; l <= P.levels; l++) {
        const uint64_t tiles = (P.m[l] + KD_TILE - 1) / KD_TILE;
        k_kd_up<<<(unsigned)tiles, KD_T, 0, st>>>(level(l), a, tabs + (uint64_t)KD_TAB * l, lv[l + 1]);
        H2B_LAUNCHED("k_kd_up");
    }
    for (int l = P.levels - 1; l >= 1; l--) {
        const uint64_t tiles = (P.m[l] + KD_TILE - 1) / KD_TILE;
        if (tiles > 1) {
            k_kd_down<<<(unsigned)(tiles - 1), KD_T, 0, st>>>(level(l), tabs + (uint64_t)KD_TAB * l, lv[l + 1]);
            H2B_LAUNCHED("k_kd_down");
        }
    }
    k_kd0_down<<<tiles0, KD_T, 0, st>>>(level(0), a, upow, lv[1]);
    H2B_LAUNCHED("k_kd0_down");
    return ok();
}

// ---- evaluation helpers ----------------------------------------------------

static uint64_t ev_blocks(uint64_t n) { return std::max<uint64_t>(1, (n + EV_TILE - 1) / EV_TILE); }

static void ev_plan(ScratchPlan& sp, uint64_t n)
{
    sp.add_n<Fr>(1);             // point
    sp.add_n<Fr>(CHAIN);         // squaring chain
    sp.add_n<Fr>(ev_blocks(n));  // CTA partials
    sp.add_n<Fr>(1);             // result
}

// result = sum_{i < n} a_i z^i with z on the device.
static RustError ev_run(const Fr* a, uint64_t n, const Fr* d_z, Fr* chain, Fr* partial, Fr* result, cudaStream_t st)
{
    k_op_chain<<<1, 32, 0, st>>>(d_z, chain);
    H2B_LAUNCHED("k_op_chain");
    const uint64_t nb = ev_blocks(n);
    k_eval_partial<<<(unsigned)nb, EV_T, 0, st>>>(a, n, chain, partial);
    H2B_LAUNCHED("k_eval_partial");
    k_eval_sum<<<1, EV_T, 0, st>>>(partial, nb, result);
    H2B_LAUNCHED("k_eval_sum");
    return ok();
}

// Multi-polynomial chunk work shared by the batch evaluation and the
// multiopen calculation: two staging slots, points, results, challenges,
// evaluation temporaries, and (multiopen) the accumulator.
struct ChunkPlan {
    static void plan(ScratchPlan& sp, uint64_t len, uint64_t batch, bool acc)
    {
        sp.add_n<Fr>(len);           // staging 0
        sp.add_n<Fr>(len);           // staging 1
        sp.add_n<Fr>(batch);         // points
        sp.add_n<Fr>(batch);         // results
        if (acc) {
            sp.add_n<Fr>(batch);     // challenges
            sp.add_n<Fr>(len);       // accumulator
        }
        sp.add_n<Fr>(CHAIN);
        sp.add_n<Fr>(ev_blocks(len));
    }
};

static RustError chunk_run(const FFITraitObject* polys, const FFITraitObject* points, const FFITraitObject* results,
                           const FFITraitObject* challenges, const FFITraitObject* acc_out, uint64_t offset,
                           uint64_t len, uint64_t batch, void* scratch, uint64_t bytes, cudaStream_t st,
                           const char* who)
{
    const bool acc = challenges != nullptr;
    ScratchArena ar(scratch, bytes);
    Fr* stage[2] = {ar.take_n<Fr>(len), ar.take_n<Fr>(len)};
    Fr* d_pts = ar.take_n<Fr>(batch);
    Fr* d_res = ar.take_n<Fr>(batch);
    Fr* d_ch = acc ? ar.take_n<Fr>(batch) : nullptr;
    Fr* d_acc = acc ? ar.take_n<Fr>(len) : nullptr;
    Fr* chain = ar.take_n<Fr>(CHAIN);
    Fr* partial = ar.take_n<Fr>(ev_blocks(len));
    if (!ar.good()) {
        ScratchPlan sp;
        ChunkPlan::plan(sp, len, batch, acc);
        return scratch_too_small(who, bytes, sp.used);
    }
    H2B_CUDA(cudaMemcpyAsync(d_pts, points->ptr, batch * 32, cudaMemcpyHostToDevice, st));
    if (acc) {
        H2B_CUDA(cudaMemcpyAsync(d_ch, challenges->ptr, batch * 32, cudaMemcpyHostToDevice, st));
        H2B_CUDA(cudaMemsetAsync(d_acc, 0, len * 32, st));
    }
    for (uint64_t i = 0; i < batch; i++) {
        Fr* slot = stage[i & 1];
        H2B_CUDA(cudaMemcpyAsync(slot, polys[i].ptr + 4 * offset, len * 32, cudaMemcpyHostToDevice, st));
        H2B_TRY(ev_run(slot, len, d_pts + i, chain, partial, d_res + i, st));
        if (acc) {
            k_op_madd<<<grid_for(len, 256), 256, 0, st>>>(d_acc, slot, d_ch + i, len);
            H2B_LAUNCHED("k_op_madd");
        }
    }
    if (acc) H2B_CUDA(cudaMemcpyAsync(acc_out->ptr + 4 * offset, d_acc, len * 32, cudaMemcpyDeviceToHost, st));
    H2B_CUDA(cudaMemcpyAsync(results->ptr, d_res, batch * 32, cudaMemcpyDeviceToHost, st));
    H2B_CUDA(cudaStreamSynchronize(st));
    return ok();
}

// ---- decode_assigned -------------------------------------------------------

struct AssignedLayout {
    uint32_t stride_bytes, num_offset, denom_offset;
};

static __device__ __forceinline__ Fr ld_unaligned_fr(const uint8_t* p)
{
    Fr r;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(p);
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = w[i];
    return r;
}

static __global__ void k_decode_assigned(Fr* __restrict__ nums, Fr* __restrict__ dens, const uint8_t* __restrict__ raw,
                                         uint64_t n, AssignedLayout L)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint8_t* rec = raw + i * L.stride_bytes;
        const uint8_t tag = rec[0];
        Fr num = Fr::zero(), den = Fr::one();
        if (tag != 0) num = ld_unaligned_fr(rec + L.num_offset);      // Trivial or Rational
        if (tag >= 2) den = ld_unaligned_fr(rec + L.denom_offset);    // Rational
        st(&nums[i], num);
        st(&dens[i], den);
    }
}

} // namespace h2b

using namespace h2b;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" uint64_t _halo2_eval_polynomial_workspace_size(uint64_t length)
{
    ScratchPlan sp;
    ev_plan(sp, length);
    return sp.used;
}

// Device polynomial, host point; *d_result_out receives the device address of
// the 32-byte result (inside scratch).  Does not synchronise.
extern "C" RustError _halo2_eval_polynomial(const void* d_poly, const FFITraitObject* point, void** d_result_out,
                                            uint64_t length, void* scratch, uint64_t scratch_bytes,
                                            cudaStream_t stream)
{
    ScratchArena ar(scratch, scratch_bytes);
    Fr* d_z = ar.take_n<Fr>(1);
    Fr* chain = ar.take_n<Fr>(CHAIN);
    Fr* partial = ar.take_n<Fr>(ev_blocks(length));
    Fr* res = ar.take_n<Fr>(1);
    if (!ar.good())
        return scratch_too_small("_halo2_eval_polynomial", scratch_bytes, _halo2_eval_polynomial_workspace_size(length));
    H2B_CUDA(cudaMemcpyAsync(d_z, point->ptr, 32, cudaMemcpyHostToDevice, stream));
    H2B_TRY(ev_run((const Fr*)d_poly, length, d_z, chain, partial, res, stream));
    *d_result_out = res;
    return ok();
}

extern "C" uint64_t _halo2_eval_polynomial_batch_workspace_size(uint64_t poly_length, uint64_t batch_size)
{
    ScratchPlan sp;
    ChunkPlan::plan(sp, poly_length, batch_size, false);
    return sp.used;
}

extern "C" uint64_t _halo2_eval_poly_batch_max_len(uint64_t poly_length, uint64_t batch_size, uint64_t free_bytes)
{
    for (uint64_t len = poly_length; len > 0; len >>= 1)
        if (_halo2_eval_polynomial_batch_workspace_size(len, batch_size) < free_bytes) return len;
    return 0;
}

// Host polynomials (chunk [offset, offset + length) of each), host points and
// results; synchronises.
extern "C" RustError _halo2_eval_polynomial_batch(const FFITraitObject* poly_in_many, const FFITraitObject* eval_points,
                                                  const FFITraitObject* eval_result, uint64_t poly_offset,
                                                  uint64_t poly_length, uint64_t batch_size, void* scratch,
                                                  uint64_t scratch_bytes, cudaStream_t stream)
{
    if (batch_size == 0) return ok();
    return chunk_run(poly_in_many, eval_points, eval_result, nullptr, nullptr, poly_offset, poly_length, batch_size,
                     scratch, scratch_bytes, stream, "_halo2_eval_polynomial_batch");
}

extern "C" uint64_t _halo2_multiopen_poly_calculation_workspace_size(uint64_t poly_length, uint64_t batch_size)
{
    ScratchPlan sp;
    ChunkPlan::plan(sp, poly_length, batch_size, true);
    return sp.used;
}

extern "C" uint64_t _halo2_multiopen_poly_max_len(uint64_t poly_length, uint64_t batch_size, uint64_t free_bytes)
{
    for (uint64_t len = poly_length; len > 0; len >>= 1)
        if (_halo2_multiopen_poly_calculation_workspace_size(len, batch_size) < free_bytes) return len;
    return 0;
}

// Per i: evaluate_result[i] = sum_k poly_i[offset + k] z_i^k, and the host
// accumulator chunk poly_acc[offset ..) = sum_i c_i poly_i[offset ..)
// (overwritten, not added to).  Synchronises.
extern "C" RustError _halo2_multiopen_poly_calculation(const FFITraitObject* poly_in_many, const FFITraitObject* poly_acc,
                                                       uint64_t poly_offset, uint64_t poly_length, uint64_t batch_size,
                                                       const FFITraitObject* challenge_point,
                                                       const FFITraitObject* evaluate_point,
                                                       const FFITraitObject* evaluate_result, void* scratch,
                                                       uint64_t scratch_bytes, cudaStream_t stream)
{
    if (batch_size == 0) return ok();
    return chunk_run(poly_in_many, evaluate_point, evaluate_result, challenge_point, poly_acc, poly_offset, poly_length,
                     batch_size, scratch, scratch_bytes, stream, "_halo2_multiopen_poly_calculation");
}

extern "C" uint64_t _halo2_kate_division_workspace_size(uint64_t n)
{
    ScratchPlan sp;
    kd_plan_scratch(sp, n);
    return sp.used;
}

// q (length n - 1) = (a - a(u)) / (X - u); all device pointers; no synchronisation.
extern "C" RustError _halo2_kate_division_device(const void* d_a, void* d_q, const void* d_u, uint64_t n, void* scratch,
                                                 uint64_t scratch_bytes, cudaStream_t stream)
{
    if (n < 2) return ok();
    return kd_run((const Fr*)d_a, (Fr*)d_q, (const Fr*)d_u, n, n - 1, scratch, scratch_bytes, stream,
                  "_halo2_kate_division_device");
}

// As above into a length-out_len buffer: q in [0, min(n - 1, out_len)), zeros after.
extern "C" RustError _halo2_kate_division_device_padded(const void* d_a, void* d_q, const void* d_u, uint64_t n,
                                                        uint64_t out_len, void* scratch, uint64_t scratch_bytes,
                                                        cudaStream_t stream)
{
    if (out_len == 0) return ok();
    const uint64_t qlen = n < 2 ? 0 : std::min<uint64_t>(n - 1, out_len);
    if (qlen < out_len) H2B_CUDA(cudaMemsetAsync((Fr*)d_q + qlen, 0, (out_len - qlen) * 32, stream));
    if (n < 2) return ok();
    return kd_run((const Fr*)d_a, (Fr*)d_q, (const Fr*)d_u, n, qlen, scratch, scratch_bytes, stream,
                  "_halo2_kate_division_device_padded");
}

// Assigned<F> records -> numerators (Zero -> 0) and denominators (Zero,
// Trivial -> 1).  Tag byte at offset 0: 0 Zero, 1 Trivial, 2 Rational.
extern "C" RustError _halo2_decode_assigned(void* d_nums, void* d_denoms, const void* d_raw, uint64_t n,
                                            AssignedLayout layout, cudaStream_t stream)
{
    if (n == 0) return ok();
    if (layout.num_offset % 4 || layout.denom_offset % 4 || layout.stride_bytes % 4)
        return err((int)cudaErrorInvalidValue, "_halo2_decode_assigned: offsets and stride must be multiples of 4");
    k_decode_assigned<<<grid_for(n, 256), 256, 0, stream>>>((Fr*)d_nums, (Fr*)d_denoms, (const uint8_t*)d_raw, n,
                                                            layout);
    H2B_LAUNCHED("k_decode_assigned");
    return ok();
}

// ---------------------------------------------------------------------------
// Many device polynomials per call (no counterpart in the reference, whose
// batch evaluation and multiopen calculation stage HOST polynomial chunks;
// a device-resident prover evaluates and combines its polynomials where they
// are).  Up to 64 polynomials of n coefficients per call; points and
// coefficients are host values carried in the kernel parameters.
// ---------------------------------------------------------------------------

extern "C" uint64_t h2b_eval_many_workspace_size(uint64_t n, uint64_t count)
{
    ScratchPlan sp;
    sp.add_n<Fr>(std::max<uint64_t>(count, 1) * CHAIN);
    sp.add_n<Fr>(std::max<uint64_t>(count, 1) * ev_blocks(n));
    return sp.used;
}

extern "C" RustError h2b_eval_many_device(const void* const* d_polys, const void* points, uint64_t count, uint64_t n,
                                          void* d_out, void* scratch, uint64_t scratch_bytes, cudaStream_t stream)
{
    if (count == 0) return ok();
    if (count > (uint64_t)MANY_MAX) return err(cudaErrorInvalidValue, "h2b_eval_many_device: more than 64 polynomials");
    if (n == 0 || !d_polys || !points || !d_out) return err(cudaErrorInvalidValue, "h2b_eval_many_device: bad arguments");
    const uint64_t need = h2b_eval_many_workspace_size(n, count);
    if (!scratch || scratch_bytes < need) return scratch_too_small("h2b_eval_many_device", scratch_bytes, need);
    static thread_local EvMany E;
    for (uint64_t i = 0; i < count; i++) {
        if (!d_polys[i]) return err(cudaErrorInvalidValue, "h2b_eval_many_device: null polynomial");
        E.p[i] = (const Fr*)d_polys[i];
        memcpy(&E.z[i], (const char*)points + 32 * i, 32);
    }
    ScratchArena ar(scratch, scratch_bytes);
    Fr* chains = ar.take_n<Fr>(count * CHAIN);
    const uint64_t nb = ev_blocks(n);
    Fr* partial = ar.take_n<Fr>(count * nb);
    k_op_chain_many<<<(unsigned)count, 32, 0, stream>>>(E, chains);
    H2B_LAUNCHED("k_op_chain_many");
    k_eval_partial_many<<<dim3((unsigned)nb, (unsigned)count), EV_T, 0, stream>>>(E, n, chains, partial, nb);
    H2B_LAUNCHED("k_eval_partial_many");
    k_eval_sum_many<<<(unsigned)count, EV_T, 0, stream>>>(partial, nb, (Fr*)d_out);
    H2B_LAUNCHED("k_eval_sum_many");
    return ok();
}

extern "C" RustError h2b_poly_linear_combination(void* d_acc, const void* const* d_polys, const void* coeffs,
                                                 uint64_t count, uint64_t n, int accumulate, cudaStream_t stream)
{
    if (n == 0) return ok();
    if (count > (uint64_t)MANY_MAX)
        return err(cudaErrorInvalidValue, "h2b_poly_linear_combination: more than 64 polynomials");
    if (!d_acc || (count && (!d_polys || !coeffs)))
        return err(cudaErrorInvalidValue, "h2b_poly_linear_combination: bad arguments");
    static thread_local LinTerms T;
    for (uint64_t t = 0; t < count; t++) {
        if (!d_polys[t]) return err(cudaErrorInvalidValue, "h2b_poly_linear_combination: null polynomial");
        T.p[t] = (const Fr*)d_polys[t];
        memcpy(&T.c[t], (const char*)coeffs + 32 * t, 32);
    }
    k_lin_comb<<<grid_for(n, 256, 148u * 16u), 256, 0, stream>>>((Fr*)d_acc, T, (uint32_t)count, n, accumulate);
    H2B_LAUNCHED("k_lin_comb");
    return ok();
}
