// Fr number-theoretic transforms behind EvaluationDomain (lagrange_to_coeff,
// coeff_to_extended, coeff_to_extended_part, extended_to_coeff) and the
// reference's `_halo2_fft_*` entry points (halo2_proofs/cuda/src/ntt.cu:21-962,
// declared at halo2_proofs/src/cuda/culib.rs:492-600).
//
// Transform conventions (identical outputs to the reference):
//   FFT (1)           A_j = sum_i a_i w^(ij), natural order in and out.
//   iFFT (2)          FFT with the caller's w (= w^-1), then * divisor.
//   cosetFFT (3)      zero-pad to 2^ext, a_i *= zeta^(i mod 3), FFT at 2^ext.
//   icosetFFT (4)     FFT at 2^ext with w, * divisor, a_i *= zeta^-(i mod 3).
//   CosetFFT_Part (6) a_i *= c^i with c carried in the divisor slot, then FFT.
//
// Structure on the device: the radix-2 network runs as a few passes, each
// pass a shared-memory tile that executes up to 9 consecutive radix-2 stages
// on groups of 2^b elements gathered at a fixed stride, so HBM is touched once
// per pass instead of once per stage.  Decimation in time (bit-reversed in,
// natural out) serves the forward transforms after a fused
// twist+bit-reversal scatter; decimation in frequency (natural in,
// bit-reversed out) serves the inverse ones, followed by a fused
// bit-reversal+scale(+untwist) pass.  Twiddles w^e, e < n/2, are generated
// into caller scratch once per call (once per batch for the *_many entries).
// Few product sites per kernel here: inline them (full product throughput).
#define H2B_INLINE_MUL 1
#include <algorithm>
#include <cstring>
#include "abi.cuh"
#include "field.cuh"
#include "hostfield.h"
#include "ntt.cuh"
#include "prof.cuh"

namespace h2b {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// lut[i] = base^(2^i), i < k.  One thread: k sequential squarings.
__global__ void k_pow2_lut(const Fr* __restrict__ base, Fr* __restrict__ lut, int k)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Fr cur = ld(base);
        for (int i = 0; i < k; i++) {
            st(&lut[i], cur);
            cur = cur * cur;
        }
    }
}

__device__ __forceinline__ Fr pow_from_lut(const Fr* __restrict__ lut, uint64_t e)
{
    Fr r = Fr::one();
    int i = 0;
    while (e) {
        if (e & 1) r = r * ldg(&lut[i]);
        e >>= 1;
        i++;
    }
    return r;
}

// tw[e] = w^e for e < half, using lut[i] = w^(2^i).  CTA b owns the tile
// [b T K, (b + 1) T K); thread t starts at w^(b T K + t) and steps by w^T, so a
// warp stores 32 consecutive twiddles per step (coalesced).
constexpr int TW_T = 256, TW_LOGT = 8, TW_K = 16;
__global__ void __launch_bounds__(TW_T) k_twiddles(const Fr* __restrict__ lut, Fr* __restrict__ tw, uint64_t half)
{
    uint64_t e = blockIdx.x * (uint64_t)(TW_T * TW_K) + threadIdx.x;
    if (e >= half) return;
    Fr p = pow_from_lut(lut, e);
    const Fr step = half > (uint64_t)TW_T ? ldg(&lut[TW_LOGT]) : Fr::one();  // lut covers bit 8 when half > 256
#pragma unroll 1
    for (int j = 0; j < TW_K && e < half; j++, e += TW_T) {
        st(&tw[e], p);
        p = p * step;
    }
}

// tw[e] = lo[e mod 2^TW2_LOG] * hi[e >> TW2_LOG] with lo[j] = w^j and
// hi[j] = w^(2^TW2_LOG j): one independent product per twiddle, both factors
// from small tables that stay in cache.
constexpr int TW2_LOG = 10;
__global__ void k_twiddles_fill(const Fr* __restrict__ lo, const Fr* __restrict__ hi, Fr* __restrict__ tw,
                                uint64_t half)
{
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < half; e += (uint64_t)gridDim.x * blockDim.x)
        st(&tw[e], ldg(&lo[e & ((1u << TW2_LOG) - 1)]) * ldg(&hi[e >> TW2_LOG]));
}

__device__ __forceinline__ uint64_t bitrev(uint64_t x, int k)
{
    return k == 0 ? 0 : (__brevll(x) >> (64 - k));
}

// Pointers of up to NTT_MAX_BATCH transforms of one size run by the same
// launches (blockIdx.y selects the transform): the polynomials of one
// `_halo2_fft_many*` call share the twiddles, the divisor and every launch,
// so small transforms fill the GPU together instead of one after another.
// src[i] may equal dst[i] (in-place transforms).
constexpr int NTT_MAX_BATCH = 32;
struct NttBatch {
    const Fr* src[NTT_MAX_BATCH];
    Fr* dst[NTT_MAX_BATCH];
};

// Forward-path input stage fused with the first DIT stage (whose twiddle is
// w^0 = 1): with a_i = in[i] * f(i) (in[i] = 0 for i >= n_in) and f
//   mode 0: 1,   mode 1: c^i (cpow[i] = c^i),   mode 2: z3[i mod 3],
// output pair (2m, 2m + 1) of the bit-reversed array holds inputs
// i0 = rev(2m) and i1 = i0 + n/2, and becomes (a_i0 + a_i1, a_i0 - a_i1).
// Threads walk the output pairs in order: stores are contiguous, the
// 32-byte input loads are scattered.  `out` must not alias `in`.
constexpr int SC_CHUNK = 8;
struct Zeta3 {
    Fr f[3];
};
__device__ __forceinline__ Fr twist_in(const Fr* __restrict__ in, uint64_t i, uint64_t n_in, int mode,
                                       const Fr* __restrict__ cpow, const Zeta3& z3)
{
    if (i >= n_in) return Fr::zero();
    const Fr v = ldg(&in[i]);
    if (mode == 1) return v * ldg(&cpow[i]);
    if (mode == 2) return v * z3.f[i % 3];
    return v;
}
__global__ void k_twist_bitrev_stage0(NttBatch B, uint64_t n_in, int log_out, int mode,
                                      const Fr* __restrict__ cpow, Zeta3 z3)
{
    const Fr* __restrict__ in = B.src[blockIdx.y];
    Fr* __restrict__ out = B.dst[blockIdx.y];
    const uint64_t half = 1ull << (log_out - 1);
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < half;
         m += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = bitrev(m, log_out - 1);   // rev(2m) over log_out bits
        const Fr a = twist_in(in, i0, n_in, mode, cpow, z3);
        const Fr b = twist_in(in, i0 + half, n_in, mode, cpow, z3);
        st(&out[2 * m], a + b);
        st(&out[2 * m + 1], a - b);
    }
}

// Coset extension from 2^k inputs to 2^(k+e) outputs (zero padding).  After
// the bit reversal over k+e bits, input i lands at rev_k(i) << e and every
// other slot of that aligned group of 2^e is zero, so the first e DIT stages
// only copy the value across the group.  This writes the twisted input
// a_i * zeta^(i mod 3) to all 2^e slots; the DIT passes then start at stage e.
// Threads walk the OUTPUT groups in order (group r holds input bitrev(r)), so
// a warp's stores form one contiguous run and only the 32-byte input loads
// are scattered.
__global__ void k_coset_spread(NttBatch B, int log_in, int e, Zeta3 z3)
{
    const Fr* __restrict__ in = B.src[blockIdx.y];
    Fr* __restrict__ out = B.dst[blockIdx.y];
    uint64_t n_in = 1ull << log_in;
    const uint64_t g = 1ull << e;
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n_in;
         r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = bitrev(r, log_in);
        Fr v = ldg(&in[i]) * z3.f[i % 3];
        Fr* dst = out + (r << e);
        for (uint64_t j = 0; j < g; j++) st(&dst[j], v);
    }
}

// In-place a_i *= c^i (mode 1, cpow[i] = c^i) or zeta^(i mod 3) factors (mode 2).
__global__ void k_twist_inplace(NttBatch B, uint64_t n, int mode, const Fr* __restrict__ cpow, Zeta3 z3)
{
    Fr* __restrict__ a = B.dst[blockIdx.y];
    uint64_t nthreads = n / SC_CHUNK + (n % SC_CHUNK ? 1 : 0);
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nthreads;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i0 = t * SC_CHUNK;
        for (int j = 0; j < SC_CHUNK && i0 + j < n; j++) {
            uint64_t i = i0 + j;
            Fr v = ld(&a[i]);
            v = v * (mode == 1 ? ldg(&cpow[i]) : z3.f[i % 3]);
            st(&a[i], v);
        }
    }
}

// In-place bit reversal; when `scale` each element landing at index i is
// multiplied by z3.f[i mod 3] (used for divisor and divisor*zeta^-(i mod 3)).
__global__ void k_bitrev_inplace(NttBatch B, int k, bool scale, Zeta3 z3)
{
    Fr* __restrict__ a = B.dst[blockIdx.y];
    uint64_t n = 1ull << k;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t j = bitrev(i, k);
        if (i < j) {
            Fr x = ld(&a[i]), y = ld(&a[j]);
            if (scale) {
                y = y * z3.f[i % 3];
                x = x * z3.f[j % 3];
            }
            st(&a[i], y);
            st(&a[j], x);
        } else if (i == j && scale) {
            Fr x = ld(&a[i]);
            st(&a[i], x * z3.f[i % 3]);
        }
    }
}

// Tiled bit reversal for 2^k arrays with k >= 10.  Index i splits as
// (h: top 5 bits, m: middle k - 10 bits, l: low 5 bits) and
// bitrev_k(i) = (rev5(l), rev_{k-10}(m), rev5(h)): the 1024 elements with
// middle index m (32 runs of 32 consecutive elements, one run per h) are
// exactly the images of the elements with middle index rev(m).  One CTA
// carries tile m and its partner tile rev(m) through shared memory, so every
// global load and store is one warp's contiguous 1 KB run instead of a
// 32-byte access n/2 away from its neighbour's.
constexpr int BR_LOG = 5, BR_SIDE = 1 << BR_LOG, BR_THREADS = 256;
constexpr int BR_MIN_LOG = 2 * BR_LOG;
constexpr int BR_TILE = BR_SIDE * BR_SIDE;
constexpr size_t BR_SMEM = 2 * BR_TILE * sizeof(Fr);  // two tiles, 64 KB

__device__ __forceinline__ uint32_t rev5(uint32_t x) { return __brev(x) >> (32 - BR_LOG); }

// slot of element (row r, column c) of a tile: the column is XOR-swizzled by
// the row, so a warp reading one column across 32 rows touches four bank
// groups per 16-byte access instead of one (two-way conflicts at most; rows
// are read and written conflict-light as well)
__device__ __forceinline__ uint32_t br_slot(uint32_t r, uint32_t c) { return r * BR_SIDE + (c ^ ((r >> 2) & 3)); }

__device__ __forceinline__ uint64_t br_index(uint32_t h, uint64_t m, uint32_t l, int k)
{
    return ((uint64_t)h << (k - BR_LOG)) | (m << BR_LOG) | l;
}

// In place: a[bitrev(j)] and a[j] swap; with `scale` the element landing at
// index j is multiplied by z3.f[j mod 3] (as k_bitrev_inplace).
__global__ void __launch_bounds__(BR_THREADS) k_bitrev_tiled(NttBatch B, int k, bool scale, Zeta3 z3)
{
    extern __shared__ uint4 br_sh[];
    Fr* tile = reinterpret_cast<Fr*>(br_sh);
    Fr* __restrict__ a = B.dst[blockIdx.y];
    const int km = k - BR_MIN_LOG;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = BR_THREADS / 32;
    for (uint64_t m = blockIdx.x; m < (1ull << km); m += gridDim.x) {
        const uint64_t mr = bitrev(m, km);
        if (m > mr) continue;  // the CTA of the partner tile moves both
        const int nt = (m == mr) ? 1 : 2;
        for (int t = 0; t < nt; t++) {
            const uint64_t mm = t ? mr : m;
            for (uint32_t h = warp; h < BR_SIDE; h += nw)
                st(&tile[t * BR_TILE + br_slot(h, lane)], ld(&a[br_index(h, mm, lane, k)]));
        }
        __syncthreads();
        // tile t holds middle index mm; its element (h, l) lands at
        // (rev5(l), rev(mm), rev5(h)), so output run h of tile rev(mm) reads
        // column rev5(h) of tile t at rows rev5(lane)
        for (int t = 0; t < nt; t++) {
            const uint64_t md = t ? m : mr;
            for (uint32_t h = warp; h < BR_SIDE; h += nw) {
                Fr v = ld(&tile[t * BR_TILE + br_slot(rev5(lane), rev5(h))]);
                const uint64_t j = br_index(h, md, lane, k);
                if (scale) v = v * z3.f[j % 3];
                st(&a[j], v);
            }
        }
        __syncthreads();
    }
}

// k_twist_bitrev_stage0 on tiles (out of place, output size 2^L, L >= 10):
// output tile m takes its inputs from input tile rev(m), twisted as they are
// loaded (twist_in), and writes the first DIT stage's pairs (l, l ^ 1) of
// each output run.
__global__ void __launch_bounds__(BR_THREADS) k_twist_bitrev_stage0_tiled(NttBatch B, uint64_t n_in, int L, int mode,
                                                                          const Fr* __restrict__ cpow, Zeta3 z3)
{
    extern __shared__ uint4 br_sh[];
    Fr* tile = reinterpret_cast<Fr*>(br_sh);
    const Fr* __restrict__ in = B.src[blockIdx.y];
    Fr* __restrict__ out = B.dst[blockIdx.y];
    const int km = L - BR_MIN_LOG;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = BR_THREADS / 32;
    for (uint64_t m = blockIdx.x; m < (1ull << km); m += gridDim.x) {
        const uint64_t mi = bitrev(m, km);
        for (uint32_t h = warp; h < BR_SIDE; h += nw)
            st(&tile[br_slot(h, lane)], twist_in(in, br_index(h, mi, lane, L), n_in, mode, cpow, z3));
        __syncthreads();
        for (uint32_t h = warp; h < BR_SIDE; h += nw) {
            // output (h, m, l) holds input (rev5(l), mi, rev5(h)); DIT stage 0
            // pairs outputs l and l ^ 1: (x_even + x_odd, x_even - x_odd)
            const Fr x = ld(&tile[br_slot(rev5(lane), rev5(h))]);
            const Fr y = ld(&tile[br_slot(rev5(lane ^ 1), rev5(h))]);
            st(&out[br_index(h, m, lane, L)], (lane & 1) ? y - x : x + y);
        }
        __syncthreads();
    }
}

// One shared-memory pass of `nst` radix-2 stages starting at stage s0.
//   DIT: stage s pairs (i, i + 2^s), twiddle w^((i mod 2^s) * n/2^(s+1)),
//        groups: 2^nst elements at stride S = 2^s0 inside blocks of S*2^nst.
//   DIF: stage s pairs (i, i + n/2^(s+1)), twiddle w^((i mod n/2^(s+1)) * 2^s),
//        groups: stride S = n / 2^(s0+nst).
// A CTA owns G = TILE >> nst consecutive groups (G * 2^nst = TILE elements).
constexpr int NTT_LOG_TILE = 10;  // at most 2^10 elements per pass tile
constexpr int NTT_THREADS = 512;

// One pass: nst consecutive stages on groups of 2^nst elements at stride
// S = 2^lS (the group's elements are g-th residue class mod S inside a block
// of S * 2^nst).  A CTA owns G = 2^lG consecutive groups.  Every size is a
// power of two, so all index arithmetic is shifts and masks on 32 bits
// (n <= 2^31).
// Blocks per SM for the pass: the FP64 product needs more live registers.
#if H2B_MUL_F64
constexpr int NTT_MIN_BLOCKS = 2;
#else
constexpr int NTT_MIN_BLOCKS = 3;
#endif

template <bool DIT>
__global__ void __launch_bounds__(NTT_THREADS, NTT_MIN_BLOCKS) k_ntt_pass(NttBatch B, const Fr* __restrict__ tw, int logn, int s0,
                                                          int nst, int lS, int lG)
{
    const Fr* src = B.src[blockIdx.y];  // the first pass of an out-of-place transform reads here
    Fr* a = B.dst[blockIdx.y];
    extern __shared__ uint4 smem_raw[];
    Fr* sm = reinterpret_cast<Fr*>(smem_raw);
    const uint32_t Smask = (1u << lS) - 1;
    const uint32_t g0 = blockIdx.x << lG;
    const uint32_t elems = 1u << (lG + nst);
    const bool wide = lS >= lG;   // the G groups of a CTA are consecutive residues

    // element idx of the tile <-> (group gl, position j) and its address
    auto locate = [&](uint32_t idx, uint32_t& slot) -> uint32_t {
        if (wide) {
            const uint32_t gl = idx & ((1u << lG) - 1), j = idx >> lG;
            const uint32_t g = g0 + gl;
            slot = (gl << nst) + j;
            return ((g >> lS) << (lS + nst)) + (j << lS) + (g & Smask);
        }
        const uint32_t bl = idx >> (lS + nst), rem = idx & ((1u << (lS + nst)) - 1);
        const uint32_t j = rem >> lS, gl = (bl << lS) + (rem & Smask);
        slot = (gl << nst) + j;
        return ((g0 >> lS) << (lS + nst)) + idx;
    };

    for (uint32_t idx = threadIdx.x; idx < elems; idx += blockDim.x) {
        uint32_t slot;
        const uint32_t addr = locate(idx, slot);
        sm[slot] = ld(&src[addr]);
    }
    __syncthreads();

    // One butterfly per thread and stage (nbf <= blockDim.x: a tile holds at
    // most 2^10 elements).  Everything that does not change with the stage is
    // computed once; addresses are 32-bit byte offsets (shift and add), so the
    // integer multiply pipe is left to the products.
    const uint32_t nbf = 1u << (lG + nst - 1);
    const uint32_t u = threadIdx.x;
    const uint32_t m = u & ((1u << (nst - 1)) - 1);
    const uint32_t gl = u >> (nst - 1);
    const uint32_t r = (g0 + gl) & Smask;
    char* const base = reinterpret_cast<char*>(sm) + ((gl << nst) << 5);
    const char* const twb = reinterpret_cast<const char*>(tw);
    for (int t = 0; t < nst; t++) {
        const int s = s0 + t;
        const int h = DIT ? t : nst - t - 1;
        const uint32_t lo = (1u << h) - 1;
        const uint32_t lowm = m & lo;
        const uint32_t q = m + (m & ~lo);                 // ((m >> h) << (h + 1)) | lowm
        const int sh = DIT ? logn - s - 1 : s;            // twiddle w^(((lowm << lS) + r) << sh)
        const uint32_t toff = (((lowm << lS) + r) << sh) << 5;
        if (u < nbf) {
            Fr* px = reinterpret_cast<Fr*>(base + (q << 5));
            Fr* py = reinterpret_cast<Fr*>(base + ((q + (1u << h)) << 5));
            const Fr x = *px, y = *py;
            const Fr w = ldg(reinterpret_cast<const Fr*>(twb + toff));
            if (DIT) {
                const Fr yw = y * w;
                *px = x + yw;
                *py = x - yw;
            } else {
                *px = x + y;
                *py = (x - y) * w;
            }
        }
        __syncthreads();
    }

    for (uint32_t idx = threadIdx.x; idx < elems; idx += blockDim.x) {
        uint32_t slot;
        const uint32_t addr = locate(idx, slot);
        st(&a[addr], sm[slot]);
    }
}

// The same pass with radix-4 steps: a thread takes four elements of a group
// at positions q, q + 2^h, q + 2^(h+1), q + 2^(h+1) + 2^h and runs two
// consecutive radix-2 stages on them in registers (four products in two
// independent pairs, three twiddle loads), so shared memory is read and
// written and the CTA synchronises once per two stages.  An odd stage count
// runs one radix-2 stage first (DIT) or last (DIF).  Same tile layout,
// twiddle indexing and outputs as k_ntt_pass.
constexpr int NTT4_THREADS = 256;
constexpr int NTT4_LOG_TILE = 11;  // radix-4 passes: up to 2^11 elements (64 KB) per tile

// The radix-4 pass keeps its tile as two planes of 16-byte halves (limbs 0-3
// of every element, then limbs 4-7), element s at the swizzled index
// s ^ (((s >> 2) ^ (s >> 3) ^ (s >> nst)) & 7).  The swizzle changes bits 0-2
// from higher bits only, so it permutes every power-of-two tile.  With it the
// eight lanes of each quarter-warp of a 16-byte access fall in eight
// different bank groups for the slot patterns the pass makes: consecutive
// slots, the stride-2/4/8 quadruples of the low-span stages and the
// stride-2^nst slots of the wide load and store loops.  With whole 32-byte
// elements at stride 32 bytes every access took 2 to 8 wavefronts instead of 1.
struct NttTile4 {
    uint4* lo;
    uint4* hi;
    int nst;
    __device__ __forceinline__ uint32_t phys(uint32_t s) const
    {
        return s ^ (((s >> 2) ^ (s >> 3) ^ (s >> nst)) & 7u);
    }
    __device__ __forceinline__ Fr get(uint32_t s) const
    {
        const uint32_t p = phys(s);
        const uint4 a = lo[p], b = hi[p];
        Fr r;
        r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
        r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
        return r;
    }
    __device__ __forceinline__ void put(uint32_t s, const Fr& x) const
    {
        const uint32_t p = phys(s);
        lo[p] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
        hi[p] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
    }
};

// Inside a radix-4 pass values stay in [0, 2p): products without their
// closing subtraction, sums and differences corrected by 2p, one
// canonicalisation per element at the store (field.cuh, residues in [0, 2p)).
__device__ __forceinline__ Fr lz_mul(const Fr& a, const Fr& b)
{
#if H2B_MUL_F64
    return mont_mul_f64_lazy<FrCfg>(a, b);
#else
    return a * b;
#endif
}
__device__ __forceinline__ Fr lz_add(const Fr& a, const Fr& b) { return add2p<FrCfg>(a, b); }
__device__ __forceinline__ Fr lz_sub(const Fr& a, const Fr& b) { return sub2p<FrCfg>(a, b); }

template <bool DIT>
__global__ void __launch_bounds__(NTT4_THREADS, 2) k_ntt_pass4(NttBatch B, const Fr* __restrict__ tw, int logn,
                                                               int s0, int nst, int lS, int lG)
{
    const Fr* src = B.src[blockIdx.y];
    Fr* a = B.dst[blockIdx.y];
    extern __shared__ uint4 smem_raw[];
    const uint32_t Smask = (1u << lS) - 1;
    const uint32_t g0 = blockIdx.x << lG;
    const uint32_t elems = 1u << (lG + nst);
    const NttTile4 T{smem_raw, smem_raw + elems, nst};
    const bool wide = lS >= lG;
    auto locate = [&](uint32_t idx, uint32_t& slot) -> uint32_t {
        if (wide) {
            const uint32_t gl = idx & ((1u << lG) - 1), j = idx >> lG;
            const uint32_t g = g0 + gl;
            slot = (gl << nst) + j;
            return ((g >> lS) << (lS + nst)) + (j << lS) + (g & Smask);
        }
        const uint32_t bl = idx >> (lS + nst), rem = idx & ((1u << (lS + nst)) - 1);
        const uint32_t j = rem >> lS, gl = (bl << lS) + (rem & Smask);
        slot = (gl << nst) + j;
        return ((g0 >> lS) << (lS + nst)) + idx;
    };
    for (uint32_t idx = threadIdx.x; idx < elems; idx += blockDim.x) {
        uint32_t slot;
        const uint32_t addr = locate(idx, slot);
        T.put(slot, ld(&src[addr]));
    }
    __syncthreads();
    const char* const twb = reinterpret_cast<const char*>(tw);
    auto twid = [&](uint32_t lowm, uint32_t r, int sh) -> Fr {
        return ldg(reinterpret_cast<const Fr*>(twb + (((((lowm << lS) + r) << sh)) << 5)));
    };
    // one radix-2 stage t
    auto stage2 = [&](int t) {
        const int s = s0 + t;
        const int h = DIT ? t : nst - t - 1;
        const uint32_t lo = (1u << h) - 1;
        const int sh = DIT ? logn - s - 1 : s;
        const uint32_t nbf = elems >> 1;
        for (uint32_t b = threadIdx.x; b < nbf; b += blockDim.x) {
            const uint32_t m = b & ((1u << (nst - 1)) - 1), gl = b >> (nst - 1);
            const uint32_t r = (g0 + gl) & Smask;
            const uint32_t lowm = m & lo, q = m + (m & ~lo);
            const uint32_t ix = (gl << nst) + q, iy = ix + (1u << h);
            const Fr x = T.get(ix), y = T.get(iy), w = twid(lowm, r, sh);
            if (DIT) {
                const Fr yw = lz_mul(y, w);
                T.put(ix, lz_add(x, yw));
                T.put(iy, lz_sub(x, yw));
            } else {
                T.put(ix, lz_add(x, y));
                T.put(iy, lz_mul(lz_sub(x, y), w));
            }
        }
        __syncthreads();
    };
    // two stages t, t + 1 as radix-4 steps
    auto stage4 = [&](int t) {
        const int h = DIT ? t : nst - t - 2;           // the smaller of the two spans is 2^h
        const uint32_t lo = (1u << h) - 1;
        const uint32_t nq = elems >> 2;
        for (uint32_t qi = threadIdx.x; qi < nq; qi += blockDim.x) {
            const uint32_t m4 = qi & ((1u << (nst - 2)) - 1), gl = qi >> (nst - 2);
            const uint32_t r = (g0 + gl) & Smask;
            const uint32_t lowm = m4 & lo, q = lowm + ((m4 >> h) << (h + 2));
            const uint32_t i0 = (gl << nst) + q, i1 = i0 + (1u << h), i2 = i0 + (2u << h), i3 = i0 + (3u << h);
            const Fr a0 = T.get(i0), a1 = T.get(i1), a2 = T.get(i2), a3 = T.get(i3);
            if (DIT) {
                // stage t (span 2^h): (i0, i1), (i2, i3) share w_h; stage t + 1 (span 2^(h+1)):
                // (i0, i2) takes lowm, (i1, i3) takes lowm + 2^h
                const int sh0 = logn - (s0 + t) - 1, sh1 = sh0 - 1;
                const Fr wh = twid(lowm, r, sh0), wa = twid(lowm, r, sh1), wb = twid(lowm + (1u << h), r, sh1);
                const Fr t1 = lz_mul(a1, wh), t3 = lz_mul(a3, wh);
                const Fr b0 = lz_add(a0, t1), b1 = lz_sub(a0, t1), b2 = lz_add(a2, t3), b3 = lz_sub(a2, t3);
                const Fr u2 = lz_mul(b2, wa), u3 = lz_mul(b3, wb);
                T.put(i0, lz_add(b0, u2));
                T.put(i2, lz_sub(b0, u2));
                T.put(i1, lz_add(b1, u3));
                T.put(i3, lz_sub(b1, u3));
            } else {
                // stage t (span 2^(h+1)): (i0, i2) takes lowm, (i1, i3) lowm + 2^h;
                // stage t + 1 (span 2^h): (i0, i1), (i2, i3) share w_h
                const int sh0 = s0 + t, sh1 = sh0 + 1;
                const Fr wa = twid(lowm, r, sh0), wb = twid(lowm + (1u << h), r, sh0), wh = twid(lowm, r, sh1);
                const Fr b0 = lz_add(a0, a2), b1 = lz_add(a1, a3);
                const Fr b2 = lz_mul(lz_sub(a0, a2), wa), b3 = lz_mul(lz_sub(a1, a3), wb);
                T.put(i0, lz_add(b0, b1));
                T.put(i1, lz_mul(lz_sub(b0, b1), wh));
                T.put(i2, lz_add(b2, b3));
                T.put(i3, lz_mul(lz_sub(b2, b3), wh));
            }
        }
        __syncthreads();
    };
    int t = 0;
    if (DIT && (nst & 1)) stage2(t++);
    for (; t + 1 < nst; t += 2) stage4(t);
    if (t < nst) stage2(t);
    for (uint32_t idx = threadIdx.x; idx < elems; idx += blockDim.x) {
        uint32_t slot;
        const uint32_t addr = locate(idx, slot);
        st(&a[addr], canon2p<FrCfg>(T.get(slot)));
    }
}

static int g_ntt_radix4 = 1;   // 1 (default): the passes run k_ntt_pass4
void ntt_set_radix4(int on) { g_ntt_radix4 = on ? 1 : 0; }
int ntt_get_radix4() { return g_ntt_radix4; }

// ---------------------------------------------------------------------------
// host-side pass planning
// ---------------------------------------------------------------------------

static int g_max_pass_stages = 9;  // tuned per k by ntt_set_pass_stages()

int ntt_pass_stages() { return g_max_pass_stages; }
int tune_value(int param, int log_n);  // tune.cu

void ntt_set_pass_stages(int b)
{
    if (b >= 1 && b <= 11) g_max_pass_stages = b;
}

// The radix-4 passes take tiles of up to 64 KB of shared memory (opt-in
// above the 48 KB default), set once per process.
static bool ntt4_smem_ready()
{
    static int state = 0;
    if (state == 0) {
        const int bytes = (1 << NTT4_LOG_TILE) * (int)sizeof(Fr);
        bool ok_ = cudaFuncSetAttribute(k_ntt_pass4<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) ==
                       cudaSuccess &&
                   cudaFuncSetAttribute(k_ntt_pass4<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) ==
                       cudaSuccess;
        state = ok_ ? 1 : 2;
    }
    return state == 1;
}

// The tiled bit reversals take 64 KB of shared memory (opt-in above the
// 48 KB default), set once per process; without it the scatter kernels run.
static bool br_smem_ready()
{
    static int state = 0;
    if (state == 0) {
        bool ok_ = cudaFuncSetAttribute(k_bitrev_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)BR_SMEM) == cudaSuccess &&
                   cudaFuncSetAttribute(k_twist_bitrev_stage0_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)BR_SMEM) == cudaSuccess;
        state = ok_ ? 1 : 2;
    }
    return state == 1;
}

static dim3 br_grid(int logn, int count)
{
    return dim3((unsigned)std::min<uint64_t>(1ull << (logn - BR_MIN_LOG), 8192), (unsigned)count);
}

// Runs radix-2 stages [first, logn) of `count` transforms in passes of at
// most g_max_pass_stages stages.  The first pass reads B.src and writes B.dst;
// the later ones work in place on B.dst.
static RustError run_passes(NttBatch B, int count, const Fr* tw, int logn, bool dit, cudaStream_t st, int first = 0)
{
    if (logn - first <= 0) return ok();
    int todo = logn - first;
    // radix-4 passes: tiles of up to 2^11 elements, 11 stages per pass unless
    // the tuning table says otherwise; radix-2 passes: at most 10
    const bool r4 = g_ntt_radix4 && ntt4_smem_ready();
    const int tile_log = r4 ? NTT4_LOG_TILE : NTT_LOG_TILE;
    const int tuned = tune_value(2, logn);
    const int max_stages = std::min(tile_log, tuned ? tuned : (r4 ? NTT4_LOG_TILE : g_max_pass_stages));
    int passes = (todo + max_stages - 1) / max_stages;
    int base = todo / passes, extra = todo % passes;
    int s0 = first;
    prof_begin(PROF_NTT_PASSES, st);
    for (int p = 0; p < passes; p++) {
        int nst = base + (p < extra ? 1 : 0);
        const int lS = dit ? s0 : logn - s0 - nst;
        // a one-stage pass runs the radix-2 kernel, whose tile stays at 2^10
        const bool pass4 = r4 && nst >= 2;
        const int lG = std::min((pass4 ? tile_log : NTT_LOG_TILE) - nst, logn - nst);
        const dim3 grid((unsigned)(1ull << (logn - nst - lG)), (unsigned)count);
        size_t smem = (size_t)(1ull << (lG + nst)) * sizeof(Fr);
        int threads = (int)std::min<uint64_t>(NTT_THREADS, std::max<uint64_t>(32, 1ull << (lG + nst - 1)));
        if (pass4) {
            threads = (int)std::min<uint64_t>(NTT4_THREADS, std::max<uint64_t>(32, 1ull << (lG + nst - 2)));
            if (dit)
                k_ntt_pass4<true><<<grid, threads, smem, st>>>(B, tw, logn, s0, nst, lS, lG);
            else
                k_ntt_pass4<false><<<grid, threads, smem, st>>>(B, tw, logn, s0, nst, lS, lG);
        } else if (dit)
            k_ntt_pass<true><<<grid, threads, smem, st>>>(B, tw, logn, s0, nst, lS, lG);
        else
            k_ntt_pass<false><<<grid, threads, smem, st>>>(B, tw, logn, s0, nst, lS, lG);
        H2B_LAUNCHED("k_ntt_pass");
        for (int i = 0; i < count; i++) B.src[i] = B.dst[i];
        s0 += nst;
    }
    prof_end(PROF_NTT_PASSES, st);
    return ok();
}

// Scratch layout for one transform family: twiddles (n/2), lut_w (64), lut_c
// (64), omega staging, (host-input variants) one data slot, then (coset
// parts) the coset powers c^i, i < n.
struct NttScratch {
    Fr* tw = nullptr;
    Fr* tw2 = nullptr;   // lo and hi factors of the two-level twiddle fill
    Fr* lut_w = nullptr;
    Fr* lut_c = nullptr;
    Fr* omega = nullptr;
    Fr* data = nullptr;
    Fr* cpow = nullptr;
};

static void plan_ntt(ScratchPlan& p, int log_size, bool data_slot, int log_data, bool coset_powers)
{
    uint64_t half = log_size == 0 ? 1 : (1ull << (log_size - 1));
    p.add_n<Fr>(half);
    p.add_n<Fr>((1ull << TW2_LOG) + (half >> TW2_LOG) + 1);
    p.add_n<Fr>(64);
    p.add_n<Fr>(64);
    p.add_n<Fr>(1);
    if (data_slot) p.add_n<Fr>(1ull << log_data);
    if (coset_powers) p.add_n<Fr>(1ull << log_size);
}

static NttScratch carve_ntt(ScratchArena& ar, int log_size, bool data_slot, int log_data, bool coset_powers)
{
    NttScratch s;
    uint64_t half = log_size == 0 ? 1 : (1ull << (log_size - 1));
    s.tw = ar.take_n<Fr>(half);
    s.tw2 = ar.take_n<Fr>((1ull << TW2_LOG) + (half >> TW2_LOG) + 1);
    s.lut_w = ar.take_n<Fr>(64);
    s.lut_c = ar.take_n<Fr>(64);
    s.omega = ar.take_n<Fr>(1);
    if (data_slot) s.data = ar.take_n<Fr>(1ull << log_data);
    if (coset_powers) s.cpow = ar.take_n<Fr>(1ull << log_size);
    return s;
}

// Builds tw[] (and lut_w) for transforms of size 2^logn from a device omega.
static RustError make_twiddles(const Fr* d_omega, NttScratch& s, int logn, cudaStream_t st)
{
    if (logn == 0) return ok();
    k_pow2_lut<<<1, 32, 0, st>>>(d_omega, s.lut_w, logn);
    H2B_LAUNCHED("k_pow2_lut");
    uint64_t half = 1ull << (logn - 1);
    const uint64_t tile = (uint64_t)TW_T * TW_K;
    if (half < (4ull << TW2_LOG)) {
        k_twiddles<<<(unsigned)((half + tile - 1) / tile), TW_T, 0, st>>>(s.lut_w, s.tw, half);
        H2B_LAUNCHED("k_twiddles");
        return ok();
    }
    // lo[j] = w^j, j < 2^TW2_LOG; hi[j] = (w^(2^TW2_LOG))^j from the same power table shifted by TW2_LOG
    const uint64_t nlo = 1ull << TW2_LOG, nhi = half >> TW2_LOG;
    Fr* lo = s.tw2;
    Fr* hi = s.tw2 + nlo;
    k_twiddles<<<(unsigned)((nlo + tile - 1) / tile), TW_T, 0, st>>>(s.lut_w, lo, nlo);
    H2B_LAUNCHED("k_twiddles");
    k_twiddles<<<(unsigned)((nhi + tile - 1) / tile), TW_T, 0, st>>>(s.lut_w + TW2_LOG, hi, nhi);
    H2B_LAUNCHED("k_twiddles");
    k_twiddles_fill<<<grid_for(half, 256, 148u * 16u), 256, 0, st>>>(lo, hi, s.tw, half);
    H2B_LAUNCHED("k_twiddles_fill");
    return ok();
}

static Zeta3 zeta_factors(const host::Fr64& scale, bool inverse)
{
    using namespace host;
    Fr64 one = fr_const(FR_ONE), z = fr_const(FR_ZETA), z2 = fr_const(FR_ZETA2);
    Fr64 f[3];
    f[0] = fr_mul(scale, one);
    // forward twist: a_i *= zeta^(i mod 3); inverse: zeta^-(i mod 3) = zeta^(2(i mod 3)).
    f[1] = fr_mul(scale, inverse ? z2 : z);
    f[2] = fr_mul(scale, inverse ? z : z2);
    Zeta3 out;
    for (int i = 0; i < 3; i++) memcpy(out.f[i].v, f[i].v, 32);
    return out;
}

static Zeta3 scale_factors(const host::Fr64& scale)
{
    Zeta3 out;
    for (int i = 0; i < 3; i++) memcpy(out.f[i].v, scale.v, 32);
    return out;
}

// In-place bit reversal (and optional scale) of `count` arrays of 2^logn.
static RustError bitrev_group(NttBatch D, int count, int logn, bool scale, Zeta3 z3, cudaStream_t st)
{
    if (logn >= BR_MIN_LOG && br_smem_ready()) {
        k_bitrev_tiled<<<br_grid(logn, count), BR_THREADS, BR_SMEM, st>>>(D, logn, scale, z3);
        H2B_LAUNCHED("k_bitrev_tiled");
    } else {
        const uint64_t n = 1ull << logn;
        k_bitrev_inplace<<<dim3(grid_for(n, 256), (unsigned)count), 256, 0, st>>>(D, logn, scale, z3);
        H2B_LAUNCHED("k_bitrev_inplace");
    }
    return ok();
}

// Core: `count` (<= NTT_MAX_BATCH) transforms of one type and size, B.src[i]
// -> B.dst[i], all on the device.  `alias`: every B.src[i] == B.dst[i].
//   log_n   : input length (and transform size except for coset types)
//   log_ext : transform size for cosetFFT / icosetFFT
static RustError transform_group(int type, int log_n, int log_ext, NttBatch B, int count, bool alias,
                                 const host::Fr64* h_divisor, NttScratch& s, cudaStream_t st)
{
    using namespace host;
    const bool coset_full = (type == 3 || type == 4);
    const int logt = coset_full ? log_ext : log_n;
    const uint64_t nt = 1ull << logt;
    const uint64_t nin = 1ull << log_n;
    Zeta3 none = scale_factors(fr_const(FR_ONE));
    NttBatch D = B;  // in place on the outputs
    for (int i = 0; i < count; i++) D.src[i] = D.dst[i];
    auto grid = [&](uint64_t work) { return dim3(grid_for(work, 256), (unsigned)count); };

    if (type == 1 || type == 6 || type == 3) {
        int mode = 0;
        Zeta3 z3 = none;
        if (type == 6) {
            // c^i for i < n once for the group (one product per element), so the
            // twist costs each polynomial one product per element
            Fr64 lut[64];
            fr_pow2_lut(*h_divisor, logt, lut);
            H2B_CUDA(cudaMemcpyAsync(s.lut_c, lut, sizeof(Fr) * logt, cudaMemcpyHostToDevice, st));
            const uint64_t tile = (uint64_t)TW_T * TW_K;
            k_twiddles<<<(unsigned)((nt + tile - 1) / tile), TW_T, 0, st>>>(s.lut_c, s.cpow, nt);
            H2B_LAUNCHED("k_twiddles");
            mode = 1;
        } else if (type == 3) {
            z3 = zeta_factors(fr_const(FR_ONE), false);
            mode = 2;
        }
        if (!alias && type == 3 && logt > log_n) {
            int e = logt - log_n;
            k_coset_spread<<<grid(nin), 256, 0, st>>>(B, log_n, e, z3);
            H2B_LAUNCHED("k_coset_spread");
            return run_passes(D, count, s.tw, logt, true, st, e);
        }
        const uint64_t nthreads = nt / SC_CHUNK + (nt % SC_CHUNK ? 1 : 0);
        if (!alias) {
            // the fused input stage also runs DIT stage 0
            if (logt >= BR_MIN_LOG && br_smem_ready()) {
                k_twist_bitrev_stage0_tiled<<<br_grid(logt, count), BR_THREADS, BR_SMEM, st>>>(
                    B, type == 3 ? nin : nt, logt, mode, s.cpow, z3);
                H2B_LAUNCHED("k_twist_bitrev_stage0_tiled");
            } else {
                k_twist_bitrev_stage0<<<grid(nt / 2), 256, 0, st>>>(B, type == 3 ? nin : nt, logt, mode, s.cpow,
                                                                      z3);
                H2B_LAUNCHED("k_twist_bitrev_stage0");
            }
            return run_passes(D, count, s.tw, logt, true, st, 1);
        } else {
            if (type == 3 && nt != nin) {
                // zero the padding in place, then twist + reverse
                for (int i = 0; i < count; i++)
                    H2B_CUDA(cudaMemsetAsync(D.dst[i] + nin, 0, (nt - nin) * sizeof(Fr), st));
            }
            if (mode != 0) {
                k_twist_inplace<<<grid(nthreads), 256, 0, st>>>(D, nt, mode, s.cpow, z3);
                H2B_LAUNCHED("k_twist_inplace");
            }
            H2B_TRY(bitrev_group(D, count, logt, false, none, st));
        }
        return run_passes(D, count, s.tw, logt, true, st);
    }
    if (type == 2 || type == 4) {
        NttBatch P = alias ? D : B;  // the first DIF pass reads the inputs
        if (type == 4) {
            for (int i = 0; i < count; i++) {
                if (!alias)
                    H2B_CUDA(cudaMemcpyAsync(D.dst[i], B.src[i], nin * sizeof(Fr), cudaMemcpyDeviceToDevice, st));
                if (nt != nin) H2B_CUDA(cudaMemsetAsync(D.dst[i] + nin, 0, (nt - nin) * sizeof(Fr), st));
            }
            P = D;
        }
        H2B_TRY(run_passes(P, count, s.tw, logt, false, st));
        Zeta3 z3 = (type == 4) ? zeta_factors(*h_divisor, true) : scale_factors(*h_divisor);
        return bitrev_group(D, count, logt, true, z3, st);
    }
    return err(-1, "unsupported ntt_type");
}

// One transform into `d_out` (device).  `in` may be host (in_host) or device,
// and may alias d_out only when it is device memory.
static RustError transform_one(int type, int log_n, int log_ext, const void* in, bool in_host, Fr* d_out,
                               const host::Fr64* h_divisor, NttScratch& s, cudaStream_t st)
{
    const Fr* din = (const Fr*)in;
    if (in_host) {
        H2B_CUDA(cudaMemcpyAsync(d_out, in, (sizeof(Fr) << log_n), cudaMemcpyHostToDevice, st));
        din = d_out;
    }
    NttBatch B;
    B.src[0] = din;
    B.dst[0] = d_out;
    return transform_group(type, log_n, log_ext, B, 1, din == d_out, h_divisor, s, st);
}

static RustError check_type(uint32_t t)
{
    if (t == 5) return err(-1, "iFFT_cosetFFT not supported");
    if (t < 1 || t > 6) return err(-6, "unsupported ntt_type");
    return ok();
}

} // namespace h2b

using namespace h2b;

// ---------------------------------------------------------------------------
// C ABI (declarations in include/halo2_gpu.h)
// ---------------------------------------------------------------------------

static int active_log(uint32_t t, uint32_t log_n, uint32_t ext) { return (t == 3 || t == 4) ? (int)ext : (int)log_n; }

extern "C" uint64_t _halo2_fft_normal_workspace_size(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n)
{
    ScratchPlan p;
    int la = active_log(ntt_type, log_n, extend_log_n);
    plan_ntt(p, la, true, la, ntt_type == 6);
    return p.used;
}

extern "C" bool _halo2_fft_normal_check_memory(uint32_t, const void*, uint32_t, uint32_t) { return true; }

extern "C" RustError _halo2_fft_normal(uint32_t ntt_type, uint32_t log_n, const void* input, void* output,
                                       const void* omega, const void* divisor, void* scratch, uint64_t scratch_bytes,
                                       cudaStream_t stream)
{
    H2B_TRY(check_type(ntt_type));
    if (log_n == 0) return err(cudaErrorInvalidValue, "_halo2_fft_normal: log_n must be >= 1");
    uint64_t need = _halo2_fft_normal_workspace_size(ntt_type, log_n, log_n);
    if (scratch_bytes < need) return scratch_too_small("_halo2_fft_normal", scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    NttScratch s = carve_ntt(ar, log_n, true, log_n, ntt_type == 6);
    if (!ar.good()) return scratch_too_small("_halo2_fft_normal", scratch_bytes, need);
    H2B_CUDA(cudaMemcpyAsync(s.omega, omega, sizeof(Fr), cudaMemcpyHostToDevice, stream));
    H2B_TRY(make_twiddles(s.omega, s, log_n, stream));
    host::Fr64 div = host::fr_from(divisor);
    H2B_TRY(transform_one(ntt_type, log_n, log_n, input, true, s.data, &div, s, stream));
    H2B_CUDA(cudaMemcpyAsync(output, s.data, sizeof(Fr) << log_n, cudaMemcpyDeviceToHost, stream));
    H2B_CUDA(cudaStreamSynchronize(stream));
    return ok();
}

extern "C" uint64_t _halo2_fft_normal_to_device_workspace_size(uint32_t ntt_type, uint32_t log_n,
                                                               uint32_t extend_log_n)
{
    ScratchPlan p;
    plan_ntt(p, active_log(ntt_type, log_n, extend_log_n), false, 0, ntt_type == 6);
    return p.used;
}

extern "C" RustError _halo2_fft_normal_to_device(uint32_t ntt_type, uint32_t log_n, const void* d_input,
                                                 void* d_output, const void* d_omega, const void* h_divisor,
                                                 void* scratch, uint64_t scratch_bytes, cudaStream_t stream)
{
    if (ntt_type != 1 && ntt_type != 2 && ntt_type != 6)
        return err(cudaErrorInvalidValue, "_halo2_fft_normal_to_device supports only FFT, iFFT, CosetFFT_Part");
    if (log_n == 0) return err(cudaErrorInvalidValue, "_halo2_fft_normal_to_device: log_n must be >= 1");
    uint64_t need = _halo2_fft_normal_to_device_workspace_size(ntt_type, log_n, log_n);
    if (scratch_bytes < need) return scratch_too_small("_halo2_fft_normal_to_device", scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    NttScratch s = carve_ntt(ar, log_n, false, 0, ntt_type == 6);
    H2B_TRY(make_twiddles((const Fr*)d_omega, s, log_n, stream));
    host::Fr64 div = host::fr_from(h_divisor);
    return transform_one(ntt_type, log_n, log_n, d_input, false, (Fr*)d_output, &div, s, stream);
}

extern "C" RustError _halo2_cosetfft(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n, const void* input,
                                     void* output, const void* omega, const void* divisor, void* scratch,
                                     uint64_t scratch_bytes, cudaStream_t stream)
{
    (void)ntt_type;
    (void)divisor;
    if (log_n == 0 || extend_log_n == 0)
        return err(cudaErrorInvalidValue, "_halo2_cosetfft: log_n and extend_log_n must be >= 1");
    if (extend_log_n < log_n) return err(cudaErrorInvalidValue, "_halo2_cosetfft: extend_log_n < log_n");
    // This entry point always runs the forward coset extension (cosetFFT).
    uint64_t need = _halo2_fft_normal_workspace_size(3, log_n, extend_log_n);
    if (scratch_bytes < need) return scratch_too_small("_halo2_cosetfft", scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    NttScratch s = carve_ntt(ar, extend_log_n, true, extend_log_n, false);
    H2B_CUDA(cudaMemcpyAsync(s.omega, omega, sizeof(Fr), cudaMemcpyHostToDevice, stream));
    H2B_TRY(make_twiddles(s.omega, s, extend_log_n, stream));
    host::Fr64 one = host::fr_const(host::FR_ONE);
    H2B_TRY(transform_one(3, log_n, extend_log_n, input, true, s.data, &one, s, stream));
    H2B_CUDA(cudaMemcpyAsync(output, s.data, sizeof(Fr) << extend_log_n, cudaMemcpyDeviceToHost, stream));
    H2B_CUDA(cudaStreamSynchronize(stream));
    return ok();
}

extern "C" uint64_t _halo2_fft_many_workspace_size(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n)
{
    ScratchPlan p;
    int la = active_log(ntt_type, log_n, extend_log_n);
    plan_ntt(p, la, true, la, ntt_type == 6);
    return p.used;
}

extern "C" uint64_t _halo2_fft_many_to_device_workspace_size(uint32_t ntt_type, uint32_t log_n,
                                                             uint32_t extend_log_n)
{
    ScratchPlan p;
    plan_ntt(p, active_log(ntt_type, log_n, extend_log_n), false, 0, ntt_type == 6);
    return p.used;
}

extern "C" bool _halo2_fft_many_check_memory(uint32_t, uint32_t, uint32_t) { return true; }

static RustError fft_many_impl(uint32_t ntt_type, uint32_t num_many, uint32_t log_n, uint32_t extend_log_n,
                               const FFITraitObject* input, const FFITraitObject* output, const void* d_omega,
                               const FFITraitObject* divisor, bool in_on_device, bool out_on_device, void* scratch,
                               uint64_t scratch_bytes, cudaStream_t stream, const char* who)
{
    if (ntt_type == 4) return err(2, "icosetFFT not supported now");
    H2B_TRY(check_type(ntt_type));
    if (log_n == 0 || extend_log_n == 0) return err(cudaErrorInvalidValue, "log_n and extend_log_n must be >= 1");
    int la = active_log(ntt_type, log_n, extend_log_n);
    uint64_t need = out_on_device ? _halo2_fft_many_to_device_workspace_size(ntt_type, log_n, extend_log_n)
                                  : _halo2_fft_many_workspace_size(ntt_type, log_n, extend_log_n);
    if (scratch_bytes < need) return scratch_too_small(who, scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    NttScratch s = carve_ntt(ar, la, !out_on_device, la, ntt_type == 6);
    H2B_TRY(make_twiddles((const Fr*)d_omega, s, la, stream));
    host::Fr64 div = (divisor && divisor->ptr) ? host::fr_from(divisor->ptr) : host::fr_const(host::FR_ONE);
    if (!out_on_device) {
        // one device slot: stage, transform and copy back one polynomial at a time
        for (uint32_t i = 0; i < num_many; i++) {
            H2B_TRY(transform_one(ntt_type, log_n, extend_log_n, input[i].ptr, !in_on_device, s.data, &div, s,
                                  stream));
            H2B_CUDA(cudaMemcpyAsync(output[i].ptr, s.data, sizeof(Fr) << la, cudaMemcpyDeviceToHost, stream));
        }
        H2B_CUDA(cudaStreamSynchronize(stream));
        return ok();
    }
    // An output that overlaps another polynomial's device input makes the
    // result depend on the order of the transforms: run them one at a time.
    bool cross = false;
    if (in_on_device) {
        const uint64_t out_b = sizeof(Fr) << la, in_b = sizeof(Fr) << log_n;
        for (uint32_t i = 0; i < num_many && !cross; i++)
            for (uint32_t j = 0; j < num_many && !cross; j++) {
                const uintptr_t o = (uintptr_t)output[i].ptr, x = (uintptr_t)input[j].ptr;
                cross = i != j && o < x + in_b && x < o + out_b;
            }
    }
    if (cross) {
        for (uint32_t i = 0; i < num_many; i++)
            H2B_TRY(transform_one(ntt_type, log_n, extend_log_n, input[i].ptr, false, (Fr*)output[i].ptr, &div, s,
                                  stream));
        return ok();
    }
    // device outputs: host inputs are staged into their outputs, then the
    // transforms run in groups (in-place ones and out-of-place ones apart)
    NttBatch grp[2];
    int cnt[2] = {0, 0};
    for (uint32_t i = 0; i < num_many; i++) {
        Fr* dst = (Fr*)output[i].ptr;
        const Fr* src = (const Fr*)input[i].ptr;
        if (!in_on_device) {
            H2B_CUDA(cudaMemcpyAsync(dst, src, sizeof(Fr) << log_n, cudaMemcpyHostToDevice, stream));
            src = dst;
        }
        const int g = src == dst ? 1 : 0;
        grp[g].src[cnt[g]] = src;
        grp[g].dst[cnt[g]] = dst;
        if (++cnt[g] == NTT_MAX_BATCH || i + 1 == num_many) {
            for (int h = 0; h < 2; h++) {
                if (cnt[h] == 0 || (h != g && i + 1 != num_many)) continue;
                H2B_TRY(transform_group(ntt_type, log_n, extend_log_n, grp[h], cnt[h], h == 1, &div, s, stream));
                cnt[h] = 0;
            }
        }
    }
    return ok();
}

extern "C" RustError _halo2_fft_many(uint32_t ntt_type, uint32_t num_many, uint32_t log_n, uint32_t extend_log_n,
                                     const FFITraitObject* input, const FFITraitObject* output, const void* d_omega,
                                     const FFITraitObject* divisor, void* scratch, uint64_t scratch_bytes,
                                     cudaStream_t stream)
{
    return fft_many_impl(ntt_type, num_many, log_n, extend_log_n, input, output, d_omega, divisor, false, false,
                         scratch, scratch_bytes, stream, "_halo2_fft_many");
}

extern "C" RustError _halo2_fft_many_to_device(uint32_t ntt_type, uint32_t num_many, uint32_t log_n,
                                               uint32_t extend_log_n, const FFITraitObject* input,
                                               const FFITraitObject* output, const void* d_omega,
                                               const FFITraitObject* divisor, bool input_on_device, void* scratch,
                                               uint64_t scratch_bytes, cudaStream_t stream)
{
    return fft_many_impl(ntt_type, num_many, log_n, extend_log_n, input, output, d_omega, divisor, input_on_device,
                         true, scratch, scratch_bytes, stream, "_halo2_fft_many_to_device");
}

extern "C" int32_t _halo2_get_fft_split_radix(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n,
                                              uint64_t free_bytes)
{
    for (uint32_t s = 0; s < log_n; s++) {
        uint64_t need = _halo2_fft_normal_workspace_size(ntt_type, log_n - s, extend_log_n - s);
        if (need < free_bytes) return (int32_t)s;
    }
    return -1;
}

// Radix-4 pass steps (1) or radix-2 stages (0, default); same results.
extern "C" void h2b_ntt_set_radix4(int on) { ntt_set_radix4(on); }
extern "C" int h2b_ntt_get_radix4(void) { return ntt_get_radix4(); }

extern "C" void h2b_ntt_set_pass_stages(int stages) { ntt_set_pass_stages(stages); }
extern "C" int h2b_ntt_get_pass_stages(void) { return ntt_pass_stages(); }
