// Batch inversion, grand-product scans and the permutation / lookup products.
//
//  * `_halo2_batch_invert` (halo2_proofs/cuda/src/polynomial/operations.cu:16-42,
//    semantics of halo2_proofs/cuda/include/kernel/inverse.h:10-63): in-place
//    x_i <- x_i^-1 with zeros preserved, Fr or Fq.  The entry point has no
//    scratch, so each CTA runs a Montgomery trick over 2048 elements with one
//    inversion (prefixes in shared memory, a product tree over the 256 thread
//    totals).  `h2b_batch_invert` adds a scratch-taking variant whose CTAs
//    publish their totals, which are inverted recursively, so the whole array
//    costs one inversion.
//  * `_halo2_grand_product{,_device_inputs}` (halo2_proofs/cuda/src/commitment/
//    grand_product.cu:45-195): out[i] = prefix * prod_{j<=i} in[j].  In-place
//    multi-level scan: each level scans tiles of 2048 level entries whose last
//    element then carries the tile total; a down-sweep multiplies every entry
//    by the final value at the end of the previous tile.  No scratch.
//  * `_halo2_commit_product{,_device_inputs}` (halo2_proofs/cuda/src/commitment/
//    commit_product.cu:51-186): (A+b)(S+g) / ((A'+b)(S'+g)) per row, fused
//    with the per-CTA inversion.
//  * `_halo2_permutation_product{,_device_inputs}` (halo2_proofs/cuda/src/
//    commitment/permutation_commit.cu:51-256): acc_r * prod_i (b*sigma_i+g+v_i)
//    inverted, times prod_i (deltaomega*delta^i*w^r*b + g + v_i); deltaomega
//    is advanced by delta^batch in place.
// Few product sites per kernel here: inline them (full product throughput).
#define H2B_INLINE_MUL 1
#include <mutex>
#include <vector>
#include "abi.cuh"
#include "field.cuh"
#include "inverse.cuh"
#include "prof.cuh"

namespace h2b {

constexpr int BI_T = 256;
constexpr int BI_E = 8;
constexpr int BI_TILE = BI_T * BI_E;  // elements per CTA
constexpr size_t BI_SMEM = (size_t)(BI_E - 1) * BI_T * 32 + (size_t)2 * BI_T * 32;

// Block Montgomery trick.  Thread t owns tile elements j*BI_T + t (j < BI_E).
//   fwd(i)   -> x_i (may stash x_i for bwd); zero is treated as one
//   bwdx(i)  -> x_i again
//   emit(i, inv_or_zero)
// The CTA's total inverse comes from *root_inv when non-null, else it is
// computed here by thread 0.
template <class C, class Fwd, class Bwdx, class Emit>
__device__ __forceinline__ void block_mont_trick(uint64_t base, uint64_t n, const Fp<C>* root_inv, Fwd fwd, Bwdx bwdx,
                                                 Emit emit)
{
    using F = Fp<C>;
    extern __shared__ uint4 bi_smem[];
    F* pre = reinterpret_cast<F*>(bi_smem);           // (E-1) x T prefixes
    F* tree = pre + (BI_E - 1) * BI_T;                 // 2T heap: tree[T + t] = thread total
    const int t = threadIdx.x;

    F acc = F::one();
#pragma unroll 1
    for (int j = 0; j < BI_E; j++) {
        uint64_t i = base + (uint64_t)j * BI_T + t;
        F x = F::one();
        if (i < n) {
            x = fwd(i);
            if (x.is_zero()) x = F::one();
        }
        acc = (j == 0) ? x : acc * x;
        if (j < BI_E - 1) pre[j * BI_T + t] = acc;
    }
    tree[BI_T + t] = acc;
    __syncthreads();
    for (int w = BI_T / 2; w >= 1; w >>= 1) {
        if (t < w) tree[w + t] = tree[2 * (w + t)] * tree[2 * (w + t) + 1];
        __syncthreads();
    }
    if (t == 0) tree[1] = root_inv ? *root_inv : finv_fast<C>(tree[1]);
    __syncthreads();
    for (int w = 1; w < BI_T; w <<= 1) {
        if (t < w) {
            int k = w + t;
            F inv = tree[k];
            F l = tree[2 * k], r = tree[2 * k + 1];
            tree[2 * k] = inv * r;
            tree[2 * k + 1] = inv * l;
        }
        __syncthreads();
    }
    // Backward: x_j^-1 = inv(prefix_j) * prefix_{j-1}; results replace the
    // consumed prefix slots, then are emitted in ascending j.
    F inv = tree[BI_T + t];
    F inv0 = F::zero();
#pragma unroll 1
    for (int j = BI_E - 1; j >= 0; j--) {
        uint64_t i = base + (uint64_t)j * BI_T + t;
        if (i >= n) continue;
        F x = bwdx(i);
        F out;
        if (x.is_zero()) {
            out = x;
        } else {
            out = (j > 0) ? inv * pre[(j - 1) * BI_T + t] : inv;
            inv = inv * x;
        }
        if (j > 0) pre[(j - 1) * BI_T + t] = out;
        else inv0 = out;
    }
#pragma unroll 1
    for (int j = 0; j < BI_E; j++) {
        uint64_t i = base + (uint64_t)j * BI_T + t;
        if (i >= n) break;
        emit(i, j == 0 ? inv0 : pre[(j - 1) * BI_T + t], j);
    }
}

template <class C>
__global__ void __launch_bounds__(BI_T) k_batch_invert(Fp<C>* __restrict__ d, uint64_t n,
                                                       const Fp<C>* __restrict__ root_inv)
{
    using F = Fp<C>;
    uint64_t base = (uint64_t)blockIdx.x * BI_TILE;
    block_mont_trick<C>(
        base, n, root_inv ? root_inv + blockIdx.x : nullptr, [&](uint64_t i) { return ld(&d[i]); },
        [&](uint64_t i) { return ld(&d[i]); }, [&](uint64_t i, const F& v, int) { st(&d[i], v); });
}

// Per-CTA product of the (zero-as-one) tile, written to totals[blockIdx.x].
template <class C>
__global__ void __launch_bounds__(BI_T) k_tile_product(const Fp<C>* __restrict__ d, uint64_t n,
                                                       Fp<C>* __restrict__ totals)
{
    using F = Fp<C>;
    __shared__ F red[BI_T];
    uint64_t base = (uint64_t)blockIdx.x * BI_TILE;
    F acc = F::one();
    for (int j = 0; j < BI_E; j++) {
        uint64_t i = base + (uint64_t)j * BI_T + threadIdx.x;
        if (i < n) {
            F x = ld(&d[i]);
            if (!x.is_zero()) acc = acc * x;
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = BI_T / 2; w >= 1; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] * red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) st(&totals[blockIdx.x], red[0]);
}

template <class Kern>
static void enable_big_smem(Kern k)
{
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BI_SMEM);
}

template <class C>
static RustError batch_invert_local(Fp<C>* d, uint64_t n, cudaStream_t st)
{
    if (n == 0) return ok();
    enable_big_smem(k_batch_invert<C>);
    uint64_t blocks = (n + BI_TILE - 1) / BI_TILE;
    k_batch_invert<C><<<(unsigned)blocks, BI_T, BI_SMEM, st>>>(d, n, nullptr);
    H2B_LAUNCHED("k_batch_invert");
    return ok();
}

static uint64_t tiles_of(uint64_t n) { return (n + BI_TILE - 1) / BI_TILE; }

static void plan_batch_invert(ScratchPlan& p, uint64_t n)
{
    while (n > BI_TILE) {
        n = tiles_of(n);
        p.add(n * 32);
    }
}

// Multi-level: tile totals -> recurse -> apply with the inverted totals.
template <class C>
static RustError batch_invert_levels(Fp<C>* d, uint64_t n, ScratchArena& ar, cudaStream_t st, bool prof = true)
{
    if (n <= BI_TILE) return batch_invert_local<C>(d, n, st);
    uint64_t nt = tiles_of(n);
    Fp<C>* tot = ar.take_n<Fp<C>>(nt);
    if (!ar.good()) return err(cudaErrorInvalidValue, "batch_invert: scratch too small");
    k_tile_product<C><<<(unsigned)nt, BI_T, 0, st>>>(d, n, tot);
    H2B_LAUNCHED("k_tile_product");
    H2B_TRY(batch_invert_levels<C>(tot, nt, ar, st, prof));
    enable_big_smem(k_batch_invert<C>);
    if (prof) prof_begin(PROF_BATCH_INVERT, st);
    k_batch_invert<C><<<(unsigned)nt, BI_T, BI_SMEM, st>>>(d, n, tot);
    if (prof) prof_end(PROF_BATCH_INVERT, st);
    H2B_LAUNCHED("k_batch_invert");
    return ok();
}

// Group form of the Montgomery trick, for the scratch entry point.  Group t
// of a level owns BI_E elements of the 1024-element tile t / 128, at stride
// 128 (bi_index), so every step of a warp touches 32 consecutive elements and
// a CTA stays inside one tile.  Up: the group product
// (zero counts as one) goes to totals[t]; the totals are inverted by the same
// scheme one level down; down: the group walks its elements backwards with
// the inverted total, two products per element, after recomputing its
// prefix products in registers.  No shared memory and no block-wide trees:
// every level is a fully parallel pass of independent threads.
constexpr int BI_GT = 128;                          // groups per tile
__device__ __forceinline__ uint64_t bi_index(uint64_t t, int j)
{
    return (t / BI_GT) * (BI_GT * BI_E) + (uint64_t)j * BI_GT + (t % BI_GT);
}

// With `pre` (an n-length array laid out like d), the up pass also stores the
// group's running products P_j (nonzero elements up to j, j < BI_E - 1) at
// pre[bi_index(t, j)], and the down pass reads P_{j-1} instead of
// recomputing it: three products per element instead of four, for one more
// write and read of the array (the passes are product-bound, the memory
// traffic overlaps).
template <class C>
__global__ void __launch_bounds__(128) k_bi_up(const Fp<C>* __restrict__ d, uint64_t n, uint64_t nt,
                                               Fp<C>* __restrict__ totals, Fp<C>* __restrict__ pre)
{
    using F = Fp<C>;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nt; t += (uint64_t)gridDim.x * blockDim.x) {
        F acc = F::one();
#pragma unroll 1
        for (int j = 0; j < BI_E; j++) {
            const uint64_t i = bi_index(t, j);
            if (i < n) {
                const F x = ld(&d[i]);
                if (!x.is_zero()) acc = acc * x;
                if (pre && j < BI_E - 1) st(&pre[i], acc);
            }
        }
        st(&totals[t], acc);
    }
}

template <class C>
__global__ void __launch_bounds__(128) k_bi_down(Fp<C>* __restrict__ d, uint64_t n, uint64_t nt,
                                                 const Fp<C>* __restrict__ inv_totals, const Fp<C>* __restrict__ stored)
{
    using F = Fp<C>;
    __shared__ F pre[BI_E][128];                           // per thread: product of the nonzero elements before j
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nt; t += (uint64_t)gridDim.x * blockDim.x) {
        if (!stored) {
            F acc = F::one();
#pragma unroll 1
            for (int j = 0; j < BI_E; j++) {
                const uint64_t i = bi_index(t, j);
                const F x = i < n ? ld(&d[i]) : F::zero();
                pre[j][threadIdx.x] = acc;
                if (!x.is_zero()) acc = acc * x;
            }
        }
        F inv = ld(&inv_totals[t]);                        // (product of all nonzero elements)^-1
#pragma unroll 1
        for (int j = BI_E - 1; j >= 0; j--) {
            const uint64_t i = bi_index(t, j);
            if (i >= n) continue;
            const F x = ld(&d[i]);                         // read again (still the input: i is written last)
            if (x.is_zero()) continue;                     // zero stays zero
            const F before = !stored ? pre[j][threadIdx.x] : (j > 0 ? ld(&stored[bi_index(t, j - 1)]) : F::one());
            const F out = inv * before;
            inv = inv * x;
            st(&d[i], out);
        }
    }
}

static uint64_t groups_of(uint64_t n) { return (n + BI_GT * BI_E - 1) / (BI_GT * BI_E) * BI_GT; }

static void plan_batch_invert_groups(ScratchPlan& p, uint64_t n)
{
    if (n > BI_TILE) p.add(n * 32);  // the top level's stored running products
    while (n > BI_TILE) {
        n = groups_of(n);
        p.add(n * 32);
    }
}

template <class C>
static RustError batch_invert_groups(Fp<C>* d, uint64_t n, ScratchArena& ar, cudaStream_t st, bool top = true)
{
    if (n <= BI_TILE) return batch_invert_local<C>(d, n, st);
    const uint64_t nt = groups_of(n);
    Fp<C>* pre = top ? ar.take_n<Fp<C>>(n) : nullptr;
    Fp<C>* tot = ar.take_n<Fp<C>>(nt);
    if (!ar.good()) return err(cudaErrorInvalidValue, "batch_invert: scratch too small");
    k_bi_up<C><<<grid_for(nt, 128, 148u * 16u), 128, 0, st>>>(d, n, nt, tot, pre);
    H2B_LAUNCHED("k_bi_up");
    H2B_TRY(batch_invert_groups<C>(tot, nt, ar, st, false));
    if (top) prof_begin(PROF_BATCH_INVERT, st);
    k_bi_down<C><<<grid_for(nt, 128, 148u * 16u), 128, 0, st>>>(d, n, nt, tot, pre);
    if (top) prof_end(PROF_BATCH_INVERT, st);
    H2B_LAUNCHED("k_bi_down");
    return ok();
}

// In-place Fq batch inversion for other kernels of this library (the MSM's
// pairing rounds): zeros stay zero; scratch from fq_batch_invert_scratch().
uint64_t fq_batch_invert_scratch(uint64_t n)
{
    ScratchPlan p;
    plan_batch_invert(p, n);
    return p.used;
}

RustError fq_batch_invert(Fq* d, uint64_t n, void* scratch, uint64_t scratch_bytes, cudaStream_t st)
{
    ScratchArena ar(scratch, scratch_bytes);
    return batch_invert_levels<FqCfg>(d, n, ar, st, false);
}

// ---------------------------------------------------------------------------
// grand product (in-place multi-level inclusive multiplicative scan)
// ---------------------------------------------------------------------------

constexpr int GP_T = 256, GP_E = 8, GP_TILE = GP_T * GP_E;

__device__ __forceinline__ uint64_t gp_pos(uint64_t m, uint64_t stride) { return (m + 1) * stride - 1; }

// Scans tiles of GP_TILE level entries (entry m lives at (m+1)*stride-1).
__global__ void __launch_bounds__(GP_T) k_gp_up(Fr* __restrict__ d, uint64_t count, uint64_t stride,
                                                 const Fr* __restrict__ prefix)
{
    __shared__ Fr tot[GP_T];
    const int t = threadIdx.x;
    const uint64_t m0 = (uint64_t)blockIdx.x * GP_TILE + (uint64_t)t * GP_E;
    Fr q[GP_E];
    Fr acc = Fr::one();
#pragma unroll
    for (int j = 0; j < GP_E; j++) {
        uint64_t m = m0 + j;
        Fr x = (m < count) ? ld(&d[gp_pos(m, stride)]) : Fr::one();
        if (m == 0 && prefix != nullptr) x = ld(prefix) * x;  // out[i] = prefix * prod_{j<=i} in[j]
        acc = (j == 0) ? x : acc * x;
        q[j] = acc;
    }
    // exclusive scan of thread totals (Hillis-Steele over 256 entries)
    tot[t] = acc;
    __syncthreads();
    for (int o = 1; o < GP_T; o <<= 1) {
        Fr v = tot[t];
        Fr u = (t >= o) ? tot[t - o] : Fr::one();
        __syncthreads();
        if (t >= o) tot[t] = u * v;
        __syncthreads();
    }
    Fr ex = (t > 0) ? tot[t - 1] : Fr::one();
#pragma unroll
    for (int j = 0; j < GP_E; j++) {
        uint64_t m = m0 + j;
        if (m < count) st(&d[gp_pos(m, stride)], t > 0 ? ex * q[j] : q[j]);
    }
}

// Entries not on a tile boundary take the final value at the end of the
// previous tile.
__global__ void k_gp_down(Fr* __restrict__ d, uint64_t count, uint64_t stride)
{
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < count;
         m += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t g = m / GP_TILE;
        if (g == 0 || ((m + 1) % GP_TILE) == 0) continue;
        Fr pre = ld(&d[gp_pos(g * GP_TILE - 1, stride)]);
        uint64_t p = gp_pos(m, stride);
        st(&d[p], pre * ld(&d[p]));
    }
}

static RustError grand_product_inplace(Fr* d, uint64_t n, const Fr* d_prefix, cudaStream_t st)
{
    if (n == 0) return ok();
    std::vector<uint64_t> strides;
    uint64_t stride = 1, count = n;
    while (true) {
        uint64_t blocks = (count + GP_TILE - 1) / GP_TILE;
        k_gp_up<<<(unsigned)blocks, GP_T, 0, st>>>(d, count, stride, stride == 1 ? d_prefix : nullptr);
        H2B_LAUNCHED("k_gp_up");
        strides.push_back(stride);
        if (count <= GP_TILE) break;
        stride *= GP_TILE;
        count = n / stride;
        if (count == 0) break;
    }
    // down-sweep from the second-highest level to level 0
    for (int l = (int)strides.size() - 2; l >= 0; l--) {
        uint64_t s = strides[l];
        uint64_t cnt = (s == 1) ? n : n / s;
        k_gp_down<<<grid_for(cnt, 256), 256, 0, st>>>(d, cnt, s);
        H2B_LAUNCHED("k_gp_down");
    }
    return ok();
}

// ---------------------------------------------------------------------------
// lookup product: (A+b)(S+g) / ((A'+b)(S'+g))
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(BI_T) k_lookup_product(Fr* __restrict__ out, const Fr* __restrict__ pa,
                                                         const Fr* __restrict__ ps, const Fr* __restrict__ ca,
                                                         const Fr* __restrict__ cs, const Fr* __restrict__ pbeta,
                                                         const Fr* __restrict__ pgamma, uint64_t n)
{
    const Fr beta = ld(pbeta), gamma = ld(pgamma);
    uint64_t base = (uint64_t)blockIdx.x * BI_TILE;
    block_mont_trick<FrCfg>(
        base, n, nullptr,
        [&](uint64_t i) {
            Fr x = (ld(&pa[i]) + beta) * (ld(&ps[i]) + gamma);
            st(&out[i], x);
            return x;
        },
        [&](uint64_t i) { return ld(&out[i]); },
        [&](uint64_t i, const Fr& inv, int) {
            Fr v = inv.is_zero() ? inv : inv * (ld(&ca[i]) + beta) * (ld(&cs[i]) + gamma);
            st(&out[i], v);
        });
}

// ---------------------------------------------------------------------------
// permutation product
// ---------------------------------------------------------------------------

constexpr int PP_MAX_COLS = 48;
struct PermCols {
    const Fr* sigma[PP_MAX_COLS];
    const Fr* value[PP_MAX_COLS];
};

__device__ __forceinline__ Fr pow_u64(const Fr& w, uint64_t e)
{
    Fr r = Fr::one(), b = w;
    while (e) {
        if (e & 1) r = r * b;
        b = b * b;
        e >>= 1;
    }
    return r;
}

// Fused device path: acc_i *= prod_c (b*sigma_c + g + v_c), invert, times
// prod_c (dw0*delta^c*w^i*b + g + v_c).
__global__ void __launch_bounds__(BI_T) k_permutation_product(Fr* __restrict__ acc, PermCols cols, int ncols,
                                                              const Fr* __restrict__ pbeta, const Fr* __restrict__ pgamma,
                                                              const Fr* __restrict__ pdelta, const Fr* __restrict__ pomega,
                                                              const Fr* __restrict__ pdeltaomega, uint64_t n)
{
    const Fr beta = ld(pbeta), gamma = ld(pgamma), delta = ld(pdelta), omega = ld(pomega);
    const Fr dw0b = ld(pdeltaomega) * beta;   // the numerator's first column term is dw0 w^i beta
    const uint64_t base = (uint64_t)blockIdx.x * BI_TILE;
    Fr wstep = pow_u64(omega, BI_T);   // emit steps i by BI_T
    Fr wib = Fr::one();
    block_mont_trick<FrCfg>(
        base, n, nullptr,
        [&](uint64_t i) {
            Fr x = ld(&acc[i]);
            for (int c = 0; c < ncols; c++) x = x * (beta * ld(&cols.sigma[c][i]) + gamma + ld(&cols.value[c][i]));
            st(&acc[i], x);
            return x;
        },
        [&](uint64_t i) { return ld(&acc[i]); },
        [&](uint64_t i, const Fr& inv, int j) {
            // column c's term is dw0 w^i delta^c beta + gamma + v_c: the
            // beta-scaled power is stepped (one product per row) and then
            // by delta per column, so a row takes 2 ncols - 1 products here
            wib = (j == 0) ? dw0b * pow_u64(omega, i) : wib * wstep;
            if (inv.is_zero()) { st(&acc[i], inv); return; }
            if (ncols == 0) { st(&acc[i], inv); return; }   // no columns: the numerator is 1
            Fr cur = wib;
            Fr num = cur + gamma + ld(&cols.value[0][i]);
            for (int c = 1; c < ncols; c++) {
                cur = cur * delta;
                num = num * (cur + gamma + ld(&cols.value[c][i]));
            }
            st(&acc[i], inv * num);
        });
}

// Host-staged path, one column per launch (the reference's 4-poly workspace):
// den_i *= b*sigma_i + g + v_i ; num_i = (first ? 1 : num_i) * (dw*w^i*b + g + v_i).
constexpr int PP_CHUNK = 8;
__global__ void k_pp_accumulate(Fr* __restrict__ den, Fr* __restrict__ num, const Fr* __restrict__ sigma,
                                const Fr* __restrict__ value, const Fr* __restrict__ pbeta,
                                const Fr* __restrict__ pgamma, const Fr* __restrict__ pomega,
                                const Fr* __restrict__ pdw, uint64_t n, bool first)
{
    const Fr beta = ld(pbeta), gamma = ld(pgamma), omega = ld(pomega), dw = ld(pdw);
    uint64_t nthreads = (n + PP_CHUNK - 1) / PP_CHUNK;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nthreads;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i0 = t * PP_CHUNK;
        Fr cur = dw * pow_u64(omega, i0);
        for (int j = 0; j < PP_CHUNK && i0 + j < n; j++) {
            uint64_t i = i0 + j;
            Fr v = ld(&value[i]);
            st(&den[i], ld(&den[i]) * (beta * ld(&sigma[i]) + gamma + v));
            Fr f = cur * beta + gamma + v;
            st(&num[i], first ? f : ld(&num[i]) * f);
            cur = cur * omega;
        }
    }
}

__global__ void __launch_bounds__(BI_T) k_pp_finish(Fr* __restrict__ den, const Fr* __restrict__ num, uint64_t n,
                                                    bool have_num)
{
    uint64_t base = (uint64_t)blockIdx.x * BI_TILE;
    block_mont_trick<FrCfg>(
        base, n, nullptr, [&](uint64_t i) { return ld(&den[i]); }, [&](uint64_t i) { return ld(&den[i]); },
        [&](uint64_t i, const Fr& inv, int) { st(&den[i], have_num ? inv * ld(&num[i]) : inv); });
}

__global__ void k_advance_deltaomega(Fr* __restrict__ dw, const Fr* __restrict__ pdelta, uint64_t batch)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        Fr x = ld(dw), d = ld(pdelta);
        for (uint64_t i = 0; i < batch; i++) x = x * d;
        st(dw, x);
    }
}

} // namespace h2b

using namespace h2b;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" RustError _halo2_batch_invert(void* d_data, uint32_t field_type, uint64_t length, cudaStream_t stream)
{
    if (field_type != 0 && field_type != 1) return err(cudaErrorInvalidValue, "Invalid scalar type");
    if (length == 0) return err(cudaErrorInvalidValue, "_halo2_batch_invert: length must be >= 1");
    if (field_type == 0) return batch_invert_local<FrCfg>((Fr*)d_data, length, stream);
    return batch_invert_local<FqCfg>((Fq*)d_data, length, stream);
}

extern "C" uint64_t h2b_batch_invert_workspace_size(uint64_t length)
{
    ScratchPlan p;
    plan_batch_invert_groups(p, length);
    return p.used;
}

extern "C" RustError h2b_batch_invert(void* d_data, uint32_t field_type, uint64_t length, void* scratch,
                                      uint64_t scratch_bytes, cudaStream_t stream)
{
    if (field_type != 0 && field_type != 1) return err(cudaErrorInvalidValue, "Invalid scalar type");
    if (length == 0) return err(cudaErrorInvalidValue, "h2b_batch_invert: length must be >= 1");
    uint64_t need = h2b_batch_invert_workspace_size(length);
    if (scratch_bytes < need) return scratch_too_small("h2b_batch_invert", scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    if (field_type == 0) return batch_invert_groups<FrCfg>((Fr*)d_data, length, ar, stream);
    return batch_invert_groups<FqCfg>((Fq*)d_data, length, ar, stream);
}

// batch_invert_assigned -------------------------------------------------------
//
// Assigned<F> columns to their values in one entry point: the composition
// halo2_proofs/src/poly.rs:364-420 (batch_invert_assigned_device) builds from
// _halo2_decode_assigned per column, one _halo2_batch_invert over every
// column's denominators and _halo2_poly_elementwise_multiply per column.
// Here: one kernel decodes the denominators of all columns into scratch, the
// scratch batch inversion inverts them all with one field inversion (zeros
// stay zero), and one kernel re-decodes each numerator and multiplies it by
// its inverted denominator into the output column, so numerators never make
// a round trip through memory.  Records: tag byte 0 Zero (value 0), 1 Trivial
// (numerator), 2 Rational (numerator / denominator; a zero denominator gives
// 0, as Assigned::invert does).

namespace h2b {
struct AssignedRec {
    uint32_t stride_bytes, num_offset, denom_offset;
};
constexpr uint32_t BIA_MAX_COLS = 64;
struct BiaCols {
    const uint8_t* raw[BIA_MAX_COLS];
    Fr* out[BIA_MAX_COLS];
};

__device__ __forceinline__ Fr ld_words_fr(const uint8_t* p)
{
    Fr r;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(p);
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = w[i];
    return r;
}

// dens[c n + i] = denominator of record i of column c (blockIdx.y = c)
__global__ void k_bia_denoms(BiaCols cols, uint64_t n, AssignedRec L, Fr* __restrict__ dens)
{
    const uint32_t c = blockIdx.y;
    const uint8_t* raw = cols.raw[c];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint8_t* rec = raw + i * L.stride_bytes;
        Fr den = rec[0] >= 2 ? ld_words_fr(rec + L.denom_offset) : Fr::one();
        st(&dens[c * n + i], den);
    }
}

// out_c[i] = numerator of record i of column c times its inverted denominator
__global__ void k_bia_apply(BiaCols cols, uint64_t n, AssignedRec L, const Fr* __restrict__ inv)
{
    const uint32_t c = blockIdx.y;
    const uint8_t* raw = cols.raw[c];
    Fr* out = cols.out[c];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint8_t* rec = raw + i * L.stride_bytes;
        Fr v = Fr::zero();
        if (rec[0] != 0) v = ld_words_fr(rec + L.num_offset) * ld(&inv[c * n + i]);
        st(&out[i], v);
    }
}
} // namespace h2b

extern "C" uint64_t h2b_batch_invert_assigned_workspace_size(uint64_t n, uint32_t n_cols)
{
    ScratchPlan p;
    uint64_t total = n * (uint64_t)n_cols;
    p.add(std::max<uint64_t>(total, 1) * sizeof(Fr));
    plan_batch_invert_groups(p, std::max<uint64_t>(total, 1));
    return p.used;
}

extern "C" RustError h2b_batch_invert_assigned(void* const* d_outs, const void* const* d_raws, uint32_t n_cols,
                                               uint64_t n, AssignedRec layout, void* scratch, uint64_t scratch_bytes,
                                               cudaStream_t stream)
{
    if (n_cols == 0 || n == 0) return ok();
    if (n_cols > BIA_MAX_COLS)
        return err(cudaErrorInvalidValue, "h2b_batch_invert_assigned: more than 64 columns per call");
    if (layout.stride_bytes % 4 || layout.num_offset % 4 || layout.denom_offset % 4 ||
        layout.num_offset + 32 > layout.stride_bytes || layout.denom_offset + 32 > layout.stride_bytes ||
        layout.num_offset == 0 || layout.denom_offset == 0)
        return err(cudaErrorInvalidValue,
                   "h2b_batch_invert_assigned: layout needs 4-byte aligned stride and offsets, payloads after the "
                   "tag byte and inside the record");
    uint64_t need = h2b_batch_invert_assigned_workspace_size(n, n_cols);
    if (scratch_bytes < need) return scratch_too_small("h2b_batch_invert_assigned", scratch_bytes, need);
    BiaCols cols;
    for (uint32_t c = 0; c < BIA_MAX_COLS; c++) {
        cols.raw[c] = c < n_cols ? (const uint8_t*)d_raws[c] : nullptr;
        cols.out[c] = c < n_cols ? (Fr*)d_outs[c] : nullptr;
    }
    ScratchArena ar(scratch, scratch_bytes);
    Fr* dens = ar.take_n<Fr>(n * n_cols);
    if (!ar.good()) return scratch_too_small("h2b_batch_invert_assigned", scratch_bytes, need);
    dim3 grid(grid_for(n, 256, 148u * 8u), n_cols);
    k_bia_denoms<<<grid, 256, 0, stream>>>(cols, n, layout, dens);
    H2B_LAUNCHED("k_bia_denoms");
    H2B_TRY(batch_invert_groups<FrCfg>(dens, n * n_cols, ar, stream));
    k_bia_apply<<<grid, 256, 0, stream>>>(cols, n, layout, dens);
    H2B_LAUNCHED("k_bia_apply");
    return ok();
}

// grand product ---------------------------------------------------------------

extern "C" uint64_t _halo2_grand_product_workspace_size(uint64_t poly_length)
{
    ScratchPlan p;
    p.add(poly_length * 32);
    p.add(32);
    return p.used;
}

extern "C" uint64_t _halo2_grand_product_max_len(uint64_t poly_length, uint64_t free_bytes)
{
    for (uint64_t l = poly_length; l > 0; l >>= 1)
        if (_halo2_grand_product_workspace_size(l) < free_bytes) return l;
    return 0;
}

extern "C" RustError _halo2_grand_product(const FFITraitObject* output, const FFITraitObject* input,
                                          const FFITraitObject* prefix, uint64_t poly_length, uint64_t poly_offset,
                                          void* scratch, uint64_t scratch_bytes, cudaStream_t stream)
{
    uint64_t need = _halo2_grand_product_workspace_size(poly_length);
    if (scratch_bytes < need) return scratch_too_small("_halo2_grand_product", scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    Fr* d = ar.take_n<Fr>(poly_length);
    Fr* dp = ar.take_n<Fr>(1);
    const uint8_t* hin = (const uint8_t*)input->ptr + poly_offset * 32;
    uint8_t* hout = (uint8_t*)output->ptr + poly_offset * 32;
    H2B_CUDA(cudaMemcpyAsync(d, hin, poly_length * 32, cudaMemcpyHostToDevice, stream));
    H2B_CUDA(cudaMemcpyAsync(dp, prefix->ptr, 32, cudaMemcpyHostToDevice, stream));
    H2B_TRY(grand_product_inplace(d, poly_length, dp, stream));
    H2B_CUDA(cudaMemcpyAsync(hout, d, poly_length * 32, cudaMemcpyDeviceToHost, stream));
    H2B_CUDA(cudaStreamSynchronize(stream));
    return ok();
}

extern "C" RustError _halo2_grand_product_device_inputs(const FFITraitObject* d_inout, const FFITraitObject* d_prefix,
                                                        uint64_t poly_length, uint64_t poly_offset, cudaStream_t stream)
{
    Fr* d = (Fr*)((uint8_t*)d_inout->ptr + poly_offset * 32);
    return grand_product_inplace(d, poly_length, (const Fr*)d_prefix->ptr, stream);
}

// lookup (commit) product -------------------------------------------------------

static RustError lookup_product_run(Fr* out, const Fr* pa, const Fr* ps, const Fr* ca, const Fr* cs, const Fr* beta,
                                    const Fr* gamma, uint64_t n, cudaStream_t st)
{
    if (n == 0) return ok();
    enable_big_smem(k_lookup_product);
    k_lookup_product<<<(unsigned)tiles_of(n), BI_T, BI_SMEM, st>>>(out, pa, ps, ca, cs, beta, gamma, n);
    H2B_LAUNCHED("k_lookup_product");
    return ok();
}

extern "C" uint64_t _halo2_commit_product_workspace_size(uint64_t poly_length)
{
    ScratchPlan p;
    for (int i = 0; i < 5; i++) p.add(poly_length * 32);
    return p.used;
}

extern "C" uint64_t _halo2_commit_product_max_len(uint64_t poly_length, uint64_t free_bytes)
{
    for (uint64_t l = poly_length; l > 0; l >>= 1)
        if (_halo2_commit_product_workspace_size(l) < free_bytes) return l;
    return 0;
}

extern "C" RustError _halo2_commit_product(const FFITraitObject* lookup_product, const FFITraitObject* permuted_input,
                                           const FFITraitObject* permuted_table,
                                           const FFITraitObject* compressed_input,
                                           const FFITraitObject* compressed_table, const void* beta_device,
                                           const void* gamma_device, uint64_t length, uint64_t offset, void* scratch,
                                           uint64_t scratch_bytes, cudaStream_t stream)
{
    uint64_t need = _halo2_commit_product_workspace_size(length);
    if (scratch_bytes < need) return scratch_too_small("_halo2_commit_product", scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    Fr* buf[5];
    for (int i = 0; i < 5; i++) buf[i] = ar.take_n<Fr>(length);
    const FFITraitObject* srcs[4] = {permuted_input, permuted_table, compressed_input, compressed_table};
    for (int i = 0; i < 4; i++)
        H2B_CUDA(cudaMemcpyAsync(buf[i + 1], (const uint8_t*)srcs[i]->ptr + offset * 32, length * 32,
                                 cudaMemcpyHostToDevice, stream));
    H2B_TRY(lookup_product_run(buf[0], buf[1], buf[2], buf[3], buf[4], (const Fr*)beta_device,
                               (const Fr*)gamma_device, length, stream));
    H2B_CUDA(cudaMemcpyAsync((uint8_t*)lookup_product->ptr + offset * 32, buf[0], length * 32,
                             cudaMemcpyDeviceToHost, stream));
    H2B_CUDA(cudaStreamSynchronize(stream));
    return ok();
}

extern "C" RustError _halo2_commit_product_device_inputs(
    const FFITraitObject* d_lookup_product, const FFITraitObject* d_permuted_input,
    const FFITraitObject* d_permuted_table, const FFITraitObject* d_compressed_input,
    const FFITraitObject* d_compressed_table, const void* beta_device, const void* gamma_device, uint64_t length,
    uint64_t offset, cudaStream_t stream)
{
    auto at = [&](const FFITraitObject* o) { return (Fr*)((uint8_t*)o->ptr + offset * 32); };
    return lookup_product_run(at(d_lookup_product), at(d_permuted_input), at(d_permuted_table),
                              at(d_compressed_input), at(d_compressed_table), (const Fr*)beta_device,
                              (const Fr*)gamma_device, length, stream);
}

// permutation product -------------------------------------------------------------

extern "C" uint64_t _halo2_permutation_product_workspace_size(uint64_t poly_length)
{
    // accumulator, numerators, and one staged (sigma, value) column pair
    ScratchPlan p;
    for (int i = 0; i < 4; i++) p.add(poly_length * 32);
    return p.used;
}

extern "C" uint64_t _halo2_permutation_product_max_len(uint64_t poly_length, uint64_t free_bytes)
{
    for (uint64_t l = poly_length; l > 0; l >>= 1)
        if (_halo2_permutation_product_workspace_size(l) < free_bytes) return l;
    return 0;
}

extern "C" RustError _halo2_permutation_product(const FFITraitObject* modified_values,
                                                const FFITraitObject* permutations, const FFITraitObject* values,
                                                const void* beta_device, const void* gamma_device,
                                                const void* delta_device, const void* omega_device,
                                                void* deltaomega_device, uint64_t length, uint64_t offset,
                                                uint64_t batch, void* scratch, uint64_t scratch_bytes,
                                                cudaStream_t stream)
{
    uint64_t need = _halo2_permutation_product_workspace_size(length);
    if (scratch_bytes < need) return scratch_too_small("_halo2_permutation_product", scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    Fr* den = ar.take_n<Fr>(length);
    Fr* num = ar.take_n<Fr>(length);
    Fr* sig = ar.take_n<Fr>(length);
    Fr* val = ar.take_n<Fr>(length);
    H2B_CUDA(cudaMemcpyAsync(den, modified_values->ptr, length * 32, cudaMemcpyHostToDevice, stream));
    for (uint64_t c = 0; c < batch; c++) {
        H2B_CUDA(cudaMemcpyAsync(sig, (const uint8_t*)permutations[c].ptr + offset * 32, length * 32,
                                 cudaMemcpyHostToDevice, stream));
        H2B_CUDA(cudaMemcpyAsync(val, (const uint8_t*)values[c].ptr + offset * 32, length * 32,
                                 cudaMemcpyHostToDevice, stream));
        if (length > 0) {
            uint64_t nthreads = (length + PP_CHUNK - 1) / PP_CHUNK;
            k_pp_accumulate<<<grid_for(nthreads, 256), 256, 0, stream>>>(
                den, num, sig, val, (const Fr*)beta_device, (const Fr*)gamma_device, (const Fr*)omega_device,
                (const Fr*)deltaomega_device, length, c == 0);
            H2B_LAUNCHED("k_pp_accumulate");
        }
        k_advance_deltaomega<<<1, 32, 0, stream>>>((Fr*)deltaomega_device, (const Fr*)delta_device, 1);
        H2B_LAUNCHED("k_advance_deltaomega");
    }
    if (length > 0) {
        enable_big_smem(k_pp_finish);
        k_pp_finish<<<(unsigned)tiles_of(length), BI_T, BI_SMEM, stream>>>(den, num, length, batch > 0);
        H2B_LAUNCHED("k_pp_finish");
    }
    H2B_CUDA(cudaMemcpyAsync(modified_values->ptr, den, length * 32, cudaMemcpyDeviceToHost, stream));
    H2B_CUDA(cudaStreamSynchronize(stream));
    return ok();
}

extern "C" uint64_t _halo2_permutation_product_device_inputs_workspace_size(uint64_t poly_length)
{
    (void)poly_length;
    return 0;
}

extern "C" RustError _halo2_permutation_product_device_inputs(
    const FFITraitObject* modified_values_device, const FFITraitObject* permutations_device,
    const FFITraitObject* values_device, const void* beta_device, const void* gamma_device, const void* delta_device,
    const void* omega_device, void* deltaomega_device, uint64_t length, uint64_t offset, uint64_t batch,
    void* scratch, uint64_t scratch_bytes, cudaStream_t stream)
{
    (void)scratch;
    (void)scratch_bytes;
    if (batch > PP_MAX_COLS) return err(cudaErrorInvalidValue, "permutation product: too many columns in one set");
    PermCols cols;
    for (uint64_t c = 0; c < batch; c++) {
        cols.sigma[c] = (const Fr*)((const uint8_t*)permutations_device[c].ptr + offset * 32);
        cols.value[c] = (const Fr*)((const uint8_t*)values_device[c].ptr + offset * 32);
    }
    Fr* acc = (Fr*)modified_values_device->ptr;
    if (length > 0) {
        enable_big_smem(k_permutation_product);
        k_permutation_product<<<(unsigned)tiles_of(length), BI_T, BI_SMEM, stream>>>(
            acc, cols, (int)batch, (const Fr*)beta_device, (const Fr*)gamma_device, (const Fr*)delta_device,
            (const Fr*)omega_device, (const Fr*)deltaomega_device, length);
        H2B_LAUNCHED("k_permutation_product");
    }
    k_advance_deltaomega<<<1, 32, 0, stream>>>((Fr*)deltaomega_device, (const Fr*)delta_device, batch);
    H2B_LAUNCHED("k_advance_deltaomega");
    return ok();
}

// ---------------------------------------------------------------------------
// Batch inversion without any allocation
// ---------------------------------------------------------------------------
// For callers that cannot allocate device memory: code that must keep the
// reference's scratch-free `_halo2_batch_invert(d, field, len, stream)` call
// shape (its Rust call sites own every device buffer and have no workspace to
// hand over), code whose device memory is entirely pre-reserved by an arena
// or pool it does not control, and code that must not trigger the
// synchronisation cudaMalloc implies.  They still get the single-inversion
// multi-level algorithm of h2b_batch_invert, with its per-tile totals kept
// in a fixed array that lives in this library's device image.
//
// Limits and rules of use:
//  * length <= 2^26 elements; larger inputs are rejected with an error.
//  * The array (1.5 MiB) is reserved on every GPU that loads this library and
//    stays reserved until the process exits.
//  * All calls share the one array: calls whose work overlaps on the GPU
//    (different streams without ordering, or several host threads) race and
//    corrupt each other's results.  Serialise them on one stream.
//  * The array keeps the previous call's contents; nothing in it needs to
//    start at zero (every tile total is written before it is read).
//  * The first call on each device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current); make that first call
//    before any stream capture.  The address is kept per device together
//    with the unique id of the CUDA context it belongs to: after the
//    device's context is destroyed and recreated (cudaDeviceReset), the
//    next call sees a new context id and looks the address up again, so a
//    stale address is never used.  No call allocates or frees memory.
namespace h2b {
constexpr uint64_t NOALLOC_SCRATCH_BYTES = 1536ull << 10;
constexpr uint64_t NOALLOC_MAX_LENGTH = 1ull << 26;
constexpr int NOALLOC_MAX_DEVICES = 64;
static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};
static unsigned long long g_noalloc_ctx[NOALLOC_MAX_DEVICES] = {};

// The unique id of the calling thread's current CUDA context (driver entry
// points cuCtxGetCurrent / cuCtxGetId, found at run time so nothing links
// against the driver library), or 0 when it cannot be read.
static unsigned long long current_context_id()
{
    typedef int (*get_current_t)(void**);
    typedef int (*get_id_t)(void*, unsigned long long*);
    static get_current_t get_current = nullptr;
    static get_id_t get_id = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            get_id = nullptr;
    }
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, &id) == 0) return id;
    return 0;
}
} // namespace h2b

extern "C" RustError h2b_batch_invert_noalloc(void* d_data, uint32_t field_type, uint64_t length, cudaStream_t stream)
{
    if (field_type != 0 && field_type != 1) return err(cudaErrorInvalidValue, "Invalid scalar type");
    if (length == 0) return err(cudaErrorInvalidValue, "h2b_batch_invert_noalloc: length must be >= 1");
    if (length > NOALLOC_MAX_LENGTH)
        return err(cudaErrorInvalidValue, "h2b_batch_invert_noalloc: length exceeds the 2^26-element maximum");
    ScratchPlan plan;                                  // the tile levels (small totals arrays)
    plan_batch_invert(plan, length);
    const uint64_t need = plan.used;
    if (need > NOALLOC_SCRATCH_BYTES)
        return err(cudaErrorInvalidValue, "h2b_batch_invert_noalloc: length needs more than the fixed scratch");
    int dev = 0;
    H2B_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return err(cudaErrorInvalidValue, "h2b_batch_invert_noalloc: device id");
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        const unsigned long long ctx = current_context_id();
        if (g_noalloc_addr[dev] == nullptr || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
            void* p = nullptr;
            cudaError_t c = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (c != cudaSuccess) return cuda_err(c, "cudaGetSymbolAddress(no-allocation scratch)");
            g_noalloc_addr[dev] = p;
            g_noalloc_ctx[dev] = ctx;
        }
        base = g_noalloc_addr[dev];
    }
    ScratchArena ar(base, NOALLOC_SCRATCH_BYTES);
    if (field_type == 0) return batch_invert_levels<FrCfg>((Fr*)d_data, length, ar, stream);
    return batch_invert_levels<FqCfg>((Fq*)d_data, length, ar, stream);
}
