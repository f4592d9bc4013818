// Lookup permute-sort: `_halo2_permute_expression_pair`
// (halo2_proofs/cuda/src/commitment/permute_expression_pair.cu:185-350), the
// device counterpart of permute_expression_pair_seq
// (halo2_proofs/src/plonk/lookup/prover.rs:787-880):
//   A' = A[0..U) sorted by canonical value (BN254 Fr ordering);
//   S'[r] = A'[r] at the first occurrence of each value; the table values not
//   consumed that way (ascending, with multiplicity) fill the repeated rows
//   from the last repeated row backwards; rows [U, n) are zero.
// An input value missing from the table is reported as an error (the host
// reference panics).
//
// Device plan (details below k_merge_pass): the distinct table values are
// found with a hash set and sorted (canonical 256-bit keys, an 8-key register
// sort per thread, then merge-path merge passes), the input is counted per
// distinct value, and A' and S' are written in row order from prefix sums
// over the distinct values.
#include <algorithm>
#include "abi.cuh"
#include "field.cuh"
#include "prof.cuh"
#include "scan_u32.cuh"

namespace h2b {

struct Key {
    uint32_t w[8];  // canonical value, little-endian words
};

__device__ __forceinline__ Key ld_key(const Key* p)
{
    Key k;
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4 a = q[0], b = q[1];
    k.w[0] = a.x; k.w[1] = a.y; k.w[2] = a.z; k.w[3] = a.w;
    k.w[4] = b.x; k.w[5] = b.y; k.w[6] = b.z; k.w[7] = b.w;
    return k;
}
__device__ __forceinline__ void st_key(Key* p, const Key& k)
{
    uint4* q = reinterpret_cast<uint4*>(p);
    q[0] = make_uint4(k.w[0], k.w[1], k.w[2], k.w[3]);
    q[1] = make_uint4(k.w[4], k.w[5], k.w[6], k.w[7]);
}

// a < b as 256-bit integers
__device__ __forceinline__ bool key_lt(const Key& a, const Key& b)
{
#pragma unroll
    for (int i = 7; i >= 0; i--) {
        if (a.w[i] != b.w[i]) return a.w[i] < b.w[i];
    }
    return false;
}
__device__ __forceinline__ bool key_eq(const Key& a, const Key& b)
{
    uint32_t d = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) d |= a.w[i] ^ b.w[i];
    return d == 0;
}

constexpr int RUN0 = 8;

__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// keys[i] = canonical(src[i]) for i < u, then each thread sorts its run of 8.
__global__ void k_keys_sort8(const Fr* __restrict__ src, Key* __restrict__ keys, uint64_t u)
{
    uint64_t nruns = (u + RUN0 - 1) / RUN0;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nruns; t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t b = t * RUN0;
        int m = (int)umin64(RUN0, u - b);
        Key k[RUN0];
        for (int j = 0; j < RUN0; j++) {
            if (j < m) {
                Fr c = from_mont(ldg(&src[b + j]));
                for (int q = 0; q < 8; q++) k[j].w[q] = c.v[q];
            }
        }
        // insertion sort (stable)
        for (int j = 1; j < m; j++) {
            Key x = k[j];
            int i = j - 1;
            while (i >= 0 && key_lt(x, k[i])) {
                k[i + 1] = k[i];
                i--;
            }
            k[i + 1] = x;
        }
        for (int j = 0; j < m; j++) st_key(&keys[b + j], k[j]);
    }
}

constexpr int MP_ITEMS = 8;

// Merge adjacent sorted runs of length `run` from src into dst (stable:
// ties take the left run first).
__global__ void k_merge_pass(const Key* __restrict__ src, Key* __restrict__ dst, uint64_t n, uint64_t run)
{
    uint64_t nthreads = (n + MP_ITEMS - 1) / MP_ITEMS;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nthreads;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t out0 = t * MP_ITEMS;
        uint64_t pair = out0 / (2 * run);
        uint64_t a0 = pair * 2 * run;
        uint64_t la = umin64(run, n - a0);
        uint64_t b0 = a0 + la;
        uint64_t lb = b0 < n ? umin64(run, n - b0) : 0;
        uint64_t d = out0 - a0;  // diagonal inside this pair
        // find i in [max(0, d - lb), min(d, la)]: A[i-1] <= B[d-i] and B[d-i-1] < A[i]
        uint64_t lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
        while (lo < hi) {
            uint64_t i = (lo + hi) >> 1;
            // take more from A while A[i] <= B[d-i-1]
            Key ai = ld_key(&src[a0 + i]);
            Key bj = ld_key(&src[b0 + d - i - 1]);
            if (!key_lt(bj, ai)) lo = i + 1;
            else hi = i;
        }
        uint64_t i = lo, j = d - lo;
        uint64_t end = umin64(out0 + MP_ITEMS, a0 + la + lb);
        for (uint64_t o = out0; o < end; o++) {
            bool take_a;
            if (i >= la) take_a = false;
            else if (j >= lb) take_a = true;
            else take_a = !key_lt(ld_key(&src[b0 + j]), ld_key(&src[a0 + i]));
            if (take_a) { st_key(&dst[o], ld_key(&src[a0 + i])); i++; }
            else { st_key(&dst[o], ld_key(&src[b0 + j])); j++; }
        }
    }
}

// Sorts u canonical keys; returns the buffer holding the result (a or b).
static Key* sort_keys(const Fr* src, uint64_t u, Key* a, Key* b, cudaStream_t st, RustError* e)
{
    uint64_t nruns = (u + RUN0 - 1) / RUN0;
    k_keys_sort8<<<grid_for(nruns, 128, 148u * 16u), 128, 0, st>>>(src, a, u);
    cudaError_t c = cudaGetLastError();
    g_kernel_launches.fetch_add(1);
    if (c != cudaSuccess) { *e = cuda_err(c, "k_keys_sort8"); return a; }
    for (uint64_t run = RUN0; run < u; run *= 2) {
        uint64_t nthreads = (u + MP_ITEMS - 1) / MP_ITEMS;
        k_merge_pass<<<grid_for(nthreads, 128, 148u * 16u), 128, 0, st>>>(a, b, u, run);
        g_kernel_launches.fetch_add(1);
        c = cudaGetLastError();
        if (c != cudaSuccess) { *e = cuda_err(c, "k_merge_pass"); return a; }
        std::swap(a, b);
    }
    *e = ok();
    return a;
}

// ---------------------------------------------------------------------------
// Distinct-value plan.  A lookup table holds few distinct values (a 2^8-entry
// range table repeated or padded over the usable rows), and equal values have
// equal Montgomery images, so:
//   1. the table rows go into a hash set keyed by their Montgomery bytes; a
//      slot holds a 32-bit fingerprint and the index of a table row with that
//      value (the row itself is the stored key, already in memory, so no
//      thread ever reads a half-written key), and a multiplicity count;
//      equal rows of a warp are merged before they touch the set;
//   2. the d distinct values are sorted by canonical value (the merge sort
//      above, on d keys) and get their ranks;
//   3. each input row is looked up (a missing value is an error) and counted
//      per rank;
//   4. prefix sums over the d ranks give, for output row i, its rank in A'
//      (a first occurrence when i starts the rank's run) and, for a repeated
//      row, its leftover: leftovers are the table multiplicities minus one
//      per value the input uses, ascending, assigned from the last repeated
//      row backwards (prover.rs:852-857).
// No per-row sort and no per-row scatter: A' and S' are written in row order.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t mont_hash(const Key& k)
{
    uint64_t a = ((uint64_t)k.w[1] << 32) | k.w[0], b = ((uint64_t)k.w[3] << 32) | k.w[2];
    uint64_t c = ((uint64_t)k.w[5] << 32) | k.w[4], d = ((uint64_t)k.w[7] << 32) | k.w[6];
    uint64_t x = a * 0x9E3779B97F4A7C15ull ^ b * 0xC2B2AE3D27D4EB4Full ^ c * 0x165667B19E3779F9ull ^
                 d * 0x27D4EB2F165667C5ull;
    x ^= x >> 29;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 32;
    return x;
}

struct HashSet {
    uint64_t* slot;      // 0 = empty, else fingerprint << 32 | (table row + 1)
    uint32_t* count;     // multiplicity of the slot's value in the table
    uint32_t* rank;      // rank of the slot's value among the distinct values
    uint64_t mask;       // slots - 1
};

enum : uint32_t { PP_ERR_MISSING = 1u, PP_ERR_FULL = 2u };

// The slot of key k, inserted with table row `row` when absent (insert) or
// ~0 when absent (lookup).  At most one pass over the slots: a full set is
// flagged and returns ~0.
__device__ __forceinline__ uint64_t hs_find(HashSet hs, const Key* __restrict__ table, const Key& k, uint32_t row,
                                            bool insert, uint32_t* errflag)
{
    uint64_t h = mont_hash(k);
    uint64_t fp = (h >> 32) & 0xffffffffull;
    uint64_t mine = (fp << 32) | ((uint64_t)row + 1);
    uint64_t s = h & hs.mask;
    for (uint64_t probe = 0; probe <= hs.mask; probe++) {
        uint64_t w = *(volatile uint64_t*)&hs.slot[s];
        if (w == 0) {
            if (!insert) return ~0ull;
            w = atomicCAS((unsigned long long*)&hs.slot[s], 0ull, (unsigned long long)mine);
            if (w == 0) return s;
        }
        if ((w >> 32) == fp && key_eq(ld_key(&table[(w & 0xffffffffull) - 1]), k)) return s;
        s = (s + 1) & hs.mask;
    }
    if (insert) atomicOr(errflag, PP_ERR_FULL);
    return ~0ull;
}

// The first row of each warp-sized group of a grid-stride loop over [0, count).
__device__ __forceinline__ uint64_t warp_base() { return (blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; }
__device__ __forceinline__ uint64_t warp_stride() { return (uint64_t)gridDim.x * (blockDim.x >> 5) * 32; }

// Table rows into the set, with their multiplicities.  Lanes holding equal
// values (same 32-bit hash, then the full key checked against the group
// leader's) add their count once.
__global__ void k_pp_insert(const Key* __restrict__ table, uint64_t u, HashSet hs, uint32_t* __restrict__ errflag)
{
    const unsigned lane = threadIdx.x & 31;
    for (uint64_t base = warp_base(); base < u; base += warp_stride()) {
        uint64_t i = base + lane;
        bool valid = i < u;
        Key k;
        if (valid) k = ld_key(&table[i]);
        else for (int q = 0; q < 8; q++) k.w[q] = 0;
        uint32_t h = valid ? (uint32_t)mont_hash(k) : 0xffffffffu;
        unsigned grp = __match_any_sync(0xffffffffu, h);
        int leader = __ffs(grp) - 1;
        Key lk;
        for (int q = 0; q < 8; q++) lk.w[q] = __shfl_sync(0xffffffffu, k.w[q], leader);
        bool same = valid && key_eq(k, lk);
        unsigned same_mask = __ballot_sync(0xffffffffu, same) & grp;
        if (!valid) continue;
        if (same) {
            if ((int)lane == leader) {
                uint64_t s = hs_find(hs, table, k, (uint32_t)i, true, errflag);
                if (s != ~0ull) atomicAdd(&hs.count[s], (uint32_t)__popc(same_mask));
            }
        } else {
            uint64_t s = hs_find(hs, table, k, (uint32_t)i, true, errflag);
            if (s != ~0ull) atomicAdd(&hs.count[s], 1u);
        }
    }
}

// Occupied slots -> the distinct values (Montgomery images, in slot order).
__global__ void k_pp_collect(const Key* __restrict__ table, HashSet hs, uint64_t nslots, Key* __restrict__ distinct,
                             uint32_t* __restrict__ dcount)
{
    const unsigned lane = threadIdx.x & 31;
    for (uint64_t base = warp_base(); base < nslots; base += warp_stride()) {
        uint64_t s = base + lane;
        uint64_t w = s < nslots ? hs.slot[s] : 0;
        unsigned occ = __ballot_sync(0xffffffffu, w != 0);
        uint32_t first = 0;
        if (lane == 0 && occ) first = atomicAdd(dcount, (uint32_t)__popc(occ));
        first = __shfl_sync(0xffffffffu, first, 0);
        if (w != 0) {
            uint32_t pos = first + __popc(occ & ((1u << lane) - 1));
            st_key(&distinct[pos], ld_key(&table[(w & 0xffffffffull) - 1]));
        }
    }
}

// Sorted canonical keys -> Montgomery images by rank, each slot's rank and
// the table multiplicity per rank.
__global__ void k_pp_rank(const Key* __restrict__ sorted, uint32_t d, const Key* __restrict__ table, HashSet hs,
                          Fr* __restrict__ dm, uint32_t* __restrict__ tcount, uint32_t* __restrict__ errflag)
{
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < d; r += gridDim.x * blockDim.x) {
        Key c = ld_key(&sorted[r]);
        Fr v;
        for (int q = 0; q < 8; q++) v.v[q] = c.w[q];
        v = to_mont(v);
        st(&dm[r], v);
        Key k;
        for (int q = 0; q < 8; q++) k.w[q] = v.v[q];
        uint64_t s = hs_find(hs, table, k, 0, false, errflag);
        if (s == ~0ull) { atomicOr(errflag, PP_ERR_FULL); tcount[r] = 0; continue; }
        hs.rank[s] = r;
        tcount[r] = hs.count[s];
    }
}

// Input rows counted per rank (equal ranks of a warp add once); a value
// absent from the table is flagged.
__global__ void k_pp_count(const Key* __restrict__ input, uint64_t u, const Key* __restrict__ table, HashSet hs,
                           uint32_t* __restrict__ acount, uint32_t* __restrict__ errflag,
                           const uint32_t* __restrict__ skip)
{
    if (skip && *skip) return;
    const unsigned lane = threadIdx.x & 31;
    for (uint64_t base = warp_base(); base < u; base += warp_stride()) {
        uint64_t i = base + lane;
        uint32_t r = 0xffffffffu;
        if (i < u) {
            Key k = ld_key(&input[i]);
            uint64_t s = hs_find(hs, table, k, 0, false, errflag);
            if (s == ~0ull) atomicOr(errflag, PP_ERR_MISSING);
            else r = hs.rank[s];
        }
        unsigned grp = __match_any_sync(0xffffffffu, r);
        if (r != 0xffffffffu && (int)lane == __ffs(grp) - 1) atomicAdd(&acount[r], (uint32_t)__popc(grp));
    }
}

// The single-CTA path's count: ranks go into a per-block histogram in shared
// memory (d <= PP_SMALL bins), each block adds its nonzero bins once, so the
// global counters see one atomic per block and rank instead of one per row.
__global__ void __launch_bounds__(256) k_pp_count_small(const Key* __restrict__ input, uint64_t u,
                                                        const Key* __restrict__ table, HashSet hs,
                                                        uint32_t* __restrict__ acount, uint32_t* __restrict__ misc);

// Per rank: used = the input holds the value; left = the table copies that
// no first occurrence takes.
__global__ void k_pp_flags(const uint32_t* __restrict__ acount, const uint32_t* __restrict__ tcount, uint32_t d,
                           uint32_t* __restrict__ used, uint32_t* __restrict__ left)
{
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < d; r += gridDim.x * blockDim.x) {
        uint32_t u1 = acount[r] > 0 ? 1u : 0u;
        used[r] = u1;
        left[r] = tcount[r] - u1;
    }
}

// Last index j < m of a non-decreasing array with a[j] <= x (given a[0] <= x).
__device__ __forceinline__ uint32_t last_le(const uint32_t* a, uint32_t m, uint32_t x)
{
    uint32_t lo = 0, hi = m;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

constexpr uint32_t PP_SMEM_RANKS = 2048;

// A' and S' in row order.  astart / lstart: exclusive scans over the d ranks
// of the input counts and of the leftovers; uexcl: exclusive scan of `used`
// (uexcl[r + 1] first occurrences lie at or before rank r's run).
__global__ void __launch_bounds__(256) k_pp_emit(const Fr* __restrict__ dm, const uint32_t* __restrict__ astart,
                                                 const uint32_t* __restrict__ uexcl,
                                                 const uint32_t* __restrict__ lstart, const uint32_t* __restrict__ pd,
                                                 uint64_t u, uint64_t n, Fr* __restrict__ pin, Fr* __restrict__ ptab,
                                                 const uint32_t* __restrict__ skip)
{
    if (skip && *skip) return;
    const uint32_t d = *pd;
    __shared__ uint32_t s_a[PP_SMEM_RANKS], s_l[PP_SMEM_RANKS];
    const bool small = d <= PP_SMEM_RANKS;
    if (small) {
        for (uint32_t r = threadIdx.x; r < d; r += blockDim.x) { s_a[r] = astart[r]; s_l[r] = lstart[r]; }
    }
    __syncthreads();
    const uint32_t* A = small ? s_a : astart;
    const uint32_t* L = small ? s_l : lstart;
    const uint32_t nrep = (uint32_t)u - uexcl[d];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (i >= u) {
            st(&pin[i], Fr::zero());
            st(&ptab[i], Fr::zero());
            continue;
        }
        uint32_t r = last_le(A, d, (uint32_t)i);
        Fr a = ld(&dm[r]);
        st(&pin[i], a);
        if ((uint32_t)i == A[r]) {
            st(&ptab[i], a);
        } else {
            uint32_t rep = (uint32_t)i - uexcl[r + 1];          // index among the repeated rows
            uint32_t j = nrep - 1 - rep;                       // the last repeated row takes leftover 0
            st(&ptab[i], ld(&dm[last_le(L, d, j)]));
        }
    }
}

// ---- few distinct values: one CTA sorts them and one CTA scans the ranks, so
// nothing waits for the host between the passes ----------------------------

constexpr uint32_t PP_SMALL = 1024;      // distinct values the single-CTA path takes
enum : int { PP_D = 0, PP_ERR = 1, PP_LARGE = 2, PP_TOT_A = 3, PP_TOT_U = 4, PP_TOT_L = 5, PP_MISC = 8 };

// Bitonic sort of the d <= PP_SMALL distinct values by canonical value in
// shared memory (indices past d act as +infinity), then per rank: the
// Montgomery image, the slot's rank, the table multiplicity, a zero input
// count.  More than PP_SMALL values set PP_LARGE and leave everything else.
__global__ void __launch_bounds__(1024) k_pp_small_sort(const Key* __restrict__ distinct, uint32_t* __restrict__ misc,
                                                        const Key* __restrict__ table, HashSet hs, Fr* __restrict__ dm,
                                                        uint32_t* __restrict__ tcount, uint32_t* __restrict__ acount)
{
    __shared__ Key sk[PP_SMALL];
    __shared__ uint16_t si[PP_SMALL];
    const uint32_t d = misc[PP_D];
    if (d > PP_SMALL) {
        if (threadIdx.x == 0) misc[PP_LARGE] = 1;
        return;
    }
    uint32_t P = 1;
    while (P < d) P <<= 1;
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
        si[i] = (uint16_t)i;
        if (i < d) {
            Fr c = from_mont(ld(reinterpret_cast<const Fr*>(&distinct[i])));
            for (int q = 0; q < 8; q++) sk[i].w[q] = c.v[q];
        }
    }
    __syncthreads();
    auto less = [&](uint32_t x, uint32_t y) -> bool {   // key x < key y, indices >= d are +infinity
        if (x >= d) return false;
        if (y >= d) return true;
        return key_lt(sk[x], sk[y]);
    };
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const uint32_t a = si[i], b = si[l];
                    const bool asc = (i & k) == 0;
                    if (asc ? less(b, a) : less(a, b)) { si[i] = (uint16_t)b; si[l] = (uint16_t)a; }
                }
            }
            __syncthreads();
        }
    }
    uint32_t* errflag = misc + PP_ERR;
    for (uint32_t r = threadIdx.x; r < d; r += blockDim.x) {
        const Key mk = ld_key(&distinct[si[r]]);          // the Montgomery image
        st_key(reinterpret_cast<Key*>(&dm[r]), mk);
        uint64_t s = hs_find(hs, table, mk, 0, false, errflag);
        acount[r] = 0;
        if (s == ~0ull) { atomicOr(errflag, PP_ERR_FULL); tcount[r] = 0; continue; }
        hs.rank[s] = r;
        tcount[r] = hs.count[s];
    }
}

// Exclusive scans over the d <= PP_SMALL ranks (one CTA of 1024 threads):
// astart of the input counts, uexcl of used = (count > 0), lstart of the
// leftovers, totals at [d] and in misc.
__global__ void __launch_bounds__(1024) k_pp_small_scan(const uint32_t* __restrict__ acount,
                                                        const uint32_t* __restrict__ tcount, uint32_t* __restrict__ misc,
                                                        uint32_t* __restrict__ astart, uint32_t* __restrict__ uexcl,
                                                        uint32_t* __restrict__ lstart)
{
    if (misc[PP_LARGE]) return;
    const uint32_t d = misc[PP_D];
    const uint32_t r = threadIdx.x, lane = r & 31, warp = r >> 5;
    const uint32_t ac = r < d ? acount[r] : 0;
    const uint32_t u1 = ac > 0 ? 1u : 0u;
    const uint32_t lf = r < d ? tcount[r] - u1 : 0;
    __shared__ uint32_t wt[3][32];
    uint32_t ia = warp_incl_scan(ac), iu = warp_incl_scan(u1), il = warp_incl_scan(lf);
    if (lane == 31) { wt[0][warp] = ia; wt[1][warp] = iu; wt[2][warp] = il; }
    __syncthreads();
    if (warp == 0) {
        for (int q = 0; q < 3; q++) {
            uint32_t v = wt[q][lane];
            uint32_t inc = warp_incl_scan(v);
            wt[q][lane] = inc - v;
            if (lane == 31) misc[PP_TOT_A + q] = inc;
        }
    }
    __syncthreads();
    if (r < d) {
        astart[r] = wt[0][warp] + ia - ac;
        uexcl[r] = wt[1][warp] + iu - u1;
        lstart[r] = wt[2][warp] + il - lf;
    }
    if (r == 0) {
        astart[d] = misc[PP_TOT_A];
        uexcl[d] = misc[PP_TOT_U];
        lstart[d] = misc[PP_TOT_L];
    }
}

__global__ void __launch_bounds__(256) k_pp_count_small(const Key* __restrict__ input, uint64_t u,
                                                        const Key* __restrict__ table, HashSet hs,
                                                        uint32_t* __restrict__ acount, uint32_t* __restrict__ misc)
{
    if (misc[PP_LARGE]) return;
    const uint32_t d = misc[PP_D];
    __shared__ uint32_t hist[PP_SMALL];
    for (uint32_t r = threadIdx.x; r < d; r += blockDim.x) hist[r] = 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < u; i += (uint64_t)gridDim.x * blockDim.x) {
        const Key k = ld_key(&input[i]);
        const uint64_t s = hs_find(hs, table, k, 0, false, misc + PP_ERR);
        if (s == ~0ull) {
            atomicOr(misc + PP_ERR, PP_ERR_MISSING);
        } else {
            const uint32_t r = hs.rank[s];
            if (r < d) atomicAdd(&hist[r], 1u);
            else atomicOr(misc + PP_ERR, PP_ERR_FULL);
        }
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < d; r += blockDim.x)
        if (hist[r]) atomicAdd(&acount[r], hist[r]);
}

static uint64_t pp_slots(uint64_t u)
{
    uint64_t s = 1024;
    while (s < 2 * u) s <<= 1;
    return s;
}

// The hash slots, their multiplicities and the misc words are one block, so
// one memset clears them.
static uint64_t pp_clear_bytes(uint64_t S) { return S * sizeof(uint64_t) + S * sizeof(uint32_t) + PP_MISC * 4; }

static void plan_permute(ScratchPlan& p, uint64_t u)
{
    uint64_t m = std::max<uint64_t>(u, 1), S = pp_slots(m);
    p.add(pp_clear_bytes(S));                              // hash slots, multiplicities, misc
    p.add_n<uint32_t>(S);                                  // ranks
    p.add(m * sizeof(Key));                                // distinct values (Montgomery), slot order
    p.add(m * sizeof(Key));                                // sort buffer A
    p.add(m * sizeof(Key));                                // sort buffer B
    p.add(m * sizeof(Fr));                                 // distinct values by rank
    for (int i = 0; i < 4; i++) p.add_n<uint32_t>(m + 1);  // table counts, input counts, used, left
    for (int i = 0; i < 3; i++) p.add_n<uint32_t>(m + 2);  // astart, uexcl, lstart
    p.add_n<uint32_t>(scan_u32_tiles(m + 1) + 1);          // scan tiles
}

} // namespace h2b

using namespace h2b;

extern "C" uint64_t _halo2_permute_expression_pair_workspace_size(uint64_t n, uint64_t usable_rows)
{
    (void)n;
    ScratchPlan p;
    plan_permute(p, usable_rows);
    return p.used;
}

extern "C" RustError _halo2_permute_expression_pair(const void* d_compressed_input, const void* d_compressed_table,
                                                    void* d_permuted_input, void* d_permuted_table, uint64_t n,
                                                    uint64_t usable_rows, void* scratch, uint64_t scratch_bytes,
                                                    cudaStream_t stream)
{
    const uint64_t u = usable_rows;
    if (u > n) return err(cudaErrorInvalidValue, "_halo2_permute_expression_pair: usable_rows > n");
    if (u >= 0x7fffffffull) return err(cudaErrorInvalidValue, "_halo2_permute_expression_pair: too many rows");
    uint64_t need = _halo2_permute_expression_pair_workspace_size(n, u);
    if (scratch_bytes < need) return scratch_too_small("_halo2_permute_expression_pair", scratch_bytes, need);
    if (n == 0) return ok();
    Fr* pin = (Fr*)d_permuted_input;
    Fr* ptab = (Fr*)d_permuted_table;
    if (u == 0) {
        H2B_CUDA(cudaMemsetAsync(pin, 0, n * sizeof(Fr), stream));
        H2B_CUDA(cudaMemsetAsync(ptab, 0, n * sizeof(Fr), stream));
        return ok();
    }
    ScratchArena ar(scratch, scratch_bytes);
    const uint64_t m = u, S = pp_slots(m);
    HashSet hs;
    char* clear = (char*)ar.take(pp_clear_bytes(S));
    hs.slot = (uint64_t*)clear;
    hs.count = (uint32_t*)(clear + S * sizeof(uint64_t));
    uint32_t* misc = (uint32_t*)(clear + S * sizeof(uint64_t) + S * sizeof(uint32_t));  // distinct count, flags, totals
    hs.rank = ar.take_n<uint32_t>(S);
    hs.mask = S - 1;
    Key* distinct = (Key*)ar.take(m * sizeof(Key));
    Key* ka = (Key*)ar.take(m * sizeof(Key));
    Key* kb = (Key*)ar.take(m * sizeof(Key));
    Fr* dm = (Fr*)ar.take(m * sizeof(Fr));
    uint32_t* tcount = ar.take_n<uint32_t>(m + 1);
    uint32_t* acount = ar.take_n<uint32_t>(m + 1);
    uint32_t* used = ar.take_n<uint32_t>(m + 1);
    uint32_t* left = ar.take_n<uint32_t>(m + 1);
    uint32_t* astart = ar.take_n<uint32_t>(m + 2);
    uint32_t* uexcl = ar.take_n<uint32_t>(m + 2);
    uint32_t* lstart = ar.take_n<uint32_t>(m + 2);
    uint32_t* tiles = ar.take_n<uint32_t>(scan_u32_tiles(m + 1) + 1);
    if (!ar.good()) return scratch_too_small("_halo2_permute_expression_pair", scratch_bytes, need);
    const Key* table = (const Key*)d_compressed_table;
    const Key* input = (const Key*)d_compressed_input;
    prof_begin(PROF_PERMUTE_SORT, stream);
    H2B_CUDA(cudaMemsetAsync(clear, 0, pp_clear_bytes(S), stream));
    k_pp_insert<<<grid_for((u + 31) / 32, 8, 148u * 16u), 256, 0, stream>>>(table, u, hs, misc + PP_ERR);
    H2B_LAUNCHED("k_pp_insert");
    k_pp_collect<<<grid_for((S + 31) / 32, 8, 148u * 16u), 256, 0, stream>>>(table, hs, S, distinct, misc + PP_D);
    H2B_LAUNCHED("k_pp_collect");
    // single-CTA path for few distinct values (skipped on the device otherwise)
    k_pp_small_sort<<<1, 1024, 0, stream>>>(distinct, misc, table, hs, dm, tcount, acount);
    H2B_LAUNCHED("k_pp_small_sort");
    k_pp_count_small<<<grid_for(u, 256, 148u * 2u), 256, 0, stream>>>(input, u, table, hs, acount, misc);
    H2B_LAUNCHED("k_pp_count_small");
    k_pp_small_scan<<<1, 1024, 0, stream>>>(acount, tcount, misc, astart, uexcl, lstart);
    H2B_LAUNCHED("k_pp_small_scan");
    k_pp_emit<<<grid_for(n, 256, 148u * 8u), 256, 0, stream>>>(dm, astart, uexcl, lstart, misc + PP_D, u, n, pin, ptab,
                                                             misc + PP_LARGE);
    H2B_LAUNCHED("k_pp_emit");
    uint32_t h[PP_MISC];
    H2B_CUDA(cudaMemcpyAsync(h, misc, sizeof(h), cudaMemcpyDeviceToHost, stream));
    H2B_CUDA(cudaStreamSynchronize(stream));
    if (h[PP_ERR] & PP_ERR_FULL) return err(cudaErrorUnknown, "permute_expression_pair: hash set overflow");
    const uint32_t d = h[PP_D];
    if (d == 0 || d > u) return err(cudaErrorUnknown, "permute_expression_pair: distinct count out of range");
    if (h[PP_LARGE]) {
        // more distinct values than one CTA sorts: merge sort of the d values,
        // then the same passes with device-wide scans
        RustError e;
        const Key* sorted = sort_keys(reinterpret_cast<const Fr*>(distinct), d, ka, kb, stream, &e);
        if (e.code) return e;
        H2B_CUDA(cudaMemsetAsync(acount, 0, (d + 1) * sizeof(uint32_t), stream));
        k_pp_rank<<<grid_for(d, 128, 148u * 8u), 128, 0, stream>>>(sorted, d, table, hs, dm, tcount, misc + PP_ERR);
        H2B_LAUNCHED("k_pp_rank");
        k_pp_count<<<grid_for((u + 31) / 32, 8, 148u * 16u), 256, 0, stream>>>(input, u, table, hs, acount,
                                                                              misc + PP_ERR, nullptr);
        H2B_LAUNCHED("k_pp_count");
        k_pp_flags<<<grid_for(d, 256, 148u * 8u), 256, 0, stream>>>(acount, tcount, d, used, left);
        H2B_LAUNCHED("k_pp_flags");
        H2B_CUDA(scan_u32(acount, d, astart, tiles, stream));
        H2B_CUDA(scan_u32(used, d, uexcl, tiles, stream));
        H2B_CUDA(scan_u32(left, d, lstart, tiles, stream));
        g_kernel_launches.fetch_add(9);
        k_pp_emit<<<grid_for(n, 256, 148u * 8u), 256, 0, stream>>>(dm, astart, uexcl, lstart, misc + PP_D, u, n, pin,
                                                                 ptab, nullptr);
        H2B_LAUNCHED("k_pp_emit");
        H2B_CUDA(cudaMemcpyAsync(&h[PP_ERR], misc + PP_ERR, 4, cudaMemcpyDeviceToHost, stream));
        H2B_CUDA(cudaMemcpyAsync(&h[PP_TOT_U], uexcl + d, 4, cudaMemcpyDeviceToHost, stream));
        H2B_CUDA(cudaMemcpyAsync(&h[PP_TOT_L], lstart + d, 4, cudaMemcpyDeviceToHost, stream));
        H2B_CUDA(cudaMemcpyAsync(&h[PP_TOT_A], astart + d, 4, cudaMemcpyDeviceToHost, stream));
        H2B_CUDA(cudaStreamSynchronize(stream));
    }
    prof_end(PROF_PERMUTE_SORT, stream);
    // A lookup input missing from the table is a constraint-system failure in
    // the reference; so is a leftover count that does not fill the repeated rows.
    if (h[PP_ERR] & PP_ERR_MISSING)
        return err(cudaErrorInvalidValue, "permute_expression_pair: input value not found in the table");
    if (h[PP_ERR]) return err(cudaErrorUnknown, "permute_expression_pair: hash set lookup failed");
    if (h[PP_TOT_A] != (uint32_t)u || h[PP_TOT_L] != (uint32_t)u - h[PP_TOT_U])
        return err(cudaErrorInvalidValue, "permute_expression_pair: leftover count mismatch");
    return ok();
}
