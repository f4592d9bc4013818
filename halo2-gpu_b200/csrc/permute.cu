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
// Device plan: canonical 256-bit keys (one Montgomery reduction each), an
// 8-key register sort per thread, then merge-path merge passes (each thread
// finds its split of the two runs by binary search on the diagonal and merges
// 8 outputs), for both A and the table.  First occurrences, consumed table
// entries (binary search of each table run head in A') and leftover /
// repeated-row positions are flags compacted by exclusive scans.
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

__device__ __forceinline__ bool key_search(const Key* __restrict__ arr, uint64_t n, const Key& k)
{
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t m = (lo + hi) >> 1;
        if (key_lt(ld_key(&arr[m]), k)) lo = m + 1; else hi = m;
    }
    return lo < n && key_eq(ld_key(&arr[lo]), k);
}

// rep[r] = A'[r] repeats A'[r-1]; left[t] = table entry t is not consumed by
// a first occurrence; err if a first-occurrence value is absent from T.
__global__ void k_flags(const Key* __restrict__ A, const Key* __restrict__ T, uint64_t u, uint32_t* __restrict__ rep,
                        uint32_t* __restrict__ left, uint32_t* __restrict__ errflag)
{
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < u; r += (uint64_t)gridDim.x * blockDim.x) {
        Key a = ld_key(&A[r]);
        bool first = (r == 0) || !key_eq(a, ld_key(&A[r - 1]));
        rep[r] = first ? 0u : 1u;
        if (first && !key_search(T, u, a)) atomicExch(errflag, 1u);
        Key t = ld_key(&T[r]);
        bool head = (r == 0) || !key_eq(t, ld_key(&T[r - 1]));
        left[r] = (head && key_search(A, u, t)) ? 0u : 1u;
    }
}

__global__ void k_leftovers(const Key* __restrict__ T, const uint32_t* __restrict__ left,
                            const uint32_t* __restrict__ lpos, uint64_t u, Key* __restrict__ L)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < u; t += (uint64_t)gridDim.x * blockDim.x)
        if (left[t]) st_key(&L[lpos[t]], ld_key(&T[t]));
}

__global__ void k_emit(const Key* __restrict__ A, const Key* __restrict__ L, const uint32_t* __restrict__ rep,
                       const uint32_t* __restrict__ rpos, uint64_t u, uint64_t n, Fr* __restrict__ pin,
                       Fr* __restrict__ ptab)
{
    const uint32_t nrep = rpos[u];
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
        if (r >= u) {
            st(&pin[r], Fr::zero());
            st(&ptab[r], Fr::zero());
            continue;
        }
        Key a = ld_key(&A[r]);
        Fr av;
        for (int q = 0; q < 8; q++) av.v[q] = a.w[q];
        av = to_mont(av);
        st(&pin[r], av);
        if (!rep[r]) {
            st(&ptab[r], av);
        } else {
            Key l = ld_key(&L[nrep - 1 - rpos[r]]);
            Fr lv;
            for (int q = 0; q < 8; q++) lv.v[q] = l.w[q];
            st(&ptab[r], to_mont(lv));
        }
    }
}

static void plan_permute(ScratchPlan& p, uint64_t u)
{
    uint64_t m = std::max<uint64_t>(u, 1);
    for (int i = 0; i < 5; i++) p.add(m * sizeof(Key));   // A, A2, T, T2, L
    p.add_n<uint32_t>(m + 1);                              // rep
    p.add_n<uint32_t>(m + 1);                              // rpos
    p.add_n<uint32_t>(m + 1);                              // left
    p.add_n<uint32_t>(m + 1);                              // lpos
    p.add_n<uint32_t>(scan_u32_tiles(m) + 1);              // scan tiles
    p.add_n<uint32_t>(2);                                  // error flag
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
    if (u >= 0xffffffffull) return err(cudaErrorInvalidValue, "_halo2_permute_expression_pair: too many rows");
    uint64_t need = _halo2_permute_expression_pair_workspace_size(n, u);
    if (scratch_bytes < need) return scratch_too_small("_halo2_permute_expression_pair", scratch_bytes, need);
    if (n == 0) return ok();
    ScratchArena ar(scratch, scratch_bytes);
    uint64_t m = std::max<uint64_t>(u, 1);
    Key* a1 = (Key*)ar.take(m * sizeof(Key));
    Key* a2 = (Key*)ar.take(m * sizeof(Key));
    Key* t1 = (Key*)ar.take(m * sizeof(Key));
    Key* t2 = (Key*)ar.take(m * sizeof(Key));
    Key* L = (Key*)ar.take(m * sizeof(Key));
    uint32_t* rep = ar.take_n<uint32_t>(m + 1);
    uint32_t* rpos = ar.take_n<uint32_t>(m + 1);
    uint32_t* left = ar.take_n<uint32_t>(m + 1);
    uint32_t* lpos = ar.take_n<uint32_t>(m + 1);
    uint32_t* tiles = ar.take_n<uint32_t>(scan_u32_tiles(m) + 1);
    uint32_t* eflag = ar.take_n<uint32_t>(2);
    Fr* pin = (Fr*)d_permuted_input;
    Fr* ptab = (Fr*)d_permuted_table;
    prof_begin(PROF_PERMUTE_SORT, stream);
    const Key* A = a1;
    const Key* T = t1;
    if (u > 0) {
        RustError e;
        A = sort_keys((const Fr*)d_compressed_input, u, a1, a2, stream, &e);
        if (e.code) return e;
        T = sort_keys((const Fr*)d_compressed_table, u, t1, t2, stream, &e);
        if (e.code) return e;
        H2B_CUDA(cudaMemsetAsync(eflag, 0, 8, stream));
        k_flags<<<grid_for(u, 256, 148u * 8u), 256, 0, stream>>>(A, T, u, rep, left, eflag);
        H2B_LAUNCHED("k_flags");
        H2B_CUDA(scan_u32(rep, u, rpos, tiles, stream));
        H2B_CUDA(scan_u32(left, u, lpos, tiles, stream));
        k_leftovers<<<grid_for(u, 256, 148u * 8u), 256, 0, stream>>>(T, left, lpos, u, L);
        H2B_LAUNCHED("k_leftovers");
    } else {
        H2B_CUDA(cudaMemsetAsync(rpos, 0, 4, stream));
        H2B_CUDA(cudaMemsetAsync(eflag, 0, 8, stream));
    }
    k_emit<<<grid_for(n, 256, 148u * 8u), 256, 0, stream>>>(A, L, rep, rpos, u, n, pin, ptab);
    H2B_LAUNCHED("k_emit");
    prof_end(PROF_PERMUTE_SORT, stream);
    // The reference treats a lookup input missing from the table as a
    // constraint-system failure; report it (and count mismatch) as an error.
    uint32_t h[2] = {0, 0};
    uint32_t tot[2] = {0, 0};
    H2B_CUDA(cudaMemcpyAsync(h, eflag, 8, cudaMemcpyDeviceToHost, stream));
    if (u > 0) {
        H2B_CUDA(cudaMemcpyAsync(&tot[0], rpos + u, 4, cudaMemcpyDeviceToHost, stream));
        H2B_CUDA(cudaMemcpyAsync(&tot[1], lpos + u, 4, cudaMemcpyDeviceToHost, stream));
    }
    H2B_CUDA(cudaStreamSynchronize(stream));
    if (h[0]) return err(cudaErrorInvalidValue, "permute_expression_pair: input value not found in the table");
    if (tot[0] != tot[1]) return err(cudaErrorInvalidValue, "permute_expression_pair: leftover count mismatch");
    return ok();
}
