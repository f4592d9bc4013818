// Device-wide exclusive scan of uint32 counts (used for MSM bucket offsets
// and the permute-sort histograms).  Three launches: per-tile sums, one CTA
// scanning the tile sums, per-tile rescan with the tile offset.  out has
// n + 1 entries; out[n] is the total.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace h2b {

constexpr int SCAN_TILE = 2048;  // elements per CTA (256 threads x 8)

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
{
    const unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (unsigned)o) v += t;
    }
    return v;
}

// Exclusive scan across a 256-thread CTA; returns the CTA total in *total.
__device__ __forceinline__ uint32_t block_excl_scan_256(uint32_t v, uint32_t* total)
{
    __shared__ uint32_t warp_tot[8];
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = warp_incl_scan(v);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < 8 ? warp_tot[lane] : 0;
        uint32_t wi = warp_incl_scan(w);
        if (lane < 8) warp_tot[lane] = wi - w;
        if (lane == 7) *total = wi;
    }
    __syncthreads();
    uint32_t res = warp_tot[warp] + inc - v;
    __syncthreads();
    return res;
}

static __global__ void k_scan_tile_sums(const uint32_t* __restrict__ in, uint64_t n, uint32_t* __restrict__ tile_sums)
{
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    uint32_t s = 0;
    for (int j = 0; j < SCAN_TILE / 256; j++) {
        uint64_t i = base + j * 256 + threadIdx.x;
        if (i < n) s += in[i];
    }
    __shared__ uint32_t tot;
    block_excl_scan_256(s, &tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// One CTA of 256 threads: exclusive scan of tile_sums in place (any length).
static __global__ void k_scan_tile_sums_single(uint32_t* __restrict__ tile_sums, uint64_t ntiles)
{
    __shared__ uint32_t carry_s;
    __shared__ uint32_t tot;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    for (uint64_t base = 0; base < ntiles; base += 256) {
        uint64_t i = base + threadIdx.x;
        uint32_t v = i < ntiles ? tile_sums[i] : 0;
        uint32_t ex = block_excl_scan_256(v, &tot);
        uint32_t carry = carry_s;
        if (i < ntiles) tile_sums[i] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry_s = carry + tot;
        __syncthreads();
    }
}

static __global__ void k_scan_apply(const uint32_t* __restrict__ in, uint64_t n, const uint32_t* __restrict__ tile_offsets,
                             uint32_t* __restrict__ out, uint64_t ntiles)
{
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * (SCAN_TILE / 256);
    uint32_t v[SCAN_TILE / 256];
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_TILE / 256; j++) {
        uint64_t i = base + j;
        v[j] = i < n ? in[i] : 0;
        s += v[j];
    }
    __shared__ uint32_t tot;
    uint32_t ex = block_excl_scan_256(s, &tot) + tile_offsets[blockIdx.x];
#pragma unroll
    for (int j = 0; j < SCAN_TILE / 256; j++) {
        uint64_t i = base + j;
        if (i < n) out[i] = ex;
        ex += v[j];
    }
    if (blockIdx.x == ntiles - 1 && threadIdx.x == 255) out[n] = ex;
}

inline uint64_t scan_u32_tiles(uint64_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }

// out[0..n] = exclusive scan of in[0..n); tile_tmp needs scan_u32_tiles(n) words.
static inline cudaError_t scan_u32(const uint32_t* in, uint64_t n, uint32_t* out, uint32_t* tile_tmp, cudaStream_t st)
{
    uint64_t nt = scan_u32_tiles(n);
    if (nt == 0) {
        return cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
    }
    k_scan_tile_sums<<<(unsigned)nt, 256, 0, st>>>(in, n, tile_tmp);
    k_scan_tile_sums_single<<<1, 256, 0, st>>>(tile_tmp, nt);
    k_scan_apply<<<(unsigned)nt, 256, 0, st>>>(in, n, tile_tmp, out, nt);
    return cudaGetLastError();
}

} // namespace h2b
