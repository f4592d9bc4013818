// Internal MSM interface shared by the C-ABI launchers and the batched /
// no-allocation entry points.
#pragma once
#include <cstdint>
#include "abi.cuh"
#include "curve.cuh"

namespace h2b {

struct MsmPlan {
    uint64_t n;
    int c;           // window bits
    int W;           // windows
    uint32_t H;      // buckets per window = 2^(c-1)
    uint64_t NB;     // W * H
    uint32_t K;      // sorted entries per accumulation chunk
    uint64_t nv;     // virtual (GLV half) scalars = 2n
    uint64_t max_entries;
    uint64_t max_chunks;
    uint32_t L;      // buckets per reduction segment
    int LOGL;        // log2(L)
    uint32_t S;      // segments per window
    int NBITS;       // log2(S)
    uint64_t max_dense;  // capacity of the dense-bucket list
    int R;               // pairing rounds before the XYZZ accumulation
    uint64_t cap[4];     // entry capacity after round r (cap[0] = max_entries)
    uint32_t Kf;         // entries per XYZZ accumulation chunk after the rounds
    uint64_t tn;         // points per window slice of a precomputed table (0: plain bases)
    int Wr;              // windows in the bucket reduction (W, or 1 with a table)
    uint32_t BP;         // CTAs per bit sum of the reduction (partials summed by a second kernel when > 1)
};

struct MsmScratch {
    G1Affine* bases_stage;
    Fr* scalar_stage;
    Fr* canon;
    uint32_t* counts;
    uint32_t* offsets;
    uint32_t* cursor;
    uint32_t* scan_tmp;
    uint32_t* sorted;
    G1Xyzz* buckets;
    G1Xyzz* heads;
    uint32_t* dense;
    G1Xyzz* pieces;
    G1Xyzz* segacc;
    G1Xyzz* segrun;
    G1Xyzz* bits;
    G1Xyzz* bitparts;    // per-part bit sums (BP > 1)
    G1Xyzz* wins;
    G1Jac* result;
    G1Affine* rbases;    // plain bases P_i, then phi(P_i), in the lazy x 2^261 form (no pairing rounds)
    G1Affine* pts[2];    // pairing-round outputs (ping-pong)
    uint32_t* roff[3];   // per-round bucket offsets (NB + 1 each)
    Fq* pr_pref;         // pairing rounds: per-job denominator prefixes
    uint2* pr_job;       // pairing rounds: per-job (input entry, output slot)
    uint32_t* pr_nj;     // pairing rounds: jobs per thread
    Fq* pr_tree;         // pairing rounds: per-CTA product trees
    Fq* pr_tot;          // pairing rounds: per-CTA totals (inverted in place)
    void* pr_inv_scratch;
    uint64_t pr_inv_bytes;
};

// Plan for an MSM that runs beside `concurrent` - 1 others (batches): same
// results; the accumulation's chunk size assumes the others share the SMs.
MsmPlan msm_plan_shared(uint64_t n, uint64_t tn, uint32_t concurrent);
MsmPlan msm_plan(uint64_t n);
// Plan for an MSM of n <= tn points over a precomputed window table built for
// tn points (window width chosen by tn; all windows share one bucket set).
MsmPlan msm_plan_table(uint64_t n, uint64_t tn);
void msm_plan_scratch(const MsmPlan& p, ScratchPlan& sp, bool scalar_host, bool bases_host);
MsmScratch msm_carve(const MsmPlan& p, ScratchArena& ar, bool scalar_host, bool bases_host);
RustError msm_run(const MsmPlan& p, const MsmScratch& s, const Fr* d_scalars, const G1Affine* d_bases,
                  cudaStream_t st);
// Merged runs: up to MSM_MERGE_MAX MSMs over one window table of tn points
// (n_total scalars in all) sorted, accumulated and reduced together, job j in
// bucket set j; each job's 96-byte result goes to outs[j].
constexpr uint32_t MSM_MERGE_MAX = 64;
MsmPlan msm_plan_merged(uint64_t n_total, uint64_t tn, uint32_t J);
RustError msm_run_merged(const MsmPlan& p, const MsmScratch& s, uint32_t J, const Fr* const* scalars,
                         const uint64_t* ns, const G1Affine* table, G1Jac* const* outs, cudaStream_t st);
void msm_set_tuning(int window_bits, int chunk);
void msm_set_pair_rounds(int rounds);

} // namespace h2b
