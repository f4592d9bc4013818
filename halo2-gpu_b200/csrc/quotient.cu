// Quotient evaluator (evaluate_h) on the extended-domain parts.
//
//  * Gate expression graph: `_halo2_quotient`, `_halo2_quotient_device_columns`,
//    `_halo2_quotient_device_columns_device_out` (halo2_proofs/cuda/src/quotient.cu:
//    309-710; kernel semantics halo2_proofs/cuda/include/kernel/quotient.h:57-303;
//    rule encoding halo2_proofs/src/plonk/evaluation.rs:107-352).  Per row r of
//    [row_start, row_end): every 128-bit rule (C1*a + C2*b)*(D ? b : 1) is
//    evaluated in order, columns read at (r + rot*rot_scale) mod num_quotient,
//    then out = Horner(prev or 0, y, value-part rules).
//  * `_halo2_quotient_permutation` (permutation_quotient.cu:23-93; CPU semantics
//    halo2_proofs/src/cpu/evaluator.rs:63-148).
//  * `_halo2_quotient_lookups` (quotient_lookups.cu:16-53; CPU semantics
//    halo2_proofs/src/cpu/arithmetic.rs:223-280).
//
// B200 design of the gate evaluator: the rule list is compiled on the host
// once per call into a compact op table whose intermediates are assigned to a
// small set of reusable slots by liveness (most intermediates die at their
// first use), rotations are pre-multiplied by rot_scale and columns are read
// in place from the caller's buffers -- no transposed copy, no per-rule global
// intermediates.  Each thread walks whole rows; every thread of a warp
// executes the same op, so there is no divergence, and column reads for
// consecutive rows are coalesced.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>
#include "abi.cuh"
#include "field.cuh"
#include "prof.cuh"

namespace h2b {

enum : uint8_t { OP_ZERO = 0, OP_COPY = 1, OP_ADD = 2, OP_SUB = 3, OP_MUL = 4, OP_NEG = 5, OP_DBL = 6 };
enum : uint8_t { SRC_FIXED = 0, SRC_INSTANCE = 1, SRC_ADVICE = 2, SRC_SLOT = 3, SRC_CONST = 4, SRC_CHALLENGE = 5,
                 SRC_NONE = 6 };

struct QOp {              // 32 bytes
    uint8_t kind, sa, sb, pad;
    uint32_t dst;
    uint32_t ia, ib;      // column (global table index), slot, constant or challenge index
    uint64_t ra, rb;      // rotation offsets in [0, num_quotient)
};

struct QVp {
    uint32_t is_const, idx;
};

// Host compilation of the reference rule encoding.
struct QProgram {
    std::vector<QOp> ops;
    std::vector<QVp> vps;
    uint32_t slots = 0;
    std::string error;
};

static inline int decode_rot(uint64_t vs)
{
    uint64_t r = (vs >> 24) & 0xffff;
    int abs = (int)(r & 0x7fff);
    return (r >> 15) & 1 ? -abs : abs;
}

static QProgram compile_rules(const uint64_t* rules, uint64_t num_rules, const uint64_t* vp, uint64_t num_vp,
                              uint64_t num_fixed, uint64_t num_instance, uint64_t num_advice, uint64_t num_constants,
                              uint64_t num_challenges, uint64_t num_quotient, uint64_t rot_scale)
{
    QProgram P;
    const uint64_t nq = num_quotient;
    // last use of each intermediate (index of the last reading rule; num_rules = read by a vp)
    std::vector<int64_t> last(num_rules, -1);
    auto note = [&](uint64_t vs, int64_t user) {
        if ((vs & 0xf) == SRC_SLOT) {
            uint64_t idx = (vs >> 4) & 0xfffff;
            if (idx < num_rules) last[idx] = std::max(last[idx], user);
        }
    };
    for (uint64_t i = 0; i < num_rules; i++) {
        note(rules[2 * i], (int64_t)i);
        note(rules[2 * i + 1], (int64_t)i);
    }
    for (uint64_t i = 0; i < num_vp; i++) note(vp[i], (int64_t)num_rules);

    std::vector<uint32_t> slot_of(num_rules, 0);
    std::vector<uint32_t> free_slots;
    auto operand = [&](uint64_t vs, uint8_t& src, uint32_t& idx, uint64_t& rot) -> bool {
        uint64_t s = vs & 0xf, i = (vs >> 4) & 0xfffff;
        int r = decode_rot(vs);
        rot = 0;
        switch (s) {
        case SRC_FIXED:
            if (i >= num_fixed) return false;
            src = SRC_FIXED; idx = (uint32_t)i;
            break;
        case SRC_INSTANCE:
            if (i >= num_instance) return false;
            src = SRC_INSTANCE; idx = (uint32_t)(num_fixed + i);
            break;
        case SRC_ADVICE:
            if (i >= num_advice) return false;
            src = SRC_ADVICE; idx = (uint32_t)(num_fixed + num_instance + i);
            break;
        case SRC_SLOT:
            if (i >= num_rules) return false;
            src = SRC_SLOT; idx = slot_of[i];
            return true;
        case SRC_CONST:
            if (i >= num_constants) return false;
            src = SRC_CONST; idx = (uint32_t)i;
            return true;
        case SRC_CHALLENGE:
            if (i >= num_challenges) return false;
            src = SRC_CHALLENGE; idx = (uint32_t)i;
            return true;
        default:
            src = SRC_NONE; idx = 0;
            return true;
        }
        int64_t off = ((int64_t)r * (int64_t)rot_scale) % (int64_t)nq;
        if (off < 0) off += (int64_t)nq;
        rot = (uint64_t)off;
        return true;
    };
    for (uint64_t i = 0; i < num_rules; i++) {
        uint64_t lo = rules[2 * i], hi = rules[2 * i + 1];
        QOp op;
        memset(&op, 0, sizeof(op));
        bool ok_a = operand(lo, op.sa, op.ia, op.ra);
        bool ok_b = operand(hi, op.sb, op.ib, op.rb);
        int c1 = (int)((lo >> 40) & 0xf), d = (int)((lo >> 44) & 0xf), c2 = (int)((hi >> 40) & 0xf);
        uint8_t kind = OP_ZERO;
        if (c1 == 1) {
            if (c2 == 0) kind = (d == 1) ? OP_MUL : OP_COPY;
            else if (c2 == 1) kind = OP_ADD;
            else if (c2 == 2) kind = OP_SUB;
        } else if (c1 == 2) {
            kind = OP_NEG;
        } else if (c1 == 3) {
            kind = OP_DBL;
        }
        bool uses_b = kind == OP_ADD || kind == OP_SUB || kind == OP_MUL;
        bool uses_a = kind != OP_ZERO;
        if ((uses_a && !ok_a) || (uses_b && !ok_b) || (uses_a && op.sa == SRC_NONE) ||
            (uses_b && op.sb == SRC_NONE)) {
            P.error = "quotient rule references an out-of-range source";
            return P;
        }
        op.kind = kind;
        // operands are read before the destination is written, so slots whose
        // last reader is this rule can be reused for its result
        auto release = [&](uint64_t vs) {
            if ((vs & 0xf) == SRC_SLOT) {
                uint64_t j = (vs >> 4) & 0xfffff;
                if (j < num_rules && last[j] == (int64_t)i) {
                    last[j] = -2;  // released once
                    free_slots.push_back(slot_of[j]);
                }
            }
        };
        release(lo);
        if (((hi >> 4) & 0xfffff) != ((lo >> 4) & 0xfffff) || (hi & 0xf) != (lo & 0xf)) release(hi);
        uint32_t s;
        if (last[i] == -1) {
            // never read: still evaluated (matches the reference) into a scratch slot
            if (free_slots.empty()) free_slots.push_back(P.slots++);
            s = free_slots.back();
        } else if (!free_slots.empty()) {
            s = free_slots.back();
            free_slots.pop_back();
        } else {
            s = P.slots++;
        }
        slot_of[i] = s;
        op.dst = s;
        P.ops.push_back(op);
    }
    for (uint64_t i = 0; i < num_vp; i++) {
        uint64_t s = vp[i] & 0xf, idx = (vp[i] >> 4) & 0xfffff;
        QVp v;
        if (s == SRC_CONST) {
            if (idx >= num_constants) { P.error = "value-part rule constant out of range"; return P; }
            v.is_const = 1; v.idx = (uint32_t)idx;
        } else {
            if (idx >= num_rules) { P.error = "value-part rule intermediate out of range"; return P; }
            v.is_const = 0; v.idx = slot_of[idx];
        }
        P.vps.push_back(v);
    }
    if (P.slots == 0) P.slots = 1;
    return P;
}

template <int MAXS>
__global__ void __launch_bounds__(128) k_quotient(const QOp* __restrict__ ops, uint32_t n_ops,
                                                  const QVp* __restrict__ vps, uint32_t n_vp,
                                                  const Fr* const* __restrict__ cols, const Fr* __restrict__ consts,
                                                  const Fr* __restrict__ chal, const Fr* __restrict__ ypt,
                                                  const Fr* __restrict__ prev, Fr* __restrict__ out, uint64_t nq,
                                                  uint64_t row_start, uint64_t rows)
{
    const Fr y = ldg(ypt);
    Fr slot[MAXS];
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t row = row_start + r;
#pragma unroll 1
        for (uint32_t i = 0; i < n_ops; i++) {
            QOp op;
            {
                const uint4* p = reinterpret_cast<const uint4*>(&ops[i]);
                uint4 u0 = __ldg(p), u1 = __ldg(p + 1);
                memcpy(&op, &u0, 16);
                memcpy(reinterpret_cast<char*>(&op) + 16, &u1, 16);
            }
            auto fetch = [&](uint8_t src, uint32_t idx, uint64_t rot) -> Fr {
                switch (src) {
                case SRC_FIXED:
                case SRC_INSTANCE:
                case SRC_ADVICE: {
                    uint64_t at = row + rot;
                    if (at >= nq) at -= nq;
                    return ldg(&cols[idx][at]);
                }
                case SRC_SLOT: return slot[idx];
                case SRC_CONST: return ldg(&consts[idx]);
                case SRC_CHALLENGE: return ldg(&chal[idx]);
                default: return Fr::zero();
                }
            };
            Fr res;
            switch (op.kind) {
            case OP_COPY: res = fetch(op.sa, op.ia, op.ra); break;
            case OP_ADD: res = fetch(op.sa, op.ia, op.ra) + fetch(op.sb, op.ib, op.rb); break;
            case OP_SUB: res = fetch(op.sa, op.ia, op.ra) - fetch(op.sb, op.ib, op.rb); break;
            case OP_MUL: res = fetch(op.sa, op.ia, op.ra) * fetch(op.sb, op.ib, op.rb); break;
            case OP_NEG: res = fneg(fetch(op.sa, op.ia, op.ra)); break;
            case OP_DBL: res = fdbl(fetch(op.sa, op.ia, op.ra)); break;
            default: res = Fr::zero();
            }
            slot[op.dst] = res;
        }
        Fr val = prev ? ld(&prev[r]) : Fr::zero();
#pragma unroll 1
        for (uint32_t i = 0; i < n_vp; i++) {
            uint2 v = __ldg(reinterpret_cast<const uint2*>(&vps[i]));
            Fr part = v.x ? ldg(&consts[v.y]) : slot[v.y];
            val = val * y + part;
        }
        st(&out[r], val);
    }
}

// Scratch layout: ops, vps, column pointer table, constants, challenges,
// expr constants, optional staged host columns, optional output staging.
struct QLayout {
    uint64_t n_cols, rows;
};

static uint64_t quotient_ws(uint64_t num_rules, uint64_t num_vp, uint64_t ncols, uint64_t num_constants,
                            uint64_t num_challenges, uint64_t rows, uint64_t stage_cols_len, bool stage_out)
{
    ScratchPlan p;
    p.add(std::max<uint64_t>(num_rules, 1) * sizeof(QOp));
    p.add(std::max<uint64_t>(num_vp, 1) * sizeof(QVp));
    p.add(std::max<uint64_t>(ncols, 1) * sizeof(void*));
    p.add(std::max<uint64_t>(num_constants, 1) * 32);
    p.add(std::max<uint64_t>(num_challenges, 1) * 32);
    p.add(5 * 32);
    if (stage_cols_len) p.add(ncols * stage_cols_len * 32);
    if (stage_out) p.add(rows * 32);
    return p.used;
}

struct QArgs {
    const void* const* fixed; uint64_t num_fixed;
    const void* const* instance; uint64_t num_instance;
    const void* const* advice; uint64_t num_advice;
    bool cols_host;
    const void* challenges; uint64_t num_challenges;
    const void* constants; uint64_t num_constants;
    const void* expr_constants;
    const uint64_t* rules; uint64_t num_rules;
    const uint64_t* vp; uint64_t num_vp;
    void* out; bool out_host;
    uint64_t num_quotient;
    const void* prev;
    uint64_t rot_scale, row_start, row_end;
    void* scratch; uint64_t scratch_bytes;
    cudaStream_t st;
};

static RustError quotient_run(const QArgs& a, const char* who)
{
    if (a.row_end < a.row_start || a.row_end > a.num_quotient)
        return err(cudaErrorInvalidValue, "quotient: row range outside [0, num_quotient]");
    const uint64_t rows = a.row_end - a.row_start;
    const uint64_t ncols = a.num_fixed + a.num_instance + a.num_advice;
    if (a.num_quotient == 0 || rows == 0) return ok();
    QProgram P = compile_rules(a.rules, a.num_rules, a.vp, a.num_vp, a.num_fixed, a.num_instance, a.num_advice,
                               a.num_constants, a.num_challenges, a.num_quotient, a.rot_scale);
    if (!P.error.empty()) return err(cudaErrorInvalidValue, P.error.c_str());
    if (P.slots > 512) return err(cudaErrorInvalidValue, "quotient: more than 512 live intermediates");
    uint64_t need = quotient_ws(a.num_rules, a.num_vp, ncols, a.num_constants, a.num_challenges, rows,
                                a.cols_host ? a.num_quotient : 0, a.out_host);
    if (a.scratch_bytes < need) return scratch_too_small(who, a.scratch_bytes, need);
    ScratchArena ar(a.scratch, a.scratch_bytes);
    QOp* d_ops = (QOp*)ar.take(std::max<uint64_t>(a.num_rules, 1) * sizeof(QOp));
    QVp* d_vps = (QVp*)ar.take(std::max<uint64_t>(a.num_vp, 1) * sizeof(QVp));
    const Fr** d_cols = (const Fr**)ar.take(std::max<uint64_t>(ncols, 1) * sizeof(void*));
    Fr* d_consts = (Fr*)ar.take(std::max<uint64_t>(a.num_constants, 1) * 32);
    Fr* d_chal = (Fr*)ar.take(std::max<uint64_t>(a.num_challenges, 1) * 32);
    Fr* d_expr = (Fr*)ar.take(5 * 32);
    Fr* d_stage = a.cols_host ? (Fr*)ar.take(ncols * a.num_quotient * 32) : nullptr;
    Fr* d_out = a.out_host ? (Fr*)ar.take(rows * 32) : (Fr*)a.out;

    std::vector<const Fr*> colptr(std::max<uint64_t>(ncols, 1), nullptr);
    uint64_t c = 0;
    auto add_cols = [&](const void* const* p, uint64_t n) -> RustError {
        for (uint64_t i = 0; i < n; i++, c++) {
            if (a.cols_host) {
                Fr* dst = d_stage + c * a.num_quotient;
                H2B_CUDA(cudaMemcpyAsync(dst, p[i], a.num_quotient * 32, cudaMemcpyHostToDevice, a.st));
                colptr[c] = dst;
            } else {
                colptr[c] = (const Fr*)p[i];
            }
        }
        return ok();
    };
    H2B_TRY(add_cols(a.fixed, a.num_fixed));
    H2B_TRY(add_cols(a.instance, a.num_instance));
    H2B_TRY(add_cols(a.advice, a.num_advice));
    if (!P.ops.empty()) H2B_CUDA(cudaMemcpyAsync(d_ops, P.ops.data(), P.ops.size() * sizeof(QOp), cudaMemcpyHostToDevice, a.st));
    if (!P.vps.empty()) H2B_CUDA(cudaMemcpyAsync(d_vps, P.vps.data(), P.vps.size() * sizeof(QVp), cudaMemcpyHostToDevice, a.st));
    H2B_CUDA(cudaMemcpyAsync(d_cols, colptr.data(), colptr.size() * sizeof(void*), cudaMemcpyHostToDevice, a.st));
    if (a.num_constants)
        H2B_CUDA(cudaMemcpyAsync(d_consts, a.constants, a.num_constants * 32, cudaMemcpyHostToDevice, a.st));
    if (a.num_challenges)
        H2B_CUDA(cudaMemcpyAsync(d_chal, a.challenges, a.num_challenges * 32, cudaMemcpyHostToDevice, a.st));
    H2B_CUDA(cudaMemcpyAsync(d_expr, a.expr_constants, 5 * 32, cudaMemcpyHostToDevice, a.st));

    unsigned grid = grid_for(rows, 128, 148u * 16u);
    prof_begin(PROF_QUOTIENT, a.st);
#define H2B_QLAUNCH(S)                                                                                         \
    k_quotient<S><<<grid, 128, 0, a.st>>>(d_ops, (uint32_t)P.ops.size(), d_vps, (uint32_t)P.vps.size(), d_cols, \
                                          d_consts, d_chal, d_expr + 4, (const Fr*)a.prev, d_out, a.num_quotient, \
                                          a.row_start, rows)
    if (P.slots <= 16) H2B_QLAUNCH(16);
    else if (P.slots <= 64) H2B_QLAUNCH(64);
    else H2B_QLAUNCH(512);
#undef H2B_QLAUNCH
    prof_end(PROF_QUOTIENT, a.st);
    H2B_LAUNCHED("k_quotient");
    if (a.out_host) {
        H2B_CUDA(cudaMemcpyAsync(a.out, d_out, rows * 32, cudaMemcpyDeviceToHost, a.st));
        H2B_CUDA(cudaStreamSynchronize(a.st));
    }
    return ok();
}

// ---------------------------------------------------------------------------
// permutation and lookup constraint kernels
// ---------------------------------------------------------------------------

constexpr int PQ_CHUNK = 8;
struct PermScalars {
    Fr beta, gamma, y, delta, delta_start, ext_omega, omega;
};

__device__ __forceinline__ uint64_t rot_index(uint64_t idx, int rot, int scale, int isize)
{
    int64_t r = ((int64_t)idx + (int64_t)rot * scale) % isize;
    if (r < 0) r += isize;
    return (uint64_t)r;
}

__device__ __forceinline__ Fr fpow_u64(Fr b, uint64_t e)
{
    Fr r = Fr::one();
    while (e) {
        if (e & 1) r = r * b;
        b = b * b;
        e >>= 1;
    }
    return r;
}

__global__ void __launch_bounds__(128) k_perm_quotient(Fr* __restrict__ values, const Fr* __restrict__ l0,
                                                       const Fr* __restrict__ l_last, const Fr* __restrict__ l_active,
                                                       const Fr* const* __restrict__ prods,
                                                       const Fr* const* __restrict__ perms,
                                                       const Fr* const* __restrict__ cols, PermScalars sc,
                                                       uint64_t n_sets, uint64_t chunk_len, uint64_t n_cols,
                                                       int last_rotation, int rot_scale, int isize, uint64_t n)
{
    const Fr one = Fr::one();
    uint64_t nthreads = (n + PQ_CHUNK - 1) / PQ_CHUNK;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nthreads;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i0 = t * PQ_CHUNK;
        Fr beta_term = sc.ext_omega * fpow_u64(sc.omega, i0);
        for (int j = 0; j < PQ_CHUNK && i0 + j < n; j++) {
            uint64_t idx = i0 + j;
            uint64_t r_next = rot_index(idx, 1, rot_scale, isize);
            uint64_t r_last = rot_index(idx, last_rotation, rot_scale, isize);
            Fr l0v = ld(&l0[idx]);
            Fr v = ld(&values[idx]);
            Fr z0 = ld(&prods[0][idx]);
            v = v * sc.y + (one - z0) * l0v;
            Fr zl = ld(&prods[n_sets - 1][idx]);
            v = v * sc.y + (zl * zl - zl) * ld(&l_last[idx]);
            for (uint64_t s = 1; s < n_sets; s++)
                v = v * sc.y + (ld(&prods[s][idx]) - ld(&prods[s - 1][r_last])) * l0v;
            Fr la = ld(&l_active[idx]);
            Fr cur_delta = sc.delta_start * beta_term;
            for (uint64_t s = 0; s < n_sets; s++) {
                uint64_t c0 = s * chunk_len, c1 = c0 + chunk_len < n_cols ? c0 + chunk_len : n_cols;
                Fr left = ld(&prods[s][r_next]);
                Fr right = ld(&prods[s][idx]);
                for (uint64_t c = c0; c < c1; c++) {
                    Fr cv = ld(&cols[c][idx]);
                    left = left * (cv + sc.beta * ld(&perms[c][idx]) + sc.gamma);
                    right = right * (cv + cur_delta + sc.gamma);
                    cur_delta = cur_delta * sc.delta;
                }
                v = v * sc.y + (left - right) * la;
            }
            st(&values[idx], v);
            beta_term = beta_term * sc.omega;
        }
    }
}

__global__ void __launch_bounds__(128) k_lookup_quotient(Fr* __restrict__ values, const Fr* __restrict__ table,
                                                         const Fr* __restrict__ z, const Fr* __restrict__ pin,
                                                         const Fr* __restrict__ ptab, const Fr* __restrict__ l0,
                                                         const Fr* __restrict__ l_last,
                                                         const Fr* __restrict__ l_active, const Fr* __restrict__ pbeta,
                                                         const Fr* __restrict__ pgamma, const Fr* __restrict__ py,
                                                         uint64_t n)
{
    const Fr one = Fr::one(), beta = ld(pbeta), gamma = ld(pgamma), y = ld(py);
    for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < n;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t nx = idx + 1 == n ? 0 : idx + 1;
        uint64_t pv = idx == 0 ? n - 1 : idx - 1;
        Fr zi = ld(&z[idx]), a = ld(&pin[idx]), s = ld(&ptab[idx]);
        Fr l0v = ld(&l0[idx]), la = ld(&l_active[idx]);
        Fr ams = a - s;
        Fr v = ld(&values[idx]);
        v = v * y + (one - zi) * l0v;
        v = v * y + (zi * zi - zi) * ld(&l_last[idx]);
        v = v * y + (ld(&z[nx]) * (a + beta) * (s + gamma) - zi * ld(&table[idx])) * la;
        v = v * y + ams * l0v;
        v = v * y + ams * (a - ld(&pin[pv])) * la;
        st(&values[idx], v);
    }
}

} // namespace h2b

using namespace h2b;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" uint64_t _halo2_quotient_workspace_size(const uint64_t* rules, uint64_t num_rules, uint64_t num_vp_rules,
                                                   uint64_t num_quotient, uint64_t num_fixed, uint64_t num_instance,
                                                   uint64_t num_advice, uint64_t num_challenges,
                                                   uint64_t num_constants, uint64_t rotation_scale,
                                                   uint64_t row_start, uint64_t row_end)
{
    (void)rules;
    (void)rotation_scale;
    uint64_t rows = row_end > row_start ? row_end - row_start : 0;
    uint64_t ncols = num_fixed + num_instance + num_advice;
    // Covers the host-column variant (staged columns + output); the device
    // variants use a prefix of the same layout.
    return quotient_ws(num_rules, num_vp_rules, ncols, num_constants, num_challenges, rows, num_quotient, true);
}

// The reference's rule decoder hook (quotient.cu:334-345): it decodes the
// rotation range of every value source for the row window and returns
// nothing, and no caller reads a result.  Kept for link compatibility; it
// walks the same encoding and has no effect.
extern "C" void _halo2_quotient_decode(uint64_t* rules, uint64_t num_rules, uint64_t num_quotient,
                                       uint64_t rotation_scale, uint64_t row_start, uint64_t row_end)
{
    (void)num_quotient; (void)row_start; (void)row_end;
    int64_t lo = 0, hi = 0;
    for (uint64_t i = 0; rules && i < 2 * num_rules; i++) {
        int64_t r = (int64_t)decode_rot(rules[i]) * (int64_t)rotation_scale;
        lo = std::min(lo, r);
        hi = std::max(hi, r);
    }
    (void)lo; (void)hi;
}

extern "C" uint64_t _halo2_evaluate_h_max_rows(const uint64_t* rules, uint64_t num_rules, uint64_t num_vp_rules,
                                               uint64_t num_quotient, uint64_t num_fixed, uint64_t num_instance,
                                               uint64_t num_advice, uint64_t num_challenges, uint64_t num_constants,
                                               uint64_t rotation_scale, uint64_t row_start, uint64_t row_end,
                                               uint64_t free_bytes)
{
    for (uint64_t rows = row_end > row_start ? row_end - row_start : 0; rows > 0; rows >>= 1) {
        if (_halo2_quotient_workspace_size(rules, num_rules, num_vp_rules, num_quotient, num_fixed, num_instance,
                                           num_advice, num_challenges, num_constants, rotation_scale, row_start,
                                           row_start + rows) < free_bytes)
            return rows;
    }
    return 0;
}

extern "C" RustError _halo2_quotient(const FFITraitObject* fixed, uint64_t num_fixed, const FFITraitObject* instance,
                                     uint64_t num_instance, const FFITraitObject* advices, uint64_t num_advice,
                                     FFITraitObject challenges, uint64_t num_challenges, FFITraitObject constants,
                                     uint64_t num_constants, FFITraitObject expr_constants, const uint64_t* rules,
                                     uint64_t num_rules, const uint64_t* value_part_rules, uint64_t num_vp_rules,
                                     FFITraitObject quotient_poly, uint64_t num_quotient, uint64_t rotation_scale,
                                     uint64_t row_start, uint64_t row_end, void* scratch, uint64_t scratch_bytes,
                                     cudaStream_t stream)
{
    std::vector<const void*> f(num_fixed), in(num_instance), adv(num_advice);
    for (uint64_t i = 0; i < num_fixed; i++) f[i] = fixed[i].ptr;
    for (uint64_t i = 0; i < num_instance; i++) in[i] = instance[i].ptr;
    for (uint64_t i = 0; i < num_advice; i++) adv[i] = advices[i].ptr;
    QArgs a{f.data(), num_fixed, in.data(), num_instance, adv.data(), num_advice, true,
            challenges.ptr, num_challenges, constants.ptr, num_constants, expr_constants.ptr,
            rules, num_rules, value_part_rules, num_vp_rules, quotient_poly.ptr, true, num_quotient, nullptr,
            rotation_scale, row_start, row_end, scratch, scratch_bytes, stream};
    return quotient_run(a, "_halo2_quotient");
}

extern "C" RustError _halo2_quotient_device_columns(
    const void* const* fixed_d_ptrs, uint64_t num_fixed, const void* const* instance_d_ptrs, uint64_t num_instance,
    const void* const* advice_d_ptrs, uint64_t num_advice, FFITraitObject challenges, uint64_t num_challenges,
    FFITraitObject constants, uint64_t num_constants, FFITraitObject expr_constants, const uint64_t* rules,
    uint64_t num_rules, const uint64_t* value_part_rules, uint64_t num_vp_rules, FFITraitObject quotient_poly,
    uint64_t num_quotient, uint64_t rotation_scale, uint64_t row_start, uint64_t row_end, void* scratch,
    uint64_t scratch_bytes, cudaStream_t stream)
{
    QArgs a{fixed_d_ptrs, num_fixed, instance_d_ptrs, num_instance, advice_d_ptrs, num_advice, false,
            challenges.ptr, num_challenges, constants.ptr, num_constants, expr_constants.ptr,
            rules, num_rules, value_part_rules, num_vp_rules, quotient_poly.ptr, true, num_quotient, nullptr,
            rotation_scale, row_start, row_end, scratch, scratch_bytes, stream};
    return quotient_run(a, "_halo2_quotient_device_columns");
}

extern "C" RustError _halo2_quotient_device_columns_device_out(
    const void* const* fixed_d_ptrs, uint64_t num_fixed, const void* const* instance_d_ptrs, uint64_t num_instance,
    const void* const* advice_d_ptrs, uint64_t num_advice, FFITraitObject challenges, uint64_t num_challenges,
    FFITraitObject constants, uint64_t num_constants, FFITraitObject expr_constants, const uint64_t* rules,
    uint64_t num_rules, const uint64_t* value_part_rules, uint64_t num_vp_rules, void* quotient_poly_device_ptr,
    uint64_t num_quotient, const void* prev_values_device_ptr, uint64_t rotation_scale, uint64_t row_start,
    uint64_t row_end, void* scratch, uint64_t scratch_bytes, cudaStream_t stream)
{
    QArgs a{fixed_d_ptrs, num_fixed, instance_d_ptrs, num_instance, advice_d_ptrs, num_advice, false,
            challenges.ptr, num_challenges, constants.ptr, num_constants, expr_constants.ptr,
            rules, num_rules, value_part_rules, num_vp_rules, quotient_poly_device_ptr, false, num_quotient,
            prev_values_device_ptr, rotation_scale, row_start, row_end, scratch, scratch_bytes, stream};
    return quotient_run(a, "_halo2_quotient_device_columns_device_out");
}

// ---------------------------------------------------------------------------
// Resident quotient programs (no counterpart in the reference, which compiles
// and uploads its rule list, constants and column table on every call): the
// program is compiled and uploaded once into caller-owned device memory,
// bound to its column buffers, and each run is a kernel launch alone -- no
// host copy, no synchronisation -- so runs can be captured in a CUDA graph
// and issued from many streams at once.
// ---------------------------------------------------------------------------

extern "C" {
typedef struct h2b_quotient_program {
    uint32_t n_ops, n_vp, slots, reserved;
    uint64_t num_quotient;
    uint64_t off_vps, off_cols, off_consts, off_chal, off_y, bytes;
} h2b_quotient_program;
}

static void qprog_layout(uint64_t num_rules, uint64_t num_vp, uint64_t ncols, uint64_t num_constants,
                         uint64_t num_challenges, h2b_quotient_program& L)
{
    ScratchPlan p;
    p.add(std::max<uint64_t>(num_rules, 1) * sizeof(QOp));
    L.off_vps = align_up(p.used);
    p.add(std::max<uint64_t>(num_vp, 1) * sizeof(QVp));
    L.off_cols = align_up(p.used);
    p.add(std::max<uint64_t>(ncols, 1) * sizeof(void*));
    L.off_consts = align_up(p.used);
    p.add(std::max<uint64_t>(num_constants, 1) * 32);
    L.off_chal = align_up(p.used);
    p.add(std::max<uint64_t>(num_challenges, 1) * 32);
    L.off_y = align_up(p.used);
    p.add(32);
    L.bytes = p.used;
}

extern "C" uint64_t h2b_quotient_program_size(uint64_t num_rules, uint64_t num_vp, uint64_t num_columns,
                                              uint64_t num_constants, uint64_t num_challenges)
{
    h2b_quotient_program L;
    qprog_layout(num_rules, num_vp, num_columns, num_constants, num_challenges, L);
    return L.bytes;
}

extern "C" RustError h2b_quotient_program_build(const uint64_t* rules, uint64_t num_rules, const uint64_t* value_part_rules,
                                               uint64_t num_vp, uint64_t num_fixed, uint64_t num_instance,
                                               uint64_t num_advice, const void* const* d_columns,
                                               const void* constants, uint64_t num_constants, const void* challenges,
                                               uint64_t num_challenges, const void* y, uint64_t num_quotient,
                                               uint64_t rotation_scale, void* d_program, uint64_t program_bytes,
                                               h2b_quotient_program* info, cudaStream_t stream)
{
    if (!info) return err(cudaErrorInvalidValue, "h2b_quotient_program_build: info is null");
    if (num_quotient == 0) return err(cudaErrorInvalidValue, "h2b_quotient_program_build: num_quotient is 0");
    const uint64_t ncols = num_fixed + num_instance + num_advice;
    QProgram P = compile_rules(rules, num_rules, value_part_rules, num_vp, num_fixed, num_instance, num_advice,
                               num_constants, num_challenges, num_quotient, rotation_scale);
    if (!P.error.empty()) return err(cudaErrorInvalidValue, P.error.c_str());
    if (P.slots > 512) return err(cudaErrorInvalidValue, "quotient: more than 512 live intermediates");
    h2b_quotient_program L;
    memset(&L, 0, sizeof(L));
    qprog_layout(num_rules, num_vp, ncols, num_constants, num_challenges, L);
    if (program_bytes < L.bytes) return scratch_too_small("h2b_quotient_program_build", program_bytes, L.bytes);
    L.n_ops = (uint32_t)P.ops.size();
    L.n_vp = (uint32_t)P.vps.size();
    L.slots = P.slots;
    L.num_quotient = num_quotient;
    char* base = (char*)d_program;
    if (!P.ops.empty())
        H2B_CUDA(cudaMemcpyAsync(base, P.ops.data(), P.ops.size() * sizeof(QOp), cudaMemcpyHostToDevice, stream));
    if (!P.vps.empty())
        H2B_CUDA(cudaMemcpyAsync(base + L.off_vps, P.vps.data(), P.vps.size() * sizeof(QVp), cudaMemcpyHostToDevice,
                                 stream));
    if (ncols)
        H2B_CUDA(cudaMemcpyAsync(base + L.off_cols, d_columns, ncols * sizeof(void*), cudaMemcpyHostToDevice, stream));
    if (num_constants)
        H2B_CUDA(cudaMemcpyAsync(base + L.off_consts, constants, num_constants * 32, cudaMemcpyHostToDevice, stream));
    if (num_challenges)
        H2B_CUDA(cudaMemcpyAsync(base + L.off_chal, challenges, num_challenges * 32, cudaMemcpyHostToDevice, stream));
    H2B_CUDA(cudaMemcpyAsync(base + L.off_y, y, 32, cudaMemcpyHostToDevice, stream));
    // the host sources are pageable and go out of scope: the copies must have read them
    H2B_CUDA(cudaStreamSynchronize(stream));
    *info = L;
    return ok();
}

extern "C" RustError h2b_quotient_program_run(const h2b_quotient_program* info, const void* d_program, void* d_out,
                                             const void* d_prev, uint64_t row_start, uint64_t row_end,
                                             cudaStream_t stream)
{
    if (!info) return err(cudaErrorInvalidValue, "h2b_quotient_program_run: info is null");
    const h2b_quotient_program& L = *info;
    if (row_end < row_start || row_end > L.num_quotient)
        return err(cudaErrorInvalidValue, "quotient: row range outside [0, num_quotient]");
    const uint64_t rows = row_end - row_start;
    if (rows == 0) return ok();
    const char* base = (const char*)d_program;
    const QOp* ops = (const QOp*)base;
    const QVp* vps = (const QVp*)(base + L.off_vps);
    const Fr* const* cols = (const Fr* const*)(base + L.off_cols);
    const Fr* consts = (const Fr*)(base + L.off_consts);
    const Fr* chal = (const Fr*)(base + L.off_chal);
    const Fr* yp = (const Fr*)(base + L.off_y);
    unsigned grid = grid_for(rows, 128, 148u * 16u);
#define H2B_QPLAUNCH(S)                                                                                           \
    k_quotient<S><<<grid, 128, 0, stream>>>(ops, L.n_ops, vps, L.n_vp, cols, consts, chal, yp, (const Fr*)d_prev, \
                                            (Fr*)d_out, L.num_quotient, row_start, rows)
    if (L.slots <= 16) H2B_QPLAUNCH(16);
    else if (L.slots <= 64) H2B_QPLAUNCH(64);
    else H2B_QPLAUNCH(512);
#undef H2B_QPLAUNCH
    H2B_LAUNCHED("k_quotient");
    return ok();
}

extern "C" RustError _halo2_quotient_lookups(void* values, const void* table_values, const void* product_coset,
                                             const void* permuted_input_coset, const void* permuted_table_coset,
                                             const void* l0, const void* l_last, const void* l_active_row,
                                             const void* beta, const void* gamma, const void* y, uint64_t poly_length,
                                             cudaStream_t stream)
{
    if (poly_length == 0) return ok();
    k_lookup_quotient<<<grid_for(poly_length, 128, 148u * 16u), 128, 0, stream>>>(
        (Fr*)values, (const Fr*)table_values, (const Fr*)product_coset, (const Fr*)permuted_input_coset,
        (const Fr*)permuted_table_coset, (const Fr*)l0, (const Fr*)l_last, (const Fr*)l_active_row, (const Fr*)beta,
        (const Fr*)gamma, (const Fr*)y, poly_length);
    H2B_LAUNCHED("k_lookup_quotient");
    return ok();
}

extern "C" RustError _halo2_quotient_permutation(void* values, const void* l0, const void* l_last,
                                                 const void* l_active_row, const void* perm_prod_cosets,
                                                 const void* perm_cosets, const void* column_values, const void* beta,
                                                 const void* gamma, const void* y, const void* delta,
                                                 const void* delta_start, const void* current_extended_omega,
                                                 const void* omega, uint64_t n_sets, uint64_t chunk_len,
                                                 uint64_t n_perm_cols, int32_t last_rotation, int32_t rot_scale,
                                                 int32_t isize_, uint64_t poly_length, cudaStream_t stream)
{
    if (n_sets == 0 || poly_length == 0) return ok();
    if (isize_ <= 0) return err(cudaErrorInvalidValue, "_halo2_quotient_permutation: isize must be positive");
    if (n_perm_cols > n_sets * chunk_len)
        return err(cudaErrorInvalidValue, "_halo2_quotient_permutation: more columns than sets * chunk_len");
    PermScalars sc;
    memcpy(&sc.beta, beta, 32);
    memcpy(&sc.gamma, gamma, 32);
    memcpy(&sc.y, y, 32);
    memcpy(&sc.delta, delta, 32);
    memcpy(&sc.delta_start, delta_start, 32);
    memcpy(&sc.ext_omega, current_extended_omega, 32);
    memcpy(&sc.omega, omega, 32);
    uint64_t nthreads = (poly_length + PQ_CHUNK - 1) / PQ_CHUNK;
    k_perm_quotient<<<grid_for(nthreads, 128, 148u * 16u), 128, 0, stream>>>(
        (Fr*)values, (const Fr*)l0, (const Fr*)l_last, (const Fr*)l_active_row, (const Fr* const*)perm_prod_cosets,
        (const Fr* const*)perm_cosets, (const Fr* const*)column_values, sc, n_sets, chunk_len, n_perm_cols,
        last_rotation, rot_scale, isize_, poly_length);
    H2B_LAUNCHED("k_perm_quotient");
    return ok();
}

// ---------------------------------------------------------------------------
// Fused extended-part quotient (no counterpart in the reference, whose
// evaluate_h runs one launcher per constraint family on each extended part:
// halo2_proofs/src/plonk/evaluation.rs:1107-1417 calls
// `_halo2_quotient_device_columns_device_out` for the gates,
// `_halo2_quotient_permutation`, and per lookup the product expression
// through `_halo2_quotient_device_columns_device_out` into `table_values`
// followed by `_halo2_quotient_lookups`).  One kernel does all of it per row:
//   value = Horner(0, y, gate value parts)
//   value = permutation constraints folded in (as _halo2_quotient_permutation)
//   per lookup: tv = Horner(0, y, its product expression's value parts),
//               value = its five constraints folded in (as _halo2_quotient_lookups)
//   out[(row - row_start) * out_stride + out_offset] = value (* scale)
// so the accumulator is written once, table_values never exist, and with
// out_stride = number of parts, out_offset = the part and scale = the part's
// 1 / (X^n - 1) value the parts land interleaved in the extended array,
// already divided by the vanishing polynomial
// (`_halo2_extended_from_lagrange_vec_device` + `_halo2_divide_by_vanishing_poly`).
// The whole program -- ops, constants, challenges, column pointers, scalars --
// is one __grid_constant__ kernel parameter block: no device program memory,
// no host synchronisation, capturable in a graph, and every op is a
// warp-uniform constant-bank read.
// ---------------------------------------------------------------------------

namespace h2b {

constexpr int FQ_MAX_OPS = 256, FQ_MAX_VPS = 64, FQ_MAX_CONSTS = 192, FQ_MAX_CHAL = 16, FQ_MAX_COLS = 64,
              FQ_MAX_SETS = 8, FQ_MAX_PCOLS = 32, FQ_MAX_LOOKUPS = 8;
constexpr unsigned FQ_THREADS = 128;

struct FqLookup {
    const Fr* z;
    const Fr* pin;
    const Fr* ptab;
    Fr beta, gamma;
    uint32_t op0, op1, vp0, vp1;
};

struct FusedParams {
    QOp ops[FQ_MAX_OPS];
    QVp vps[FQ_MAX_VPS];
    Fr consts[FQ_MAX_CONSTS];
    Fr chal[FQ_MAX_CHAL];
    const Fr* cols[FQ_MAX_COLS];
    const Fr* prods[FQ_MAX_SETS];
    const Fr* sigmas[FQ_MAX_PCOLS];
    const Fr* pcols[FQ_MAX_PCOLS];
    FqLookup lk[FQ_MAX_LOOKUPS];
    const Fr* l0;
    const Fr* l_last;
    const Fr* l_active;
    Fr* out;
    Fr y, beta, gamma, delta, delta_start, ext_omega, omega, scale;
    uint64_t nq, isize, off_next, off_last, out_stride, out_offset;
    uint32_t gate_ops, gate_vps, n_sets, chunk_len, n_pcols, n_lookups, has_scale, pad;
};

// The fused pass keeps its intermediates in [0, 2p): products without their
// closing subtraction, sums and differences corrected by 2p, the row's value
// made canonical once before the store (field.cuh, residues in [0, 2p)).
// Columns, constants and scalars enter canonical.
__device__ __forceinline__ Fr zm(const Fr& a, const Fr& b) { return mont_mul_lazy_outline<FrCfg>(a, b); }
__device__ __forceinline__ Fr za(const Fr& a, const Fr& b) { return add2p<FrCfg>(a, b); }
__device__ __forceinline__ Fr zs(const Fr& a, const Fr& b) { return sub2p<FrCfg>(a, b); }

__device__ __forceinline__ Fr fq_fetch(const FusedParams& P, const Fr* slot, uint8_t src, uint32_t idx, uint64_t rot,
                                       uint64_t row)
{
    switch (src) {
    case SRC_FIXED:
    case SRC_INSTANCE:
    case SRC_ADVICE: {
        uint64_t at = row + rot;
        if (at >= P.nq) at -= P.nq;
        return ldg(&P.cols[idx][at]);
    }
    case SRC_SLOT: return slot[idx];
    case SRC_CONST: return P.consts[idx];
    case SRC_CHALLENGE: return P.chal[idx];
    default: return Fr::zero();
    }
}

// ops [i0, i1) of the program on one row, then Horner(0, y, value parts [v0, v1))
__device__ __forceinline__ Fr fq_run(const FusedParams& P, Fr* slot, uint32_t i0, uint32_t i1, uint32_t v0,
                                     uint32_t v1, uint64_t row)
{
#pragma unroll 1
    for (uint32_t i = i0; i < i1; i++) {
        const QOp& op = P.ops[i];
        const uint8_t kind = op.kind;
        Fr res;
        switch (kind) {
        case OP_COPY: res = fq_fetch(P, slot, op.sa, op.ia, op.ra, row); break;
        case OP_ADD: res = za(fq_fetch(P, slot, op.sa, op.ia, op.ra, row), fq_fetch(P, slot, op.sb, op.ib, op.rb, row)); break;
        case OP_SUB: res = zs(fq_fetch(P, slot, op.sa, op.ia, op.ra, row), fq_fetch(P, slot, op.sb, op.ib, op.rb, row)); break;
        case OP_MUL: res = zm(fq_fetch(P, slot, op.sa, op.ia, op.ra, row), fq_fetch(P, slot, op.sb, op.ib, op.rb, row)); break;
        case OP_NEG: res = zs(Fr::zero(), fq_fetch(P, slot, op.sa, op.ia, op.ra, row)); break;
        case OP_DBL: { const Fr x = fq_fetch(P, slot, op.sa, op.ia, op.ra, row); res = za(x, x); } break;
        default: res = Fr::zero();
        }
        slot[op.dst] = res;
    }
    Fr val = Fr::zero();
#pragma unroll 1
    for (uint32_t i = v0; i < v1; i++) {
        const QVp v = P.vps[i];
        val = za(zm(val, P.y), v.is_const ? P.consts[v.idx] : slot[v.idx]);
    }
    return val;
}

template <int MAXS, int MINB>
__global__ void __launch_bounds__(FQ_THREADS, MINB) k_quotient_fused(const __grid_constant__ FusedParams P,
                                                                     uint64_t row_start, uint64_t rows)
{
    Fr slot[MAXS];
    const Fr one = Fr::one();
    const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
    // omega^step, the factor between a thread's consecutive rows, once per block
    __shared__ Fr s_wstep;
    if (P.n_sets && threadIdx.x == 0) s_wstep = fpow_u64(P.omega, step);
    __syncthreads();
    const Fr wstep = P.n_sets ? s_wstep : one;
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    // X-dependent factor of the identity permutation on this thread's first
    // row, ext_omega * omega^row
    Fr bt = P.n_sets ? P.ext_omega * fpow_u64(P.omega, row_start + r) : one;   // canonical
    for (; r < rows; r += step) {
        const uint64_t row = row_start + r;
        Fr v = fq_run(P, slot, 0, P.gate_ops, 0, P.gate_vps, row);
        if (P.n_sets) {
            uint64_t rn = row + P.off_next, rl = row + P.off_last;
            if (rn >= P.isize) rn -= P.isize;
            if (rl >= P.isize) rl -= P.isize;
            const Fr l0v = ld(&P.l0[row]);
            const Fr z0 = ld(&P.prods[0][row]);
            v = za(zm(v, P.y), zm(zs(one, z0), l0v));
            const Fr zl = P.n_sets == 1 ? z0 : ld(&P.prods[P.n_sets - 1][row]);
            v = za(zm(v, P.y), zm(zs(zm(zl, zl), zl), ld(&P.l_last[row])));
            for (uint32_t s = 1; s < P.n_sets; s++)
                v = za(zm(v, P.y), zm(zs(ld(&P.prods[s][row]), ld(&P.prods[s - 1][rl])), l0v));
            const Fr la = ld(&P.l_active[row]);
            Fr cur = zm(P.delta_start, bt);
            for (uint32_t s = 0; s < P.n_sets; s++) {
                const uint32_t c0 = s * P.chunk_len;
                const uint32_t c1 = c0 + P.chunk_len < P.n_pcols ? c0 + P.chunk_len : P.n_pcols;
                Fr left = ld(&P.prods[s][rn]);
                Fr right = ld(&P.prods[s][row]);
                for (uint32_t c = c0; c < c1; c++) {
                    const Fr cv = ld(&P.pcols[c][row]);
                    left = zm(left, za(za(cv, zm(P.beta, ld(&P.sigmas[c][row]))), P.gamma));
                    right = zm(right, za(za(cv, cur), P.gamma));
                    cur = zm(cur, P.delta);
                }
                v = za(zm(v, P.y), zm(zs(left, right), la));
            }
            bt = bt * wstep;
        }
        if (P.n_lookups) {
            const uint64_t nx = row + 1 == P.nq ? 0 : row + 1;
            const uint64_t pv = row == 0 ? P.nq - 1 : row - 1;
            const Fr l0v = ld(&P.l0[row]), llast = ld(&P.l_last[row]), la = ld(&P.l_active[row]);
            for (uint32_t l = 0; l < P.n_lookups; l++) {
                const FqLookup& L = P.lk[l];
                const Fr tv = fq_run(P, slot, L.op0, L.op1, L.vp0, L.vp1, row);
                const Fr zi = ld(&L.z[row]), a = ld(&L.pin[row]), s = ld(&L.ptab[row]);
                const Fr ams = zs(a, s);
                v = za(zm(v, P.y), zm(zs(one, zi), l0v));
                v = za(zm(v, P.y), zm(zs(zm(zi, zi), zi), llast));
                v = za(zm(v, P.y), zm(zs(zm(zm(ld(&L.z[nx]), za(a, L.beta)), za(s, L.gamma)), zm(zi, tv)), la));
                v = za(zm(v, P.y), zm(ams, l0v));
                v = za(zm(v, P.y), zm(zm(ams, zs(a, ld(&L.pin[pv]))), la));
            }
        }
        if (P.has_scale) v = zm(v, P.scale);
        st(&P.out[r * P.out_stride + P.out_offset], canon2p<FrCfg>(v));
    }
}

} // namespace h2b

extern "C" {
typedef struct h2b_quotient_rules {
    const uint64_t* rules;
    uint64_t num_rules;
    const uint64_t* value_part_rules;
    uint64_t num_vp;
    const void* constants;
    uint64_t num_constants;
    const void* challenges;
    uint64_t num_challenges;
} h2b_quotient_rules;

typedef struct h2b_quotient_permutation_args {
    uint64_t n_sets, chunk_len, n_columns;
    const void* const* product_cosets;
    const void* const* sigma_cosets;
    const void* const* column_values;
    const void* beta;
    const void* gamma;
    const void* delta;
    const void* delta_start;
    const void* current_extended_omega;
    const void* omega;
    int32_t last_rotation, rot_scale, isize, reserved;
} h2b_quotient_permutation_args;

typedef struct h2b_quotient_lookup_args {
    h2b_quotient_rules product;
    const void* product_coset;
    const void* permuted_input_coset;
    const void* permuted_table_coset;
    const void* beta;
    const void* gamma;
} h2b_quotient_lookup_args;
}

namespace {

// Appends one compiled rule list to the parameter block: constants and
// challenges get their own ranges, ops and value parts are relocated to them.
RustError fq_append(FusedParams& P, uint32_t& n_ops, uint32_t& n_vps, uint32_t& n_consts, uint32_t& n_chal,
                    const h2b_quotient_rules& R, uint64_t num_fixed, uint64_t num_instance, uint64_t num_advice,
                    uint64_t nq, uint64_t rot_scale, uint32_t& slots, uint32_t& op0, uint32_t& op1, uint32_t& vp0,
                    uint32_t& vp1)
{
    if (R.num_rules && !R.rules) return err(cudaErrorInvalidValue, "h2b_quotient_fused: rules pointer is null");
    if (R.num_vp && !R.value_part_rules)
        return err(cudaErrorInvalidValue, "h2b_quotient_fused: value part rules pointer is null");
    QProgram Q = compile_rules(R.rules, R.num_rules, R.value_part_rules, R.num_vp, num_fixed, num_instance,
                               num_advice, R.num_constants, R.num_challenges, nq, rot_scale);
    if (!Q.error.empty()) return err(cudaErrorInvalidValue, Q.error.c_str());
    if (n_ops + Q.ops.size() > (size_t)FQ_MAX_OPS || n_vps + Q.vps.size() > (size_t)FQ_MAX_VPS ||
        n_consts + R.num_constants > (uint64_t)FQ_MAX_CONSTS || n_chal + R.num_challenges > (uint64_t)FQ_MAX_CHAL)
        return err(cudaErrorInvalidValue,
                   "h2b_quotient_fused: program larger than the fused kernel's parameter block "
                   "(256 ops, 64 value parts, 192 constants, 16 challenges)");
    if (R.num_constants && !R.constants) return err(cudaErrorInvalidValue, "h2b_quotient_fused: constants pointer is null");
    if (R.num_challenges && !R.challenges)
        return err(cudaErrorInvalidValue, "h2b_quotient_fused: challenges pointer is null");
    memcpy(&P.consts[n_consts], R.constants, R.num_constants * 32);
    memcpy(&P.chal[n_chal], R.challenges, R.num_challenges * 32);
    op0 = n_ops;
    for (QOp op : Q.ops) {
        if (op.sa == SRC_CONST) op.ia += n_consts;
        if (op.sb == SRC_CONST) op.ib += n_consts;
        if (op.sa == SRC_CHALLENGE) op.ia += n_chal;
        if (op.sb == SRC_CHALLENGE) op.ib += n_chal;
        P.ops[n_ops++] = op;
    }
    op1 = n_ops;
    vp0 = n_vps;
    for (QVp v : Q.vps) {
        if (v.is_const) v.idx += n_consts;
        P.vps[n_vps++] = v;
    }
    vp1 = n_vps;
    n_consts += (uint32_t)R.num_constants;
    n_chal += (uint32_t)R.num_challenges;
    slots = std::max(slots, Q.slots);
    return ok();
}

Fr fr_from(const void* p)
{
    Fr r;
    memcpy(&r, p, 32);
    return r;
}

} // namespace

// Register budget of the fused kernel, in blocks of 128 threads per SM: 3
// (162 registers, no spills; the default), 4 (128 registers, a few spills)
// or 5 (96 registers, more spills).  2^20 rows of a config-3 part: 1.416,
// 1.500 and 1.489 ms (1.54 ms uncapped at 198 registers; the reference's
// four per-part launches 1.50 ms).  Same results.
static int g_fq_blocks = 3;
extern "C" void h2b_quotient_fused_set_blocks(int blocks_per_sm)
{
    if (blocks_per_sm >= 3 && blocks_per_sm <= 5) g_fq_blocks = blocks_per_sm;
}
extern "C" int h2b_quotient_fused_get_blocks(void) { return g_fq_blocks; }

extern "C" RustError h2b_quotient_fused(const void* const* fixed, uint64_t num_fixed, const void* const* instance,
                                        uint64_t num_instance, const void* const* advice, uint64_t num_advice,
                                        const h2b_quotient_rules* gates, const void* y, const void* l0,
                                        const void* l_last, const void* l_active_row,
                                        const h2b_quotient_permutation_args* perm,
                                        const h2b_quotient_lookup_args* lookups, uint64_t num_lookups,
                                        uint64_t num_quotient, uint64_t rotation_scale, uint64_t row_start,
                                        uint64_t row_end, void* out, uint64_t out_stride, uint64_t out_offset,
                                        const void* scale, cudaStream_t stream)
{
    if (num_quotient == 0) return err(cudaErrorInvalidValue, "h2b_quotient_fused: num_quotient is 0");
    if (row_end < row_start || row_end > num_quotient)
        return err(cudaErrorInvalidValue, "h2b_quotient_fused: row range outside [0, num_quotient]");
    const uint64_t rows = row_end - row_start;
    if (rows == 0) return ok();
    if (!gates || !y || !out || out_stride == 0)
        return err(cudaErrorInvalidValue, "h2b_quotient_fused: gates, y and out are required, out_stride >= 1");
    const uint64_t ncols = num_fixed + num_instance + num_advice;
    if (ncols > (uint64_t)FQ_MAX_COLS) return err(cudaErrorInvalidValue, "h2b_quotient_fused: more than 64 columns");
    if (num_lookups > (uint64_t)FQ_MAX_LOOKUPS)
        return err(cudaErrorInvalidValue, "h2b_quotient_fused: more than 8 lookups");
    if (num_lookups && !lookups) return err(cudaErrorInvalidValue, "h2b_quotient_fused: lookups pointer is null");
    const bool has_perm = perm && perm->n_sets;
    if ((has_perm || num_lookups) && (!l0 || !l_last || !l_active_row))
        return err(cudaErrorInvalidValue, "h2b_quotient_fused: l0, l_last and l_active are required");

    static thread_local FusedParams P;   // about 18 KB: kept off the stack
    memset(&P, 0, sizeof(P));
    uint64_t c = 0;
    for (uint64_t i = 0; i < num_fixed; i++) P.cols[c++] = (const Fr*)fixed[i];
    for (uint64_t i = 0; i < num_instance; i++) P.cols[c++] = (const Fr*)instance[i];
    for (uint64_t i = 0; i < num_advice; i++) P.cols[c++] = (const Fr*)advice[i];
    for (uint64_t i = 0; i < ncols; i++)
        if (!P.cols[i]) return err(cudaErrorInvalidValue, "h2b_quotient_fused: null column pointer");

    uint32_t n_ops = 0, n_vps = 0, n_consts = 0, n_chal = 0, slots = 1, op0, op1, vp0, vp1;
    H2B_TRY(fq_append(P, n_ops, n_vps, n_consts, n_chal, *gates, num_fixed, num_instance, num_advice, num_quotient,
                      rotation_scale, slots, op0, op1, vp0, vp1));
    P.gate_ops = op1;
    P.gate_vps = vp1;
    for (uint64_t l = 0; l < num_lookups; l++) {
        const h2b_quotient_lookup_args& A = lookups[l];
        if (!A.product_coset || !A.permuted_input_coset || !A.permuted_table_coset || !A.beta || !A.gamma)
            return err(cudaErrorInvalidValue, "h2b_quotient_fused: incomplete lookup arguments");
        FqLookup& L = P.lk[l];
        H2B_TRY(fq_append(P, n_ops, n_vps, n_consts, n_chal, A.product, num_fixed, num_instance, num_advice,
                          num_quotient, rotation_scale, slots, L.op0, L.op1, L.vp0, L.vp1));
        L.z = (const Fr*)A.product_coset;
        L.pin = (const Fr*)A.permuted_input_coset;
        L.ptab = (const Fr*)A.permuted_table_coset;
        L.beta = fr_from(A.beta);
        L.gamma = fr_from(A.gamma);
    }
    P.n_lookups = (uint32_t)num_lookups;
    if (slots > 64)
        return err(cudaErrorInvalidValue, "h2b_quotient_fused: more than 64 live intermediates");

    if (has_perm) {
        const h2b_quotient_permutation_args& A = *perm;
        if (A.n_sets > (uint64_t)FQ_MAX_SETS || A.n_columns > (uint64_t)FQ_MAX_PCOLS || A.chunk_len == 0 ||
            A.n_columns > A.n_sets * A.chunk_len)
            return err(cudaErrorInvalidValue,
                       "h2b_quotient_fused: permutation shape (at most 8 sets, 32 columns, columns <= sets * chunk_len)");
        if (A.isize <= 0 || row_end > (uint64_t)A.isize)
            return err(cudaErrorInvalidValue, "h2b_quotient_fused: permutation isize must cover the rows");
        if (!A.product_cosets || (A.n_columns && (!A.sigma_cosets || !A.column_values)) || !A.beta || !A.gamma ||
            !A.delta || !A.delta_start || !A.current_extended_omega || !A.omega)
            return err(cudaErrorInvalidValue, "h2b_quotient_fused: incomplete permutation arguments");
        for (uint64_t s = 0; s < A.n_sets; s++) {
            P.prods[s] = (const Fr*)A.product_cosets[s];
            if (!P.prods[s]) return err(cudaErrorInvalidValue, "h2b_quotient_fused: null product coset");
        }
        for (uint64_t i = 0; i < A.n_columns; i++) {
            P.sigmas[i] = (const Fr*)A.sigma_cosets[i];
            P.pcols[i] = (const Fr*)A.column_values[i];
            if (!P.sigmas[i] || !P.pcols[i]) return err(cudaErrorInvalidValue, "h2b_quotient_fused: null permutation column");
        }
        P.n_sets = (uint32_t)A.n_sets;
        P.chunk_len = (uint32_t)A.chunk_len;
        P.n_pcols = (uint32_t)A.n_columns;
        P.isize = (uint64_t)A.isize;
        auto wrap = [&](int64_t rot) -> uint64_t {
            int64_t o = (rot * (int64_t)A.rot_scale) % (int64_t)A.isize;
            return (uint64_t)(o < 0 ? o + A.isize : o);
        };
        P.off_next = wrap(1);
        P.off_last = wrap(A.last_rotation);
        P.beta = fr_from(A.beta);
        P.gamma = fr_from(A.gamma);
        P.delta = fr_from(A.delta);
        P.delta_start = fr_from(A.delta_start);
        P.ext_omega = fr_from(A.current_extended_omega);
        P.omega = fr_from(A.omega);
    }
    P.l0 = (const Fr*)l0;
    P.l_last = (const Fr*)l_last;
    P.l_active = (const Fr*)l_active_row;
    P.out = (Fr*)out;
    P.y = fr_from(y);
    P.nq = num_quotient;
    P.out_stride = out_stride;
    P.out_offset = out_offset;
    if (scale) {
        P.has_scale = 1;
        P.scale = fr_from(scale);
    }
    const unsigned grid = grid_for(rows, FQ_THREADS, 148u * 8u);
    prof_begin(PROF_QUOTIENT, stream);
#define H2B_FQ_LAUNCH(B)                                                                      \
    do {                                                                                      \
        if (slots <= 16) k_quotient_fused<16, B><<<grid, FQ_THREADS, 0, stream>>>(P, row_start, rows); \
        else k_quotient_fused<64, B><<<grid, FQ_THREADS, 0, stream>>>(P, row_start, rows);   \
    } while (0)
    if (g_fq_blocks == 3) H2B_FQ_LAUNCH(3);
    else if (g_fq_blocks == 5) H2B_FQ_LAUNCH(5);
    else H2B_FQ_LAUNCH(4);
#undef H2B_FQ_LAUNCH
    prof_end(PROF_QUOTIENT, stream);
    H2B_LAUNCHED("k_quotient_fused");
    return ok();
}
