// C-ABI plumbing shared by every launcher.
//
// Wire types match the reference's FFI exactly so the Rust crate can link this
// library in place of libhalo2_gpu:
//  * RustError {int code; char* message} is returned by value; the message is
//    strdup'd here and freed by the caller (halo2_proofs/cuda/include/common/
//    halo2_ffi.h:27-49, halo2_proofs/src/cuda/error.rs:17-50).  code 0 = ok.
//  * FFITraitObject {uint64_t* ptr} is one machine word that carries a host or
//    a device address depending on the entry point (halo2_ffi.h:56-60,
//    halo2_proofs/src/cuda/utils.rs:98-117).
//  * Caller-owned scratch is (void* scratch, uint64_t bytes), sized by a pure
//    host `_workspace_size` preflight; launchers never allocate
//    (halo2_ffi.h:9-19).  ScratchArena carves it with 256-byte alignment and
//    reports overflow as an error code instead of trapping.
#pragma once
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>

extern "C" {
typedef struct RustError {
    int code;
    char* message;
} RustError;

typedef struct FFITraitObject {
    uint64_t* ptr;
} FFITraitObject;
}

namespace h2b {

inline RustError ok() { RustError e; e.code = 0; e.message = nullptr; return e; }

inline RustError err(int code, const char* msg)
{
    RustError e;
    e.code = code;
    e.message = msg ? strdup(msg) : nullptr;
    return e;
}

inline RustError cuda_err(cudaError_t c, const char* where)
{
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(c));
    return err((int)c, buf);
}

#define H2B_CUDA(expr)                                             \
    do {                                                           \
        cudaError_t _c = (expr);                                   \
        if (_c != cudaSuccess) return ::h2b::cuda_err(_c, #expr);  \
    } while (0)

// Every kernel launch site is followed by H2B_LAUNCHED, which also counts the
// launch (read with h2b_launch_count()).
inline std::atomic<uint64_t> g_kernel_launches{0};

#define H2B_LAUNCHED(where)                                        \
    do {                                                           \
        ::h2b::g_kernel_launches.fetch_add(1, std::memory_order_relaxed); \
        cudaError_t _c = cudaGetLastError();                       \
        if (_c != cudaSuccess) return ::h2b::cuda_err(_c, where);  \
    } while (0)

#define H2B_TRY(expr)                                              \
    do {                                                           \
        RustError _e = (expr);                                     \
        if (_e.code != 0) return _e;                               \
    } while (0)

static constexpr uint64_t kAlign = 256;

inline uint64_t align_up(uint64_t x, uint64_t a = kAlign) { return (x + a - 1) / a * a; }

// Bump allocator over caller-provided scratch.  `take` returns nullptr once
// the span is exhausted; launchers check `ok()` before launching anything.
struct ScratchArena {
    uint8_t* base;
    uint64_t bytes;
    uint64_t used = 0;
    bool overflow = false;
    ScratchArena(void* p, uint64_t n) : base((uint8_t*)p), bytes(n) {}
    void* take(uint64_t n)
    {
        uint64_t off = align_up(used);
        if (off + n > bytes || (n > 0 && base == nullptr)) { overflow = true; return nullptr; }
        used = off + align_up(n);
        return base + off;
    }
    template <class T> T* take_n(uint64_t count) { return (T*)take(count * sizeof(T)); }
    bool good() const { return !overflow; }
};

// Size accumulator with the same rounding as ScratchArena::take.
struct ScratchPlan {
    uint64_t used = 0;
    void add(uint64_t n) { used = align_up(used) + align_up(n); }
    template <class T> void add_n(uint64_t count) { add(count * sizeof(T)); }
};

inline RustError scratch_too_small(const char* who, uint64_t have, uint64_t need)
{
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: scratch too small (%llu bytes given, %llu needed)", who,
             (unsigned long long)have, (unsigned long long)need);
    return err((int)cudaErrorInvalidValue, buf);
}

inline unsigned grid_for(uint64_t work, unsigned threads, unsigned cap = 148u * 64u)
{
    uint64_t g = (work + threads - 1) / threads;
    if (g == 0) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

} // namespace h2b
