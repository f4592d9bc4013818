// Batch execution helpers for serving many independent jobs of uneven size
// (many MSMs, NTTs and quotient evaluations of k = 14..22) on one GPU.  No
// counterpart in the reference, which runs one launcher at a time on one
// stream.
//
//  * h2b_exec_fork / h2b_exec_join: N internal non-blocking streams ordered
//    after / before the caller's stream through events, so jobs issued on
//    them overlap on the device while the caller keeps one stream of record.
//    The streams and events are created once per device (first fork on that
//    device) and live until process exit.
//  * h2b_graph_begin / h2b_graph_end / h2b_graph_launch / h2b_graph_destroy:
//    capture everything issued on the caller's stream (and on streams forked
//    from it) into a CUDA graph and replay it; the pointers and sizes of the
//    captured calls are baked in.  Only entry points that issue no host
//    copies and no synchronisation can be captured (the device-resident MSM,
//    NTT types 1-4 and the device-column quotient are such).
//  * h2b_msm_batch: `count` device-resident MSMs spread over `streams`
//    forked streams, longest job first onto the least-loaded stream, each
//    stream with its own slice of the caller's scratch.
#include <algorithm>
#include <map>
#include <numeric>
#include <vector>
#include "abi.cuh"
#include "curve.cuh"
#include "msm.cuh"

namespace h2b {

namespace {
constexpr uint32_t EXEC_MAX_STREAMS = 32;

struct DevExec {
    std::vector<cudaStream_t> streams;
    cudaEvent_t fork_ev = nullptr;
    std::vector<cudaEvent_t> join_ev;
};
// Per calling thread: callers on different threads (one per served request,
// say) never share forked streams or events, so their forks and joins cannot
// interleave.
thread_local std::map<int, DevExec> t_exec;

// Streams and events of the current device and thread, created on first use.
RustError exec_get(uint32_t n, DevExec** out)
{
    if (n == 0 || n > EXEC_MAX_STREAMS) return err((int)cudaErrorInvalidValue, "exec: streams must be in 1..32");
    int dev = 0;
    H2B_CUDA(cudaGetDevice(&dev));
    DevExec& d = t_exec[dev];
    if (!d.fork_ev) H2B_CUDA(cudaEventCreateWithFlags(&d.fork_ev, cudaEventDisableTiming));
    while (d.streams.size() < n) {
        cudaStream_t s;
        H2B_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        d.streams.push_back(s);
        cudaEvent_t e;
        H2B_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        d.join_ev.push_back(e);
    }
    *out = &d;
    return ok();
}

struct GraphHandle {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

// Plan of one job: plain bases, or a precomputed window table of table_n points.
MsmPlan job_plan(uint64_t n, uint64_t table_n, uint32_t concurrent)
{
    return msm_plan_shared(n, table_n, concurrent);
}

// Scratch of one MSM slot (device scalars and bases), 256-byte aligned.
uint64_t msm_slot_bytes(uint64_t n, uint64_t table_n, uint32_t concurrent)
{
    MsmPlan p = job_plan(n, table_n, concurrent);
    ScratchPlan sp;
    msm_plan_scratch(p, sp, false, false);
    return align_up(sp.used);
}
} // namespace

} // namespace h2b

using namespace h2b;

extern "C" RustError h2b_exec_fork(cudaStream_t parent, uint32_t n, cudaStream_t* out)
{
    DevExec* d = nullptr;
    H2B_TRY(exec_get(n, &d));
    H2B_CUDA(cudaEventRecord(d->fork_ev, parent));
    for (uint32_t i = 0; i < n; i++) {
        H2B_CUDA(cudaStreamWaitEvent(d->streams[i], d->fork_ev, 0));
        out[i] = d->streams[i];
    }
    return ok();
}

extern "C" RustError h2b_exec_join(cudaStream_t parent, uint32_t n)
{
    DevExec* d = nullptr;
    H2B_TRY(exec_get(n, &d));
    for (uint32_t i = 0; i < n; i++) {
        H2B_CUDA(cudaEventRecord(d->join_ev[i], d->streams[i]));
        H2B_CUDA(cudaStreamWaitEvent(parent, d->join_ev[i], 0));
    }
    return ok();
}

// Stream-ordered upload of a small host buffer (pageable memory is staged by
// the driver before this returns, so the source may be reused at once); unlike
// a synchronous copy it does not wait for the work already queued on `s`.
extern "C" RustError h2b_upload(void* d_dst, const void* h_src, uint64_t bytes, cudaStream_t s)
{
    if (bytes == 0) return ok();
    if (!d_dst || !h_src) return err((int)cudaErrorInvalidValue, "h2b_upload: null pointer");
    H2B_CUDA(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, s));
    return ok();
}

extern "C" RustError h2b_graph_begin(cudaStream_t s)
{
    H2B_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    return ok();
}

extern "C" RustError h2b_graph_end(cudaStream_t s, void** handle)
{
    GraphHandle* g = new GraphHandle;
    cudaError_t e = cudaStreamEndCapture(s, &g->graph);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) {
        if (g->graph) cudaGraphDestroy(g->graph);
        delete g;
        return cuda_err(e, "h2b_graph_end");
    }
    *handle = g;
    return ok();
}

extern "C" RustError h2b_graph_launch(void* handle, cudaStream_t s)
{
    if (!handle) return err((int)cudaErrorInvalidValue, "h2b_graph_launch: null handle");
    H2B_CUDA(cudaGraphLaunch(static_cast<GraphHandle*>(handle)->exec, s));
    return ok();
}

extern "C" void h2b_graph_destroy(void* handle)
{
    GraphHandle* g = static_cast<GraphHandle*>(handle);
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

// ---- batched MSM --------------------------------------------------------------

typedef struct h2b_msm_job {
    const void* d_scalars;  // n Montgomery Fr (device)
    const void* d_bases;    // n affine G1, or a window table built for table_n bases (device)
    void* d_out;            // 96-byte Jacobian image (device)
    uint64_t n;
    uint64_t table_n;       // 0: d_bases are plain bases
} h2b_msm_job;

// MSMs of a batch that run at the same time: one per forked stream.
static uint32_t batch_concurrency(uint64_t count, uint32_t streams)
{
    return (uint32_t)std::min<uint64_t>(count, streams);
}

static uint64_t batch_slot(const h2b_msm_job* jobs, uint64_t count, uint32_t concurrent)
{
    uint64_t mx = 0;
    for (uint64_t i = 0; i < count; i++) mx = std::max(mx, msm_slot_bytes(jobs[i].n, jobs[i].table_n, concurrent));
    return mx;
}

// One scratch slot per stream, each sized for the largest job.
extern "C" uint64_t h2b_msm_batch_workspace_size(const h2b_msm_job* jobs, uint64_t count, uint32_t streams)
{
    if (streams == 0 || streams > EXEC_MAX_STREAMS) return 0;
    return (uint64_t)streams * batch_slot(jobs, count, batch_concurrency(count, streams));
}

extern "C" RustError h2b_msm_batch(const h2b_msm_job* jobs, uint64_t count, uint32_t streams, void* scratch,
                                   uint64_t scratch_bytes, cudaStream_t stream)
{
    if (count == 0) return ok();
    if (streams == 0 || streams > EXEC_MAX_STREAMS)
        return err((int)cudaErrorInvalidValue, "h2b_msm_batch: streams must be in 1..32");
    for (uint64_t i = 0; i < count; i++) {
        if (jobs[i].n > 0 && (!jobs[i].d_scalars || !jobs[i].d_bases))
            return err((int)cudaErrorInvalidValue, "h2b_msm_batch: null input pointer");
        if (!jobs[i].d_out) return err((int)cudaErrorInvalidValue, "h2b_msm_batch: null output pointer");
        if (jobs[i].table_n && jobs[i].n > jobs[i].table_n)
            return err((int)cudaErrorInvalidValue, "h2b_msm_batch: job longer than its table");
    }
    const uint32_t conc = batch_concurrency(count, streams);
    const uint64_t slot = batch_slot(jobs, count, conc);
    if (scratch_bytes < slot * streams || !scratch)
        return scratch_too_small("h2b_msm_batch", scratch_bytes, slot * streams);
    // longest job first onto the least-loaded stream
    std::vector<uint64_t> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return jobs[a].n > jobs[b].n; });
    std::vector<uint64_t> load(streams, 0);
    cudaStream_t sub[EXEC_MAX_STREAMS];
    H2B_TRY(h2b_exec_fork(stream, streams, sub));
    for (uint64_t j : order) {
        const uint32_t k = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
        load[k] += jobs[j].n + 4096;  // fixed cost per job: launch and tail latency
        const MsmPlan p = job_plan(jobs[j].n, jobs[j].table_n, conc);
        ScratchArena ar((uint8_t*)scratch + (uint64_t)k * slot, slot);
        const MsmScratch s = msm_carve(p, ar, false, false);
        if (!ar.good()) return err((int)cudaErrorInvalidValue, "h2b_msm_batch: slot carving failed");
        H2B_TRY(msm_run(p, s, (const Fr*)jobs[j].d_scalars, (const G1Affine*)jobs[j].d_bases, sub[k]));
        H2B_CUDA(cudaMemcpyAsync(jobs[j].d_out, s.result, sizeof(G1Jac), cudaMemcpyDeviceToDevice, sub[k]));
    }
    return h2b_exec_join(stream, streams);
}

// Merged MSMs over one window table (no counterpart in the reference, whose
// prover commits one polynomial per `_halo2_multiexp*` call): every job must
// name the same table (d_bases, table_n > 0); up to 64 jobs of any lengths
// up to table_n run as one MSM whose bucket sets are the jobs'.  Results are
// those of h2b_msm_device_table per job.
static RustError merged_check(const h2b_msm_job* jobs, uint64_t count, uint64_t& n_total)
{
    if (count == 0 || count > MSM_MERGE_MAX)
        return err((int)cudaErrorInvalidValue, "h2b_msm_merged: 1 to 64 jobs");
    n_total = 0;
    for (uint64_t i = 0; i < count; i++) {
        if (jobs[i].table_n == 0 || jobs[i].d_bases != jobs[0].d_bases || jobs[i].table_n != jobs[0].table_n)
            return err((int)cudaErrorInvalidValue, "h2b_msm_merged: jobs must share one window table");
        if (jobs[i].n > jobs[i].table_n)
            return err((int)cudaErrorInvalidValue, "h2b_msm_merged: job longer than its table");
        if (!jobs[i].d_out || (jobs[i].n > 0 && !jobs[i].d_scalars))
            return err((int)cudaErrorInvalidValue, "h2b_msm_merged: null pointer");
        n_total += jobs[i].n;
    }
    return ok();
}

extern "C" uint64_t h2b_msm_merged_workspace_size(const h2b_msm_job* jobs, uint64_t count)
{
    uint64_t n_total = 0;
    RustError e = merged_check(jobs, count, n_total);
    if (e.code) {
        free(e.message);
        return 0;
    }
    const MsmPlan p = msm_plan_merged(std::max<uint64_t>(n_total, 1), jobs[0].table_n, (uint32_t)count);
    ScratchPlan sp;
    msm_plan_scratch(p, sp, false, false);
    return sp.used;
}

extern "C" RustError h2b_msm_merged(const h2b_msm_job* jobs, uint64_t count, void* scratch, uint64_t scratch_bytes,
                                    cudaStream_t stream)
{
    uint64_t n_total = 0;
    H2B_TRY(merged_check(jobs, count, n_total));
    const MsmPlan p = msm_plan_merged(std::max<uint64_t>(n_total, 1), jobs[0].table_n, (uint32_t)count);
    ScratchPlan sp;
    msm_plan_scratch(p, sp, false, false);
    if (!scratch || scratch_bytes < sp.used) return scratch_too_small("h2b_msm_merged", scratch_bytes, sp.used);
    ScratchArena ar(scratch, scratch_bytes);
    const MsmScratch s = msm_carve(p, ar, false, false);
    if (!ar.good()) return err((int)cudaErrorInvalidValue, "h2b_msm_merged: scratch carving failed");
    const Fr* sc[MSM_MERGE_MAX];
    uint64_t ns[MSM_MERGE_MAX];
    G1Jac* outs[MSM_MERGE_MAX];
    for (uint64_t i = 0; i < count; i++) {
        sc[i] = (const Fr*)jobs[i].d_scalars;
        ns[i] = jobs[i].n;
        outs[i] = (G1Jac*)jobs[i].d_out;
    }
    return msm_run_merged(p, s, (uint32_t)count, sc, ns, (const G1Affine*)jobs[0].d_bases, outs, stream);
}
