"""Batch execution: many MSMs and NTTs of uneven size overlapped on forked
streams and replayed from a captured CUDA graph give the same bytes as the
same jobs run one at a time (the batched-prover pattern: 64 jobs of k drawn
from {14, 16, 18, 20}; smaller sizes here)."""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def _single_msm(h2b, d_sc, d_b, n):
    out = h2b.dev_empty(96)
    ws = h2b.msm_workspace(n)
    h2b.msm_device(d_sc, d_b, out, n, ws)
    torch.cuda.synchronize()
    return out.cpu().numpy().tobytes()


@pytest.fixture(scope="module")
def msm_jobs(h2b, cuda):
    lengths = [1, 0, 100, 1 << 10, 1 << 12, 3000, 1 << 14, 1 << 12, 17, 1 << 16, 5, 1 << 13]
    srs = h2b.srs_device(0xBA7C, 1 << 16)
    d_sc = [h2b.random_fr_device(max(n, 1), 100 + i, i % 2) for i, n in enumerate(lengths)]
    d_b = [srs for _ in lengths]
    want = [_single_msm(h2b, d_sc[i], d_b[i], n) for i, n in enumerate(lengths)]
    return lengths, d_sc, d_b, want


@pytest.mark.parametrize("streams", [1, 4, 8])
def test_msm_batch_matches_single(h2b, cuda, msm_jobs, streams):
    lengths, d_sc, d_b, want = msm_jobs
    outs = [h2b.dev_empty(96) for _ in lengths]
    jobs = h2b.msm_batch_jobs(d_sc, d_b, outs, lengths)
    ws = h2b.msm_batch_workspace(jobs, len(lengths), streams)
    for _ in range(2):  # twice in a row: slots are reused
        for o in outs:
            o.zero_()
        h2b.msm_batch(jobs, len(lengths), streams, ws)
        torch.cuda.synchronize()
        assert [o.cpu().numpy().tobytes() for o in outs] == want


def test_msm_batch_argument_errors(h2b, cuda, msm_jobs):
    lengths, d_sc, d_b, _ = msm_jobs
    outs = [h2b.dev_empty(96) for _ in lengths]
    jobs = h2b.msm_batch_jobs(d_sc, d_b, outs, lengths)
    ws = h2b.msm_batch_workspace(jobs, len(lengths), 2)
    with pytest.raises(h2b.Halo2GpuError):
        h2b.msm_batch(jobs, len(lengths), 33, ws)
    small = h2b.dev_empty(1024)
    with pytest.raises(h2b.Halo2GpuError):
        h2b.msm_batch(jobs, len(lengths), 2, small)


def _coset_jobs(h2b, logs, seed):
    ins, outs = [], []
    for i, k in enumerate(logs):
        ins.append(h2b.random_fr_device(1 << k, seed + i, 0))
        outs.append(h2b.dev_empty(32 << (k + 2)))
    return ins, outs


def test_forked_streams_and_graph_replay(h2b, cuda, msm_jobs):
    """MSMs (batched) plus coset extensions on forked streams, captured once
    and replayed twice over new input contents in the same buffers."""
    f = h2b.fields
    lengths, d_sc, d_b, _ = msm_jobs
    logs = [10, 12, 14, 11]
    ins, outs = _coset_jobs(h2b, logs, 500)
    doms = [f.EvaluationDomain(3, k) for k in logs]
    ntt_ws = [h2b.dev_empty(h2b.lib()._halo2_fft_many_to_device_workspace_size(3, k, k + 2)) for k in logs]
    msm_outs = [h2b.dev_empty(96) for _ in lengths]
    jobs = h2b.msm_batch_jobs(d_sc, d_b, msm_outs, lengths)
    msm_ws = h2b.msm_batch_workspace(jobs, len(lengths), 4)

    def reference():
        got_ntt = []
        for i, k in enumerate(logs):
            o = h2b.dev_empty(32 << (k + 2))
            h2b.fft_many_to_device(3, k, k + 2, [ins[i]], [o], doms[i].extended_omega, 1)
            got_ntt.append(o.cpu().numpy().tobytes())
        got_msm = [_single_msm(h2b, d_sc[i], d_b[i], n) for i, n in enumerate(lengths)]
        return got_ntt, got_msm

    # everything the capture needs is allocated before it (no allocation or
    # host copy may run while the stream is being captured)
    d_oms = [h2b.to_dev(f.fr_mont_limbs([d.extended_omega])) for d in doms]
    one = f.fr_mont_limbs([1])
    one_ffi = h2b.host_ffi(one)
    tables = [(h2b.ffi_array([ins[i].data_ptr()]), h2b.ffi_array([outs[i].data_ptr()])) for i in range(len(logs))]

    def coset(i, k, stream):
        h2b.call("_halo2_fft_many_to_device", 3, 1, k, k + 2, tables[i][0], tables[i][1], h2b.ptr(d_oms[i]),
                 ctypes.byref(one_ffi), True, h2b.ptr(ntt_ws[i]), ntt_ws[i].numel(), h2b.stream_handle(stream))

    side = torch.cuda.Stream()
    # warm-up outside capture: creates the forked streams and loads every kernel
    subs = h2b.exec_fork(len(logs), side)
    for i, k in enumerate(logs):
        coset(i, k, subs[i])
    h2b.exec_join(len(logs), side)
    h2b.msm_batch(jobs, len(lengths), 4, msm_ws, stream=side)
    torch.cuda.synchronize()
    g = h2b.Graph(side)
    g.begin()
    subs = h2b.exec_fork(len(logs), side)
    for i, k in enumerate(logs):
        coset(i, k, subs[i])
    h2b.exec_join(len(logs), side)
    h2b.msm_batch(jobs, len(lengths), 4, msm_ws, stream=side)
    g.end()
    try:
        for rnd in range(2):
            for i, k in enumerate(logs):   # new contents, same buffers
                ins[i].copy_(h2b.random_fr_device(1 << k, 900 + 10 * rnd + i, 0))
            for i, n in enumerate(lengths):
                d_sc[i].copy_(h2b.random_fr_device(max(n, 1), 700 + 10 * rnd + i, 1))
            torch.cuda.synchronize()
            g.launch(side)
            side.synchronize()
            want_ntt, want_msm = reference()
            assert [o.cpu().numpy().tobytes() for o in outs] == want_ntt
            assert [o.cpu().numpy().tobytes() for o in msm_outs] == want_msm
    finally:
        g.close()
