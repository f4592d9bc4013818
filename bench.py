#!/usr/bin/env python3
"""Benchmark of the BN254 prover hot path at k = 22 (one GPU per process).

A step is one pass of the full-size single-kernel workload:
  * MSM over 2^22 SRS points [tau^i] G (seeded tau) with the witness-like
    scalar mix 50% uniform / 30% < 2^64 / 20% in {0, 1};
  * coeff_to_extended: coset NTT 2^22 -> 2^24 (extension factor 4);
  * batch_invert over 2^24 nonzero uniform Fr.
The headline metric is MSM points/s; NTT GB/s (algorithmic bytes
2^22*32 + 2^24*32 per transform) and batch-invert elements/s are reported
beside it from the same timed steps.  Inputs (128 MB scalars + 256 MB bases,
512 MB NTT output, 512 MB inversion array) exceed the 126 MB L2, so no flush
is needed between steps.

`--impl reference` times the CPU restatement of the reference's CPU path
(best_multiexp_cpu, the radix-2 FFT, the chunked Montgomery trick) with all
host threads: each of its K timed steps (after W untimed ones) is the CPU MSM
over a 2^20-point sample of the same workload (SRS points, the same scalar
mix), and its value is the points/s those steps measured; the coset NTT
2^22 -> 2^24 and the batch inversion of 2^24 elements are each timed once at
full size beside it (`cpu_rows`).

The dominant kernel's roofline is its binding resource, the field products:
the FP64-form product (five 52-bit limbs, exact FMA splits) issues, per 32
products, 430 warp instructions of which 211 go to the integer ALU pipe and
155 to the FP64 pipe (ncu, profiles/product_probe_fp64.md); with B200's 4
issue slots and 2 ALU and 2 FP64 warp instructions per clock per SM, issue
bounds it at 148 x 4 / 430 x 32 products per clock (the ALU pipe within 2 %).
That ceiling, at the SM clock sampled during the run, is `roofline.peak`;
the HBM figures sit beside it in `roofline.hbm`.
"""
import argparse
import ctypes
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
K_MSM, K_NTT, K_EXT, K_BI = 22, 22, 24, 24
METRIC = "MSM pts/s at k=22 (step: MSM 2^22 + coset NTT 2^22->2^24 + batch_invert 2^24)"
UNIT = "points/s"
WORKLOAD = {
    "workload": "k22_single_kernels",
    "msm_points": 1 << K_MSM,
    "msm_scalar_mix": "50% uniform Fr / 30% < 2^64 / 20% {0,1}",
    "ntt": "coset 2^22 -> 2^24",
    "batch_invert": 1 << K_BI,
    "l2": "inputs larger than L2 (no flush)",
}


def load_pkg():
    name = "halo2_gpu_b200"
    pkg = os.path.join(ROOT, "halo2-gpu_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def max_over_ranks(values, dist, device):
    """Element-wise maximum of per-rank timings over all ranks (the slowest
    rank sets every whole-job figure); values unchanged without a process
    group."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def whole_job_points_per_s(world, points_per_rank, ms):
    """Weak scaling: every rank runs its own MSM of `points_per_rank` points;
    the job's throughput is all points over the slowest rank's time."""
    return world * points_per_rank / (ms * 1e-3)


# Per 32 products of the FP64-form field product (ncu on h2b_probe_modmul's
# kernel, profiles/product_probe_fp64.md): warp instructions issued, and those
# executed by the integer ALU pipe and the FP64 pipe.
PRODUCT_WARP_INST = {"issue": 430, "alu": 211, "fp64": 155}
# B200 warp instructions per clock per SM: issue slots (4 schedulers), ALU and
# FP64 pipes (16 lanes per scheduler each)
SM_RATE = {"issue": 4, "alu": 2, "fp64": 2}
NUM_SMS = 148


def product_ceiling(sm_mhz):
    """Products/s ceilings of the FP64-form field product at `sm_mhz`: per
    resource, SMs x rate / (warp instructions per 32 products) x 32; the
    lowest binds."""
    ceilings = {r: NUM_SMS * SM_RATE[r] / PRODUCT_WARP_INST[r] * 32 * sm_mhz * 1e6 / 1e9 for r in SM_RATE}
    bind = min(ceilings, key=ceilings.get)
    return {"peak_gproducts_per_s": ceilings[bind], "binding": bind,
            "ceilings": {r: round(v, 2) for r, v in ceilings.items()},
            "source": f"{bind} pipe: {NUM_SMS} SMs x {SM_RATE[bind]} warp instr/clk / "
                      f"{PRODUCT_WARP_INST[bind]} per 32 products at {sm_mhz:.0f} MHz (sampled SM clock)"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class UtilSampler:
    """nvidia-smi GPU utilisation (the fraction of time a kernel ran) sampled
    every 100 ms while a serving trace runs."""

    def __init__(self, gpu_index):
        self.gpu, self.proc, self.vals = gpu_index, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=utilization.gpu",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            try:
                self.vals.append(float(line.strip()))
            except ValueError:
                pass

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        v = sorted(self.vals)
        return {"median_pct": v[len(v) // 2], "mean_pct": round(sum(v) / len(v), 1), "samples": len(v)} if v else None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region.

    start() returns once the first sample has arrived (nvidia-smi takes a
    moment to begin), so the timed region is sampled from its start; begin()
    and end() mark the region, and stop() reports the samples that arrived
    inside it (all samples when the region was shorter than one interval)."""

    INTERVAL_MS = 50

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.first = threading.Event()
        self.t_begin = self.t_end = None

    def start(self, wait_s=5.0):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.first.wait(wait_s)
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))
            self.first.set()

    def begin(self):
        self.t_begin = time.monotonic()

    def end(self):
        self.t_end = time.monotonic()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(2 * self.INTERVAL_MS / 1000)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        lines = self.lines
        inside = []
        if self.t_begin is not None and self.t_end is not None:
            inside = [x for x in lines if self.t_begin <= x[0] <= self.t_end + self.INTERVAL_MS / 1000]
            lines = inside or lines
        sms, mx, reasons = [], None, set()
        for _, ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        sms.sort()
        med = sms[len(sms) // 2] if sms else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sms),
                "interval_ms": self.INTERVAL_MS, "samples_inside_timed_region": bool(inside)}


def ncu_traffic(name):
    """DRAM bytes per launch from a committed ncu summary (profiles/<name>), or None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch_full_size:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


REF_LOG_N = 20


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    return orc


def _fields():
    return load_pkg().fields if "halo2_gpu_b200" not in sys.modules else sys.modules["halo2_gpu_b200"].fields


def cpu_msm_inputs(log_n):
    """A 2^log_n sample of the k=22 MSM workload on the host: SRS points
    [tau^i] G and scalars with the witness-like mix (50% uniform, 30% < 2^64,
    20% in {0, 1})."""
    import numpy as np
    orc, f = _oracle(), _fields()
    n = 1 << log_n
    bases = orc.srs(f.fr_mont_limbs([0x5EED]), n)
    sc = orc.chacha_fr(22, n)
    rng = np.random.default_rng(22)
    cls = rng.integers(0, 10, n)
    small = rng.integers(0, 2**63, n, dtype=np.uint64)
    sc_plain = np.zeros((n, 4), np.uint64)
    sc_plain[:, 0] = np.where(cls >= 8, small & np.uint64(1), small)
    smallm = np.zeros_like(sc_plain)
    orc.lib().o_to_mont(0, sc_plain.ctypes.data, smallm.ctypes.data, n)
    return np.ascontiguousarray(np.where((cls < 5)[:, None], sc, smallm)), bases


def cpu_threads():
    orc = _oracle()
    try:
        avail = len(os.sched_getaffinity(0))
    except AttributeError:
        avail = os.cpu_count()
    return orc.num_threads(), avail


def cpu_baseline_msm(log_n=REF_LOG_N, min_runs=3, budget_s=10.0):
    """The oracle's best_multiexp_cpu restatement (oracle/oracle.c: contiguous
    chunks per thread, c = ceil(ln n) unsigned windows, affine bases added into
    Jacobian buckets by mixed addition) over a 2^log_n sample, all host
    threads; at least `min_runs` runs, more while under `budget_s`."""
    orc = _oracle()
    sc, bases = cpu_msm_inputs(log_n)
    threads, avail = cpu_threads()
    orc.msm(sc[:1024], bases[:1024], threads)
    times = []
    t0 = time.perf_counter()
    while len(times) < min_runs or time.perf_counter() - t0 < budget_s:
        t = time.perf_counter()
        orc.msm(sc, bases, threads)
        times.append(time.perf_counter() - t)
    n = 1 << log_n
    times.sort()
    return {"value": n * len(times) / sum(times), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"best_multiexp_cpu restatement (oracle/oracle.c) over 2^{log_n} SRS points with the same "
                      f"scalar mix, {len(times)} runs",
            "run_ms": {"min": round(times[0] * 1e3, 2), "median": round(times[len(times) // 2] * 1e3, 2),
                       "max": round(times[-1] * 1e3, 2)},
            "threads_available": avail}


def cpu_rows(threads):
    """The other CPU paths of the k=22 step, each timed once at full size with
    all host threads: the radix-2 coset NTT 2^22 -> 2^24 (best_fft's
    structure: bit reversal, then stages split over the threads) and the
    chunked Montgomery-trick batch inversion of 2^24 elements
    (halo2_proofs/src/arithmetic.rs:113-150: one chunk and one inversion per
    thread)."""
    orc, f = _oracle(), _fields()
    dom = f.EvaluationDomain(5, K_NTT)
    a = orc.chacha_fr(2000, 1 << K_NTT)
    t = time.perf_counter()
    orc.ntt(3, K_NTT, K_EXT, a, f.fr_mont_limbs([dom.extended_omega]), f.fr_mont_limbs([1]))
    ntt_s = time.perf_counter() - t
    del a
    x = orc.chacha_fr(3000, 1 << K_BI)
    t = time.perf_counter()
    orc.batch_invert_par(x, 0, threads)
    bi_s = time.perf_counter() - t
    ntt_bytes = 32 * (1 << K_NTT) + 32 * (1 << K_EXT)
    return {"coset_ntt_22_24": {"ms": round(ntt_s * 1e3, 1), "GB_per_s": ntt_bytes / ntt_s / 1e9,
                                "elements_per_s": (1 << K_EXT) / ntt_s},
            "batch_invert_24": {"ms": round(bi_s * 1e3, 1), "elements_per_s": (1 << K_BI) / bi_s},
            "cores": threads}


def run_reference(args, rank):
    """The reference arm: the CPU path, rank 0 only.  Every step is timed:
    W untimed then K timed CPU MSMs over the same 2^20-point sample."""
    if rank != 0:
        return
    wall0 = time.perf_counter()
    orc = _oracle()
    sc, bases = cpu_msm_inputs(REF_LOG_N)
    threads, avail = cpu_threads()
    for _ in range(args.warmup):
        orc.msm(sc, bases, threads)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        orc.msm(sc, bases, threads)
        times.append(time.perf_counter() - t)
    n = 1 << REF_LOG_N
    value = n * len(times) / sum(times)
    srt = sorted(times)
    rows = cpu_rows(threads)
    sample = (f"each step: best_multiexp_cpu restatement (oracle/oracle.c) over a 2^{REF_LOG_N}-point sample of the "
              f"k=22 MSM (SRS points, same scalar mix); {args.steps} timed steps after {args.warmup} untimed")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(times) / len(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64-limb Montgomery Fr/Fq (exact)", "data": "synthetic (seeded SRS and scalars)",
            "config": dict(WORKLOAD, reference_step=f"CPU MSM over a 2^{REF_LOG_N}-point sample of the same "
                                                    f"workload; value is points/s over the timed steps"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "threads_available": avail,
                             "step_ms": {"min": round(srt[0] * 1e3, 2), "median": round(srt[len(srt) // 2] * 1e3, 2),
                                         "max": round(srt[-1] * 1e3, 2)}},
            "cpu_rows": rows,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": round(time.perf_counter() - wall0, 2)}
    print(json.dumps(line), flush=True)


def rows_section(h2b, torch, hbm_gbs, product_peak, k=20, reps=5):
    """Every other row of the hot path at the k = 20 proof size, timed with
    CUDA events around the public entry point (as a caller would call it).
    For each: ms per call, units/s, algorithmic GB/s and its fraction of the
    measured HBM peak, and (where the product count per unit is fixed) the
    fraction of the measured field-product throughput (register-resident
    chains of the same operator*, h2b_probe_modmul)."""
    import numpy as np
    rules_mod = importlib.util.spec_from_file_location("h2b_rules", os.path.join(ROOT, "halo2-gpu_b200", "rules.py"))
    R = importlib.util.module_from_spec(rules_mod)
    rules_mod.loader.exec_module(R)
    f = h2b.fields
    L = h2b.lib()
    n = 1 << k
    side = torch.cuda.Stream()
    rnd = lambda m, s: h2b.random_fr_device(m, s, 0)  # noqa: E731
    out = {}

    def timed(name, fn, units, unit, bytes_per_unit, products_per_unit=None):
        with torch.cuda.stream(side):
            fn()
            side.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(side)
            for _ in range(reps):
                fn()
            e1.record(side)
        side.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gbs = units * bytes_per_unit / (ms * 1e-3) / 1e9
        r = {"ms": round(ms, 4), f"{unit}_per_s": units / (ms * 1e-3), "GB_per_s": round(gbs, 1),
             "hbm_frac": round(gbs / hbm_gbs, 4)}
        if products_per_unit:
            r["product_frac"] = round(units * products_per_unit / (ms * 1e-3) / product_peak, 4)
        out[name] = r

    # a7: quotient evaluator, PLONK + Fibonacci gates over one extended part (rot_scale 4)
    g = R.Graph()
    parts = R.plonk_and_fibonacci(g)
    rules = np.array(g.rules, dtype=np.uint64)
    prods = sum(1 for i in range(0, len(rules), 2) if (int(rules[i]) >> 44) & 1) + len(parts)
    fixed, inst, adv = [rnd(n, 10 + i) for i in range(3)], [rnd(n, 20)], [rnd(n, 30 + i) for i in range(4)]
    ch = f.fr_mont_limbs([0xC4A1])
    consts = f.fr_mont_limbs(g.constants)
    vp = np.array(parts, dtype=np.uint64)
    d_q = h2b.dev_empty(32 * n)
    timed("quotient_plonk_fib", lambda: h2b.quotient_device(fixed, inst, adv, ch, consts, 0x1234, rules, vp, n, 4, 0,
                                                            n, d_q, None, stream=side),
          n, "rows", 9 * 32, prods)
    # a8: permutation quotient (4 columns, chunk 2 -> 2 sets)
    vals, l0, ll, la = (rnd(n, 40 + i) for i in range(4))
    pprods, perms, cols = [rnd(n, 50 + i) for i in range(2)], [rnd(n, 60 + i) for i in range(4)], \
        [rnd(n, 70 + i) for i in range(4)]
    sc = lambda s: f.fr_mont_limbs([s])  # noqa: E731
    dom = f.EvaluationDomain(4, k)
    timed("permutation_quotient_4col", lambda: h2b.quotient_permutation_device(
        vals, l0, ll, la, pprods, perms, cols, sc(3), sc(5), sc(7), f.fr_mont_limbs([f.DELTA]), sc(11),
        f.fr_mont_limbs([pow(dom.extended_omega, 3, f.R_MOD)]), f.fr_mont_limbs([dom.extended_omega]), 2, -5, 4, n, n,
        stream=side), n, "rows", 15 * 32)
    # a9: lookup quotient
    arrs = [rnd(n, 80 + i) for i in range(8)]
    d_b, d_g, d_y = (h2b.to_dev(sc(s)) for s in (3, 5, 7))
    timed("lookup_quotient", lambda: h2b.quotient_lookups_device(*arrs, d_b, d_g, d_y, n, stream=side), n, "rows",
          9 * 32)
    # a7-a9 together on one config-3 extended part: the reference's four per-part
    # launches (gates, permutation, lookup expression, lookup constraints)
    # against one h2b_quotient_fused launch; 20 arrays of 32 B per row are read
    # once and one written by the fused pass (3 fixed, instance, 4 advice,
    # 4 sigma, l0 / l_last / l_active, 2 permutation products, the lookup
    # product and A' / S')
    C = importlib.import_module(h2b.__name__ + ".circuit")
    g_rules, g_parts, g_consts = C.gate_graph()
    l_rules, l_parts, l_consts = C.lookup_product_graph()
    qf, qi, qa = [rnd(n, 200 + i) for i in range(3)], [rnd(n, 210)], [rnd(n, 220 + i) for i in range(4)]
    zs, sg = [rnd(n, 230 + i) for i in range(2)], [rnd(n, 240 + i) for i in range(4)]
    zl, pa, ps = (rnd(n, 250 + i) for i in range(3))
    lag3 = [rnd(n, 260 + i) for i in range(3)]
    beta, gamma, yv = 0x1234567, 0x7654321, 0xABCDEF
    pcols = [qa[0], qa[1], qa[2], qi[0]]
    shift = pow(dom.extended_omega, 3, f.R_MOD)
    dstart = beta * f.ZETA % f.R_MOD
    bg = f.fr_mont_limbs([beta, gamma])
    hj, tv, fo = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
    d_bt, d_gm, d_yv = (h2b.to_dev(sc(s)) for s in (beta, gamma, yv))
    last = -(C.BLINDING_FACTORS + 1)

    def chain():
        h2b.quotient_device(qf, qi, qa, [], g_consts, yv, g_rules, g_parts, n, 1, 0, n, hj, stream=side)
        h2b.quotient_permutation_device(hj, *lag3, zs, sg, pcols, beta, gamma, yv, f.DELTA, dstart, shift, dom.omega,
                                        C.CHUNK_LEN, last, 1, n, n, stream=side)
        h2b.quotient_device(qf, qi, qa, bg, l_consts, yv, l_rules, l_parts, n, 1, 0, n, tv, stream=side)
        h2b.quotient_lookups_device(hj, tv, zl, pa, ps, *lag3, d_bt, d_gm, d_yv, n, stream=side)

    perm = dict(prods=zs, sigmas=sg, cols=pcols, beta=beta, gamma=gamma, delta=f.DELTA, delta_start=dstart,
                ext_omega=shift, omega=dom.omega, chunk_len=C.CHUNK_LEN, last_rotation=last, rot_scale=1, isize=n)
    look = [dict(rules=(bg, l_consts, l_rules, l_parts), z=zl, pin=pa, ptab=ps, beta=beta, gamma=gamma)]
    no_ch = np.zeros((0, 4), np.uint64)
    timed("quotient_part_chain", chain, n, "rows", 21 * 32)
    timed("quotient_part_fused", lambda: h2b.quotient_fused_device(
        qf, qi, qa, (no_ch, g_consts, g_rules, g_parts), yv, *lag3, perm, look, n, 1, 0, n, fo, stream=side),
        n, "rows", 21 * 32)
    torch.cuda.synchronize()
    out["quotient_part_fused"]["identical_to_chain"] = bool(torch.equal(hj, fo))
    out["quotient_part_fused"]["speedup_over_chain"] = round(out["quotient_part_chain"]["ms"] /
                                                             out["quotient_part_fused"]["ms"], 3)
    # a10: permutation grand product (4 columns)
    mod = rnd(n, 90)
    pv, pp = [rnd(n, 91 + i) for i in range(4)], [rnd(n, 95 + i) for i in range(4)]
    d_delta, d_om, d_dw = h2b.to_dev(f.fr_mont_limbs([f.DELTA])), h2b.to_dev(f.fr_mont_limbs([dom.omega])), \
        h2b.to_dev(sc(1))
    timed("permutation_product_4col", lambda: h2b.permutation_product_device(
        mod, pp, pv, d_b, d_g, d_delta, d_om, d_dw, n, stream=side), n, "rows", 9 * 32 + 32)
    # a11: lookup grand product
    lo = h2b.dev_empty(32 * n)
    lk = [rnd(n, 100 + i) for i in range(4)]
    timed("lookup_product", lambda: h2b.lookup_product_device(lo, *lk, d_b, d_g, n, stream=side), n, "rows", 5 * 32)
    # grand product scan
    gp = rnd(n, 110)
    d_pre = h2b.to_dev(sc(1))
    timed("grand_product", lambda: h2b.grand_product_device(gp, d_pre, n, stream=side), n, "elements", 64, 2)
    # a12: batch inversion at the proof size
    bi = rnd(n, 120)
    bws = h2b.dev_empty(L.h2b_batch_invert_workspace_size(n))
    timed("batch_invert", lambda: h2b.call("h2b_batch_invert", h2b.ptr(bi), 0, n, h2b.ptr(bws), bws.numel(),
                                           h2b.stream_handle(side)), n, "elements", 64, 4)
    # a13: lookup permute-sort, 2^8-entry table
    tab = rnd(256, 130)
    idx = torch.randint(0, 256, (n,), device="cuda")
    d_in = tab.view(256, 32)[idx].reshape(-1).contiguous()
    d_pa, d_ps = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
    d_tab = torch.zeros(32 * n, dtype=torch.uint8, device="cuda")
    d_tab[: 32 * 256] = tab
    pws = h2b.dev_empty(L._halo2_permute_expression_pair_workspace_size(n, n - 10))
    timed("permute_pair_t256", lambda: h2b.call("_halo2_permute_expression_pair", h2b.ptr(d_in), h2b.ptr(d_tab),
                                                h2b.ptr(d_pa), h2b.ptr(d_ps), n, n - 10, h2b.ptr(pws), pws.numel(),
                                                h2b.stream_handle(side)), n, "rows", 4 * 32)
    # a5: coset extension parts (CosetFFT_Part) for 8 polynomials, one part
    polys = [rnd(n, 140 + i) for i in range(8)]
    outs = [h2b.dev_empty(32 * n) for _ in polys]
    cf = f.ZETA * dom.extended_omega % f.R_MOD
    nws = h2b.dev_empty(L._halo2_fft_many_to_device_workspace_size(6, k, k))
    timed("coset_part_ntt_x8", lambda: h2b.fft_many_to_device(6, k, k, polys, outs, dom.omega, cf, ws=nws,
                                                              stream=side), 8 * n, "elements", 64, k / 2 + 1)
    # a6: divide_by_vanishing over the extended domain (4 * 2^k)
    ext = rnd(4 * n, 150)
    d_t = h2b.to_dev(f.fr_mont_limbs(dom.t_evaluations))
    timed("divide_by_vanishing_ext", lambda: h2b.call("_halo2_divide_by_vanishing_poly", h2b.ptr(ext), h2b.ptr(d_t),
                                                      len(dom.t_evaluations), 4 * n, h2b.stream_handle(side)),
          4 * n, "elements", 64, 1)
    # opening: Kate division and Horner evaluation
    a = rnd(n, 160)
    dqq = h2b.dev_empty(32 * n)
    d_u = h2b.to_dev(sc(0xABCDEF))
    timed("kate_division", lambda: h2b.kate_division_device(a, dqq, d_u, n, stream=side), n, "coefficients", 64, 5)
    ews = h2b.dev_empty(L._halo2_eval_polynomial_workspace_size(n))
    pt = f.fr_mont_limbs([0x5A5A5A])
    res = ctypes.c_void_p()
    timed("eval_polynomial", lambda: h2b.call("_halo2_eval_polynomial", h2b.ptr(a), ctypes.byref(h2b.host_ffi(pt)),
                                              ctypes.byref(res), n, h2b.ptr(ews), ews.numel(),
                                              h2b.stream_handle(side)), n, "coefficients", 32, 1.5)
    # twiddles: omega^i for i < 2^k
    tw = h2b.dev_empty(32 * n)
    d_w = h2b.to_dev(f.fr_mont_limbs([dom.omega]))
    tws = h2b.dev_empty(L._halo2_generate_omega_powers_workspace_size(k))
    timed("omega_powers", lambda: h2b.call("_halo2_generate_omega_powers", h2b.ptr(tw), h2b.ptr(d_w), k,
                                           h2b.ptr(tws), tws.numel(), h2b.stream_handle(side)), n, "elements", 32)
    return {"k": k, "rows": out}


def table_section(h2b, torch, d_srs, d_sc, n, reps):
    """The same k=22 MSM over the SRS kept resident with its window multiples
    (h2b_msm_table_precompute once, then h2b_msm_device_table): one bucket
    set for all windows and no final doubling chain.  The result must equal
    the plain MSM's."""
    side = torch.cuda.Stream()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    with torch.cuda.stream(side):
        e[0].record(side)
        table = h2b.msm_table_precompute(d_srs, n, stream=side)
        e[1].record(side)
        ws = h2b.dev_empty(h2b.lib().h2b_msm_table_workspace_size(n, n))
        out_t, out_p = h2b.dev_empty(96), h2b.dev_empty(96)
        h2b.msm_device(d_sc, d_srs, out_p, n, h2b.msm_workspace(n), stream=side)
        for _ in range(2):
            h2b.msm_device_table(d_sc, table, n, out_t, n, ws=ws, stream=side)
        e[2].record(side)
        for _ in range(reps):
            h2b.msm_device_table(d_sc, table, n, out_t, n, ws=ws, stream=side)
        e[3].record(side)
    side.synchronize()
    ms = e[2].elapsed_time(e[3]) / reps
    same = out_t.cpu().numpy().tobytes() == out_p.cpu().numpy().tobytes()
    res = {"ms": ms, "points_per_s": n / (ms * 1e-3), "precompute_ms": e[0].elapsed_time(e[1]),
           "table_GB": table.numel() / 1e9, "identical_to_plain": same}
    del table, ws
    torch.cuda.empty_cache()
    return res


def serving_section(h2b, torch, count=24, slots=4, kmax=22, seed=9, loads=(0.5, 1.0, 1.5)):
    """The config-3 circuit's prover (halo2-gpu_b200/prover.py: a satisfying
    witness synthesised on the device, create_proof's phases with the
    Fiat-Shamir transcript, the SHPLONK opening; every proof verifies) served
    from one GPU.  The service time of one request alone is measured first
    for each k (untimed warm-up request before it; the median of three
    single requests), and the first of those proofs is verified
    (verify.verify_proof, untimed); `prove_k20` is the k = 20 time as
    proofs/s.  Then, for each load factor, a seeded Poisson trace of `count`
    requests with k in {16, 18, 20, 22} (weights .4/.3/.2/.1) arrives at
    load x the rate the one-at-a-time prover sustains, and runs plain (one
    slot) and served (`slots` worker streams under an HBM budget that counts
    the resident state).  Reports proofs/s over the makespan, p50/p99 latency
    (arrival to completion, host clock) and the device-memory high-water mark
    of the run.  `concurrency_by_k` times a burst of same-k requests plain and
    served; with each k's share of the plain prover's time it gives the
    served/plain gain the mixed trace can reach at saturation."""
    P = importlib.import_module(h2b.__name__ + ".prover")
    V = importlib.import_module(h2b.__name__ + ".verify")
    res = P.Resident(h2b, kmax)
    ks, weights = (16, 18, 20, 22), (0.4, 0.3, 0.2, 0.1)
    budget = 120 << 30
    plain = P.Server(res, 1, budget, transcript=True)
    served = P.Server(res, slots, budget, transcript=True)
    service, verified = {}, {}
    for k in ks:
        plain.serve([(0.0, k, 7 + k)])
        torch.cuda.reset_peak_memory_stats()
        r = plain.serve([(0.0, k, 8 + k)], keep_outputs=True)
        # the service time alone: median of three single requests (one alone is noisy)
        lat = sorted([float(r["latency_s"][0])] + [float(plain.serve([(0.0, k, 20 + k + j)])["latency_s"][0])
                                                  for j in range(2)])
        service[k] = (lat[1], torch.cuda.max_memory_allocated() / 1e9)
        _, _, proof, public = r["outputs"][0]
        verified[str(k)] = bool(V.verify_proof(res.verifying_key(k), public, proof, res.verifier_params()))
    served.serve([(0.0, k, 9 + k) for k in ks for _ in range(slots)])   # untimed: every worker's pools warm
    mean_s = sum(w * service[k][0] for k, w in zip(ks, weights))
    # what concurrency buys per k: a burst of same-k requests one at a time
    # against the worker streams; with each k's share of the plain prover's
    # time this bounds the served/plain gain of the mixed trace
    conc = {}
    for k in ks:
        burst = [(0.0, k, 300 + 10 * k + i) for i in range(8 if k < 22 else 4)]
        t_plain = plain.serve(burst)["makespan_s"]
        t_served = served.serve(burst)["makespan_s"]
        conc[str(k)] = {"requests": len(burst), "plain_s": round(t_plain, 4), "served_s": round(t_served, 4),
                        "speedup": round(t_plain / t_served, 3)}
    share = {k: w * service[k][0] / mean_s for k, w in zip(ks, weights)}
    bound = 1.0 / sum(share[k] / conc[str(k)]["speedup"] for k in ks)
    out = {"requests": count, "slots": slots, "hbm_budget_GB": budget >> 30,
           "resident_GB": round(res.device_bytes() / 1e9, 2),
           "service_ms_alone": {str(k): round(v[0] * 1e3, 2) for k, v in service.items()},
           "proof_verifies": verified,
           "prove_k20": {"proofs_per_s": round(1.0 / service[20][0], 3), "ms": round(service[20][0] * 1e3, 2),
                         "hbm_peak_GB": round(service[20][1], 2)},
           "capacity_plain_per_s": round(1.0 / mean_s, 3),
           "concurrency_by_k": conc, "plain_time_share_by_k": {str(k): round(v, 3) for k, v in share.items()},
           "served_over_plain_bound_from_bursts": round(bound, 3), "loads": {}}
    for load in loads:
        reqs = P.requests(count, load / mean_s, seed, ks, weights)
        row = {"arrival_rate_per_s": round(load / mean_s, 3)}
        for name, srv in (("plain", plain), ("served", served)):
            torch.cuda.reset_peak_memory_stats()
            util = UtilSampler(torch.cuda.current_device()).start()
            row[name] = P.summary(reqs, srv.serve(reqs))
            row[name]["gpu_utilisation"] = util.stop()
            row[name]["hbm_peak_GB"] = round(torch.cuda.max_memory_allocated() / 1e9, 2)
        out["loads"][str(load)] = row
    plain.close()
    served.close()
    return out


def batch_section(h2b, torch, n_jobs=64, streams=16, reps=3, seed=4):
    """Batched jobs of uneven size (the 64-job configuration): n_jobs jobs with
    k drawn from {14, 16, 18, 20} (weights .4/.3/.2/.1, seeded); each job is
    one MSM with uniform scalars against a shared 2^20 SRS, one forward Fr
    NTT of its 2^k polynomial, one coset extension 2^k -> 2^(k+2), and one
    evaluation of the config-3 gate set (PLONK + Fibonacci gates, rules.py)
    over that extended coset (rot_scale 4; the job's extension as its advice
    columns, fixed and instance columns shared per k).  Plain: one job after
    another on one stream (h2b_msm_device, _halo2_fft_many_to_device per
    transform, the resident quotient program).  Batched: the NTTs of all jobs
    of one size as one launch per transform type (up to 32 polynomials each)
    on that size's forked stream, followed there by the size's quotient
    runs; the MSMs through h2b_msm_batch over the forked streams; captured
    once into a CUDA graph and replayed.  Outputs of both must be identical;
    times are CUDA events."""
    import random
    import numpy as np
    f = h2b.fields
    L = h2b.lib()
    spec = importlib.util.spec_from_file_location("h2b_rules_b", os.path.join(ROOT, "halo2-gpu_b200", "rules.py"))
    R = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(R)
    rng = random.Random(seed)
    ks = rng.choices([14, 16, 18, 20], weights=[4, 3, 2, 1], k=n_jobs)
    sizes = sorted(set(ks))
    srs = h2b.srs_device(0x5EED20, 1 << 20)
    d_sc = [h2b.random_fr_device(1 << k, 5000 + i, 0) for i, k in enumerate(ks)]
    d_in = [h2b.random_fr_device(1 << k, 6000 + i, 0) for i, k in enumerate(ks)]
    outs = {name: [h2b.dev_empty(sz(k)) for k in ks] for name, sz in
            (("msm", lambda k: 96), ("fwd", lambda k: 32 << k), ("ext", lambda k: 32 << (k + 2)),
             ("q", lambda k: 32 << (k + 2)))}
    plain_outs = {name: [h2b.dev_empty(t.numel()) for t in v] for name, v in outs.items()}
    doms = {k: f.EvaluationDomain(3, k) for k in sizes}
    one = f.fr_mont_limbs([1])
    one_ffi = h2b.host_ffi(one)
    d_om = {k: h2b.to_dev(f.fr_mont_limbs([doms[k].omega])) for k in sizes}
    d_omx = {k: h2b.to_dev(f.fr_mont_limbs([doms[k].extended_omega])) for k in sizes}
    # the gate set and its shared columns per size
    g = R.Graph()
    vps = np.array(R.plonk_and_fibonacci(g), dtype=np.uint64)
    rules = np.array(g.rules, dtype=np.uint64)
    consts = f.fr_mont_limbs(g.constants)
    chal = f.fr_mont_limbs([0xC4A11])
    shared = {k: ([h2b.random_fr_device(1 << (k + 2), 7000 + 10 * k + j, 0) for j in range(3)],
                  [h2b.random_fr_device(1 << (k + 2), 7005 + 10 * k, 0)]) for k in sizes}
    progs = {}
    for which in ("batched", "plain"):
        ext = outs["ext"] if which == "batched" else plain_outs["ext"]
        progs[which] = [h2b.ResidentQuotient(shared[k][0], shared[k][1], [ext[i]] * 4, chal, consts, 0x1234567,
                                             rules, vps, 1 << (k + 2), 4) for i, k in enumerate(ks)]
    side = torch.cuda.Stream()
    ws1 = {k: h2b.dev_empty(L._halo2_fft_many_to_device_workspace_size(1, k, k)) for k in sizes}
    ws3 = {k: h2b.dev_empty(L._halo2_fft_many_to_device_workspace_size(3, k, k + 2)) for k in sizes}
    msm_ws = h2b.msm_workspace(1 << max(ks))

    def ntt_many(typ, k, ins, outs_, st):
        for c in range(0, len(ins), 32):
            a, b = ins[c:c + 32], outs_[c:c + 32]
            om = d_om[k] if typ == 1 else d_omx[k]
            ws = ws1[k] if typ == 1 else ws3[k]
            h2b.call("_halo2_fft_many_to_device", typ, len(a), k, k + 2 if typ == 3 else k,
                     h2b.ffi_array([t.data_ptr() for t in a]), h2b.ffi_array([t.data_ptr() for t in b]),
                     h2b.ptr(om), ctypes.byref(one_ffi), True, h2b.ptr(ws), ws.numel(), h2b.stream_handle(st))

    def plain():
        for i, k in enumerate(ks):
            h2b.call("h2b_msm_device", h2b.ptr(d_sc[i]), h2b.ptr(srs), h2b.ptr(plain_outs["msm"][i]), 1 << k,
                     h2b.ptr(msm_ws), msm_ws.numel(), h2b.stream_handle(side))
            ntt_many(1, k, [d_in[i]], [plain_outs["fwd"][i]], side)
            ntt_many(3, k, [d_in[i]], [plain_outs["ext"][i]], side)
            progs["plain"][i].run(plain_outs["q"][i], stream=side)

    groups = {k: [i for i in range(n_jobs) if ks[i] == k] for k in sizes}

    def batched(bases, table_n=0, merged=False):
        subs = h2b.exec_fork(streams, side)
        for gi, k in enumerate(sorted(sizes, reverse=True)):
            st = subs[gi]
            idx = groups[k]
            ntt_many(1, k, [d_in[i] for i in idx], [outs["fwd"][i] for i in idx], st)
            ntt_many(3, k, [d_in[i] for i in idx], [outs["ext"][i] for i in idx], st)
            for i in idx:
                progs["batched"][i].run(outs["q"][i], stream=st)
        jobs = h2b.msm_batch_jobs(d_sc, [bases] * n_jobs, outs["msm"], [1 << k for k in ks], table_n=table_n)
        if merged:
            # all 64 MSMs as one run over the table, beside the transforms
            h2b.msm_merged(jobs, n_jobs, bws["merged"], stream=subs[len(sizes)])
            h2b.exec_join(streams, side)
        else:
            h2b.msm_batch(jobs, n_jobs, streams, bws[table_n], stream=side)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(side)
        for _ in range(reps):
            fn()
        e1.record(side)
        side.synchronize()
        return e0.elapsed_time(e1) / reps

    def graph_time(bases, table_n=0, merged=False):
        batched(bases, table_n, merged)      # warm-up: forked streams, kernels loaded
        side.synchronize()
        gr = h2b.Graph(side)
        gr.begin()
        batched(bases, table_n, merged)
        gr.end()
        try:
            gr.launch(side)
            side.synchronize()
            return timed(lambda: gr.launch(side))
        finally:
            gr.close()

    def identical():
        torch.cuda.synchronize()
        return all(torch.equal(outs[nm][i], plain_outs[nm][i]) for nm in outs for i in range(n_jobs))

    jobs0 = h2b.msm_batch_jobs(d_sc, [srs] * n_jobs, outs["msm"], [1 << k for k in ks])
    bws = {0: h2b.msm_batch_workspace(jobs0, n_jobs, streams)}
    plain()
    side.synchronize()
    t_plain = timed(plain)
    t_streams = timed(lambda: batched(srs))
    t_graph = graph_time(srs)
    same = identical()
    # served form: the shared SRS kept resident with its window multiples
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(side)
    table = h2b.msm_table_precompute(srs, 1 << 20, stream=side)
    e1.record(side)
    side.synchronize()
    t_pre = e0.elapsed_time(e1)
    for o in outs["msm"]:
        o.zero_()
    jobs_t = h2b.msm_batch_jobs(d_sc, [table] * n_jobs, outs["msm"], [1 << k for k in ks], table_n=1 << 20)
    bws[1 << 20] = h2b.msm_batch_workspace(jobs_t, n_jobs, streams)
    t_table = graph_time(table, 1 << 20)
    same = same and identical()
    # the 64 MSMs over the table as one merged run (h2b_msm_merged)
    for o in outs["msm"]:
        o.zero_()
    bws["merged"] = h2b.dev_empty(h2b.msm_merged_workspace_bytes(jobs_t, n_jobs))
    t_merged = graph_time(table, 1 << 20, merged=True)
    same = same and identical()
    return {"workload": f"{n_jobs} jobs, k in {{14,16,18,20}} w .4/.3/.2/.1 (seed {seed}): MSM vs shared 2^20 SRS "
                        f"+ forward NTT + coset extension x4 + config-3 gate quotient over the extended coset",
            "k_counts": {k: ks.count(k) for k in sizes},
            "msm_points": sum(1 << k for k in ks), "streams": streams,
            "plain_ms": t_plain, "batched_streams_ms": t_streams, "batched_graph_ms": t_graph,
            "plain_jobs_per_s": n_jobs / (t_plain * 1e-3), "batched_jobs_per_s": n_jobs / (t_graph * 1e-3),
            "speedup": t_plain / t_graph, "table_precompute_ms": t_pre, "batched_table_graph_ms": t_table,
            "batched_table_jobs_per_s": n_jobs / (t_table * 1e-3), "table_speedup": t_plain / t_table,
            "batched_table_merged_graph_ms": t_merged, "batched_table_merged_jobs_per_s": n_jobs / (t_merged * 1e-3),
            "table_merged_speedup": t_plain / t_merged, "identical_outputs": same}


def run_case(args):
    """One kernel family at 2^log_n, warmup + steps, nothing else (for ncu)."""
    import torch
    torch.cuda.set_device(0)
    h2b = load_pkg()
    L = h2b.lib()
    f = h2b.fields
    sh = h2b.stream_handle()
    n = 1 << args.log_n
    if args.case == "permute":
        tab = h2b.random_fr_device(256, 130, 0)
        d_tab = torch.zeros(32 * n, dtype=torch.uint8, device="cuda")
        d_tab[: 32 * 256] = tab
        idx = torch.randint(0, 256, (n,), device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
        d_in = tab.view(256, 32)[idx].reshape(-1).contiguous()
        d_pa, d_ps = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
        pws = h2b.dev_empty(L._halo2_permute_expression_pair_workspace_size(n, n - 10))
        fn = lambda: h2b.call("_halo2_permute_expression_pair", h2b.ptr(d_in), h2b.ptr(d_tab),  # noqa: E731
                              h2b.ptr(d_pa), h2b.ptr(d_ps), n, n - 10, h2b.ptr(pws), pws.numel(), sh)
    elif args.case == "probe":
        sink = h2b.dev_empty(4 * 148 * 64)
        fn = lambda: h2b.call("h2b_probe_modmul", 148 * 8, 256, 64, h2b.ptr(sink), sh)  # noqa: E731
    elif args.case == "msm":
        d_srs = h2b.srs_device(0x5EED, n)
        d_sc = h2b.random_fr_device(n, 1000, 1)
        d_out = h2b.dev_empty(96)
        ws = h2b.msm_workspace(n)
        fn = lambda: h2b.call("h2b_msm_device", h2b.ptr(d_sc), h2b.ptr(d_srs), h2b.ptr(d_out), n, h2b.ptr(ws),
                              ws.numel(), sh)
    elif args.case == "ntt":
        dom = f.EvaluationDomain(5, args.log_n)
        ek = dom.extended_k
        d_in = h2b.random_fr_device(n, 2000, 0)
        d_ext = h2b.dev_empty(32 << ek)
        ws = h2b.dev_empty(L._halo2_fft_many_to_device_workspace_size(3, args.log_n, ek))
        d_om = h2b.to_dev(f.fr_mont_limbs([dom.extended_omega]))
        one = f.fr_mont_limbs([1])
        one_ffi = h2b.host_ffi(one)
        ins, outs = h2b.ffi_array([d_in.data_ptr()]), h2b.ffi_array([d_ext.data_ptr()])
        fn = lambda: h2b.call("_halo2_fft_many_to_device", 3, 1, args.log_n, ek, ins, outs, h2b.ptr(d_om),
                              ctypes.byref(one_ffi), True, h2b.ptr(ws), ws.numel(), sh)
    elif args.case == "quotient":
        # one config-3 extended part through h2b_quotient_fused
        C = importlib.import_module(h2b.__name__ + ".circuit")
        import numpy as np
        g_rules, g_parts, g_consts = C.gate_graph()
        l_rules, l_parts, l_consts = C.lookup_product_graph()
        rnd = lambda s: h2b.random_fr_device(n, s, 0)  # noqa: E731
        qf, qi, qa = [rnd(200 + i) for i in range(3)], [rnd(210)], [rnd(220 + i) for i in range(4)]
        lag3 = [rnd(260 + i) for i in range(3)]
        dom = f.EvaluationDomain(4, args.log_n)
        perm = dict(prods=[rnd(230), rnd(231)], sigmas=[rnd(240 + i) for i in range(4)],
                    cols=[qa[0], qa[1], qa[2], qi[0]], beta=3, gamma=5, delta=f.DELTA, delta_start=11,
                    ext_omega=dom.extended_omega, omega=dom.omega, chunk_len=C.CHUNK_LEN,
                    last_rotation=-(C.BLINDING_FACTORS + 1), rot_scale=1, isize=n)
        look = [dict(rules=(f.fr_mont_limbs([3, 5]), l_consts, l_rules, l_parts), z=rnd(250), pin=rnd(251),
                     ptab=rnd(252), beta=3, gamma=5)]
        gates = (np.zeros((0, 4), np.uint64), g_consts, g_rules, g_parts)
        d_out = h2b.dev_empty(32 * n)
        fn = lambda: h2b.quotient_fused_device(qf, qi, qa, gates, 7, *lag3, perm, look, n, 1, 0, n,  # noqa: E731
                                               d_out)
    else:
        d = h2b.random_fr_device(n, 3000, 0)
        ws = h2b.dev_empty(L.h2b_batch_invert_workspace_size(n))
        fn = lambda: h2b.call("h2b_batch_invert", h2b.ptr(d), 0, n, h2b.ptr(ws), ws.numel(), sh)
    for _ in range(args.warmup + args.steps):
        fn()
    torch.cuda.synchronize()
    print(json.dumps({"case": args.case, "log_n": args.log_n, "runs": args.warmup + args.steps}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-jobs section")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-prover section")
    ap.add_argument("--case", choices=["msm", "ntt", "bi", "serve", "probe", "rows", "batch", "permute", "quotient",
                                       "prove", "table_widths"],
                    help="run one kernel family (profiling runs) or the served-prover section only")
    ap.add_argument("--log-n", type=int, default=21, help="size for --case")
    ap.add_argument("--widths", default="10,12,13,14,15,16,17,18",
                    help="window widths for --case table_widths")
    ap.add_argument("--tables", default="10,11,12,13,14,15,16,17,18,19,20",
                    help="log2 table sizes for --case table_widths")
    ap.add_argument("--requests", type=int, default=24, help="requests per trace for --case serve")
    ap.add_argument("--loads", default="0.5,1.0,1.5", help="load factors (x plain capacity) for --case serve")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the built-in MSM window / chunk and NTT pass settings (no autotuner)")
    args = ap.parse_args()
    if args.case == "batch":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"case": "batch", "batch": batch_section(load_pkg(), torch)}))
        return
    if args.case == "rows":
        import torch
        torch.cuda.set_device(0)
        h2b = load_pkg()
        sink = h2b.dev_empty(4 * 148 * 64)
        sh = h2b.stream_handle()
        h2b.call("h2b_probe_modmul", 148 * 8, 256, 8, h2b.ptr(sink), sh)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        h2b.call("h2b_probe_modmul", 148 * 8, 256, 64, h2b.ptr(sink), sh)
        e1.record()
        torch.cuda.synchronize()
        probe = 148 * 8 * 256 * 64 * 4 / (e0.elapsed_time(e1) * 1e-3)
        print(json.dumps({"case": "rows", "rows_k20": rows_section(h2b, torch, peaks()[0], probe)}))
        return
    if args.case == "serve":
        import torch
        torch.cuda.set_device(0)
        loads = tuple(float(x) for x in args.loads.split(","))
        print(json.dumps({"case": "serve", "serving": serving_section(load_pkg(), torch, count=args.requests,
                                                                      loads=loads)}))
        return
    if args.case == "table_widths":
        # MSMs over window tables (--tables, log2 sizes) built at each window
        # width (--widths): uniform and witness-mix scalars at the table's
        # size, uniform at 1/16 of it, and 2^16 uniform scalars over tables
        # above 2^18 points (a small proof's commitments over a served SRS);
        # outputs must agree across widths
        import hashlib
        import torch
        torch.cuda.set_device(0)
        h2b = load_pkg()
        L = h2b.lib()
        out_rows = {}
        for lg in [int(x) for x in args.tables.split(",")]:
            tn = 1 << lg
            srs = h2b.srs_device(0x7AB1E + lg, tn)
            scs = {(tn, 1): h2b.random_fr_device(tn, 60 + lg, 1), (tn, 0): h2b.random_fr_device(tn, 70 + lg, 0),
                   (max(tn >> 4, 1), 0): h2b.random_fr_device(max(tn >> 4, 1), 80 + lg, 0)}
            if lg > 18:
                scs[(1 << 16, 0)] = h2b.random_fr_device(1 << 16, 90 + lg, 0)
            ref = {}
            for c in [int(x) for x in args.widths.split(",")]:
                L.h2b_msm_set_tuning(c, 0)
                table = h2b.msm_table_precompute(srs, tn)
                row = {}
                for (n, mix), sc in scs.items():
                    out = h2b.dev_empty(96)
                    ws = h2b.dev_empty(L.h2b_msm_table_workspace_size(n, tn))
                    for _ in range(2):
                        h2b.msm_device_table(sc, table, tn, out, n, ws=ws)
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(5):
                        h2b.msm_device_table(sc, table, tn, out, n, ws=ws)
                    e1.record()
                    torch.cuda.synchronize()
                    key = f"n=2^{n.bit_length() - 1} {'mix' if mix else 'uniform'}"
                    digest = hashlib.sha256(out.cpu().numpy().tobytes()).hexdigest()
                    ref.setdefault(key, digest)
                    row[key] = {"ms": round(e0.elapsed_time(e1) / 5, 3), "same": digest == ref[key]}
                out_rows[f"2^{lg} table, c={c}"] = row
                print(json.dumps({f"2^{lg} table, c={c}": row}), file=sys.stderr, flush=True)
                del table
                torch.cuda.empty_cache()
            L.h2b_msm_set_tuning(0, 0)
        print(json.dumps({"case": "table_widths", "rows": out_rows}))
        return
    if args.case == "prove":
        # config-3 proofs at 2^log_n one after another (transcript on), for
        # launch lists of a whole proof: warmup untimed, then steps timed
        import torch
        torch.cuda.set_device(0)
        h2b = load_pkg()
        P = importlib.import_module(h2b.__name__ + ".prover")
        res = P.Resident(h2b, args.log_n)
        res.key_cosets(args.log_n)
        res.lagrange_table(args.log_n)
        st = torch.cuda.Stream()
        ms = []
        for i in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            if i == args.warmup:
                torch.cuda.profiler.start()   # `ncu --profile-from-start off` sees the timed proofs only
            t0 = time.perf_counter()
            P.ProofWorkload(res, args.log_n, 500 + i, transcript=True).run(st)
            st.synchronize()
            if i >= args.warmup:
                ms.append(round((time.perf_counter() - t0) * 1e3, 2))
        torch.cuda.profiler.stop()
        print(json.dumps({"case": "prove", "log_n": args.log_n, "proof_ms": ms}))
        return
    if args.case:
        run_case(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    h2b = load_pkg()
    L = h2b.lib()
    f = h2b.fields
    stream = torch.cuda.current_stream()
    sh = h2b.stream_handle(stream)

    # ---- setup (untimed) ----
    n_msm, n_ntt, n_ext, n_bi = 1 << K_MSM, 1 << K_NTT, 1 << K_EXT, 1 << K_BI
    dom = f.EvaluationDomain(5, K_NTT)
    assert dom.extended_k == K_EXT
    d_srs = h2b.srs_device(0x5EED + 0x1000 * rank, n_msm)
    # per-(op, k) settings from the autotuner's cache for this GPU and build
    # (tuned here when absent), before any scratch is sized
    tuning = None
    if not args.no_tune:
        at = importlib.import_module("halo2_gpu_b200.autotune")
        r = at.autotune(h2b, msm_ks=(14, 16, 18, 20, 22), ntt_ks=tuple(range(14, 25)), d_bases=d_srs)
        tuning = {"cache": "tuned" if r["tuned"] else "cached", "key": r["key"],
                  "msm": {k: {x: e[x] for x in ("window", "chunk", "auto_window", "ms", "auto_ms")}
                          for k, e in r["msm"].items()},
                  "ntt": {k: {x: e[x] for x in ("stages", "auto_stages", "ms", "auto_ms")} for k, e in r["ntt"].items()}}
    d_sc = h2b.random_fr_device(n_msm, 1000 + rank, 1)
    d_ntt_in = h2b.random_fr_device(n_ntt, 2000 + rank, 0)
    d_ext = h2b.dev_empty(32 * n_ext)
    d_bi = h2b.random_fr_device(n_bi, 3000 + rank, 0)
    d_msm_out = h2b.dev_empty(96)
    ws_msm = h2b.msm_workspace(n_msm)
    ws_ntt = h2b.dev_empty(L._halo2_fft_many_to_device_workspace_size(3, K_NTT, K_EXT))
    ws_bi = h2b.dev_empty(L.h2b_batch_invert_workspace_size(n_bi))
    d_om = h2b.to_dev(f.fr_mont_limbs([dom.extended_omega]))
    one = f.fr_mont_limbs([1])
    one_ffi = h2b.host_ffi(one)
    ins = h2b.ffi_array([d_ntt_in.data_ptr()])
    outs = h2b.ffi_array([d_ext.data_ptr()])
    d_cnt = h2b.dev_empty(8)
    h2b.call("h2b_msm_count_entries", h2b.ptr(d_sc), n_msm, h2b.ptr(d_cnt), sh)
    torch.cuda.synchronize()
    entries = int(d_cnt.cpu().numpy().view("uint64")[0])

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        h2b.call("h2b_msm_device", h2b.ptr(d_sc), h2b.ptr(d_srs), h2b.ptr(d_msm_out), n_msm, h2b.ptr(ws_msm),
                 ws_msm.numel(), sh)
        if ev is not None:
            ev[1].record(stream)
        h2b.call("_halo2_fft_many_to_device", 3, 1, K_NTT, K_EXT, ins, outs, h2b.ptr(d_om), ctypes.byref(one_ffi),
                 True, h2b.ptr(ws_ntt), ws_ntt.numel(), sh)
        if ev is not None:
            ev[2].record(stream)
        h2b.call("h2b_batch_invert", h2b.ptr(d_bi), 0, n_bi, h2b.ptr(ws_bi), ws_bi.numel(), sh)
        if ev is not None:
            ev[3].record(stream)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    # IMAD / modmul pipe probes (untimed), for the roofline denominators
    sink = h2b.dev_empty(4 * 148 * 64)
    probe = {}
    for name, iters, per in (("h2b_probe_imad", 4096, 16), ("h2b_probe_modmul", 64, 4)):
        h2b.call(name, 148 * 8, 256, 8, h2b.ptr(sink), sh)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h2b.call(name, 148 * 8, 256, iters, h2b.ptr(sink), sh)
        e1.record(stream)
        torch.cuda.synchronize()
        probe[name] = 148 * 8 * 256 * iters * per / (e0.elapsed_time(e1) * 1e-3)

    # ---- timed region ----
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    launches0 = L.h2b_launch_count()
    L.h2b_prof_enable(1)
    clocks = ClockSampler(local)
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    clocks.begin()
    t0.record(stream)
    for i in range(args.steps):
        step(evs[i])
    t1.record(stream)
    torch.cuda.synchronize()
    clocks.end()
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    launches = L.h2b_launch_count() - launches0
    total_ms = t0.elapsed_time(t1)
    msm_ms = sum(e[0].elapsed_time(e[1]) for e in evs) / args.steps
    ntt_ms = sum(e[1].elapsed_time(e[2]) for e in evs) / args.steps
    bi_ms = sum(e[2].elapsed_time(e[3]) for e in evs) / args.steps
    acc_ms, acc_cnt = h2b.prof_read(h2b.PROF_MSM_ACCUMULATE)
    nttp_ms, nttp_cnt = h2b.prof_read(h2b.PROF_NTT_PASSES)
    bik_ms, bik_cnt = h2b.prof_read(h2b.PROF_BATCH_INVERT)
    L.h2b_prof_enable(0)

    step_ms = total_ms / args.steps
    step_ms, msm_ms, ntt_ms, bi_ms = max_over_ranks([step_ms, msm_ms, ntt_ms, bi_ms], dist, "cuda")

    ntt_bytes = 32 * n_ntt + 32 * n_ext
    value = whole_job_points_per_s(world, n_msm, msm_ms)
    hbm, hbm_kind = peaks()
    # dominant kernel: MSM bucket accumulation (one launch per MSM)
    acc_avg_ms = acc_ms / max(acc_cnt, 1)
    acc_bytes = entries * (4 + 64) + (1 << 19) * 128          # sorted ids + affine points + bucket sums
    acc_modmul = entries * 10                                  # XYZZ mixed add 8M + 2S
    # the accumulation is bound by its field products (about 0.25 products per
    # byte of traffic), so the roofline is the FP64-form product's pipe ceiling
    sm_mhz = clk.get("sm_mhz") or 1965.0
    ceil = product_ceiling(sm_mhz)
    acc_gps = acc_modmul / (acc_avg_ms * 1e-3) / 1e9
    hbm_achieved = acc_bytes / (acc_avg_ms * 1e-3) / 1e9
    roofline = {"bound": f"{ceil['binding']} (FP64-form field products)", "kernel": "k_msm_accumulate_d",
                "achieved": acc_gps, "peak": ceil["peak_gproducts_per_s"], "unit": "G products/s",
                "frac": acc_gps / ceil["peak_gproducts_per_s"],
                "peak_source": ceil["source"], "ceilings_gproducts_per_s": ceil["ceilings"],
                "traffic": ncu_traffic("msm_accumulate_d_k22.md"),
                "products_per_launch": acc_modmul, "launch_ms": acc_avg_ms,
                "hbm": {"achieved_GB_per_s": hbm_achieved, "peak_GB_per_s": hbm,
                        "frac": hbm_achieved / hbm,
                        "peak_source": ("measured: MEASURED_PEAKS.json hbm_gbs" if hbm_kind == "measured" else
                                        "fallback: MEASURED_PEAKS.json absent, 6.65 TB/s measured earlier on this pool"),
                        "algorithmic_bytes_per_launch": acc_bytes}}
    # beside it: the same product in register-resident chains (h2b_probe_modmul)
    products = {"kernel": "k_msm_accumulate_d", "modmul_per_launch": acc_modmul,
                "achieved_products_per_s": acc_modmul / (acc_avg_ms * 1e-3),
                "peak_products_per_s": probe["h2b_probe_modmul"],
                "peak_source": "measured h2b_probe_modmul (operator*, FP64 product, four chains per thread)",
                "imad_ops_per_s_probe": probe["h2b_probe_imad"]}
    products["frac"] = products["achieved_products_per_s"] / products["peak_products_per_s"]
    ntt_kernel_ms = nttp_ms / max(nttp_cnt, 1)
    ntt_modmul = (n_ext // 2) * K_NTT   # the first K_EXT - K_NTT stages are broadcasts
    bi_kernel_ms = bik_ms / max(bik_cnt, 1)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "Montgomery Fr/Fq, exact integer (52-bit limbs in f64 for products, u32 words in memory)",
        "data": "synthetic (seeded SRS [tau^i]G and scalars; generated on device)",
        "config": dict(WORKLOAD, parallelism=f"replicas x{world}"),
        "msm": {"ms": msm_ms, "points_per_s": n_msm / (msm_ms * 1e-3), "entries": entries,
                "window_bits": L.h2b_msm_window_bits(n_msm)},
        "ntt": {"ms": ntt_ms, "GB_per_s": ntt_bytes / (ntt_ms * 1e-3) / 1e9,
                "elements_per_s": n_ext / (ntt_ms * 1e-3), "pass_kernels_ms": ntt_kernel_ms,
                "product_frac_passes": ntt_modmul / (ntt_kernel_ms * 1e-3) / probe["h2b_probe_modmul"]},
        "batch_invert": {"ms": bi_ms, "elements_per_s": n_bi / (bi_ms * 1e-3), "apply_kernel_ms": bi_kernel_ms},
        "roofline": roofline, "product_roofline": products, "clocks": clk, "gpu_launches": launches,
        "tuning": tuning,
    }

    # ---- end to end through the reference-facing C ABI with host buffers ----
    if not args.no_e2e:
        import numpy as np
        h_sc = torch.empty(32 * n_msm, dtype=torch.uint8).pin_memory()
        h_sc.copy_(d_sc.cpu())
        h_ntt = torch.empty(32 * n_ntt, dtype=torch.uint8).pin_memory()
        h_ntt.copy_(d_ntt_in.cpu())
        h_ext = torch.empty(32 * n_ext, dtype=torch.uint8).pin_memory()
        h_bi = torch.empty(32 * n_bi, dtype=torch.uint8).pin_memory()
        h_bi.copy_(d_bi.cpu())
        h_out = np.zeros(12, np.uint64)
        ws_e2e_msm = h2b.dev_empty(L._halo2_multiexp_device_bases_workspace_size(n_msm))
        ws_e2e_ntt = h2b.dev_empty(L._halo2_fft_normal_workspace_size(3, K_NTT, K_EXT))
        sc_ffi = h2b.FFITraitObject(ctypes.c_void_p(h_sc.data_ptr()))
        out_ffi = h2b.host_ffi(h_out)
        h_om = f.fr_mont_limbs([dom.extended_omega])

        def e2e_step(ev=None):
            if ev is not None:
                ev[0].record(stream)
            h2b.call("_halo2_multiexp_device_bases", ctypes.byref(sc_ffi), h2b.ptr(d_srs), ctypes.byref(out_ffi),
                     n_msm, h2b.ptr(ws_e2e_msm), ws_e2e_msm.numel(), sh)
            if ev is not None:
                ev[1].record(stream)
            h2b.call("_halo2_cosetfft", 3, K_NTT, K_EXT, ctypes.c_void_p(h_ntt.data_ptr()),
                     ctypes.c_void_p(h_ext.data_ptr()), h_om.ctypes.data, one.ctypes.data, h2b.ptr(ws_e2e_ntt),
                     ws_e2e_ntt.numel(), sh)
            d_bi.copy_(h_bi, non_blocking=True)
            h2b.call("h2b_batch_invert", h2b.ptr(d_bi), 0, n_bi, h2b.ptr(ws_bi), ws_bi.numel(), sh)
            h_bi.copy_(d_bi, non_blocking=True)
            if ev is not None:
                ev[2].record(stream)

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        eevs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
        for i in range(args.steps):
            e2e_step(eevs[i])
        torch.cuda.synchronize()
        e_msm = sum(e[0].elapsed_time(e[1]) for e in eevs) / args.steps
        e_rest = sum(e[1].elapsed_time(e[2]) for e in eevs) / args.steps
        e_step = sum(e[0].elapsed_time(e[2]) for e in eevs) / args.steps
        e_msm, e_rest, e_step = max_over_ranks([e_msm, e_rest, e_step], dist, "cuda")
        # the metric's e2e: the MSM through _halo2_multiexp_device_bases with
        # pinned host scalars (copied inside the call) and the 96-byte result
        # read back to the host; the bytes are that call's
        line["e2e"] = {"value": whole_job_points_per_s(world, n_msm, e_msm), "unit": UNIT,
                       "h2d_bytes_per_step": 32 * n_msm, "d2h_bytes_per_step": 96, "ms": e_msm,
                       "api": "_halo2_multiexp_device_bases (host scalars, resident bases, host result)",
                       "step": {"ms": e_step, "h2d_bytes": 32 * n_msm + 32 * n_ntt + 32 * n_bi,
                                "d2h_bytes": 96 + 32 * n_ext + 32 * n_bi,
                                "ntt_and_batch_invert_ms": e_rest,
                                "api": "the MSM above, then _halo2_cosetfft (host in/out) and h2b_batch_invert "
                                       "with pinned H2D/D2H"}}

    if not args.no_batch:
        line["msm_table"] = table_section(h2b, torch, d_srs, d_sc, n_msm, args.steps)
        line["rows_k20"] = rows_section(h2b, torch, hbm, probe["h2b_probe_modmul"])
        line["batch"] = batch_section(h2b, torch)
    if world == 1 and not args.no_serve:
        line["serving"] = serving_section(h2b, torch)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_msm()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
