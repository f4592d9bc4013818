"""Autotuner for the library's per-size tuning table, cached per (op, k).

The reference fixes its MSM window width by a formula of n
(halo2_proofs/cuda/src/multiexp.cu:260-300) and its NTT stage split by a
constant block size (halo2_proofs/cuda/include/kernel/ntt_combine.h:90-94).
Here those choices are entries of a table inside libhalo2_gpu.so
(h2b_tune_set / h2b_tune_get, csrc/tune.cu): for each (op, k) this module
times candidate settings on the GPU it runs on and keeps the fastest:

* op "msm", k = log2 of the MSM length: the signed-digit window width
  (automatic width - 1, automatic, + 1, within 10..16), then the sorted
  entries per accumulation chunk (automatic, 32, 64, 128, 256) at the chosen
  width.  Timed on the witness-like scalar mix (50 % uniform, 30 % < 2^64,
  20 % {0, 1}) over a prefix of a synthetic SRS.
* op "ntt", k = log2 of the transform size: stages per shared-memory pass
  (6..11; 11 only with the radix-4 pass kernel, whose tiles hold 2^11
  elements), timed on a forward FFT of uniform random coefficients; the
  setting then applies to every transform of that size (FFT, iFFT, coset
  extension passes).

Each candidate runs once untimed, then `reps` times between CUDA events on
one stream; its time is the median.  Every candidate's output must equal the
automatic setting's output bit for bit (a setting never changes results), or
the tuner raises.  A candidate replaces the automatic setting only when it is
more than `margin` (default 1 %) faster, so noise keeps the built-in choice.

Winners are stored in a JSON cache keyed by the device (name, SM count) and
the library build (SHA-1 of libhalo2_gpu.so), so a new GPU model or a new
build is tuned afresh, and are loaded into the library with h2b_tune_set.
The cache path is $H2B_TUNE_CACHE, else ~/.cache/halo2_gpu_b200/tune.json.
"""
import hashlib
import json
import os
import statistics

PARAM_WINDOW, PARAM_CHUNK, PARAM_STAGES = 0, 1, 2
WINDOW_RANGE = (10, 16)
CHUNK_CANDIDATES = (0, 32, 64, 128, 256)
STAGE_CANDIDATES = (6, 7, 8, 9, 10, 11)
CACHE_VERSION = 1


def default_cache_path():
    return os.environ.get("H2B_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "halo2_gpu_b200", "tune.json"))


def library_digest(path):
    h = hashlib.sha1()
    with open(path, "rb") as f:
        for block in iter(lambda: f.read(1 << 20), b""):
            h.update(block)
    return h.hexdigest()[:16]


def device_key(gpu_name, sm_count, lib_digest):
    return f"{gpu_name}|sm{sm_count}|lib-{lib_digest}"


def load_cache(path):
    """The cache as a dict ({"version", "devices": {key: {op: {k: entry}}}}); empty when absent or stale."""
    try:
        with open(path) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return {"version": CACHE_VERSION, "devices": {}}
    if not isinstance(d, dict) or d.get("version") != CACHE_VERSION or not isinstance(d.get("devices"), dict):
        return {"version": CACHE_VERSION, "devices": {}}
    return d


def save_cache(path, cache):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def pick(timings, auto, margin=0.01):
    """The candidate with the smallest median time; `auto` (the built-in
    setting) wins unless the best is more than `margin` faster than it.
    timings: {candidate: [ms, ...]} (must include `auto`)."""
    med = {c: statistics.median(v) for c, v in timings.items()}
    best = min(med, key=lambda c: (med[c], c != auto))
    if med[best] < med[auto] * (1.0 - margin):
        return best, med
    return auto, med


def window_candidates(auto_c):
    lo, hi = WINDOW_RANGE
    return [c for c in (auto_c - 1, auto_c, auto_c + 1) if lo <= c <= hi]


def apply_entries(set_fn, entries):
    """Loads cached entries ({op: {k: entry}}) through set_fn(param, k, value)
    (h2b_tune_set); raises if the library rejects one."""
    for k, e in entries.get("msm", {}).items():
        for param, key in ((PARAM_WINDOW, "window"), (PARAM_CHUNK, "chunk")):
            if set_fn(param, int(k), int(e.get(key, 0))) != 0:
                raise ValueError(f"tuning table rejected msm k={k} {key}={e.get(key)}")
    for k, e in entries.get("ntt", {}).items():
        if set_fn(PARAM_STAGES, int(k), int(e.get("stages", 0))) != 0:
            raise ValueError(f"tuning table rejected ntt k={k} stages={e.get('stages')}")


# --- GPU measurement ------------------------------------------------------------

def _time(torch, fn, reps):
    stream = torch.cuda.current_stream()
    fn()
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def tune_msm(h2b, k, d_bases, reps=3, margin=0.01, seed=0x7A11):
    """Chooses window width and chunk size for MSMs of 2^k points over the
    first 2^k of `d_bases`; returns the cache entry."""
    import torch
    L = h2b.lib()
    n = 1 << k
    d_sc = h2b.random_fr_device(n, seed + k, 1)
    d_out = h2b.dev_empty(96)
    L.h2b_tune_set(PARAM_WINDOW, k, 0)
    L.h2b_tune_set(PARAM_CHUNK, k, 0)
    auto_c = L.h2b_msm_window_bits(n)
    ref = None

    def run_with(c, chunk):
        nonlocal ref
        if L.h2b_tune_set(PARAM_WINDOW, k, c) != 0 or L.h2b_tune_set(PARAM_CHUNK, k, chunk) != 0:
            raise ValueError(f"tuning table rejected msm k={k} window={c} chunk={chunk}")
        ws = h2b.msm_workspace(n)
        t = _time(torch, lambda: h2b.msm_device(d_sc, d_bases, d_out, n, ws), reps)
        got = d_out.clone()
        if ref is None:
            ref = got
        elif not torch.equal(got, ref):
            raise RuntimeError(f"msm k={k}: window {c} chunk {chunk} changed the result")
        del ws
        return t

    times_c = {0: run_with(0, 0)}
    for c in window_candidates(auto_c):
        if c != auto_c:
            times_c[c] = run_with(c, 0)
    best_c, med_c = pick(times_c, 0, margin)
    times_k = {0: times_c[best_c]}
    for chunk in CHUNK_CANDIDATES:
        if chunk:
            times_k[chunk] = run_with(best_c, chunk)
    best_k, med_k = pick(times_k, 0, margin)
    L.h2b_tune_set(PARAM_WINDOW, k, best_c)
    L.h2b_tune_set(PARAM_CHUNK, k, best_k)
    return {"window": best_c, "chunk": best_k, "auto_window": auto_c, "ms": med_k[best_k], "auto_ms": med_c[0],
            "candidates_ms": {**{f"w{c or auto_c}": round(v, 4) for c, v in med_c.items()},
                              **{f"K{c or 'auto'}": round(v, 4) for c, v in med_k.items()}}}


def tune_ntt(h2b, k, reps=3, margin=0.01, seed=0x7A12):
    """Chooses the radix-2 stages per pass for transforms of 2^k points;
    returns the cache entry."""
    import torch
    from . import fields as f
    L = h2b.lib()
    n = 1 << k
    dom = f.EvaluationDomain(2, k)
    d_in = h2b.random_fr_device(n, seed + k, 0)
    d_out = h2b.dev_empty(32 * n)
    d_om = h2b.to_dev(f.fr_mont_limbs([dom.omega]))
    one = f.fr_mont_limbs([1]).reshape(4)
    ws = h2b.dev_empty(L._halo2_fft_normal_to_device_workspace_size(1, k, k))

    def fft():
        h2b.call("_halo2_fft_normal_to_device", 1, k, h2b.ptr(d_in), h2b.ptr(d_out), h2b.ptr(d_om),
                 one.ctypes.data, h2b.ptr(ws), ws.numel(), h2b.stream_handle())
    L.h2b_tune_set(PARAM_STAGES, k, 0)
    auto = L.h2b_ntt_get_pass_stages()
    ref = None

    def run_with(st):
        nonlocal ref
        if L.h2b_tune_set(PARAM_STAGES, k, st) != 0:
            raise ValueError(f"tuning table rejected ntt k={k} stages={st}")
        t = _time(torch, fft, reps)
        got = d_out.clone()
        if ref is None:
            ref = got
        elif not torch.equal(got, ref):
            raise RuntimeError(f"ntt k={k}: {st} stages per pass changed the result")
        return t

    times = {0: run_with(0)}
    for st in STAGE_CANDIDATES:
        if st != auto and st <= k:
            times[st] = run_with(st)
    best, med = pick(times, 0, margin)
    L.h2b_tune_set(PARAM_STAGES, k, best)
    return {"stages": best, "auto_stages": auto, "ms": med[best], "auto_ms": med[0],
            "candidates_ms": {f"s{s or auto}": round(v, 4) for s, v in med.items()}}


def autotune(h2b, msm_ks=(), ntt_ks=(), cache_path=None, reps=3, force=False, d_bases=None):
    """Loads the cached settings for this GPU and build, tunes the (op, k)
    pairs the cache lacks (all of them with `force`), stores them, and leaves
    every requested entry applied in the library.  Returns
    {"key", "msm": {k: entry}, "ntt": {k: entry}, "tuned": [...], "cached": [...]}."""
    import torch
    L = h2b.lib()
    path = cache_path or default_cache_path()
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    key = device_key(props.name, props.multi_processor_count, library_digest(h2b.LIB_PATH))
    cache = load_cache(path)
    dev = cache["devices"].setdefault(key, {"msm": {}, "ntt": {}})
    apply_entries(L.h2b_tune_set, dev)
    tuned, cached = [], []
    need_msm = [k for k in msm_ks if force or str(k) not in dev["msm"]]
    if need_msm:
        n_max = 1 << max(need_msm)
        bases = d_bases if d_bases is not None and d_bases.numel() >= 64 * n_max else h2b.srs_device(0x7A10, n_max)
        for k in need_msm:
            dev["msm"][str(k)] = tune_msm(h2b, k, bases, reps)
            tuned.append(("msm", k))
        del bases
    for k in ntt_ks:
        if force or str(k) not in dev["ntt"]:
            dev["ntt"][str(k)] = tune_ntt(h2b, k, reps)
            tuned.append(("ntt", k))
    cached = [(op, k) for op, ks in (("msm", msm_ks), ("ntt", ntt_ks)) for k in ks if (op, k) not in tuned]
    if tuned:
        save_cache(path, cache)
    return {"key": key, "msm": {k: dev["msm"][str(k)] for k in msm_ks}, "ntt": {k: dev["ntt"][str(k)] for k in ntt_ks},
            "tuned": tuned, "cached": cached, "path": path}
