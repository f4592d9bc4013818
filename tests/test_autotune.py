"""Per-size tuning table and autotuner.

CPU: the selection rule, the cache file, loading entries, and the table's
host-side checks and effects on the MSM plan (window width, workspace size,
window-table layout untouched).  GPU: every setting the table accepts leaves
MSM and NTT outputs bit-exact with the oracle, and an autotune run over small
sizes writes a cache that a second run reads back without re-timing."""
import json
import os

import pytest

from conftest import assert_limbs_equal


@pytest.fixture()
def at(h2b):
    import importlib
    return importlib.import_module("halo2_gpu_b200.autotune")


@pytest.fixture()
def clean_table(built_lib):
    built_lib.h2b_tune_clear()
    yield built_lib
    built_lib.h2b_tune_clear()


def test_pick_keeps_automatic_within_margin(at):
    assert at.pick({0: [1.00, 1.02, 0.99], 7: [0.995, 0.995]}, 0)[0] == 0
    assert at.pick({0: [1.00, 1.00], 7: [0.90, 0.95, 0.91], 8: [0.92]}, 0)[0] == 7
    best, med = at.pick({0: [2.0, 1.0, 3.0], 5: [1.5]}, 0)
    assert med[0] == 2.0 and best == 5


def test_window_candidates_stay_in_range(at):
    assert at.window_candidates(16) == [15, 16]
    assert at.window_candidates(12) == [11, 12, 13]
    assert at.window_candidates(10) == [10, 11]


def test_cache_round_trip_and_stale_versions(at, tmp_path):
    p = str(tmp_path / "sub" / "tune.json")
    assert at.load_cache(p) == {"version": at.CACHE_VERSION, "devices": {}}
    cache = {"version": at.CACHE_VERSION, "devices": {"k": {"msm": {"20": {"window": 15, "chunk": 64}}, "ntt": {}}}}
    at.save_cache(p, cache)
    assert at.load_cache(p) == cache
    json.dump({"version": 0, "devices": {"k": {}}}, open(p, "w"))
    assert at.load_cache(p)["devices"] == {}
    open(p, "w").write("{not json")
    assert at.load_cache(p)["devices"] == {}
    assert at.device_key("NVIDIA B200", 148, "abc") == "NVIDIA B200|sm148|lib-abc"


def test_apply_entries_sets_and_rejects(at):
    calls = []

    def fake_set(param, k, v):
        calls.append((param, k, v))
        return 0 if v != 99 else -1

    at.apply_entries(fake_set, {"msm": {"20": {"window": 15, "chunk": 64}}, "ntt": {"22": {"stages": 8}}})
    assert calls == [(at.PARAM_WINDOW, 20, 15), (at.PARAM_CHUNK, 20, 64), (at.PARAM_STAGES, 22, 8)]
    with pytest.raises(ValueError):
        at.apply_entries(fake_set, {"ntt": {"22": {"stages": 99}}})


def test_table_validates_values(clean_table):
    L = clean_table
    assert L.h2b_tune_set(0, 22, 15) == 0 and L.h2b_tune_get(0, 22) == 15
    for param, bad in ((0, 9), (0, 17), (1, 7), (1, 513), (2, 12), (3, 1)):
        assert L.h2b_tune_set(param, 20, bad) == -1
    assert L.h2b_tune_set(0, 33, 12) == -1
    assert L.h2b_tune_get(0, 22) == 15 and L.h2b_tune_get(0, 20) == 0
    L.h2b_tune_clear()
    assert L.h2b_tune_get(0, 22) == 0


def test_table_drives_plain_msm_plan_only(clean_table):
    L = clean_table
    n = 1 << 20
    auto_c = L.h2b_msm_window_bits(n)
    auto_c21 = L.h2b_msm_window_bits(2 * n)
    ws_auto = L._halo2_multiexp_device_scalars_device_bases_workspace_size(n)
    table_pts = L.h2b_msm_table_points(n)
    assert L.h2b_tune_set(0, 20, auto_c - 1) == 0
    assert L.h2b_msm_window_bits(n) == auto_c - 1
    assert L.h2b_msm_window_bits(n + 12345) == auto_c - 1        # floor(log2 n) selects the entry
    assert L.h2b_msm_window_bits(2 * n) == auto_c21                # other sizes keep their own entry
    assert L.h2b_msm_table_points(n) == table_pts                # a window table's layout never changes
    L.h2b_tune_set(0, 20, 0)
    assert L.h2b_tune_set(1, 20, 16) == 0                        # smaller chunks: more chunk heads
    assert L._halo2_multiexp_device_scalars_device_bases_workspace_size(n) > ws_auto
    L.h2b_tune_clear()
    assert L._halo2_multiexp_device_scalars_device_bases_workspace_size(n) == ws_auto


@pytest.mark.gpu
def test_every_msm_setting_is_bit_exact(h2b, orc, cuda, clean_table):
    L = clean_table
    n = 3000
    tau = h2b.fields.fr_mont_limbs([0x5151])
    bases = orc.srs(tau, n)
    sc = orc.chacha_fr(0x5152, n)
    sc[::7] = 0
    want = orc.msm(sc, bases)
    d_b, d_s = h2b.to_dev(bases), h2b.to_dev(sc)
    for c in (10, 11, 12, 13, 14, 15, 16):
        for chunk in (0, 8, 37, 256):
            assert L.h2b_tune_set(0, 11, c) == 0 and L.h2b_tune_set(1, 11, chunk) == 0
            got = h2b.multiexp_gpu_device_scalars_device_bases(d_s, d_b, n)
            assert_limbs_equal(got, want, f"window {c} chunk {chunk}")


@pytest.mark.gpu
def test_every_ntt_setting_is_bit_exact(h2b, orc, cuda, clean_table):
    L = clean_table
    f = h2b.fields
    for k in (10, 13):
        d = f.EvaluationDomain(3, k)
        a = orc.chacha_fr(0x5153 + k, 1 << k)
        c = d.g_coset * d.extended_omega % f.R_MOD
        cases = [(1, d.omega, 1), (2, d.omega_inv, d.ifft_divisor), (6, d.omega, c)]
        wants = [orc.ntt(t, k, k, a, f.fr_mont_limbs([om]), f.fr_mont_limbs([dv])) for t, om, dv in cases]
        for st in range(1, 12):
            assert L.h2b_tune_set(2, k, st) == 0
            for (t, om, dv), want in zip(cases, wants):
                assert_limbs_equal(h2b.fft_normal(t, k, a, om, dv), want, f"k={k} type {t} stages {st}")


@pytest.mark.gpu
def test_autotune_writes_and_reuses_cache(h2b, at, cuda, clean_table, tmp_path):
    L = clean_table
    p = str(tmp_path / "tune.json")
    r1 = at.autotune(h2b, msm_ks=(11, 12), ntt_ks=(12,), cache_path=p, reps=2)
    assert sorted(r1["tuned"]) == [("msm", 11), ("msm", 12), ("ntt", 12)] and r1["cached"] == []
    for k in (11, 12):
        e = r1["msm"][k]
        assert L.h2b_tune_get(0, k) == e["window"] and L.h2b_tune_get(1, k) == e["chunk"]
        assert e["ms"] <= e["auto_ms"] * 1.2
    assert L.h2b_tune_get(2, 12) == r1["ntt"][12]["stages"]
    assert os.path.exists(p)
    L.h2b_tune_clear()
    r2 = at.autotune(h2b, msm_ks=(11, 12), ntt_ks=(12,), cache_path=p, reps=2)
    assert r2["tuned"] == [] and sorted(r2["cached"]) == [("msm", 11), ("msm", 12), ("ntt", 12)]
    assert r2["msm"] == r1["msm"] and r2["ntt"] == r1["ntt"]
    assert L.h2b_tune_get(0, 12) == r1["msm"][12]["window"]
    assert L.h2b_tune_get(2, 12) == r1["ntt"][12]["stages"]
    # the tuned MSM still matches the automatic one
    n = 1 << 12
    d_b = h2b.srs_device(0x99, n)
    d_s = h2b.random_fr_device(n, 0x98, 1)
    tuned = h2b.multiexp_gpu_device_scalars_device_bases(d_s, d_b, n)
    L.h2b_tune_clear()
    assert_limbs_equal(tuned, h2b.multiexp_gpu_device_scalars_device_bases(d_s, d_b, n), "tuned vs automatic")
