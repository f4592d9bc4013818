"""C-ABI checks that need no GPU: the library loads, exports every symbol the
public header declares, and the pure-host preflights / argument checks behave
like the reference's (no device work is issued by any call here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b((?:_halo2|h2b)_\w+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_reference_entry_points():
    names = declared_symbols()
    for must in ("_halo2_multiexp", "_halo2_fft_normal", "_halo2_batch_invert", "_halo2_grand_product",
                 "_halo2_permute_expression_pair", "_halo2_quotient_device_columns_device_out",
                 "_halo2_quotient_permutation", "_halo2_quotient_lookups", "_halo2_commit_product_device_inputs"):
        assert must in names


def test_library_exports_every_declared_symbol(built_lib):
    missing = [n for n in declared_symbols() if not hasattr(built_lib, n)]
    assert not missing, f"not exported: {missing}"


def test_python_mirror_binds_every_declared_symbol(h2b, built_lib):
    bound = set(h2b._SIGS)
    missing = [n for n in declared_symbols() if n not in bound]
    assert not missing, f"python mirror lacks: {missing}"


def test_workspace_preflights_are_pure_host(h2b, built_lib):
    L = built_lib
    for k in (1, 10, 16, 22):
        a = L._halo2_fft_normal_workspace_size(1, k, k)
        b = L._halo2_fft_normal_to_device_workspace_size(1, k, k)
        assert a > b > 0
        assert L._halo2_fft_many_workspace_size(3, k, k + 2) >= (32 << (k + 2))
    assert L._halo2_multiexp_workspace_size(1 << 16) > L._halo2_multiexp_device_bases_workspace_size(1 << 16)
    assert L._halo2_msm_max_length(1 << 40) == 1 << 27
    assert L._halo2_msm_max_length(1 << 20) < (1 << 20)
    assert L._halo2_fft_normal_check_memory(1, None, 10, 10)
    assert L._halo2_fft_many_check_memory(1, 10, 10)
    assert L._halo2_get_fft_split_radix(1, 20, 20, 1 << 40) == 0
    assert L._halo2_get_fft_split_radix(1, 20, 20, 1) == -1
    assert L._halo2_grand_product_max_len(1 << 20, 1 << 40) == 1 << 20
    assert L._halo2_commit_product_max_len(1 << 20, 1 << 10) < (1 << 20)


def test_argument_errors_match_reference(h2b, built_lib):
    import numpy as np
    z = np.zeros(4, np.uint64)
    # iFFT_cosetFFT is rejected with -1 before any device work (ntt.cu:74,93-94)
    e = built_lib._halo2_fft_normal(5, 4, z.ctypes.data, z.ctypes.data, z.ctypes.data, z.ctypes.data, None, 0, None)
    assert e.code == -1
    # log_n == 0 -> cudaErrorInvalidValue (1)
    e = built_lib._halo2_fft_normal(1, 0, z.ctypes.data, z.ctypes.data, z.ctypes.data, z.ctypes.data, None, 0, None)
    assert e.code == 1
    # icosetFFT is refused by the many-FFT entries with code 2 (ntt.cu:837)
    e = built_lib._halo2_fft_many(4, 1, 4, 4, None, None, None, None, None, 0, None)
    assert e.code == 2
    # bad field type / empty batch invert
    assert built_lib._halo2_batch_invert(None, 7, 8, None).code == 1
    assert built_lib._halo2_batch_invert(None, 0, 0, None).code == 1
    # scratch too small is an error code, not a trap
    e = built_lib._halo2_fft_normal_to_device(1, 10, None, None, None, z.ctypes.data, None, 0, None)
    assert e.code == 1
    with pytest.raises(h2b.Halo2GpuError):
        h2b.check(built_lib._halo2_batch_invert(None, 9, 8, None), "batch_invert")


def test_twiddle_preflights_and_argument_errors(h2b, built_lib):
    import numpy as np
    L = built_lib
    assert L._halo2_power_of_omega_workspace_size(31) >= 32 * 34
    assert L._halo2_power_of_omega_workspace_size(32) == 0
    assert L._halo2_generate_omega_powers_workspace_size(22) > 0
    assert L._halo2_generate_omega_lut_workspace_size(9) == 0
    assert L._halo2_generate_omega_lut_workspace_size(20) >= 32 * ((1 << 10) + (1 << 10))
    assert L._halo2_generate_omegadelta_workspace_size(20, 0, 100, 5, 0) > 0
    z = np.zeros(4, np.uint64)
    o = h2b.host_ffi(z)
    # pow >= 2^log_n and log_n >= 32 are refused before any device work (omega.cu:40-43)
    assert L._halo2_power_of_omega(ctypes.byref(o), ctypes.byref(o), ctypes.byref(o), 4, 16, None, 0, None).code == 1
    assert L._halo2_power_of_omega(ctypes.byref(o), ctypes.byref(o), ctypes.byref(o), 32, 1, None, 0, None).code == 1
    # log_n outside [DENSE_POWER_DEGREE, DENSE_POWER_DEGREE + 32) (omega.cu:118-120,181-183)
    assert L._halo2_generate_omega_lut(ctypes.byref(o), ctypes.byref(o), 9, None, 0, None).code == 1
    assert L._halo2_generate_omegadelta(None, None, z.ctypes.data, z.ctypes.data, 42, 0, 1, 1, 0, None, 0,
                                        None).code == 1
    # undersized scratch is an error code
    assert L._halo2_power_of_omega(ctypes.byref(o), ctypes.byref(o), ctypes.byref(o), 4, 3, None, 0, None).code == 1
    # the decode hook has no outputs and accepts any rule list
    rules = np.zeros(4, np.uint64)
    L._halo2_quotient_decode(rules.ctypes.data, 2, 1 << 10, 1, 0, 1 << 10)


def test_window_table_layouts(h2b, built_lib):
    """A window table holds 2 W tn points (W slices of 2^(c w) P and their
    endomorphism images); the width c follows the table size: 10 bits up to
    2^12 points, 13 bits from 2^13, 16 bits from 2^17 (one shared bucket set
    per table, so narrow windows make long buckets).  W covers the 127-bit
    GLV halves with room for the top digit's carry.  Pure host: the layout
    preflight and the MSM's window width for plain bases."""
    L = built_lib
    L.h2b_msm_table_points.restype = ctypes.c_uint64
    L.h2b_msm_table_points.argtypes = [ctypes.c_uint64]

    def windows(c):
        w = (127 + c - 1) // c
        return w + 1 if 127 - c * (w - 1) > c - 1 else w

    for lg, c in ((10, 10), (12, 10), (13, 13), (16, 13), (17, 16), (20, 16), (22, 16)):
        tn = 1 << lg
        assert L.h2b_msm_table_points(tn) == 2 * windows(c) * tn, (lg, c)
    assert windows(10) == 13 and windows(13) == 10 and windows(16) == 8
    assert L.h2b_msm_table_points(1 << 28) == 0          # entries must stay 31-bit


def test_fused_quotient_and_merged_msm_reject_on_the_host(h2b, built_lib):
    """h2b_quotient_fused and h2b_msm_merged check their arguments before any
    device work: each bad call below returns cudaErrorInvalidValue with a
    message (device pointers are stand-ins and never dereferenced)."""
    import numpy as np
    L = built_lib
    fake = [ctypes.c_void_p(0x10000 + 0x1000 * i) for i in range(70)]
    cols = (ctypes.c_void_p * 70)(*fake)
    y = np.zeros(4, np.uint64)
    rules = np.zeros(2, np.uint64)                        # one OP_ZERO rule
    vp = np.array([3 | (0 << 4)], np.uint64)              # value part: intermediate 0
    g = h2b.QuotientRules(rules.ctypes.data, 1, vp.ctypes.data, 1, None, 0, None, 0)

    def fused(n_fixed=1, nq=1024, r0=0, r1=1024, gates=ctypes.byref(g), lookups=None, n_lookups=0, perm=None,
              lag=True):
        la = lookups if lookups is not None else (h2b.QuotientLookupArgs * 1)()
        l = fake[60] if lag else None
        return L.h2b_quotient_fused(cols, n_fixed, None, 0, None, 0, gates, y.ctypes.data, l, l, l, perm, la,
                                    n_lookups, nq, 1, r0, r1, fake[61], 1, 0, None, None)

    def bad(e, text):
        assert e.code == 1, text
        msg = ctypes.string_at(e.message).decode()
        h2b._libc.free(e.message)
        assert text in msg, msg

    bad(fused(nq=0), "num_quotient is 0")
    bad(fused(r0=10, r1=1025), "row range")
    bad(fused(gates=None), "gates, y and out are required")
    bad(fused(n_fixed=65), "more than 64 columns")
    bad(fused(n_lookups=9, lookups=(h2b.QuotientLookupArgs * 9)()), "more than 8 lookups")
    bad(fused(n_lookups=1, lag=False), "l0, l_last and l_active are required")
    big_rules = np.zeros(2 * 300, np.uint64)
    gbig = h2b.QuotientRules(big_rules.ctypes.data, 300, vp.ctypes.data, 1, None, 0, None, 0)
    bad(fused(gates=ctypes.byref(gbig)), "parameter block")
    pa = h2b.QuotientPermutationArgs(2, 1, 4, ctypes.addressof(cols), ctypes.addressof(cols), ctypes.addressof(cols),
                                     *[y.ctypes.data] * 6, -6, 1, 1024, 0)
    bad(fused(perm=ctypes.byref(pa)), "permutation shape")
    # merged MSMs: one table, at most 64 jobs, each no longer than the table
    jobs = (h2b.MsmJob * 2)()
    for i in range(2):
        jobs[i].d_scalars, jobs[i].d_bases, jobs[i].d_out, jobs[i].n, jobs[i].table_n = fake[i], fake[10], fake[20 + i], 8, 16
    assert L.h2b_msm_merged_workspace_size(jobs, 2) > 0
    jobs[1].d_bases = fake[11]
    assert L.h2b_msm_merged_workspace_size(jobs, 2) == 0
    bad(L.h2b_msm_merged(jobs, 2, fake[30], 1 << 30, None), "jobs must share one window table")
    jobs[1].d_bases, jobs[1].n = fake[10], 17
    bad(L.h2b_msm_merged(jobs, 2, fake[30], 1 << 30, None), "job longer than its table")
    jobs[1].n = 8
    bad(L.h2b_msm_merged(jobs, 2, fake[30], 16, None), "h2b_msm_merged")      # scratch too small
