"""halo2-gpu_b200: B200-native BN254 Halo2/KZG prover hot path.

Python host mirror of the reference's GPU wrappers
(halo2_proofs/src/cuda/funcs/*.rs, halo2_proofs/src/poly/domain.rs) over the
C ABI in libhalo2_gpu.so (declared in include/halo2_gpu.h).  PyTorch provides
device memory and streams only; every field operation runs in this package's
CUDA kernels.  There is no CPU fallback: if the shared library is missing the
import of `lib()` raises.

Array conventions: field elements are numpy uint64 arrays of shape (n, 4) in
Montgomery form (the halo2curves memory image); G1 affine points are (n, 8)
(x limbs then y limbs); an MSM result is the (12,) Jacobian image
{X, Y, Z} with Z = 1 (or (0, 1, 0) for infinity).
"""
import ctypes
import os

import numpy as np

from . import fields  # noqa: F401  (re-exported helper module)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhalo2_gpu.so")

NTT_FFT, NTT_IFFT, NTT_COSET, NTT_ICOSET, NTT_IFFT_COSET, NTT_COSET_PART = 1, 2, 3, 4, 5, 6


class RustError(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int), ("message", ctypes.c_void_p)]


class FFITraitObject(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p)]


class AssignedLayout(ctypes.Structure):
    """Byte layout of the Rust Assigned<F> records (culib.rs:22-26)."""
    _fields_ = [("stride_bytes", ctypes.c_uint32), ("num_offset", ctypes.c_uint32), ("denom_offset", ctypes.c_uint32)]


class MsmJob(ctypes.Structure):
    """One job of h2b_msm_batch (device scalars, device bases, device 96-byte output, length)."""
    _fields_ = [("d_scalars", ctypes.c_void_p), ("d_bases", ctypes.c_void_p), ("d_out", ctypes.c_void_p),
                ("n", ctypes.c_uint64), ("table_n", ctypes.c_uint64)]


class QuotientProgram(ctypes.Structure):
    """h2b_quotient_program: a compiled quotient program's host-side header."""
    _fields_ = [("n_ops", ctypes.c_uint32), ("n_vp", ctypes.c_uint32), ("slots", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("num_quotient", ctypes.c_uint64), ("off_vps", ctypes.c_uint64),
                ("off_cols", ctypes.c_uint64), ("off_consts", ctypes.c_uint64), ("off_chal", ctypes.c_uint64),
                ("off_y", ctypes.c_uint64), ("bytes", ctypes.c_uint64)]


class QuotientRules(ctypes.Structure):
    """h2b_quotient_rules: one expression graph in the reference's rule encoding, host data."""
    _fields_ = [("rules", ctypes.c_void_p), ("num_rules", ctypes.c_uint64), ("value_part_rules", ctypes.c_void_p),
                ("num_vp", ctypes.c_uint64), ("constants", ctypes.c_void_p), ("num_constants", ctypes.c_uint64),
                ("challenges", ctypes.c_void_p), ("num_challenges", ctypes.c_uint64)]


class QuotientPermutationArgs(ctypes.Structure):
    """h2b_quotient_permutation_args: the permutation argument of one extended part."""
    _fields_ = [("n_sets", ctypes.c_uint64), ("chunk_len", ctypes.c_uint64), ("n_columns", ctypes.c_uint64),
                ("product_cosets", ctypes.c_void_p), ("sigma_cosets", ctypes.c_void_p),
                ("column_values", ctypes.c_void_p), ("beta", ctypes.c_void_p), ("gamma", ctypes.c_void_p),
                ("delta", ctypes.c_void_p), ("delta_start", ctypes.c_void_p),
                ("current_extended_omega", ctypes.c_void_p), ("omega", ctypes.c_void_p),
                ("last_rotation", ctypes.c_int32), ("rot_scale", ctypes.c_int32), ("isize", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class QuotientLookupArgs(ctypes.Structure):
    """h2b_quotient_lookup_args: one lookup of one extended part."""
    _fields_ = [("product", QuotientRules), ("product_coset", ctypes.c_void_p),
                ("permuted_input_coset", ctypes.c_void_p), ("permuted_table_coset", ctypes.c_void_p),
                ("beta", ctypes.c_void_p), ("gamma", ctypes.c_void_p)]


class Halo2GpuError(RuntimeError):
    def __init__(self, code, message, who):
        super().__init__(f"{who}: code {code}: {message}")
        self.code = code
        self.message = message


_u64, _u32, _i32, _vp, _b = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_bool
_ffi = ctypes.POINTER(FFITraitObject)

# name -> (restype, argtypes)
_SIGS = {
    "_halo2_msm_max_length": (_u64, [_u64]),
    "_halo2_multiexp_workspace_size": (_u64, [_u64]),
    "_halo2_multiexp": (RustError, [_ffi, _ffi, _ffi, _u64, _vp, _u64, _vp]),
    "_halo2_multiexp_device_bases_workspace_size": (_u64, [_u64]),
    "_halo2_multiexp_device_bases": (RustError, [_ffi, _vp, _ffi, _u64, _vp, _u64, _vp]),
    "_halo2_multiexp_device_scalars_device_bases_workspace_size": (_u64, [_u64]),
    "_halo2_multiexp_device_scalars_device_bases": (RustError, [_vp, _vp, _ffi, _u64, _vp, _u64, _vp]),
    "_halo2_batch_invert": (RustError, [_vp, _u32, _u64, _vp]),
    "_halo2_commit_product_max_len": (_u64, [_u64, _u64]),
    "_halo2_commit_product_workspace_size": (_u64, [_u64]),
    "_halo2_commit_product": (RustError, [_ffi, _ffi, _ffi, _ffi, _ffi, _vp, _vp, _u64, _u64, _vp, _u64, _vp]),
    "_halo2_commit_product_device_inputs": (RustError, [_ffi, _ffi, _ffi, _ffi, _ffi, _vp, _vp, _u64, _u64, _vp]),
    "_halo2_permutation_product_max_len": (_u64, [_u64, _u64]),
    "_halo2_permutation_product_workspace_size": (_u64, [_u64]),
    "_halo2_permutation_product": (RustError, [_ffi, _ffi, _ffi, _vp, _vp, _vp, _vp, _vp, _u64, _u64, _u64, _vp,
                                               _u64, _vp]),
    "_halo2_permutation_product_device_inputs_workspace_size": (_u64, [_u64]),
    "_halo2_permutation_product_device_inputs": (RustError, [_ffi, _ffi, _ffi, _vp, _vp, _vp, _vp, _vp, _u64, _u64,
                                                             _u64, _vp, _u64, _vp]),
    "_halo2_grand_product_max_len": (_u64, [_u64, _u64]),
    "_halo2_grand_product_workspace_size": (_u64, [_u64]),
    "_halo2_grand_product": (RustError, [_ffi, _ffi, _ffi, _u64, _u64, _vp, _u64, _vp]),
    "_halo2_grand_product_device_inputs": (RustError, [_ffi, _ffi, _u64, _u64, _vp]),
    "_halo2_permute_expression_pair_workspace_size": (_u64, [_u64, _u64]),
    "_halo2_permute_expression_pair": (RustError, [_vp, _vp, _vp, _vp, _u64, _u64, _vp, _u64, _vp]),
    "_halo2_poly_multiply_add": (RustError, [_vp, _vp, _vp, _u64, _vp]),
    "_halo2_poly_elementwise_multiply": (RustError, [_vp, _vp, _vp, _u64, _vp]),
    "_halo2_poly_fill_one": (RustError, [_vp, _u64, _vp]),
    "_halo2_divide_by_vanishing_poly": (RustError, [_vp, _vp, _u32, _u64, _vp]),
    "_halo2_poly_sub_short_inplace": (RustError, [_vp, _vp, _u64, _vp]),
    "_halo2_poly_sub_short_out_of_place": (RustError, [_vp, _vp, _vp, _u64, _u64, _vp]),
    "_halo2_poly_sub_scalar_at_zero": (RustError, [_vp, _vp, _vp]),
    "_halo2_extended_from_lagrange_vec_device": (RustError, [_vp, _vp, _u32, _u64, _vp]),
    "_halo2_distribute_powers_zeta": (RustError, [_vp, _vp, _u32, _u64, _vp]),
    "_halo2_eval_polynomial_workspace_size": (_u64, [_u64]),
    "_halo2_eval_polynomial": (RustError, [_vp, _ffi, ctypes.POINTER(ctypes.c_void_p), _u64, _vp, _u64, _vp]),
    "_halo2_eval_poly_batch_max_len": (_u64, [_u64, _u64, _u64]),
    "_halo2_eval_polynomial_batch_workspace_size": (_u64, [_u64, _u64]),
    "_halo2_eval_polynomial_batch": (RustError, [_ffi, _ffi, _ffi, _u64, _u64, _u64, _vp, _u64, _vp]),
    "_halo2_kate_division_workspace_size": (_u64, [_u64]),
    "_halo2_kate_division_device": (RustError, [_vp, _vp, _vp, _u64, _vp, _u64, _vp]),
    "_halo2_kate_division_device_padded": (RustError, [_vp, _vp, _vp, _u64, _u64, _vp, _u64, _vp]),
    "_halo2_multiopen_poly_max_len": (_u64, [_u64, _u64, _u64]),
    "_halo2_multiopen_poly_calculation_workspace_size": (_u64, [_u64, _u64]),
    "_halo2_multiopen_poly_calculation": (RustError, [_ffi, _ffi, _u64, _u64, _u64, _ffi, _ffi, _ffi, _vp, _u64,
                                                      _vp]),
    "_halo2_decode_assigned": (RustError, [_vp, _vp, _vp, _u64, AssignedLayout, _vp]),
    "_halo2_fft_normal_workspace_size": (_u64, [_u32, _u32, _u32]),
    "_halo2_fft_normal": (RustError, [_u32, _u32, _vp, _vp, _vp, _vp, _vp, _u64, _vp]),
    "_halo2_fft_normal_check_memory": (_b, [_u32, _vp, _u32, _u32]),
    "_halo2_fft_normal_to_device_workspace_size": (_u64, [_u32, _u32, _u32]),
    "_halo2_fft_normal_to_device": (RustError, [_u32, _u32, _vp, _vp, _vp, _vp, _vp, _u64, _vp]),
    "_halo2_cosetfft": (RustError, [_u32, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _u64, _vp]),
    "_halo2_fft_many_workspace_size": (_u64, [_u32, _u32, _u32]),
    "_halo2_fft_many_to_device_workspace_size": (_u64, [_u32, _u32, _u32]),
    "_halo2_fft_many": (RustError, [_u32, _u32, _u32, _u32, _ffi, _ffi, _vp, _ffi, _vp, _u64, _vp]),
    "_halo2_fft_many_to_device": (RustError, [_u32, _u32, _u32, _u32, _ffi, _ffi, _vp, _ffi, _b, _vp, _u64, _vp]),
    "_halo2_fft_many_check_memory": (_b, [_u32, _u32, _u32]),
    "_halo2_get_fft_split_radix": (_i32, [_u32, _u32, _u32, _u64]),
    "_halo2_power_of_omega_workspace_size": (_u64, [_u32]),
    "_halo2_power_of_omega": (RustError, [_ffi, _ffi, _ffi, _u32, _u32, _vp, _u64, _vp]),
    "_halo2_generate_omega_powers_workspace_size": (_u64, [_u32]),
    "_halo2_generate_omega_powers": (RustError, [_vp, _vp, _u32, _vp, _u64, _vp]),
    "_halo2_generate_omega_lut_workspace_size": (_u64, [_u32]),
    "_halo2_generate_omega_lut": (RustError, [_ffi, _ffi, _u32, _vp, _u64, _vp]),
    "_halo2_generate_omegadelta_workspace_size": (_u64, [_u32, _u32, _u32, _u32, _u32]),
    "_halo2_generate_omegadelta": (RustError, [_vp, _vp, _vp, _vp, _u32, _u32, _u32, _u32, _u32, _vp, _u64, _vp]),
    "_halo2_quotient_decode": (None, [_vp, _u64, _u64, _u64, _u64, _u64]),
    "_halo2_evaluate_h_max_rows": (_u64, [_vp, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _u64,
                                          _u64]),
    "_halo2_quotient_workspace_size": (_u64, [_vp, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _u64,
                                              _u64]),
    "_halo2_quotient": (RustError, [_ffi, _u64, _ffi, _u64, _ffi, _u64, FFITraitObject, _u64, FFITraitObject, _u64,
                                    FFITraitObject, _vp, _u64, _vp, _u64, FFITraitObject, _u64, _u64, _u64, _u64, _vp,
                                    _u64, _vp]),
    "_halo2_quotient_device_columns_device_out": (RustError, [_vp, _u64, _vp, _u64, _vp, _u64, FFITraitObject, _u64,
                                                              FFITraitObject, _u64, FFITraitObject, _vp, _u64, _vp,
                                                              _u64, _vp, _u64, _vp, _u64, _u64, _u64, _vp, _u64, _vp]),
    "_halo2_quotient_device_columns": (RustError, [_vp, _u64, _vp, _u64, _vp, _u64, FFITraitObject, _u64,
                                                   FFITraitObject, _u64, FFITraitObject, _vp, _u64, _vp, _u64,
                                                   FFITraitObject, _u64, _u64, _u64, _u64, _vp, _u64, _vp]),
    "_halo2_quotient_lookups": (RustError, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u64, _vp]),
    "_halo2_quotient_permutation": (RustError, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                                _vp, _u64, _u64, _u64, _i32, _i32, _i32, _u64, _vp]),
    "h2b_msm_device": (RustError, [_vp, _vp, _vp, _u64, _vp, _u64, _vp]),
    "h2b_msm_set_tuning": (None, [ctypes.c_int, ctypes.c_int]),
    "h2b_msm_set_accumulate_variant": (None, [ctypes.c_int]),
    "h2b_msm_set_pair_rounds": (None, [ctypes.c_int]),
    "h2b_msm_get_accumulate_variant": (ctypes.c_int, []),
    "h2b_msm_get_pair_rounds": (ctypes.c_int, []),
    "h2b_msm_set_prefetch": (None, [ctypes.c_int]),
    "h2b_msm_get_prefetch": (ctypes.c_int, []),
    "h2b_exec_fork": (RustError, [_vp, _u32, ctypes.POINTER(ctypes.c_void_p)]),
    "h2b_exec_join": (RustError, [_vp, _u32]),
    "h2b_upload": (RustError, [_vp, _vp, _u64, _vp]),
    "h2b_graph_begin": (RustError, [_vp]),
    "h2b_graph_end": (RustError, [_vp, ctypes.POINTER(ctypes.c_void_p)]),
    "h2b_graph_launch": (RustError, [_vp, _vp]),
    "h2b_graph_destroy": (None, [_vp]),
    "h2b_msm_batch_workspace_size": (_u64, [ctypes.POINTER(MsmJob), _u64, _u32]),
    "h2b_msm_table_points": (_u64, [_u64]),
    "h2b_msm_table_precompute_workspace_size": (_u64, [_u64]),
    "h2b_msm_table_precompute": (RustError, [_vp, _u64, _vp, _vp, _u64, _vp]),
    "h2b_msm_table_workspace_size": (_u64, [_u64, _u64]),
    "h2b_msm_device_table": (RustError, [_vp, _vp, _u64, _vp, _u64, _vp, _u64, _vp]),
    "h2b_msm_batch": (RustError, [ctypes.POINTER(MsmJob), _u64, _u32, _vp, _u64, _vp]),
    "h2b_msm_merged_workspace_size": (_u64, [ctypes.POINTER(MsmJob), _u64]),
    "h2b_msm_merged": (RustError, [ctypes.POINTER(MsmJob), _u64, _vp, _u64, _vp]),
    "h2b_batch_invert_workspace_size": (_u64, [_u64]),
    "h2b_batch_invert": (RustError, [_vp, _u32, _u64, _vp, _u64, _vp]),
    "h2b_ntt_set_pass_stages": (None, [ctypes.c_int]),
    "h2b_ntt_get_pass_stages": (ctypes.c_int, []),
    "h2b_ntt_set_radix4": (None, [ctypes.c_int]),
    "h2b_ntt_get_radix4": (ctypes.c_int, []),
    "h2b_random_fr": (RustError, [_vp, _u64, _u64, ctypes.c_int, _vp]),
    "h2b_powers": (RustError, [_vp, _u64, _vp, _vp]),
    "h2b_fibonacci_fr": (RustError, [_vp, _u64, _vp, _vp]),
    "h2b_gather_fr": (RustError, [_vp, _vp, _u64, _vp, _u64, _vp]),
    "h2b_eval_many_workspace_size": (_u64, [_u64, _u64]),
    "h2b_eval_many_device": (RustError, [_vp, _vp, _u64, _u64, _vp, _vp, _u64, _vp]),
    "h2b_poly_linear_combination": (RustError, [_vp, _vp, _vp, _u64, _u64, ctypes.c_int, _vp]),
    "h2b_srs_from_powers": (RustError, [_vp, _vp, _u64, _vp, _vp]),
    "h2b_prof_enable": (None, [ctypes.c_int]),
    "h2b_prof_read": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]),
    "h2b_probe_imad": (RustError, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "h2b_probe_modmul": (RustError, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "h2b_probe_imad_form": (RustError, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "h2b_probe_modmul_impl": (RustError, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "h2b_fr_mul_batch": (RustError, [ctypes.c_int, _vp, _vp, _vp, _u64, _vp]),
    "h2b_launch_count": (_u64, []),
    "h2b_msm_count_entries": (RustError, [_vp, _u64, _vp, _vp]),
    "h2b_msm_window_bits": (ctypes.c_int, [_u64]),
    "h2b_batch_invert_noalloc": (RustError, [_vp, _u32, _u64, _vp]),
    "h2b_batch_invert_assigned_workspace_size": (_u64, [_u64, _u32]),
    "h2b_quotient_program_size": (_u64, [_u64, _u64, _u64, _u64, _u64]),
    "h2b_quotient_program_build": (RustError, [_vp, _u64, _vp, _u64, _u64, _u64, _u64, _vp, _vp, _u64, _vp, _u64,
                                               _vp, _u64, _u64, _vp, _u64, ctypes.POINTER(QuotientProgram), _vp]),
    "h2b_quotient_program_run": (RustError, [ctypes.POINTER(QuotientProgram), _vp, _vp, _vp, _u64, _u64, _vp]),
    "h2b_quotient_fused": (RustError, [_vp, _u64, _vp, _u64, _vp, _u64, ctypes.POINTER(QuotientRules), _vp, _vp, _vp,
                                       _vp, ctypes.POINTER(QuotientPermutationArgs),
                                       ctypes.POINTER(QuotientLookupArgs), _u64, _u64, _u64, _u64, _u64, _vp, _u64,
                                       _u64, _vp, _vp]),
    "h2b_quotient_fused_set_blocks": (None, [ctypes.c_int]),
    "h2b_quotient_fused_get_blocks": (ctypes.c_int, []),
    "h2b_batch_invert_assigned": (RustError, [_vp, _vp, _u32, _u64, AssignedLayout, _vp, _u64, _vp]),
    "h2b_tune_set": (_i32, [_u32, _u32, _i32]),
    "h2b_tune_get": (_i32, [_u32, _u32]),
    "h2b_tune_clear": (None, []),
}

PROF_MSM_ACCUMULATE, PROF_MSM_TOTAL, PROF_NTT_PASSES, PROF_BATCH_INVERT, PROF_QUOTIENT, PROF_PERMUTE_SORT = range(6)


def prof_read(prof_id):
    ms, cnt = ctypes.c_double(), ctypes.c_int()
    lib().h2b_prof_read(prof_id, ctypes.byref(ms), ctypes.byref(cnt))
    return ms.value, cnt.value

_lib = None


def lib():
    """Loads libhalo2_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing; run `python halo2-gpu_b200/build.py` "
                                    "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return [n for n in _SIGS if hasattr(lib(), n)]


_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def check(err, who):
    if err.code != 0:
        msg = ctypes.string_at(err.message).decode(errors="replace") if err.message else ""
        if err.message:
            _libc.free(err.message)
        raise Halo2GpuError(err.code, msg, who)
    if err.message:
        _libc.free(err.message)


def call(name, *args):
    """Calls a RustError-returning entry point and raises on a non-zero code."""
    check(getattr(lib(), name)(*args), name)


# --- device memory helpers (torch as the allocator) ---------------------------

def _torch():
    import torch
    return torch


def stream_handle(stream=None):
    """cudaStream_t of a torch stream (current stream by default), or a raw handle (c_void_p / int)."""
    if isinstance(stream, ctypes.c_void_p):
        return stream
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def dev_empty(nbytes):
    torch = _torch()
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")


def to_dev(arr, stream=None):
    """numpy (any dtype) -> torch uint8 device tensor with the same bytes.
    With a `stream`, the copy is queued there (h2b_upload) without waiting for
    the work already queued on it, and is ordered only with that stream's
    later work.  Without one, it runs on the current stream and is complete
    when this returns (usable from any stream)."""
    torch = _torch()
    a = np.ascontiguousarray(arr)
    nbytes = a.nbytes
    t = torch.empty(max(nbytes, 1), dtype=torch.uint8, device="cuda")
    if nbytes:
        call("h2b_upload", ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(a.ctypes.data), nbytes,
             stream_handle(stream))
        if stream is None:
            torch.cuda.current_stream().synchronize()
    return t[:nbytes] if nbytes else t[:0]


def to_host(t, shape=None):
    a = t.cpu().numpy().view(np.uint64)
    return a.reshape(shape) if shape is not None else a.reshape(-1, 4)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def ffi(p):
    return FFITraitObject(ctypes.c_void_p(p) if isinstance(p, int) else p)


def host_ffi(arr):
    """FFITraitObject carrying the address of a numpy array (kept alive by caller)."""
    return FFITraitObject(ctypes.c_void_p(arr.ctypes.data))


def ffi_array(ptrs):
    arr = (FFITraitObject * max(len(ptrs), 1))()
    for i, p in enumerate(ptrs):
        arr[i].ptr = p if isinstance(p, int) else p.value
    return arr


def _scalar_bytes(x):
    """Accepts a python int (plain value) or 32 Montgomery bytes / (1,4) limbs."""
    if isinstance(x, int):
        return np.frombuffer(fields.fr_scalar(x), dtype=np.uint64).copy()
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint64).reshape(4))


# --- MSM (halo2_proofs/src/cuda/funcs/multiexp.rs) -------------------------------

def multiexp_gpu(scalars, bases, stream=None):
    """_halo2_multiexp: host scalars (n,4) and host bases (n,8) -> (12,) Jacobian."""
    torch = _torch()
    n = int(scalars.shape[0])
    sc = np.ascontiguousarray(scalars, dtype=np.uint64)
    bs = np.ascontiguousarray(bases, dtype=np.uint64)
    out = np.zeros(12, dtype=np.uint64)
    ws = dev_empty(lib()._halo2_multiexp_workspace_size(n))
    a, b, o = host_ffi(sc), host_ffi(bs), host_ffi(out)
    call("_halo2_multiexp", ctypes.byref(a), ctypes.byref(b), ctypes.byref(o), n, ptr(ws), ws.numel(),
         stream_handle(stream))
    del torch
    return out


def multiexp_gpu_device_bases(scalars, d_bases, n=None, stream=None):
    n = int(scalars.shape[0]) if n is None else n
    sc = np.ascontiguousarray(scalars, dtype=np.uint64)
    out = np.zeros(12, dtype=np.uint64)
    ws = dev_empty(lib()._halo2_multiexp_device_bases_workspace_size(n))
    a, o = host_ffi(sc), host_ffi(out)
    call("_halo2_multiexp_device_bases", ctypes.byref(a), ptr(d_bases), ctypes.byref(o), n, ptr(ws), ws.numel(),
         stream_handle(stream))
    return out


def multiexp_gpu_device_scalars_device_bases(d_scalars, d_bases, n, ws=None, stream=None):
    out = np.zeros(12, dtype=np.uint64)
    need = lib()._halo2_multiexp_device_scalars_device_bases_workspace_size(n)
    if ws is None or ws.numel() < need:
        ws = dev_empty(need)
    o = host_ffi(out)
    call("_halo2_multiexp_device_scalars_device_bases", ptr(d_scalars), ptr(d_bases), ctypes.byref(o), n, ptr(ws),
         ws.numel(), stream_handle(stream))
    return out


def msm_device(d_scalars, d_bases, d_out, n, ws, stream=None):
    call("h2b_msm_device", ptr(d_scalars), ptr(d_bases), ptr(d_out), n, ptr(ws), ws.numel(), stream_handle(stream))


def msm_workspace(n):
    return dev_empty(lib()._halo2_multiexp_device_scalars_device_bases_workspace_size(n))


# --- batch execution (no reference counterpart) ---------------------------------

def msm_batch_jobs(d_scalars, d_bases, d_outs, lengths, table_n=0):
    """Job array for h2b_msm_batch; table_n > 0 when d_bases are window tables built for table_n bases."""
    jobs = (MsmJob * max(len(lengths), 1))()
    for i, n in enumerate(lengths):
        jobs[i].d_scalars = d_scalars[i].data_ptr()
        jobs[i].d_bases = d_bases[i].data_ptr()
        jobs[i].d_out = d_outs[i].data_ptr()
        jobs[i].n = int(n)
        jobs[i].table_n = int(table_n)
    return jobs


def msm_batch_workspace(jobs, count, streams):
    return dev_empty(lib().h2b_msm_batch_workspace_size(jobs, count, streams))


def msm_table_precompute(d_bases, n, stream=None):
    """Window table [2^(c w)] P_i for the n device bases (resident SRS form); returns the device table."""
    pts = lib().h2b_msm_table_points(n)
    if pts == 0:
        raise ValueError(f"no window table for {n} bases")
    table = dev_empty(64 * pts)
    ws = dev_empty(lib().h2b_msm_table_precompute_workspace_size(n))
    call("h2b_msm_table_precompute", ptr(d_bases), n, ptr(table), ptr(ws), ws.numel(), stream_handle(stream))
    return table


def msm_device_table(d_scalars, d_table, table_n, d_out, n, ws=None, stream=None):
    need = lib().h2b_msm_table_workspace_size(n, table_n)
    if ws is None or ws.numel() < need:
        ws = dev_empty(need)
    call("h2b_msm_device_table", ptr(d_scalars), ptr(d_table), table_n, ptr(d_out), n, ptr(ws), ws.numel(),
         stream_handle(stream))
    return d_out


def msm_batch(jobs, count, streams, ws, stream=None):
    """h2b_msm_batch: count device MSMs overlapped on `streams` forked streams."""
    call("h2b_msm_batch", jobs, count, streams, ptr(ws), ws.numel(), stream_handle(stream))


def msm_merged_workspace_bytes(jobs, count):
    return lib().h2b_msm_merged_workspace_size(jobs, count)


def msm_merged(jobs, count, ws, stream=None):
    """h2b_msm_merged: up to 64 MSMs over one window table as one sorted,
    accumulated and reduced run (job i's result in jobs[i].d_out)."""
    call("h2b_msm_merged", jobs, count, ptr(ws), ws.numel(), stream_handle(stream))


def exec_fork(n, stream=None):
    out = (ctypes.c_void_p * n)()
    call("h2b_exec_fork", stream_handle(stream), n, out)
    return [ctypes.c_void_p(out[i]) for i in range(n)]


def exec_join(n, stream=None):
    call("h2b_exec_join", stream_handle(stream), n)


class Graph:
    """A CUDA graph captured from everything issued on `stream` between begin() and end()."""

    def __init__(self, stream=None):
        self.stream = stream
        self.handle = None

    def begin(self):
        call("h2b_graph_begin", stream_handle(self.stream))

    def end(self):
        h = ctypes.c_void_p()
        call("h2b_graph_end", stream_handle(self.stream), ctypes.byref(h))
        self.handle = h

    def launch(self, stream=None):
        call("h2b_graph_launch", self.handle, stream_handle(stream if stream is not None else self.stream))

    def close(self):
        if self.handle is not None:
            lib().h2b_graph_destroy(self.handle)
            self.handle = None


# --- NTT (halo2_proofs/src/cuda/funcs/ntt.rs, poly/domain.rs) ----------------------

def fft_normal(ntt_type, log_n, values, omega, divisor, stream=None):
    """_halo2_fft_normal: host in/out (types 1,2,3,4,6 with extend = log_n)."""
    inp = np.ascontiguousarray(values, dtype=np.uint64)
    out = np.zeros_like(inp)
    om, dv = _scalar_bytes(omega), _scalar_bytes(divisor)
    ws = dev_empty(lib()._halo2_fft_normal_workspace_size(ntt_type, log_n, log_n))
    call("_halo2_fft_normal", ntt_type, log_n, inp.ctypes.data, out.ctypes.data, om.ctypes.data, dv.ctypes.data,
         ptr(ws), ws.numel(), stream_handle(stream))
    return out


def fft_normal_to_device(ntt_type, log_n, d_in, d_out, omega, divisor, ws=None, stream=None):
    d_om = to_dev(_scalar_bytes(omega), stream)
    dv = _scalar_bytes(divisor)
    need = lib()._halo2_fft_normal_to_device_workspace_size(ntt_type, log_n, log_n)
    if ws is None or ws.numel() < need:
        ws = dev_empty(need)
    call("_halo2_fft_normal_to_device", ntt_type, log_n, ptr(d_in), ptr(d_out), ptr(d_om), dv.ctypes.data, ptr(ws),
         ws.numel(), stream_handle(stream))
    return d_out


def cosetfft(log_n, extend_log_n, values, extended_omega, stream=None):
    inp = np.ascontiguousarray(values, dtype=np.uint64)
    out = np.zeros((1 << extend_log_n, 4), dtype=np.uint64)
    om = _scalar_bytes(extended_omega)
    one = _scalar_bytes(1)
    ws = dev_empty(lib()._halo2_fft_normal_workspace_size(NTT_COSET, log_n, extend_log_n))
    call("_halo2_cosetfft", NTT_COSET, log_n, extend_log_n, inp.ctypes.data, out.ctypes.data, om.ctypes.data,
         one.ctypes.data, ptr(ws), ws.numel(), stream_handle(stream))
    return out


# --- opening-phase polynomials (halo2_proofs/src/cuda/funcs/polynomial_ops.rs) ----

def eval_polynomial_device(d_poly, n, point, stream=None):
    """eval_polynomial_device (polynomial_ops.rs:441-480): sum_i poly[i] point^i, result read back."""
    torch = _torch()
    pt = _scalar_bytes(point)
    ws = dev_empty(lib()._halo2_eval_polynomial_workspace_size(n))
    res = ctypes.c_void_p()
    call("_halo2_eval_polynomial", ptr(d_poly), ctypes.byref(host_ffi(pt)), ctypes.byref(res), n, ptr(ws),
         ws.numel(), stream_handle(stream))
    out = np.zeros(4, dtype=np.uint64)
    torch.cuda.synchronize()
    base = ws.data_ptr()
    off = res.value - base
    assert 0 <= off <= ws.numel() - 32, "result must lie inside the scratch"
    out[:] = ws[off:off + 32].cpu().numpy().view(np.uint64)
    return out


def batch_eval_polynomial_gpu(polys, points, poly_offset, poly_length, stream=None):
    """basic_batch_eval_polynomial_gpu (polynomial_ops.rs:32-70): host polys, chunk-local exponents."""
    ps = [np.ascontiguousarray(p, dtype=np.uint64) for p in polys]
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.uint64).reshape(-1, 4))
    res = np.zeros((len(ps), 4), dtype=np.uint64)
    ws = dev_empty(lib()._halo2_eval_polynomial_batch_workspace_size(poly_length, len(ps)))
    call("_halo2_eval_polynomial_batch", ffi_array([p.ctypes.data for p in ps]), ctypes.byref(host_ffi(pts)),
         ctypes.byref(host_ffi(res)), poly_offset, poly_length, len(ps), ptr(ws), ws.numel(), stream_handle(stream))
    return res


def kate_division_device(d_a, d_q, d_u, n, out_len=None, stream=None):
    """kate_division_device (polynomial_ops.rs:541-583); out_len selects the padded entry."""
    ws = dev_empty(lib()._halo2_kate_division_workspace_size(n))
    if out_len is None:
        call("_halo2_kate_division_device", ptr(d_a), ptr(d_q), ptr(d_u), n, ptr(ws), ws.numel(),
             stream_handle(stream))
    else:
        call("_halo2_kate_division_device_padded", ptr(d_a), ptr(d_q), ptr(d_u), n, out_len, ptr(ws), ws.numel(),
             stream_handle(stream))
    return d_q


def multiopen_poly_calculation(polys, acc, challenges, points, poly_offset, poly_length, stream=None):
    """_halo2_multiopen_poly_calculation: evaluations of each chunk, and acc chunk = sum c_i * chunk_i."""
    ps = [np.ascontiguousarray(p, dtype=np.uint64) for p in polys]
    ch = np.ascontiguousarray(np.asarray(challenges, dtype=np.uint64).reshape(-1, 4))
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.uint64).reshape(-1, 4))
    res = np.zeros((len(ps), 4), dtype=np.uint64)
    ws = dev_empty(lib()._halo2_multiopen_poly_calculation_workspace_size(poly_length, len(ps)))
    call("_halo2_multiopen_poly_calculation", ffi_array([p.ctypes.data for p in ps]), ctypes.byref(host_ffi(acc)),
         poly_offset, poly_length, len(ps), ctypes.byref(host_ffi(ch)), ctypes.byref(host_ffi(pts)),
         ctypes.byref(host_ffi(res)), ptr(ws), ws.numel(), stream_handle(stream))
    return res


def decode_assigned_device(d_nums, d_denoms, d_raw, n, stride_bytes, num_offset, denom_offset, stream=None):
    """decode_assigned_to_num_denom_device (polynomial_ops.rs): Assigned<F> records -> (nums, denoms)."""
    call("_halo2_decode_assigned", ptr(d_nums), ptr(d_denoms), ptr(d_raw), n,
         AssignedLayout(stride_bytes, num_offset, denom_offset), stream_handle(stream))


def batch_invert_assigned_device(d_outs, d_raws, n, stride_bytes, num_offset, denom_offset, stream=None):
    """batch_invert_assigned_device (halo2_proofs/src/poly.rs:364-420) as one call:
    each device column of Assigned<F> records -> its values in the matching output."""
    ncols = len(d_raws)
    ws = dev_empty(lib().h2b_batch_invert_assigned_workspace_size(n, ncols))
    call("h2b_batch_invert_assigned", _ptr_table(d_outs), _ptr_table(d_raws), ncols, n,
         AssignedLayout(stride_bytes, num_offset, denom_offset), ptr(ws), ws.numel(), stream_handle(stream))
    _keep_until_done([ws], stream)


# --- twiddle tables (halo2_proofs/src/cuda/funcs/omega.rs) -----------------------

def power_of_omega_gpu(omega, log_n, pow_, stream=None):
    """power_of_omega_gpu (omega.rs:15-49): returns (omega^pow, log table of log_n + 1 limbs)."""
    om = _scalar_bytes(omega)
    res = np.zeros((1, 4), dtype=np.uint64)
    lut = np.zeros((log_n + 1, 4), dtype=np.uint64)
    ws = dev_empty(lib()._halo2_power_of_omega_workspace_size(log_n))
    call("_halo2_power_of_omega", ctypes.byref(host_ffi(res)), ctypes.byref(host_ffi(lut)),
         ctypes.byref(host_ffi(om)), log_n, pow_, ptr(ws), ws.numel(), stream_handle(stream))
    return res, lut


def generate_omega_powers_gpu(omega, log_n, output_num=None, stream=None):
    """generate_omega_powers_gpu (omega.rs:51-103): first output_num of omega^i, i < 2^log_n, to host."""
    torch = _torch()
    d_om = to_dev(_scalar_bytes(omega), stream)
    d_out = dev_empty(32 << log_n)
    ws = dev_empty(lib()._halo2_generate_omega_powers_workspace_size(log_n))
    call("_halo2_generate_omega_powers", ptr(d_out), ptr(d_om), log_n, ptr(ws), ws.numel(), stream_handle(stream))
    torch.cuda.synchronize()
    out = to_host(d_out)
    return out if output_num is None else out[:output_num]


def generate_omega_lut_gpu(omega, log_n, stream=None):
    """generate_omega_lut_gpu (omega.rs:105-136): the 2^10 + 2^(log_n-10) two-level table."""
    om = _scalar_bytes(omega)
    out = np.zeros(((1 << 10) + (1 << (log_n - 10)), 4), dtype=np.uint64)
    ws = dev_empty(lib()._halo2_generate_omega_lut_workspace_size(log_n))
    call("_halo2_generate_omega_lut", ctypes.byref(host_ffi(out)), ctypes.byref(host_ffi(om)), log_n, ptr(ws),
         ws.numel(), stream_handle(stream))
    return out


def generate_omegadelta_device(d_out, d_mapping, omega, delta, log_n, start, end, colnum, coloffset=0, stream=None):
    """_halo2_generate_omegadelta: d_out[i] = omega^row * delta^col over mapping[start..=end]."""
    om, de = _scalar_bytes(omega), _scalar_bytes(delta)
    ws = dev_empty(lib()._halo2_generate_omegadelta_workspace_size(log_n, start, end, colnum, coloffset))
    call("_halo2_generate_omegadelta", ptr(d_out), ptr(d_mapping), om.ctypes.data, de.ctypes.data, log_n, start,
         end, colnum, coloffset, ptr(ws), ws.numel(), stream_handle(stream))
    return d_out


def fft_many(ntt_type, log_n, extend_log_n, polys, omega, divisor, stream=None):
    """_halo2_fft_many: list of host polys -> list of host outputs."""
    ins = [np.ascontiguousarray(p, dtype=np.uint64) for p in polys]
    la = extend_log_n if ntt_type in (NTT_COSET, NTT_ICOSET) else log_n
    outs = [np.zeros((1 << la, 4), dtype=np.uint64) for _ in polys]
    d_om = to_dev(_scalar_bytes(omega), stream)
    dv = _scalar_bytes(divisor)
    dvo = host_ffi(dv)
    ws = dev_empty(lib()._halo2_fft_many_workspace_size(ntt_type, log_n, extend_log_n))
    call("_halo2_fft_many", ntt_type, len(ins), log_n, extend_log_n, ffi_array([a.ctypes.data for a in ins]),
         ffi_array([a.ctypes.data for a in outs]), ptr(d_om), ctypes.byref(dvo), ptr(ws), ws.numel(),
         stream_handle(stream))
    return outs


def fft_many_to_device(ntt_type, log_n, extend_log_n, d_ins, d_outs, omega, divisor, input_on_device=True,
                       ws=None, stream=None):
    d_om = to_dev(_scalar_bytes(omega), stream)
    dv = _scalar_bytes(divisor)
    dvo = host_ffi(dv)
    need = lib()._halo2_fft_many_to_device_workspace_size(ntt_type, log_n, extend_log_n)
    if ws is None or ws.numel() < need:
        ws = dev_empty(need)
    ins = [t.data_ptr() if hasattr(t, "data_ptr") else t.ctypes.data for t in d_ins]
    call("_halo2_fft_many_to_device", ntt_type, len(d_ins), log_n, extend_log_n, ffi_array(ins),
         ffi_array([t.data_ptr() for t in d_outs]), ptr(d_om), ctypes.byref(dvo), bool(input_on_device), ptr(ws),
         ws.numel(), stream_handle(stream))
    return d_outs


# --- batch inversion and products --------------------------------------------------

def batch_invert_device(d, n, field_type=0, stream=None):
    call("_halo2_batch_invert", ptr(d), field_type, n, stream_handle(stream))


def batch_invert_device_scratch(d, n, field_type=0, ws=None, stream=None):
    need = lib().h2b_batch_invert_workspace_size(n)
    if ws is None or ws.numel() < need:
        ws = dev_empty(need)
    call("h2b_batch_invert", ptr(d), field_type, n, ptr(ws), ws.numel(), stream_handle(stream))


def grand_product(inp, prefix, offset=0, length=None, stream=None):
    a = np.ascontiguousarray(inp, dtype=np.uint64)
    length = a.shape[0] - offset if length is None else length
    out = np.zeros_like(a)
    pf = _scalar_bytes(prefix)
    ws = dev_empty(lib()._halo2_grand_product_workspace_size(length))
    o, i, p = host_ffi(out), host_ffi(a), host_ffi(pf)
    call("_halo2_grand_product", ctypes.byref(o), ctypes.byref(i), ctypes.byref(p), length, offset, ptr(ws),
         ws.numel(), stream_handle(stream))
    return out


def grand_product_device(d_inout, d_prefix, length, offset=0, stream=None):
    a, p = ffi(d_inout.data_ptr()), ffi(d_prefix.data_ptr())
    call("_halo2_grand_product_device_inputs", ctypes.byref(a), ctypes.byref(p), length, offset,
         stream_handle(stream))


def lookup_product(permuted_input, permuted_table, compressed_input, compressed_table, beta, gamma, offset=0,
                   length=None, stream=None):
    arrs = [np.ascontiguousarray(x, dtype=np.uint64) for x in
            (permuted_input, permuted_table, compressed_input, compressed_table)]
    length = arrs[0].shape[0] - offset if length is None else length
    out = np.zeros_like(arrs[0])
    d_b, d_g = to_dev(_scalar_bytes(beta), stream), to_dev(_scalar_bytes(gamma), stream)
    ws = dev_empty(lib()._halo2_commit_product_workspace_size(length))
    objs = [host_ffi(out)] + [host_ffi(a) for a in arrs]
    call("_halo2_commit_product", *[ctypes.byref(o) for o in objs], ptr(d_b), ptr(d_g), length, offset, ptr(ws),
         ws.numel(), stream_handle(stream))
    return out


def lookup_product_device(d_out, d_pin, d_ptab, d_cin, d_ctab, d_beta, d_gamma, length, offset=0, stream=None):
    objs = [ffi(t.data_ptr()) for t in (d_out, d_pin, d_ptab, d_cin, d_ctab)]
    call("_halo2_commit_product_device_inputs", *[ctypes.byref(o) for o in objs], ptr(d_beta), ptr(d_gamma), length,
         offset, stream_handle(stream))


def permutation_product(modified_values, permutations, values, beta, gamma, delta, omega, deltaomega, offset=0,
                        length=None, stream=None):
    """Host variant; returns (modified_values, advanced deltaomega limbs)."""
    mv = np.ascontiguousarray(modified_values, dtype=np.uint64).copy()
    perms = [np.ascontiguousarray(p, dtype=np.uint64) for p in permutations]
    vals = [np.ascontiguousarray(v, dtype=np.uint64) for v in values]
    length = mv.shape[0] if length is None else length
    d_sc = [to_dev(_scalar_bytes(x), stream) for x in (beta, gamma, delta, omega, deltaomega)]
    ws = dev_empty(lib()._halo2_permutation_product_workspace_size(length))
    m = host_ffi(mv)
    call("_halo2_permutation_product", ctypes.byref(m), ffi_array([p.ctypes.data for p in perms]),
         ffi_array([v.ctypes.data for v in vals]), *[ptr(t) for t in d_sc], length, offset, len(perms), ptr(ws),
         ws.numel(), stream_handle(stream))
    return mv, to_host(d_sc[4])[0]


def permutation_product_device(d_mod, d_perms, d_vals, d_beta, d_gamma, d_delta, d_omega, d_deltaomega, length,
                               offset=0, stream=None):
    m = ffi(d_mod.data_ptr())
    call("_halo2_permutation_product_device_inputs", ctypes.byref(m), ffi_array([t.data_ptr() for t in d_perms]),
         ffi_array([t.data_ptr() for t in d_vals]), ptr(d_beta), ptr(d_gamma), ptr(d_delta), ptr(d_omega),
         ptr(d_deltaomega), length, offset, len(d_perms), None, 0, stream_handle(stream))


def permute_expression_pair_device(d_in, d_table, d_pin, d_ptab, n, usable_rows, stream=None):
    ws = dev_empty(lib()._halo2_permute_expression_pair_workspace_size(n, usable_rows))
    call("_halo2_permute_expression_pair", ptr(d_in), ptr(d_table), ptr(d_pin), ptr(d_ptab), n, usable_rows,
         ptr(ws), ws.numel(), stream_handle(stream))


# --- device-side generators ------------------------------------------------------

def random_fr_device(n, seed, mix=0, stream=None):
    d = dev_empty(32 * n)
    call("h2b_random_fr", ptr(d), n, seed, mix, stream_handle(stream))
    return d


def powers_device(x, n, stream=None):
    d = dev_empty(32 * n)
    call("h2b_powers", ptr(d), n, ptr(to_dev(_scalar_bytes(x), stream)), stream_handle(stream))
    return d


def fibonacci_device(s0, s1, n, stream=None):
    """out[0] = s0, out[1] = s1, out[i + 2] = out[i + 1] + out[i] (Fr, device)."""
    d = dev_empty(32 * n)
    seeds = np.concatenate([_scalar_bytes(s0), _scalar_bytes(s1)])
    call("h2b_fibonacci_fr", ptr(d), n, ptr(to_dev(seeds, stream)), stream_handle(stream))
    return d


def gather_fr_device(d_table, d_idx, stream=None):
    """out[i] = table[idx[i]] for 32-byte elements (h2b_gather_fr); d_idx is a
    device int64 tensor, indices outside the table give zero."""
    torch = _torch()
    idx = d_idx.contiguous()
    if idx.dtype != torch.int64:
        raise TypeError("gather_fr_device: indices must be int64")
    n = idx.numel()
    out = dev_empty(32 * n)
    call("h2b_gather_fr", ptr(out), ptr(d_table), d_table.numel() // 32, ptr(idx), n, stream_handle(stream))
    return out


def eval_many_device(d_polys, points, n, d_out=None, ws=None, stream=None):
    """[p_i(z_i)] for up to 64 device polynomials of n coefficients
    (h2b_eval_many_device); points are ints; returns the device results
    (32 bytes each) without synchronising."""
    count = len(d_polys)
    pts = np.ascontiguousarray(fields.fr_mont_limbs([int(z) % fields.R_MOD for z in points]))
    if d_out is None:
        d_out = dev_empty(32 * count)
    need = lib().h2b_eval_many_workspace_size(n, count)
    if ws is None or ws.numel() < need:
        ws = dev_empty(need)
    call("h2b_eval_many_device", _ptr_table(d_polys), pts.ctypes.data, count, n, ptr(d_out), ptr(ws), ws.numel(),
         stream_handle(stream))
    return d_out


def linear_combination_device(d_acc, d_polys, coeffs, n, accumulate=True, stream=None):
    """acc = (acc if accumulate else 0) + sum_t coeffs[t] polys[t] over n
    coefficients (h2b_poly_linear_combination; up to 64 terms; coefficients
    are ints)."""
    cs = np.ascontiguousarray(fields.fr_mont_limbs([int(c) % fields.R_MOD for c in coeffs])) if len(coeffs) else \
        np.zeros((1, 4), np.uint64)
    call("h2b_poly_linear_combination", ptr(d_acc), _ptr_table(d_polys), cs.ctypes.data, len(coeffs), n,
         1 if accumulate else 0, stream_handle(stream))
    return d_acc


def srs_device(tau, n, stream=None):
    """[tau^i] G, i < n, as a device tensor of n affine points (64 bytes each)."""
    pw = powers_device(tau, n, stream)
    table = to_dev(fields.g1_pow2_table(256), stream)
    out = dev_empty(64 * n)
    call("h2b_srs_from_powers", ptr(out), ptr(pw), n, ptr(table), stream_handle(stream))
    return out


# --- quotient (halo2_proofs/src/plonk/evaluation.rs:916-1054) -----------------

def _expr_constants(y):
    f = fields
    yv = y if isinstance(y, int) else f.fr_from_mont_limbs(np.asarray(y).reshape(1, 4))[0]
    return f.fr_mont_limbs([0, 1, f.R_MOD - 1, 2, yv])


def _ptr_table(tensors):
    arr = (ctypes.c_void_p * max(len(tensors), 1))()
    for i, t in enumerate(tensors):
        arr[i] = t.data_ptr()
    return arr


def quotient_device(d_fixed, d_instance, d_advice, challenges, constants, y, rules, vp_rules, num_quotient,
                    rot_scale, row_start, row_end, d_out, d_prev=None, stream=None):
    """_halo2_quotient_device_columns_device_out: device columns in, device rows out."""
    ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 4) if len(challenges) else \
        np.zeros((1, 4), np.uint64)
    cs = np.ascontiguousarray(constants, dtype=np.uint64).reshape(-1, 4)
    ec = _expr_constants(y)
    r = np.ascontiguousarray(rules, dtype=np.uint64)
    vp = np.ascontiguousarray(vp_rules, dtype=np.uint64)
    nf, ni, na = len(d_fixed), len(d_instance), len(d_advice)
    ws = dev_empty(lib()._halo2_quotient_workspace_size(r.ctypes.data, len(r) // 2, len(vp), num_quotient, nf, ni,
                                                        na, len(challenges), cs.shape[0], rot_scale, row_start,
                                                        row_end))
    call("_halo2_quotient_device_columns_device_out", _ptr_table(d_fixed), nf, _ptr_table(d_instance), ni,
         _ptr_table(d_advice), na, host_ffi(ch), len(challenges), host_ffi(cs), cs.shape[0], host_ffi(ec),
         r.ctypes.data, len(r) // 2, vp.ctypes.data, len(vp), ptr(d_out), num_quotient,
         ptr(d_prev) if d_prev is not None else None, rot_scale, row_start, row_end, ptr(ws), ws.numel(),
         stream_handle(stream))
    return d_out


def quotient_host(fixed, instance, advice, challenges, constants, y, rules, vp_rules, num_quotient, rot_scale,
                  row_start, row_end, stream=None):
    """_halo2_quotient: host columns in, host rows out."""
    fx = [np.ascontiguousarray(c, dtype=np.uint64) for c in fixed]
    ins = [np.ascontiguousarray(c, dtype=np.uint64) for c in instance]
    adv = [np.ascontiguousarray(c, dtype=np.uint64) for c in advice]
    ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 4) if len(challenges) else \
        np.zeros((1, 4), np.uint64)
    cs = np.ascontiguousarray(constants, dtype=np.uint64).reshape(-1, 4)
    ec = _expr_constants(y)
    r = np.ascontiguousarray(rules, dtype=np.uint64)
    vp = np.ascontiguousarray(vp_rules, dtype=np.uint64)
    out = np.zeros((row_end - row_start, 4), dtype=np.uint64)
    ws = dev_empty(lib()._halo2_quotient_workspace_size(r.ctypes.data, len(r) // 2, len(vp), num_quotient, len(fx),
                                                        len(ins), len(adv), len(challenges), cs.shape[0], rot_scale,
                                                        row_start, row_end))
    call("_halo2_quotient", ffi_array([a.ctypes.data for a in fx]), len(fx), ffi_array([a.ctypes.data for a in ins]),
         len(ins), ffi_array([a.ctypes.data for a in adv]), len(adv), host_ffi(ch), len(challenges), host_ffi(cs),
         cs.shape[0], host_ffi(ec), r.ctypes.data, len(r) // 2, vp.ctypes.data, len(vp), host_ffi(out),
         num_quotient, rot_scale, row_start, row_end, ptr(ws), ws.numel(), stream_handle(stream))
    return out


class ResidentQuotient:
    """A quotient program compiled once and kept on the device, bound to its
    columns (h2b_quotient_program_build); run() is a kernel launch alone."""

    def __init__(self, d_fixed, d_instance, d_advice, challenges, constants, y, rules, vp_rules, num_quotient,
                 rot_scale, stream=None):
        ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 4) if len(challenges) else \
            np.zeros((1, 4), np.uint64)
        cs = np.ascontiguousarray(constants, dtype=np.uint64).reshape(-1, 4)
        yv = _scalar_bytes(y)
        r = np.ascontiguousarray(rules, dtype=np.uint64)
        vp = np.ascontiguousarray(vp_rules, dtype=np.uint64)
        cols = list(d_fixed) + list(d_instance) + list(d_advice)
        self.columns = cols                      # kept alive: the program holds their addresses
        nb = lib().h2b_quotient_program_size(len(r) // 2, len(vp), len(cols), cs.shape[0], len(challenges))
        self.d_prog = dev_empty(nb)
        self.info = QuotientProgram()
        call("h2b_quotient_program_build", r.ctypes.data, len(r) // 2, vp.ctypes.data, len(vp), len(d_fixed),
             len(d_instance), len(d_advice), _ptr_table(cols), cs.ctypes.data, cs.shape[0], ch.ctypes.data,
             len(challenges), yv.ctypes.data, num_quotient, rot_scale, ptr(self.d_prog), nb, ctypes.byref(self.info),
             stream_handle(stream))

    def run(self, d_out, d_prev=None, row_start=0, row_end=None, stream=None):
        row_end = self.info.num_quotient if row_end is None else row_end
        call("h2b_quotient_program_run", ctypes.byref(self.info), ptr(self.d_prog), ptr(d_out),
             ptr(d_prev) if d_prev is not None else None, row_start, row_end, stream_handle(stream))
        return d_out


def _rules_struct(graph, keep):
    """QuotientRules for (challenges, constants, rules, value_part_rules); the
    numpy arrays it points into are appended to `keep`."""
    challenges, constants, rules, vp_rules = graph
    ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 4) if len(challenges) else \
        np.zeros((1, 4), np.uint64)
    cs = np.ascontiguousarray(constants, dtype=np.uint64).reshape(-1, 4) if len(constants) else \
        np.zeros((1, 4), np.uint64)
    r = np.ascontiguousarray(rules, dtype=np.uint64)
    vp = np.ascontiguousarray(vp_rules, dtype=np.uint64)
    keep += [ch, cs, r, vp]
    return QuotientRules(r.ctypes.data, len(r) // 2, vp.ctypes.data, len(vp), cs.ctypes.data,
                         len(constants) and cs.shape[0], ch.ctypes.data, len(challenges))


def quotient_fused_device(d_fixed, d_instance, d_advice, gates, y, d_l0, d_llast, d_lactive, perm, lookups,
                          num_quotient, rot_scale, row_start, row_end, d_out, out_stride=1, out_offset=0, scale=None,
                          stream=None):
    """h2b_quotient_fused: gates, permutation and lookups of one extended part in
    one kernel.  `gates` and each lookup's `rules` are (challenges, constants,
    rules, value_part_rules); `perm` is None or a dict with prods, sigmas, cols
    (device tensors), beta, gamma, delta, delta_start, ext_omega, omega (ints),
    chunk_len, last_rotation, rot_scale, isize; each lookup is a dict with rules,
    z, pin, ptab (device tensors), beta, gamma (ints).  Scalars are integers."""
    keep = []
    g = _rules_struct(gates, keep)
    yv = _scalar_bytes(y)
    keep.append(yv)
    pa = None
    if perm is not None:
        tabs = [_ptr_table(perm[k]) for k in ("prods", "sigmas", "cols")]
        sc = [_scalar_bytes(perm[k]) for k in ("beta", "gamma", "delta", "delta_start", "ext_omega", "omega")]
        keep += tabs + sc
        pa = QuotientPermutationArgs(len(perm["prods"]), perm["chunk_len"], len(perm["cols"]),
                                     ctypes.addressof(tabs[0]), ctypes.addressof(tabs[1]), ctypes.addressof(tabs[2]),
                                     *[x.ctypes.data for x in sc], perm["last_rotation"], perm["rot_scale"],
                                     perm["isize"], 0)
    la = (QuotientLookupArgs * max(len(lookups), 1))()
    for i, lk in enumerate(lookups):
        bt, gm = _scalar_bytes(lk["beta"]), _scalar_bytes(lk["gamma"])
        keep += [bt, gm]
        la[i] = QuotientLookupArgs(_rules_struct(lk["rules"], keep), ptr(lk["z"]), ptr(lk["pin"]), ptr(lk["ptab"]),
                                   bt.ctypes.data, gm.ctypes.data)
    sv = None
    if scale is not None:
        sv = _scalar_bytes(scale)
        keep.append(sv)
    call("h2b_quotient_fused", _ptr_table(d_fixed), len(d_fixed), _ptr_table(d_instance), len(d_instance),
         _ptr_table(d_advice), len(d_advice), ctypes.byref(g), yv.ctypes.data,
         ptr(d_l0) if d_l0 is not None else None, ptr(d_llast) if d_llast is not None else None,
         ptr(d_lactive) if d_lactive is not None else None, ctypes.byref(pa) if pa is not None else None, la,
         len(lookups), num_quotient, rot_scale, row_start, row_end, ptr(d_out), out_stride, out_offset,
         sv.ctypes.data if sv is not None else None, stream_handle(stream))
    return d_out


def quotient_lookups_device(d_values, d_table, d_z, d_pin, d_ptab, d_l0, d_llast, d_lactive, d_beta, d_gamma, d_y,
                            n, stream=None):
    call("_halo2_quotient_lookups", *[ptr(t) for t in (d_values, d_table, d_z, d_pin, d_ptab, d_l0, d_llast,
                                                       d_lactive, d_beta, d_gamma, d_y)], n, stream_handle(stream))


def quotient_permutation_device(d_values, d_l0, d_llast, d_lactive, d_prods, d_perms, d_cols, beta, gamma, y, delta,
                                delta_start, ext_omega, omega, chunk_len, last_rotation, rot_scale, isize, n,
                                stream=None):
    tabs = [to_dev(np.array([t.data_ptr() for t in lst], dtype=np.uint64), stream) for lst in (d_prods, d_perms, d_cols)]
    scal = [_scalar_bytes(x) for x in (beta, gamma, y, delta, delta_start, ext_omega, omega)]
    call("_halo2_quotient_permutation", ptr(d_values), ptr(d_l0), ptr(d_llast), ptr(d_lactive), ptr(tabs[0]),
         ptr(tabs[1]), ptr(tabs[2]), *[s.ctypes.data for s in scal], len(d_prods), chunk_len, len(d_cols),
         last_rotation, rot_scale, isize, n, stream_handle(stream))
    _keep_until_done(tabs, stream)


def _keep_until_done(tensors, stream):
    """Device tensors that a kernel queued on `stream` reads must not be
    reused before it ran: for a torch stream the caching allocator is told so
    (record_stream); for a raw handle the call waits for the stream."""
    torch = _torch()
    if stream is None or isinstance(stream, torch.cuda.Stream):
        s = stream if stream is not None else torch.cuda.current_stream()
        for t in tensors:
            t.record_stream(s)
    else:
        torch.cuda.synchronize()
