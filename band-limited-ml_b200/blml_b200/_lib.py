"""ctypes binding of libblml_b200.so (the C ABI declared in include/blml_b200.h).

The library is the only compute path: there is no CPU fallback. Loading fails loudly when the shared library is
missing, and every call raises BLMLError when the library returns an error status."""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libblml_b200.so')

F64, F32 = 0, 1
ENGINE_SIMT, ENGINE_TC = 0, 1
ROUTE_AUTO, ROUTE_CONTRACT, ROUTE_FFT = 0, 1, 2


class BLMLError(RuntimeError):
    pass


class Tables(C.Structure):
    """blml_tables: the pair kernels' value tables (device pointers)."""
    _fields_ = [('d', C.c_int), ('U', C.c_int), ('G', C.c_int), ('nW', C.c_int), ('LR', C.c_int), ('f32', C.c_int),
                ('nT', C.c_int64), ('ndT', C.c_int64),
                ('T', C.c_void_p), ('base', C.c_void_p), ('Jk', C.c_void_p), ('mk', C.c_void_p),
                ('kinds', C.c_void_p), ('nbins', C.c_void_p), ('grp', C.c_void_p), ('RT', C.c_void_p),
                ('dim_unit', C.c_void_p), ('grp_unit', C.c_void_p), ('dT', C.c_void_p), ('dbase', C.c_void_p),
                ('dR', C.c_void_p), ('wunit', C.c_void_p), ('wcol', C.c_void_p), ('wgrp', C.c_void_p),
                ('T32', C.c_void_p), ('RT32', C.c_void_p), ('dT32', C.c_void_p), ('dR32', C.c_void_p)]


class PointCol(C.Structure):
    """blml_point_col: one column's exact kernel for blml_point_rows."""
    _fields_ = [('kind', C.c_int), ('M', C.c_int), ('Mi', C.c_int), ('f', C.c_double), ('fi', C.c_double),
                ('P', C.c_double)]


PT_SINC, PT_SLITS, PT_DIRICHLET, PT_BALL = 0, 1, 2, 3
SEG_SPLIT_BLOCKS = 2048                 # BLML_SEG_SPLIT_BLOCKS: the history kernels' blocks, shared out by fit size

_P, _I, _L, _D = C.c_void_p, C.c_int, C.c_int64, C.c_double
_SIGS = {
    'blml_last_error': (C.c_char_p, []),
    'blml_abi_version': (_I, []),
    'blml_reduce_blocks': (_I, []),
    'blml_launch_count': (_L, []),
    'blml_plan_create': (_I, [_I, _P, _P, _P, _P, _I, _I, C.POINTER(_P)]),
    'blml_plan_destroy': (_I, [_P]),
    'blml_plan_status': (_I, [_P]),
    'blml_matvec_workspace': (_L, [_P, _I]),
    'blml_matvec': (_I, [_P, _P, _P, _I, _I, _P, _L, _P]),
    'blml_group_create': (_I, [_I, _P, _P, _I, _P, _P, _P, _P, C.POINTER(_P)]),
    'blml_group_matvec': (_I, [_P, _P]),
    'blml_group_destroy': (_I, [_P]),
    'blml_spectrum_workspace': (_L, [_P, _I]),
    'blml_spectrum': (_I, [_P, _P, _P, _I, _I, _P, _L, _P]),
    'blml_planewave_points': (_I, [_I, _I, _P, _P, _P, _L, _P, _P, _P]),
    'blml_plan_set_route': (_I, [_P, _I]),
    'blml_plan_route': (_I, [_P]),
    'blml_group_set_route': (_I, [_P, _I]),
    'blml_group_route': (_I, [_P]),
    'blml_fft_set_shape': (_I, [_I, _I]),
    'blml_fft_get_shape': (_I, [_P, _P]),
    'blml_seg_blocks': (_I, []),
    'blml_seg_start_root': (_I, [_I, _I, _P, _P, _P, _P, _P, _P]),
    'blml_seg_update_real1': (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    'blml_seg_merit': (_I, [_I, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    'blml_seg_resid': (_I, [_I, _I, _P, _I, _P, _P, _P, _P, _P, _P, _P]),
    'blml_seg_dots': (_I, [_I, _I, _P, _I, _I, _P, _P, _P, _P, _P]),
    'blml_seg_lincomb': (_I, [_I, _I, _P, _I, _P, _I, _P, _P, _P]),
    'blml_seg_lgrad_weights': (_I, [_I, _I, _P, _I, _P, _P, _P, _P, _P, _P, _P]),
    'blml_seg_lgrad_finish': (_I, [_I, _I, _P, _I, _P, _P, _P, _P, _P, _P]),
    'blml_seg_trials': (_I, [_I, _I, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    'blml_seg_axpy2': (_I, [_I, _I, _P, _I, _P, _P, _P, _P, _P, _P]),
    'blml_seg_finish': (_I, [_I, _I, _P, _I, _P, _P, _P, _P, _P, _P, _P]),
    'blml_seg_log_score': (_I, [_I, _I, _P, _I, _P, _P, _P, _D, _P, _P, _P]),
    'blml_seg_val_score': (_I, [_I, _I, _P, _P, _P, _P, _P, _P]),
    'blml_seg_phases': (_I, [_I, _I, _P, _D, _P, _P, _P]),
    'blml_seg_real_to_complex': (_I, [_I, _I, _P, _P, _P, _P, _P]),
    'blml_seg_cert_weights': (_I, [_I, _I, _P, _P, _P, _P, _P]),
    'blml_seg_append_mode': (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    'blml_group_matvec_masked': (_I, [_P, _P, _I, _P, _P]),
    'blml_seg_dots2': (_I, [_I, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    'blml_nn_gemm_bf16': (_I, [_P, _P, _P, _I, _I, _I, _I, _P, _P]),
    'blml_nn_im2col': (_I, [_P, _I, _I, _I, _I, _I, _I, _P, _I, _P]),
    'blml_nn_col2im': (_I, [_P, _I, _I, _I, _I, _P, _I, _I, _P]),
    'blml_nn_bias_act': (_I, [_P, _I, _L, _I, _P, _I, _P, _I, _I, _P]),
    'blml_nn_relu_bwd': (_I, [_P, _I, _I, _P, _I, _I, _L, _I, _P, _P, _P]),
    'blml_nn_bias_grad': (_I, [_P, _I, _I, _P, _I, _I, _L, _I, _I, _I, _P, _P, _P]),
    'blml_nn_sum_splits': (_I, [_P, _I, _L, _P, _P]),
    'blml_nn_pool_fwd': (_I, [_P, _I, _I, _I, _I, _I, _I, _P, _I, _I, _P]),
    'blml_nn_pool_bwd_add': (_I, [_P, _I, _I, _I, _I, _P, _I, _I, _P]),
    'blml_nn_up_fwd': (_I, [_P, _I, _I, _I, _I, _P, _I, _I, _P]),
    'blml_nn_up_bwd': (_I, [_P, _I, _I, _I, _I, _I, _I, _P, _P]),
    'blml_nn_head_fwd': (_I, [_P, _L, _I, _P, _P, _I, _P, _P]),
    'blml_nn_head_bwd': (_I, [_P, _P, _L, _I, _I, _P, _P, _I, _P, _P, _P]),
    'blml_nn_phase_loss': (_I, [_P, _P, _L, _I, _P, _P, _P, _P]),
    'blml_nn_adam': (_I, [_P, _P, _P, _P, _L, C.c_float, C.c_float, C.c_float, C.c_float, _I, _P, _P, _I, _I, _P]),
    'blml_nn_to_bf16': (_I, [_P, _L, _P, _P, _I, _I, _P]),
    'blml_lbfgs_batch_create': (_I, [_I, _I, _P, _P, _I, _D, _D, _L, _P, _P, _P, _P, _P, C.POINTER(_P)]),
    'blml_lbfgs_batch_set_caps': (_I, [_P, _P]),
    'blml_lbfgs_batch_set_history': (_I, [_P, _I]),
    'blml_seg_dots2_h32': (_I, [_I, _P, _P, _I, _P, _P, _P, _P, _P, _P, _P]),
    'blml_seg_split_ints': (_L, [_I]),
    'blml_seg_lincomb_h32': (_I, [_I, _P, _P, _P, _I, _I, _P, _P, C.c_uint64, _P]),
    'blml_lanczos_coef': (_I, [_I, _I, _P, _P, _P, _I, _P]),
    'blml_lanczos_beta': (_I, [_I, _P, _P, _P, _P]),
    'blml_lbfgs_batch_run': (_I, [_P, _P]),
    'blml_lbfgs_batch_result': (_I, [_P, _P, _P, _P, _P, _P]),
    'blml_lbfgs_batch_stats': (_I, [_P, _P]),
    'blml_lbfgs_batch_destroy': (_I, [_P]),
    'blml_start_batch_create': (_I, [_I, _P, _P, _I, _D, _L, _L, _P, _P, _P, _P, _P, C.POINTER(_P)]),
    'blml_start_batch_run': (_I, [_P, _P]),
    'blml_start_batch_result': (_I, [_P, _P, _P]),
    'blml_start_batch_stats': (_I, [_P, _P]),
    'blml_start_batch_destroy': (_I, [_P]),
    'blml_jacobi_update': (_I, [_I, _I, _L, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    'blml_merit_terms': (_I, [_I, _I, _L, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    'blml_resid': (_I, [_I, _I, _L, _I, _P, _P, _P, _D, _P, _P, _P]),
    'blml_dots': (_I, [_I, _L, _I, _P, _P, _P, _P, _P]),
    'blml_lincomb': (_I, [_I, _L, _P, _I, _P, _P, _P]),
    'blml_mul_bins': (_I, [_I, _I, _L, _I, _P, _P, _P, _P]),
    'blml_lgrad_weights': (_I, [_I, _I, _L, _I, _P, _P, _D, _P, _P, _P, _P]),
    'blml_lgrad_finish': (_I, [_I, _I, _L, _I, _P, _P, _P, _D, _P, _P]),
    'blml_pgrad_weights': (_I, [_I, _I, _L, _I, _P, _P, _D, _P, _P, _P, _P]),
    'blml_hvp_inner': (_I, [_I, _I, _L, _I, _P, _P, _P, _P, _P]),
    'blml_mixed_terms': (_I, [_I, _I, _L, _I, _P, _I, _P, _P, _P, _P, _P]),
    'blml_hvp_real1': (_I, [_I, _L, _P, _P, _P, _P, _P, _P]),
    'blml_counts_axpy': (_I, [_I, _L, _D, _P, _D, _P, _I, _P, _P]),
    'blml_bin_ratio': (_I, [_I, _L, _P, _P, _P, _P]),
    'blml_new_bins': (_I, [_I, _I, _L, _I, _P, _P, _P, _P, _P]),
    'blml_gain_sums': (_I, [_I, _L, _P, _D, _P, _D, _P, _D, _P, _P, _P]),
    'blml_point_rows': (_I, [_L, _I, _P, _L, _P, _P, _P, _P, _P]),
    'blml_point_rows_multi': (_I, [_L, _I, _P, _L, _P, _P, _I, _P, _P, _I, _P, _P, _P]),
    'blml_block_root': (_I, [_I, _P, _L, _P, _P, _P, _D, _P, _P]),
    'blml_block_search': (_I, [_I, _P, _L, _P, _P, _P, _P, _P, _P, _P]),
    'blml_block_apply': (_I, [_I, _P, _L, _P, _D, _P, _P]),
    'blml_gather_rows_i64': (_I, [_I, _I, _P, _P, _L, _P, _P]),
    'blml_lbfgs_trial': (_I, [_I, _I, _L, _I, _P, _P, _P, _P, _P, _D, _P, _P, _P, _P, _P]),
    'blml_finish': (_I, [_I, _I, _L, _I, _P, _P, _D, _P, _P, _P, _P]),
    'blml_log_score': (_I, [_I, _I, _L, _I, _P, _P, _D, _D, _P, _P, _P]),
    'blml_start_root': (_I, [_I, _L, _P, _P, _D, _P, _P]),
    'blml_fill_modes': (_I, [_I, _I, _L, _I, _I, _I, _D, _P, _P, _P]),
    'blml_cert_weights': (_I, [_I, _I, _L, _I, _P, _P, _P, _P]),
    'blml_rows': (_I, [C.POINTER(Tables), _P, _L, _P, _L, _P, _I, _P, _P, _P]),
    'blml_rows_multi': (_I, [C.POINTER(Tables), _P, _L, _P, _L, _P, _I, _P, _P, _P]),
    'blml_cols': (_I, [C.POINTER(Tables), _P, _L, _P, _L, _P, _I, _P]),
    'blml_cols_dep': (_I, [C.POINTER(Tables), _P, _L, _P, _L, _L, _P, _P, _I, _P]),
    'blml_lattice_coords': (_I, [_P, _L, _I, _P, _P, _P]),
    'blml_rows_plan_create': (_I, [C.POINTER(Tables), _P, _L, _P, C.POINTER(_P)]),
    'blml_rows_plan_workspace': (_L, [_P, _L, _L]),
    'blml_rows_plan_run': (_I, [_P, _P, _L, _P, _L, _P, _P, _P, _L, _P]),
    'blml_rows_plan_destroy': (_I, [_P]),
    'blml_rows_noalloc': (_I, [C.POINTER(Tables), _P, _L, _P, _L, _P, _P, _P]),
}
EXPORTS = tuple(_SIGS)

_lib = None


def lib():
    """The loaded library (raises when it was not built: python -m blml_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BLMLError(f'{LIB_PATH} is missing: build it with `python -m blml_b200.build` (no CPU fallback)')
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
        _apply_tuning(L)
    return _lib


TUNING_PATH = os.path.join(_HERE, 'fft_tuning.json')


def _apply_tuning(L):
    """The FFT route's launch shape from the autotuner's table (bench.py --tune writes it), if the package has one."""
    if os.path.exists(TUNING_PATH):
        import json
        t = json.load(open(TUNING_PATH))
        if L.blml_fft_set_shape(int(t['cta_bytes']), int(t['max_cols'])) != 0:
            raise BLMLError(f'{TUNING_PATH}: {L.blml_last_error().decode(errors="replace")}')


def check(rc, what):
    if rc != 0:
        msg = lib().blml_last_error().decode(errors='replace')
        raise BLMLError(f'{what} failed ({rc}): {msg}')


def call(name, *args):
    check(getattr(lib(), name)(*args), name)


def ptrs(arrs):
    """A ctypes array of device pointers from tensors (or raw ints)."""
    vals = [a if isinstance(a, int) else a.data_ptr() for a in arrs]
    return (C.c_void_p * max(len(vals), 1))(*vals)


def dbl(vals):
    vals = [float(v) for v in vals]
    return (C.c_double * max(len(vals), 1))(*vals)


def host_ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def i64(vals):
    return np.ascontiguousarray(vals, np.int64)
