"""ctypes binding of ``libfastlpr_b200.so`` (the C ABI in include/fastlpr_b200.h).

The library is mandatory: importing the GPU entry points without it raises,
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from typing import Dict, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("FASTLPR_B200_LIB", os.path.join(_HERE, "libfastlpr_b200.so"))

FLPR_PREC_F32 = 0
FLPR_PREC_F64 = 1

# (name, restype, argtypes) for every exported symbol of include/fastlpr_b200.h
_VP, _I, _I64, _D, _SZ = C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_size_t
_PI, _PD = C.POINTER(C.c_int), C.POINTER(C.c_double)
_PVP = C.POINTER(C.c_void_p)
SIGNATURES = [
    ("flpr_last_error", C.c_char_p, []),
    ("flpr_version", _I, []),
    ("flpr_launch_count", _I64, []),
    ("flpr_set_tuning", _I, [_I, _I]),
    ("flpr_get_tuning", _I, [_I]),
    ("flpr_create", _I, [C.POINTER(_VP), _I]),
    ("flpr_destroy", _I, [_VP]),
    ("flpr_point_stats_ws", _SZ, [_I, _I64]),
    ("flpr_point_stats", _I, [_I, _I64, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_point_stats_noalloc", _I, [_I, _I64, _VP, _VP, _VP]),
    ("flpr_spread_ws", _SZ, [_I, _I64, _PI, _I, _I, _I]),
    ("flpr_spread", _I, [_I, _I64, _VP, _PD, _PI, _I, _PD, _I, _I, _PVP, _VP, _I, _VP, _SZ, _VP]),
    ("flpr_spread_dkmap", _I, [_I, _I64, _VP, _VP, _PD, _PI, _I, _PD, _I, _I, _PVP, _VP, _I, _VP,
                               _SZ, _VP]),
    ("flpr_spread_grid64", _I, [_I, _I64, _PI, _I, _I, _VP, _SZ, _VP, _VP]),
    ("flpr_spread_grid64_channels", _I, [_I, _I64, _PI, _I, _I, _I, _VP, _SZ, _VP, _VP]),
    ("flpr_knot_map", _I, [_I, _I64, _VP, _PD, _PD, _PD, _VP, _VP]),
    ("flpr_forward_fft_ws", _SZ, [_VP, _I, _PI, _I, _I]),
    ("flpr_forward_fft", _I, [_VP, _I, _PI, _I, _VP, _VP, _I, _VP, _SZ, _VP]),
    ("flpr_oversample_crop", _I, [_I, _PI, _PI, _I, _PD, _I, _VP, _VP, _I, _VP]),
    ("flpr_kernel_factors_ws", _SZ, [_VP, _I, _PI, _I, _I]),
    ("flpr_kernel_factors", _I, [_VP, _I, _PI, _PI, _PD, _PD, _I, _VP, _I, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_kernel_spectra_ws", _SZ, [_VP, _I, _PI, _I]),
    ("flpr_kernel_spectra", _I, [_VP, _I, _PI, _PI, _PD, _PD, _I, _I, _VP, _I, _PI, _VP, _VP,
                                 _SZ, _VP]),
    ("flpr_conv_full", _I, [_VP, _I, _PI, _PI, _PI, _I, _VP, _VP, _I, _PI, _PI, _D, _I, _VP, _I,
                            _VP, _SZ, _VP]),
    ("flpr_conv_ws", _SZ, [_VP, _I, _PI, _I, _I]),
    ("flpr_conv2d_sep_ws", _SZ, [_VP, _PI, _PI, _I, _I]),
    ("flpr_conv2d_sep", _I, [_VP, _PI, _PI, _PI, _I, _I, _VP, _VP, _I, _PI, _PI, _PI, _D, _I, _VP,
                             _I, _VP, _SZ, _VP]),
    ("flpr_conv", _I, [_VP, _I, _PI, _PI, _PI, _I, _I, _VP, _VP, _I, _PI, _PI, _PI, _D, _I, _VP,
                       _I, _VP, _SZ, _VP]),
    ("flpr_solve", _I, [_I, _I, _I, _I, _I64, _I, _VP, _VP, _D, _VP, _VP, _I, _VP]),
    ("flpr_solve_reduce", _I, [_I, _I, _I, _I, _I64, _I, _VP, _VP, _D, _I, _VP, _VP, _VP, _VP,
                               _I, _VP]),
    ("flpr_solve_reduce_given", _I, [_I, _I, _I, _I, _I64, _I, _VP, _VP, _D, _I, _VP, _VP, _VP,
                                     _VP, _I, _VP]),
    ("flpr_scalar_of", _I, [_I, _I, _I, _I64, _VP, _I, _VP, _VP, _VP]),
    ("flpr_deposit", _I, [_I, _I64, _VP, _PD, _PI, _I, _PVP, _VP, _VP, _VP, _VP]),
    ("flpr_deposit_sorted_ws", _SZ, [_I, _I64, _PI, _I, _I]),
    ("flpr_deposit_sorted", _I, [_I, _I64, _VP, _PI, _I, _I, _I, _PVP, _VP, _SZ, _PD, _PI, _PI,
                                 _VP, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_stencil_quad", _I, [_I, _PI, _I, _I, _VP, _VP, _VP, _VP]),
    ("flpr_stencil_quad_fixed_ws", _SZ, [_I, _PI, _I, _I]),
    ("flpr_stencil_quad_fixed", _I, [_I, _PI, _I, _I, _VP, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_lpr2d_fused_supported", _I, [_PI, _PI, _PI, _I, _I, _I]),
    ("flpr_lpr2d_fused_ws", _SZ, [_PI, _PI, _PI, _I, _I, _I]),
    ("flpr_lpr2d_fused", _I, [_PI, _PI, _PI, _I, _I, _I, _I, _I, _VP, _VP, _D, _VP, _D, _VP, _VP,
                              _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_lpr2d_fused_floor", _I, [_PI, _PI, _PI, _I, _I, _I, _I, _I, _VP, _VP, _D, _VP, _D,
                                    _VP, _VP, _VP, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_lpr2d_fused_t", _I, [_PI, _PI, _PI, _I, _I, _I, _I, _I, _VP, _VP, _D, _VP, _D, _VP,
                                _VP, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_lpr2d_fused_ex_supported", _I, [_I, _PI, _PI, _PI, _I, _I, _I]),
    ("flpr_lpr2d_fused_ex_ws", _SZ, [_I, _PI, _PI, _PI, _I, _I, _I]),
    ("flpr_lpr2d_fused_ex", _I, [_I, _I, _PI, _PI, _PI, _I, _I, _I, _I, _I, _VP, _VP, _D, _VP,
                                 _D, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_interp_reduce_ws", _SZ, [_I64, _I, _I, _I]),
    ("flpr_interp_reduce", _I, [_I, _I64, _VP, _PD, _PI, _I, _I, _I, _VP, _PVP, _PVP, _VP, _VP,
                                _VP, _VP, _SZ, _VP]),
    ("flpr_interp_eval", _I, [_I, _I64, _VP, _PD, _PI, _I, _VP, _VP, _VP]),
    ("flpr_interp_eval_extrap", _I, [_I, _I64, _VP, _PD, _PI, _I, _VP, _VP, _VP]),
    ("flpr_spline_prefilter", _I, [_I, _PI, _I64, _I, _VP, _VP, _VP]),
    ("flpr_gcv_select", _I, [_I, _I, _I, _I, _I, _I, _D, _D, _VP, _VP, _VP, _VP, _VP]),
    ("flpr_select_grid", _I, [_I64, _I, _I, _I, _VP, _VP, _I, _VP, _VP, _VP, _VP]),
    ("flpr_spline_reduce", _I, [_I, _I64, _VP, _VP, _PI, _I, _I, _I, _VP, _PVP, _PVP, _VP, _VP,
                                _VP, _VP]),
    ("flpr_spline_eval", _I, [_I, _I64, _VP, _VP, _PI, _I, _VP, _VP, _VP]),
    ("flpr_kde_ws", _SZ, [_I64, _I, _I64]),
    ("flpr_kde_lcv", _I, [_I, _I64, _VP, _PD, _PI, _I, _VP, _D, _PD, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_log_shift", _I, [_I64, _VP, _D, _VP, _VP]),
    ("flpr_exp_weighted_sum", _I, [_I64, _VP, _VP, _VP, _VP]),
    ("flpr_bin_moments", _I, [_I, _I64, _VP, _VP, _VP, _VP, _VP]),
    ("flpr_learned_features", _I, [_I, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    ("flpr_learned_window", _I, [_I, _VP, _D, _D, _I, _VP, _I, _VP, _VP, _I, _VP, _VP, _VP]),
    ("flpr_copy_rows", _I, [_VP, _VP, _I64, _I, _VP, _VP]),
    ("flpr_mlp_gemm", _I, [_I, _I, _I, _VP, _I, _I, _VP, _I, _I, _VP, _I, _VP, _I, _VP, _VP, _I,
                           _VP]),
    ("flpr_mlp_param_count", _I64, [_I, _PI]),
    ("flpr_mlp_ws", _SZ, [_I, _PI, _I]),
    ("flpr_mlp_fwd", _I, [_I, _PI, _VP, _VP, _I, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_mlp_bwd", _I, [_I, _PI, _VP, _I, _VP, _VP, _VP, _VP, _SZ, _VP]),
    ("flpr_mlp_step", _I, [_I64, _VP, _VP, _VP, _VP, _VP, C.c_float, C.c_float, C.c_float,
                           C.c_float, C.c_float, _I, _VP]),
    ("flpr_mlp_mse", _I, [_I, _VP, _VP, _VP, _VP, _VP]),
    ("flpr_to_bf16", _I, [_I64, _VP, _VP, _VP]),
    ("flpr_mlp_infer_supported", _I, [_I, _PI]),
    ("flpr_mlp_infer", _I, [_I, _PI, _VP, _VP, _I, _VP, _VP, _VP, _VP]),
]


class FastLPRError(RuntimeError):
    """Error status returned by the CUDA library."""


_lib: Optional[C.CDLL] = None
_lib_lock = threading.Lock()


def load() -> C.CDLL:
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"fastlpr_b200 CUDA library not found at {LIB_PATH}; build it with "
                    "`python -m fastlpr_b200.build` (there is no CPU fallback)")
            lib = C.CDLL(LIB_PATH)
            for name, res, args in SIGNATURES:
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = load().flpr_last_error().decode(errors="replace")
        raise FastLPRError(f"{what} failed with status {status}: {msg}")


def _carray(vals, np_type, c_type):
    # one conversion pass in numpy and one copy into the ctypes array (a
    # Python-level loop per element costs more than the calls it feeds)
    a = np.ascontiguousarray(vals, dtype=np_type).reshape(-1)
    if a.size == 0:
        a = np.zeros(1, dtype=np_type)
    return (c_type * a.size).from_buffer_copy(a)


def ivec(vals: Sequence[int]):
    return _carray(vals, np.int32, C.c_int)


def dvec(vals: Sequence[float]):
    return _carray(vals, np.float64, C.c_double)


def pvec(ptrs: Sequence[int]):
    return _carray([int(p) for p in ptrs], np.uint64, C.c_void_p)


_handles: Dict[int, C.c_void_p] = {}


def handle(device: int) -> C.c_void_p:
    """Per-device library handle (owns the cuFFT plan cache)."""
    h = _handles.get(device)
    if h is None:
        h = C.c_void_p()
        check(load().flpr_create(C.byref(h), device), "flpr_create")
        _handles[device] = h
    return h
