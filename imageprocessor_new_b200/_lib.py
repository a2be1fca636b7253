"""ctypes binding of libsubpx_b200.so, the package's only compute backend.

There is no CPU fallback: importing the binding on a machine without the built library or without a
CUDA device raises immediately, with the reason.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_longlong, c_size_t, c_void_p
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libsubpx_b200.so"

# Pixel dtype codes (include/subpx_b200.h).
DTYPES = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.float32): 2, np.dtype(np.float64): 3}

REFINE_CODES = {"none": 0, "weighted": 1, "logquad": 2, "logquadratic": 2, "edge_gradmoment": 3,
                "edge_moment": 3, "edges_centered": 3, "auto": 4}

STATUS_NAMES = ("ok", "no_signal", "insufficient_cell_pixels", "insufficient_fit_pixels", "singular_fit",
                "non_gaussian_fit", "contour_outside_cell", "incomplete_rays", "fit_diverged",
                "center_outside_cell", "edge_at_cell_border", "region_at_cell_border")

_P = c_void_p
_I = c_int
_D = c_double
_S = c_size_t

class BgMap(ctypes.Structure):
    """spx_bgmap (include/subpx_b200.h)."""

    _fields_ = [("rows", c_void_p), ("j1", c_void_p), ("t", c_void_p), ("ny", c_int), ("width", c_int),
                ("fixed", c_double), ("mode", c_int)]


class MethodOut(ctypes.Structure):
    """spx_method_out (include/subpx_b200.h)."""

    _fields_ = [("centers", c_void_p), ("contours", c_void_p), ("status", c_void_p), ("metrics", c_void_p),
                ("center_local", c_void_p), ("edge_px", c_void_p), ("eigenvalues", c_void_p), ("axes", c_void_p),
                ("n_metrics", c_int), ("metric_col_stride", c_longlong)]


class GemmEpilogue(ctypes.Structure):
    """spx_gemm_epilogue."""

    _fields_ = [("scale", ctypes.c_float), ("bias", c_void_p), ("relu", c_int), ("mask_act", c_void_p),
                ("ld_mask", c_int), ("out_f32", c_void_p), ("ld_f32", c_int), ("accumulate", c_int),
                ("out_bf16", c_void_p), ("ld_bf16", c_int), ("out_bf16_t", c_void_p), ("ld_t", c_int)]


class FitOptions(ctypes.Structure):
    """spx_fit_options: LM arithmetic (FIT_F64 / FIT_F32), the plain fits' relative cost tolerance and
    the rows per image of a stack (0: one image)."""
    _fields_ = [("precision", c_int), ("cost_tol", c_double), ("rows_per_image", c_int)]


FIT_F64, FIT_F32 = 0, 1
_BG = POINTER(BgMap)
_FO = POINTER(FitOptions)
_MO = POINTER(MethodOut)

# name -> (restype, argtypes)
SIGNATURES = {
    "spx_last_error": (ctypes.c_char_p, []),
    "spx_version": (_I, []),
    "spx_launch_count": (ctypes.c_ulonglong, []),
    "spx_device_info": (_I, [POINTER(c_int), POINTER(c_int)]),
    "spx_fp64_fma_rate": (_I, [_I, _I, _P, POINTER(c_double), _P]),
    "spx_otsu_workspace_bytes": (_S, [_I]),
    "spx_otsu": (_I, [_P, _I, _I, _I, _I, _P, _P, _S, _P]),
    "spx_otsu_static": (_I, [_P, _I, _I, _I, _I, _P, _P]),
    "spx_triangle": (_I, [_P, _I, _I, _I, _P, _P, _S, _P]),
    "spx_ccl_workspace_bytes": (_S, [_I, _I]),
    "spx_gemm_bf16": (_I, [_P, _I, _P, _I, _I, _I, _I, POINTER(GemmEpilogue), _P, _P]),
    "spx_deblend_initial_warm": (_I, [_P, _I, _D, _I, _I, _P, _P, _P, _P, _I, _I, _I, _I, _D, _I, _I, _P, _P, _D, _P,
                                      _P, _P, _P, _P, _P, _FO, _P, _S, _P]),
    "spx_mlp_loss_grad": (_I, [_P, _P, _P, _I, _I, _I, _P, _P, _P, _P]),
    "spx_rowsum_bf16": (_I, [_P, _I, _I, _P, _P]),
    "spx_adamw": (_I, [_P, _P, _P, _P, _I, _I, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                       ctypes.c_float, _P, _I, _P, _I, _P]),
    "spx_transpose_bf16": (_I, [_P, _I, _I, _P, _P]),
    "spx_mlp_outputs_to_params": (_I, [_P, _P, _P, _P, _P, _I, _P, _P, _P]),
    "spx_extract_patches": (_I, [_P, _I, _D, _I, _I, _P, _I, _P, _P, _P]),
    "spx_extract_patches_stack": (_I, [_P, _I, _D, _I, _I, _I, _P, _P, _I, _P, _P, _P]),
    "spx_hole_coverage": (_I, [_I, _I, _P, _P, _P, _I, _I, _D, _I, _P, _P]),
    "spx_page_finish": (_I, [_P, c_longlong, _D, _D, _D, ctypes.c_ulonglong, _P, _P]),
    "spx_tune_set": (_I, [ctypes.c_char_p, _I]),
    "spx_tune_get": (_I, [ctypes.c_char_p, POINTER(c_int)]),
    "spx_histogram": (_I, [_P, _I, _I, _I, _I, _P, _P, _P]),
    "spx_otsu_from_histogram": (_I, [_P, _I, _P, c_longlong, _P, _P, _S, _P]),
    "spx_binarize": (_I, [_P, _I, _I, _I, _P, _D, _I, _P, _P]),
    "spx_morphology": (_I, [_P, _I, _I, _I, _I, _P, _P]),
    "spx_ccl_label": (_I, [_P, _I, _I, _I, _P, _D, _I, _I, _P, _P, _P, _S, _P]),
    "spx_ccl_finish": (_I, [_P, _I, _I, _I, _I, _P, _P, _P, _S, _P]),
    "spx_select_workspace_bytes": (_S, [_I]),
    "spx_select_components": (_I, [_P, _I, _I, _I, _I, _D, _P, _P, _P, _P, _S, _P]),
    "spx_component_rows": (_I, [_P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _S, _P]),
    "spx_status_name": (ctypes.c_char_p, [_I]),
    "spx_status_text": (_I, [_P, _I, _P, _P]),
    "spx_refine_centers_counted": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _I, _I, _P, _P]),
    "spx_refine_centers": (_I, [_P, _I, _I, _I, _P, _P, _P, _I, _I, _P, _P]),
    "spx_keep_band_workspace_bytes": (_S, [_I]),
    "spx_keep_band": (_I, [_P, _I, _D, _D, _D, _P, _P, _I, _P, _S, _P]),
    "spx_dedupe_workspace_bytes": (_S, [_I, _D, _D, _D, _D, _D]),
    "spx_dedupe_centers": (_I, [_P, _I, _D, _D, _D, _D, _D, _P, _P, _P, _S, _P]),
    "spx_voronoi_workspace_bytes": (_S, [_I, _I, _I]),
    "spx_voronoi_labels": (_I, [_P, _I, _I, _I, _P, _P, _S, _P]),
    "spx_seed_distance_map": (_I, [_P, _I, _I, _I, _P, _P, _S, _P]),
    "spx_nearest_distances": (_I, [_P, _I, _P, _I, _I, _I, _I, _P, _P, _S, _P]),
    "spx_cells_setup": (_I, [_P, _I, _I, _I, _I, _P, _P, _P, _P, _P]),
    "spx_fit_workspace_bytes": (_S, [_I]),
    "spx_deblend_initial": (_I, [_P, _I, _D, _I, _I, _P, _P, _P, _P, _I, _I, _I, _I, _D, _I, _I, _P, _P, _P, _P,
                                 _S, _P]),
    "spx_deblend_iteration": (_I, [_P, _I, _D, _I, _I, _P, _P, _P, _I, _I, _I, _I, _BG, _P, _I, _P, _D, _I, _P,
                                   _P, _P, _P, _FO, _P, _S, _P]),
    "spx_render_workspace_bytes": (_S, [_I, _I, _I]),
    "spx_render_model": (_I, [_P, _P, _I, _I, _I, _I, _P, _P, _S, _P]),
    "spx_render_overflow": (_I, [_P, _I, _I, _I, POINTER(c_int), _I, _P]),
    "spx_quantiles": (_I, [_P, _I, _P, _P]),
    "spx_cell_stats": (_I, [_P, _P, _I, _P, _P, _P]),
    "spx_background_at": (_I, [_BG, _I, _I, _P, _I, _D, _P, _P]),
    "spx_clean_cells": (_I, [_P, _I, _D, _I, _I, _P, _P, _P, _I, _BG, _P, _P, _I, _I, _I, _P, _P]),
    "spx_tile_medians": (_I, [_P, _I, _D, _I, _I, _P, _P, _P, _I, _D, _D, _I, _P, _P, _P]),
    "spx_background_rows": (_I, [_P, _I, _I, _I, _I, _P, _P]),
    "spx_residual": (_I, [_P, _I, _D, _I, _I, _BG, _P, _P, _P]),
    "spx_gaussian_filter": (_I, [_P, _I, _I, _P, _I, _P, _P, _P]),
    "spx_maximum_filter": (_I, [_P, _I, _I, _I, _P, _P, _P]),
    "spx_find_peaks": (_I, [_P, _P, _P, _I, _I, _D, _P, _I, _P, _P]),
    "spx_label_mask": (_I, [_P, _P, _I, _I, _I, _P, _P, _P]),
    "spx_gaussian_method": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _MO, _P]),
    "spx_logquad_cd": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _D, _MO, _P]),
    "spx_projection_cd": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _D, _P, _P, _I, _P, _P, _I, _MO, _P]),
    "spx_half_area_workspace_bytes": (_S, [_I, _I, _I]),
    "spx_half_area_cd": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _P, _P, _I, _D, _I, _I, _I, _MO, _MO, _P, _S, _P]),
    "spx_wide_cells_workspace_bytes": (_S, [_I, _I, _I, _I, _D]),
    "spx_wide_cells": (_I, [_P, _I, _D, _I, _I, _BG, _P, _P, _P, _I, _I, _I, _P, _I, _I, _D, _D, _P, _P, _P, _P, _P,
                            _P, _P, _S, _P]),
    "spx_tail_area_workspace_bytes": (_S, [_I, _I, _I]),
    "spx_tail_area_cd": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _I, _P, _P, _I, _D, _I, _I, _P, _MO, _MO, _MO, _MO, _MO,
                              _P, _S, _P]),
    "spx_radial_workspace_bytes": (_S, [_I, _I, _I]),
    "spx_radial_cd": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _D, _P, _I, _MO, _MO, _P, _S, _P]),
    "spx_minimum_filter": (_I, [_P, _I, _I, _I, _P, _P, _P]),
    "spx_support_labels": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _P, _P, _P]),
    "spx_clean_masked": (_I, [_P, _I, _D, _I, _I, _P, _P, _P, _I, _BG, _P, _I, _I, _I, _P, _P]),
    "spx_rebuild_contours": (_I, [_I, _P, _P, _P, _P, _P, _P, _I, _I, _P, _P]),
    "spx_signal_image": (_I, [_P, _I, _D, _I, _I, _P, _P]),
    "spx_pitch_workspace_bytes": (_S, [_I, _I, _I]),
    "spx_pitch_crop": (_I, [_P, _I, _D, _I, _I, _I, _P, _P, _S, _P]),
    "spx_pitch_from_autocorrelation": (_I, [_P, _I, _I, _I, _P, _P, _S, _P]),
    "spx_peak_workspace_bytes": (_S, [_I, _I]),
    "spx_peak_candidates": (_I, [_P, _P, _P, _I, _I, _P, _P, _I, _P, _P, _S, _P]),
    "spx_peak_select_workspace_bytes": (_S, [_I]),
    "spx_peak_select": (_I, [_P, _P, _I, _P, _D, _P, _I, _I, _P, _P, _P, _S, _P]),
}

class QuantileReq(ctypes.Structure):
    """The request struct of spx_quantiles."""

    _fields_ = [("values", c_void_p), ("stride", c_int), ("mask", c_void_p), ("finite_only", c_int), ("n", c_int),
                ("mode", c_int), ("q", c_double)]


BG_MAP, BG_FIXED = 0, 1
TILE_FREE, TILE_USABLE, TILE_ALL = 0, 1, 2


class LibraryError(RuntimeError):
    """A libsubpx_b200 entry point returned an error status."""


def load_library(path: Path | str = LIB_PATH) -> ctypes.CDLL:
    """Loads the shared library and declares every exported entry point (no GPU needed)."""
    path = Path(path)
    if not path.exists():
        raise RuntimeError(f"{path.name} is not built; run `python -m imageprocessor_new_b200.build`")
    lib = ctypes.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """The loaded library, after checking that a CUDA device is usable."""
    global _LIB
    if _LIB is None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("imageprocessor_new_b200 needs a CUDA device (B200, sm_100a); none is visible")
        _LIB = load_library()
    return _LIB


def call(name: str, *args) -> int:
    """Calls an entry point and raises LibraryError with spx_last_error() on a non-zero status."""
    fn = getattr(lib(), name)
    status = fn(*args)
    if status != 0:
        msg = lib().spx_last_error().decode(errors="replace")
        raise LibraryError(f"{name}: {msg} (status {status})")
    return status


def size(name: str, *args) -> int:
    return int(getattr(lib(), name)(*args))
