"""ctypes binding of the C ABI in ``include/aldvc_b200.h``.

The structs mirror the header field for field; every entry point returns an int that
:func:`check` turns into a ``RuntimeError`` carrying ``aldvc_last_error()``.  There is no
fallback: if the library is missing, loading raises.
"""

from __future__ import annotations

import ctypes
import os

from .build import LIB

ALDVC_OK = 0
BATCHED = 0
PLAIN = 1
NCC_TILED = 0
NCC_PLAIN = 1
NCC_FFT = 2
NCC_FFT_STOCKHAM = 3
NCC_FFT_CLUSTER = 4

_p = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_d = ctypes.c_double
_sz = ctypes.c_size_t


class Volumes(ctypes.Structure):
    _fields_ = [("f", _p), ("gx", _p), ("gy", _p), ("gz", _p), ("mask", _p), ("g", _p), ("nz", _i64), ("ny", _i64),
                ("nx", _i64), ("g4", _p)]


class Subset(ctypes.Structure):
    _fields_ = [("hx", _i32), ("hy", _i32), ("hz", _i32), ("stride", _i32), ("mode", _i32), ("reserved", _i32),
                ("split_index", _p), ("split_keep", _p), ("keep_bytes", _i64), ("node_half", _p)]


class IcgnParams(ctypes.Structure):
    _fields_ = [("tol", _d), ("dp_tol", _d), ("max_iter", _i32), ("patience", _i32), ("noise_gain", _d),
                ("predictive", _i32), ("variant", _i32), ("threads", _i32), ("brick_floats", _i32), ("mu", _d),
                ("n_full", _d), ("sweep_rows", _i32), ("reserved", _i32), ("node_order", _p)]


class Hex8Mesh(ctypes.Structure):
    _fields_ = [("nx", _i64), ("ny", _i64), ("nz", _i64), ("sx", _d), ("sy", _d), ("sz", _d), ("elem_active", _p),
                ("gauss_order", _i32), ("reserved", _i32)]


# name -> (restype, argtypes); the full exported surface of include/aldvc_b200.h
PROTOTYPES = {
    "aldvc_abi_version": (_i32, []),
    "aldvc_last_error": (ctypes.c_char_p, []),
    "aldvc_launch_count": (ctypes.c_ulonglong, []),
    "aldvc_kernel_timing": (_i32, [_i32]),
    "aldvc_kernel_timing_read": (_i32, [_i32, _p, _i32, _p, _p]),
    "aldvc_device_info": (_i32, [ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "aldvc_gradients": (_i32, [_p, _i64, _i64, _i64, _i32, _p, _p, _p, _p]),
    "aldvc_precompute_grid_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _i64]),
    "aldvc_precompute_grid": (_i32, [ctypes.POINTER(Volumes), ctypes.POINTER(Subset), _p, _i64, _p, _i64, _p, _i64, _d, _d, _p, _p, _p,
                                     _p, _p, _p, _p, _sz, _p]),
    "aldvc_precompute": (_i32, [ctypes.POINTER(Volumes), ctypes.POINTER(Subset), _p, _i64, _d, _d, _p, _p, _p, _p, _p, _p,
                                _p]),
    "aldvc_icgn_workspace_size": (_sz, [ctypes.POINTER(Subset), _i64, ctypes.POINTER(IcgnParams)]),
    "aldvc_icgn12": (_i32, [ctypes.POINTER(Volumes), ctypes.POINTER(Subset), _p, _i64, _p, _p, _p, _p, _p, _p,
                            ctypes.POINTER(IcgnParams), _p, _sz, _p, _p, _p, _p, _p]),
    "aldvc_icgn3": (_i32, [ctypes.POINTER(Volumes), ctypes.POINTER(Subset), _p, _i64, _p, _p, _p, _p, _p, _p, _p,
                           ctypes.POINTER(IcgnParams), _p, _sz, _p, _p, _p, _p, _p]),
    "aldvc_ncc_map": (_i32, [_p, _p, _i64, _i64, _i64, _p, _i64, _i32, _i32, _i32, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p]),
    "aldvc_ncc_search_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _i32, _i32, _i32, _i32, _i32, _i32, _i32]),
    "aldvc_ncc_search": (_i32, [_p, _p, _i64, _i64, _i64, _p, _i64, _i32, _i32, _i32, _i32, _i32, _i32, _p, _i32, _p, _sz, _p, _p,
                                _p, _p, _p, _p]),
    "aldvc_global_rhs": (_i32, [ctypes.POINTER(Hex8Mesh), _d, _d, _d, _p, _p, _p, _p, _p, _p]),
    "aldvc_pcg_workspace_size": (_sz, [ctypes.POINTER(Hex8Mesh)]),
    "aldvc_pcg_hex8": (_i32, [ctypes.POINTER(Hex8Mesh), _d, _d, _d, _p, _p, _d, _i32, _p, _sz, _p, _p, _p, _p]),
    "aldvc_pcg_hex8_noalloc_max_nodes": (_i64, []),
    "aldvc_test_set_barrier": (_i32, [_i32, _i64]),
    "aldvc_pcg_hex8_noalloc": (_i32, [ctypes.POINTER(Hex8Mesh), _d, _d, _d, _p, _p, _d, _i32, _p, _p, _p, _p]),
    "aldvc_nodal_gradient": (_i32, [ctypes.POINTER(Hex8Mesh), _p, _p, _p]),
    "aldvc_znssd_forward": (_i32, [ctypes.POINTER(Volumes), _p, _i64, _i32, _i32, _i32, _i32, _p, _p, _p, _p]),
    "aldvc_znssd_backward": (_i32, [ctypes.POINTER(Volumes), _p, _i64, _i32, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p]),
    "aldvc_normalize_workspace_size": (_sz, []),
    "aldvc_normalize": (_i32, [_p, _i32, _i64, _d, _p, _p, _p, _sz, _p]),
    "aldvc_sep_filter": (_i32, [_p, _p, _i64, _i64, _i64, _i32, _p, _i32, _i32, _p]),
    "aldvc_mask_fill": (_i32, [_p, _p, _i64, ctypes.c_float, _p]),
    "aldvc_make_quads": (_i32, [_p, _i64, _p, _p]),
    "aldvc_gradient_plane_fit": (_i32, [_p, _p, _i64, _i64, _i64, _d, _d, _d, _i32, _i32, _i32, _p, _p, _p]),
    "aldvc_gradient_fd": (_i32, [_p, _p, _i64, _i64, _i64, _d, _d, _d, _p, _p, _p]),
    "aldvc_grid_smooth_workspace_size": (_sz, [_i64, _i64, _i64]),
    "aldvc_grid_smooth": (_i32, [_p, _p, _i64, _i64, _i64, _p, _i32, _p, _p, _sz, _p]),
    "aldvc_grid_interp_workspace_size": (_sz, [_i64, _i64, _i64, _i32, _i32, _i32, _i32]),
    "aldvc_displacement_uncertainty": (_i32, [_p, _p, _p, _p, _p, _p, _i64, _p, _d, _d, _i32, _p, _p]),
    "aldvc_grid_interp": (_i32, [_p, _i64, _i64, _i64, _i32, _p, _p, _p, _i32, _i32, _i32, _d, _d, _d, _d, _d, _d, _p, _i64, _i32, _p,
                                 _p, _sz, _p]),
    "aldvc_strain_measures": (_i32, [_p, _i64, _i32, _p, _p, _p, _p, _p, _p, _p, _p]),
    "aldvc_stats_workspace_size": (_sz, []),
    "aldvc_volume_stats": (_i32, [_p, _i32, _i64, _i64, _i64, _p, _d, _p, _p, _sz, _p]),
    "aldvc_normalize_voi": (_i32, [_p, _i32, _i64, _i64, _i64, _p, _d, _p, _p, _p, _sz, _p]),
    "aldvc_volume_moments": (_i32, [_p, _i32, _i64, _d, _p, _p, _sz, _p]),
    "aldvc_normalize_sums": (_i32, [_p, _i32, _i64, _p, _i64, _d, _p, _p, _p]),
    "aldvc_block_downsample": (_i32, [_p, _i64, _i64, _i64, _i32, _p, _p]),
    "aldvc_phase_correlation_workspace_size": (_sz, [_i64, _i64, _i64]),
    "aldvc_phase_correlation": (_i32, [_p, _p, _i64, _i64, _i64, _p, _p, _sz, _p]),
    "aldvc_render_beads": (_i32, [_p, _i64, _i64, _i64, _p, _p, _i64, _d, _i32, _p]),
    "aldvc_inpaint_workspace_size": (_sz, [_i64, _i64, _i64, _i32]),
    "aldvc_inpaint": (_i32, [_p, _i64, _i64, _i64, _i32, _p, _d, _i32, _p, _sz, _p, _p, _p]),
    "aldvc_median_test_workspace_size": (_sz, [_i64, _i64, _i64, _i32]),
    "aldvc_median_test": (_i32, [_p, _i64, _i64, _i64, _i32, _p, _d, _d, _p, _p, _sz, _p, _p]),
}

_lib = None


def load(path: str | None = None):
    """Load (building first if needed) and type the library; raises if it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB
    if not os.path.exists(path):
        from .build import build

        build()
    L = ctypes.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.aldvc_abi_version() != 1:
        raise RuntimeError("aldvc_b200 ABI version mismatch")
    _lib = L
    return L


def check(rc: int, what: str) -> None:
    if rc != ALDVC_OK:
        msg = load().aldvc_last_error()
        raise RuntimeError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")
