"""B200-native ES-DGSEM shallow-water engine (drop-in for ESDGSEM_MPIOCCA's
OCCA device path).

The compute path is libesdg_b200.so (hand-written CUDA for sm_100a behind a
C ABI, include/esdg_b200.h).  This package only loads it and mirrors the
reference's host-side call surface for Python callers; it has no CPU
fallback: if the library is missing or fails to load, importing
``esdgsem_mpiocca_b200.lib`` raises.
"""
from __future__ import annotations

import ctypes
import os

from . import build_ext

_LIB = None

_D = ctypes.c_double
_I = ctypes.c_int
_PD = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p


def _declare(lib):
    sig = {
        "esdg_deviceclass_create": (_I, [_I, _I, ctypes.POINTER(_VP)]),
        "esdg_init_device_variables": (_I, [_VP, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _D, _D, _D, _D, _D, _D,
                                            _I, _I, _I, _D, _I, _I, _I, _I, _I]),
        "esdg_copy_device_variables": (_I, [_VP, _I, _I] + [_PD] * 22 + [_PI] * 5),
        "esdg_build_device_kernels": (_I, [_VP, _I, _I, _I, _I, _I, _I, _I, _I, _I]),
        "esdg_dg_timeloop": (_I, [_VP, _I, _I, _I, _PD, _PD, _PD, _D, _D, _D, _D, _I, _I, _I, _I, _I, _D, _I, _I,
                                  _I, _I, _I, _PD, _PI]),
        "esdg_copy_q_to_host": (_I, [_VP, _PD]),
        "esdg_copy_q_from_host": (_I, [_VP, _PD]),
        "esdg_copy_visc_to_host": (_I, [_VP, _PD]),
        "esdg_copy_arrival_times": (_I, [_VP, _PD]),
        "esdg_copy_maximum_elevation": (_I, [_VP, _PD]),
        "esdg_bytes_allocated": (ctypes.c_longlong, [_VP]),
        "esdg_kernel_launches": (ctypes.c_longlong, [_VP]),
        "esdg_free_occa_vars": (_I, [_VP, _I, _I, _I]),
        "esdg_deviceclass_destroy": (_I, [_VP]),
        "esdg_last_error": (ctypes.c_char_p, [_VP]),
        "esdg_compute_rhs": (_I, [_VP, _PD, _PD]),
        "esdg_set_stream": (_I, [_VP, _VP]),
        "esdg_advance": (_I, [_VP, _I, _D, _PD, _PI]),
        "esdg_profile_steps": (_I, [_VP, _I, _PD, _PD]),
        "esdg_debug_bulk_wait_test": (_I, [_VP, ctypes.c_longlong, _I]),
        "esdg_set_pause": (_I, [_VP, _D]),
        "esdg_set_indicator_every_stage": (_I, [_VP, _I]),
        "esdg_okada_uplift": (_I, [ctypes.c_longlong, _VP, _VP, _PD, _I, _I, _VP, _VP]),
        "esdg_mesh_element_curves": (_I, [_VP, _PI, _PD, _PI, _PD]),
        "esdg_geometry_device": (_I, [_I, _I, _I] + [_VP] * 13 + [_VP]),
        "esdg_ensemble_set_indicator_every_stage": (_I, [_VP, _I]),
        "esdg_resume": (_I, [_VP, _PD, _PI]),
        "esdg_compute_rhs_noalloc": (_I, [_I, _I, _I, _I, _I, _D, _D] + [_VP] * 17 + [_VP, _VP]),
        "esdg_basis": (_I, [_I, _I] + [_PD] * 9),
        "esdg_basis_fd": (_I, [_I, _PD, _PD, _PD]),
        "esdg_copy_partial_dry_data": (_I, [_VP, _PD, _PD, _PD]),
        "esdg_mesh_cartesian": (_I, [_I, _D, _D, _D, _D, _I, _I, _I, _I, ctypes.POINTER(_VP)]),
        "esdg_mesh_mapped": (_I, [_I, _D, _D, _D, _D, _I, _I, _D, _I, ctypes.c_uint, ctypes.POINTER(_VP)]),
        "esdg_mesh_read_ism2": (_I, [_I, ctypes.c_char_p, _I, _I, ctypes.POINTER(_VP)]),
        "esdg_mesh_write_ism2": (_I, [_VP, ctypes.c_char_p]),
        "esdg_mesh_sizes": (_I, [_VP, _PI, _PI]),
        "esdg_mesh_pack": (_I, [_VP] + [_PD] * 11 + [_PI] * 5),
        "esdg_mesh_free": (None, [_VP]),
        "esdg_bottom_derivatives": (_I, [_I, _I] + [_PD] * 9),
        "esdg_element_sizes": (_I, [_I, _I, _PD, _PD, _PD, _PD]),
        "esdg_rk_coefficients": (_I, [_I, _I, _PD, _PD, _PD, _PI]),
        "esdg_diagnostics": (_I, [_I, _I, _PD, _PD, _PD, _PD, _PD, _D, _PD, _PD, _PD, _PD]),
        "esdg_ensemble_create": (_I, [_I, _I, _I, _I, _I, _I, _I, _D, _D, _I, _D, _D, _D, _I, _I, _I,
                                      ctypes.POINTER(_VP)]),
        "esdg_ensemble_add": (_I, [_VP, _I, _I] + [_PD] * 13 + [_PI] * 4 + [_D, _I, _D, _D, _D, _PI]),
        "esdg_ensemble_remove": (_I, [_VP, _I]),
        "esdg_ensemble_advance": (_I, [_VP, _I]),
        "esdg_ensemble_launch": (_I, [_VP, _I]),
        "esdg_ensemble_sync": (_I, [_VP]),
        "esdg_ensemble_status": (_I, [_VP, _I, _PD, _PI, _PI, _PI]),
        "esdg_ensemble_copy_q": (_I, [_VP, _I, _PD]),
        "esdg_ensemble_free_capacity": (_I, [_VP, _PI, _PI, _PI]),
        "esdg_ensemble_bytes": (ctypes.c_longlong, [_VP]),
        "esdg_ensemble_kernel_launches": (ctypes.c_longlong, [_VP]),
        "esdg_ensemble_set_stream": (_I, [_VP, _VP]),
        "esdg_ensemble_last_error": (ctypes.c_char_p, [_VP]),
        "esdg_ensemble_destroy": (_I, [_VP]),
        "esdg_state_pointers": (_I, [_VP, ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(_VP)]),
        "esdg_tuned_config": (_I, [_VP, _PI, _PI, ctypes.POINTER(ctypes.c_float)]),
        "esdg_element_variants": (_I, [_VP, _PI, _PI, ctypes.POINTER(ctypes.c_float), _PI, _I]),
        "esdg_set_element_variant": (_I, [_VP, _I]),
        "esdg_ensemble_element_variants": (_I, [_VP, _PI, _PI, ctypes.POINTER(ctypes.c_float), _PI, _I]),
        "esdg_ensemble_set_element_variant": (_I, [_VP, _I]),
        "esdg_set_indicator": (_I, [_VP, _I, ctypes.POINTER(ctypes.c_float), _I, ctypes.c_float]),
        "esdg_indicator_stats": (_I, [_VP, ctypes.POINTER(ctypes.c_ulonglong), _I]),
        "esdg_ensemble_set_indicator": (_I, [_VP, _I, ctypes.POINTER(ctypes.c_float), _I, ctypes.c_float]),
        "esdg_ensemble_indicator_stats": (_I, [_VP, ctypes.POINTER(ctypes.c_ulonglong), _I]),
        "esdg_mlp_layout": (_I, [_I, _PI]),
        "esdg_mlp_features": (_I, [_I, _I, _VP, _VP, _VP, _D, _VP, _VP, _VP, _VP]),
        "esdg_mlp_cast": (_I, [_I, _VP, _VP, _VP]),
        "esdg_mlp_forward": (_I, [_I, _I, _VP, _VP, _VP, _VP, _I, _VP]),
        "esdg_mlp_backward": (_I, [_I, _I, _VP, _VP, _VP, _VP, _VP, _I, _VP]),
        "esdg_mlp_adam": (_I, [_I, _I, _VP, _VP, _VP, _VP, _VP, _VP, ctypes.c_float, ctypes.c_float,
                               ctypes.c_float, ctypes.c_float, _I, _VP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def library_path() -> str:
    return build_ext.LIB


def lib(build: bool = False):
    """The loaded engine library (compiled first when build=True)."""
    global _LIB
    if _LIB is None:
        if build:
            build_ext.build()
        path = build_ext.LIB
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: run `python -m esdgsem_mpiocca_b200.build_ext` (the engine has no CPU fallback)")
        _LIB = _declare(ctypes.CDLL(path))
    return _LIB
