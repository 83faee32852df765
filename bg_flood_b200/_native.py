"""Loader for the in-tree native library (bg_flood_b200/_lib/libbgflood_b200.so).

The library holds the sm_100a kernels and the C ABI declared in
include/bg_flood_b200.h.  There is no fallback: if the library is missing or a
symbol is absent, loading fails loudly.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libbgflood_b200.so")

_lib = None

c_int_p = ctypes.POINTER(ctypes.c_int)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_void_p = ctypes.c_void_p

# every symbol of include/bg_flood_b200.h with its ctypes signature
SIGNATURES = {
    "bgf_param_default": (None, [c_void_p]),
    "bgf_strerror": (ctypes.c_char_p, [ctypes.c_int]),
    "bgf_last_error": (ctypes.c_char_p, []),
    "bgf_device_supported": (ctypes.c_int, [ctypes.c_int]),
    "bgf_create": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, ctypes.POINTER(c_void_p)]),
    "bgf_destroy": (ctypes.c_int, [c_void_p]),
    "bgf_set_blocks": (ctypes.c_int, [c_void_p, c_void_p]),
    "bgf_set_bed": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int_p]),
    "bgf_add_bnd_segment": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, c_double_p, c_double_p, c_int_p,
                                           ctypes.POINTER(c_int_p)]),
    "bgf_set_rain_series": (ctypes.c_int, [c_void_p, ctypes.c_int, c_double_p, c_double_p]),
    "bgf_set_state": (ctypes.c_int, [c_void_p, c_void_p]),
    "bgf_get_state": (ctypes.c_int, [c_void_p, c_void_p]),
    "bgf_init_dt": (ctypes.c_int, [c_void_p, c_void_p]),
    "bgf_flow_step": (ctypes.c_int, [c_void_p, c_void_p]),
    "bgf_run": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int, c_int_p]),
    "bgf_volume": (ctypes.c_int, [c_void_p, c_double_p]),
    "bgf_kernel_launches": (ctypes.c_int64, [c_void_p]),
    "bgf_set_profiling": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "bgf_kernel_timing": (ctypes.c_int, [c_void_p, c_double_p, c_double_p, ctypes.POINTER(ctypes.c_int64)]),
    "bgf_run_timing": (ctypes.c_int, [c_void_p, c_double_p, ctypes.POINTER(ctypes.c_int64)]),
    "bgf_flow_step_noalloc": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "bgf_mesh_uniform": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, c_void_p, c_int_p, c_int_p,
                                        c_int_p, c_double_p, c_double_p, ctypes.c_int]),
    "bgf_set_bathy": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, c_void_p]),
    "bgf_adapt_flags": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "bgf_adapt": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_int_p]),
    "bgf_get_blocks": (ctypes.c_int, [c_void_p, c_int_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "bgf_get_bed": (ctypes.c_int, [c_void_p, c_void_p]),
    "bgf_set_grid": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "bgf_set_kernel_layout": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "bgf_set_gauges": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, c_void_p, c_void_p]),
    "bgf_read_gauges": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "bgf_pool_set_gauges": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, c_void_p, c_void_p, c_void_p]),
    "bgf_pool_read_gauges": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, c_void_p, c_void_p, c_void_p]),
    "bgf_pool_create": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_void_p,
                                       ctypes.POINTER(c_void_p)]),
    "bgf_pool_destroy": (ctypes.c_int, [c_void_p]),
    "bgf_pool_admit": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                      c_int_p]),
    "bgf_pool_retire": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, c_int_p]),
    "bgf_pool_run": (ctypes.c_int, [c_void_p, ctypes.c_int, c_int_p]),
    "bgf_pool_query": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, c_int_p, ctypes.POINTER(ctypes.c_int64)]),
    "bgf_pool_get_depth": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, c_void_p]),
    "bgf_pool_timing": (ctypes.c_int, [c_void_p, c_double_p, ctypes.POINTER(ctypes.c_int64), c_int_p]),
    "bgf_pool_set_grid": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "bgf_pool_set_kernel_layout": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "bgf_pool_run_async": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "bgf_set_adapt_mode": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "bgf_pool_wait": (ctypes.c_int, [c_void_p, c_int_p]),
    "bgf_pool_prepare": (ctypes.c_int, [c_void_p]),
    "bgf_pool_finish": (ctypes.c_int, [c_void_p, ctypes.c_int, c_int_p, c_void_p, c_void_p, c_void_p,
                                       ctypes.POINTER(ctypes.c_int64), c_int_p]),
    "bgf_autotune": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_int_p, c_double_p]),
    "bgf_add_target_level_map": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double, c_int_p]),
    "bgf_clear_target_level_maps": (ctypes.c_int, [c_void_p]),
    "bgf_pool_autotune": (ctypes.c_int, [c_void_p, ctypes.c_int, c_int_p, c_double_p]),
    "bgf_set_rain_map": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_double, c_void_p]),
    "bgf_add_river": (ctypes.c_int, [c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, c_double_p, c_double_p, c_double_p]),
    "bgf_read_asc_head": (ctypes.c_int, [ctypes.c_char_p, c_int_p, c_int_p, c_double_p, c_double_p, c_double_p,
                                         c_double_p]),
    "bgf_read_asc": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, c_void_p]),
    "bgf_mask_blocks": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double, c_void_p, c_int_p]),
    "bgf_interp_bathy": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, c_void_p]),
    "bgf_refine_sanity": (ctypes.c_int, [ctypes.c_int, c_int_p, c_int_p, c_int_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, c_void_p, c_void_p]),
    "bgf_refine_tables": (ctypes.c_int, [c_int_p, c_int_p, c_int_p, c_int_p, c_double_p, c_double_p, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_int, c_void_p, c_int_p]),
    "bgf_adapt_sanity": (ctypes.c_int, [ctypes.c_int, c_int_p, c_int_p, c_int_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, c_double_p, c_double_p, ctypes.c_double, ctypes.c_int,
                                        c_void_p, c_void_p]),
    "bgf_adapt_tables": (ctypes.c_int, [c_int_p, c_int_p, c_int_p, c_int_p, c_double_p, c_double_p, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_int, c_void_p, c_void_p, c_int_p, c_int_p]),
}


def lib() -> ctypes.CDLL:
    """Returns the loaded native library (built by bg_flood_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"native library not built: {LIB_PATH} (run bg_flood_b200.build.build())")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(l, name)  # AttributeError if the symbol is missing
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib
