"""ctypes binding of the C ABI in include/phox.h (libphox.so, built in-tree).

Importing this module loads the shared library; there is no fallback path: if the library
is missing or fails to load, an ImportError says why.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# PHX_LIB selects another build of the same library (used to time compile-time variants)
LIB_PATH = os.environ.get("PHX_LIB", os.path.join(HERE, "libphox.so"))


class PhxGeometry(C.Structure):
    _fields_ = [
        ("node", C.c_void_p), ("num_node", C.c_int32),
        ("prim", C.c_void_p), ("num_prim", C.c_int32),
        ("solid", C.c_void_p), ("num_solid", C.c_int32),
        ("inst", C.c_void_p), ("num_inst", C.c_int32),
        ("itra", C.c_void_p), ("num_itra", C.c_int32),
        ("plan", C.c_void_p), ("num_plan", C.c_int32),
    ]


class PhxPhysics(C.Structure):
    _fields_ = [
        ("bnd", C.c_void_p), ("num_bnd", C.c_int32), ("num_wl", C.c_int32),
        ("wl_low", C.c_float), ("wl_step", C.c_float),
        ("optical", C.c_void_p),
        ("icdf", C.c_void_p), ("icdf_layers", C.c_int32), ("icdf_width", C.c_int32), ("hd_factor", C.c_int32),
    ]


class PhxConfig(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64), ("offset", C.c_uint64), ("skipahead_event_offset", C.c_uint64),
        ("max_photon", C.c_int64), ("max_bounce", C.c_int32), ("max_time", C.c_float),
        ("propagate_epsilon", C.c_float), ("propagate_epsilon0", C.c_float),
        ("epsilon0_mask", C.c_uint32), ("hit_mask", C.c_uint32),
        ("root_polish", C.c_int32), ("num_sensor", C.c_int32),
        ("kernel_mode", C.c_int32), ("block", C.c_int32), ("regroup", C.c_int32), ("chunk", C.c_int32),
        ("use_graph", C.c_int32), ("wave_pool", C.c_int64),
        ("wave_refill", C.c_int32), ("wave_rounds", C.c_int32), ("wave_tail", C.c_int64),
        ("adj_wave_rounds", C.c_int32),
    ]


class PhxOutputs(C.Structure):
    _fields_ = [
        ("photon", C.c_void_p), ("seq", C.c_void_p), ("hit", C.c_void_p), ("hit_capacity", C.c_int64),
        ("sensor_hits", C.c_void_p),
        ("num_photon", C.c_int64), ("num_hit", C.c_int64), ("status", C.c_uint32),
    ]


# every symbol the header declares, with its ctypes signature
SIGNATURES = {
    "phx_config_default": (None, [C.POINTER(PhxConfig)]),
    "phx_last_error": (C.c_char_p, []),
    "phx_version": (C.c_char_p, []),
    "phx_create": (C.c_int, [C.POINTER(PhxGeometry), C.POINTER(PhxPhysics), C.POINTER(PhxConfig), C.c_int, C.POINTER(C.c_void_p)]),
    "phx_destroy": (C.c_int, [C.c_void_p]),
    "phx_trim": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "phx_set_launch_config": (C.c_int, [C.c_void_p, C.POINTER(PhxConfig)]),
    "phx_count_photons": (C.c_int64, [C.c_void_p, C.c_int32]),
    "phx_simulate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(PhxOutputs)]),
    "phx_simulate_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.c_int64, C.POINTER(PhxOutputs),
                                      C.c_void_p]),
    "phx_simulate_device_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.c_int64,
                                              C.POINTER(PhxOutputs), C.c_void_p]),
    "phx_simulate_batched_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.c_int32,
                                              C.c_int32, C.c_int32, C.c_void_p, C.POINTER(PhxOutputs), C.c_void_p]),
    "phx_csg_scan": (C.c_int, [C.c_void_p, C.c_int32, C.c_float, C.c_void_p, C.c_int64, C.c_void_p]),
    "phx_csg_scan_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_float, C.c_void_p, C.c_int64, C.c_void_p, C.c_int32, C.c_void_p]),
    "phx_trace": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float, C.c_void_p, C.POINTER(C.c_uint32)]),
    "phx_trace_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float, C.c_void_p, C.POINTER(C.c_uint32),
                                   C.c_void_p]),
    "phx_rng_sequence": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_int64, C.c_int32, C.c_void_p]),
    "phx_adjoint_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.c_void_p, C.c_int32,
                                     C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "phx_merge_hits_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_uint32, C.c_float, C.c_void_p,
                                        C.c_int64, C.POINTER(C.c_int64), C.c_void_p]),
    "phx_merge_hits": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_uint32, C.c_float, C.c_void_p, C.c_int64,
                                 C.POINTER(C.c_int64)]),
    "phx_last_call_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "phx_set_input_photon": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "phx_planck_icdf": (C.c_int, [C.c_void_p, C.c_int]),
    "phx_set_input_photon_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
}


def load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"libphox.so not found at {path}: build it with `python -m opticks_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().phx_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")
