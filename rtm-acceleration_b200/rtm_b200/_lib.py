"""ctypes declarations of librtm_b200.so (include/rtm_b200.h).

The library is built in-tree (``make -C rtm-acceleration_b200``) into
``rtm-acceleration_b200/lib/librtm_b200.so``.  There is no fallback: if the
library is missing or cannot be loaded, importing the engine raises.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.environ.get("RTM_B200_LIBRARY") or os.path.join(ROOT_DIR, "lib", "librtm_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(ROOT_DIR), "include", "rtm_b200.h")

OK, EINVAL, ENOMEM, ECUDA, ESTATE, ETIMEOUT, EUNSUPPORTED, EREJECTED, ENOTFOUND = 0, -1, -2, -3, -4, -5, -6, -7, -8
STATUS_NAMES = {0: "OK", -1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ESTATE", -5: "ETIMEOUT",
                -6: "EUNSUPPORTED", -7: "EREJECTED", -8: "ENOTFOUND"}

MODE_PLAIN, MODE_BATCH, MODE_SERVE = 0, 1, 2
SNAP_F32, SNAP_BF16, SNAP_F16, SNAP_RECON = 0, 1, 2, 3
ARITH_IEEE, ARITH_FMA, ARITH_FP64, ARITH_AUTO = 0, 1, 2, 3
ACC_PLAIN, ACC_COMPENSATED = 0, 1


class Config(C.Structure):
    _fields_ = [("struct_size", C.c_int), ("mode", C.c_int), ("device", C.c_int), ("nb", C.c_int),
                ("order", C.c_int), ("sponge_alpha", C.c_float), ("store_interval", C.c_int),
                ("f0", C.c_float), ("verbose", C.c_int), ("snap_precision", C.c_int),
                ("arithmetic", C.c_int), ("accumulation", C.c_int), ("max_shots_in_flight", C.c_int),
                ("device_mem_budget", C.c_longlong), ("tile_cols", C.c_int), ("chunk_steps", C.c_int),
                ("serve_max_nx", C.c_int), ("serve_max_nz", C.c_int)]


class Shot(C.Structure):
    _fields_ = [("sx", C.c_float), ("sz", C.c_float), ("nrec", C.c_int), ("nt", C.c_int), ("dt", C.c_float),
                ("rx", C.POINTER(C.c_float)), ("rz", C.POINTER(C.c_float)), ("traces", C.POINTER(C.c_float)),
                ("window_x0", C.c_int), ("window_nx", C.c_int)]


class Times(C.Structure):
    _fields_ = [("io", C.c_double), ("forward", C.c_double), ("backward", C.c_double), ("imaging", C.c_double),
                ("total", C.c_double), ("h2d", C.c_double), ("kernel", C.c_double), ("d2h", C.c_double),
                ("cell_updates", C.c_double), ("algorithmic_bytes", C.c_double), ("h2d_bytes", C.c_double),
                ("d2h_bytes", C.c_double), ("kernel_launches", C.c_int), ("shots", C.c_int)]


class Request(C.Structure):
    _fields_ = [("vel", C.POINTER(C.c_float)), ("nx", C.c_int), ("nz", C.c_int), ("dx", C.c_float),
                ("dz", C.c_float), ("ox", C.c_float), ("oz", C.c_float), ("order", C.c_int), ("f0", C.c_float),
                ("nt", C.c_int), ("dt", C.c_float), ("store_interval", C.c_int), ("nshots", C.c_int),
                ("shots", C.POINTER(Shot)), ("arrival_time", C.c_double)]


class StaticProblem(C.Structure):
    _fields_ = [("vel", C.POINTER(C.c_float)), ("nx", C.c_int), ("nz", C.c_int), ("dx", C.c_float),
                ("dz", C.c_float), ("ox", C.c_float), ("oz", C.c_float), ("nb", C.c_int), ("order", C.c_int),
                ("sponge_alpha", C.c_float), ("f0", C.c_float), ("nt", C.c_int), ("dt", C.c_float),
                ("device", C.c_int)]


class RequestStatus(C.Structure):
    _fields_ = [("state", C.c_int), ("shots_done", C.c_int), ("submit_time", C.c_double),
                ("start_time", C.c_double), ("finish_time", C.c_double), ("snapshot_bytes", C.c_double)]


_lib = None


def load():
    """Load librtm_b200.so and declare its signatures; raises if unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"librtm_b200.so is not built ({LIB_PATH}); run `make -C {ROOT_DIR} lib` "
                           "or __graft_entry__.build()")
    lib = C.CDLL(LIB_PATH)
    fp, dp, vp = C.POINTER(C.c_float), C.POINTER(C.c_double), C.c_void_p
    E = vp   # opaque engine handle
    sig = {
        "rtm_b200_config_init": (None, [C.POINTER(Config)]),
        "rtm_b200_create": (C.c_int, [C.POINTER(Config), C.POINTER(vp)]),
        "rtm_b200_destroy": (C.c_int, [E]),
        "rtm_b200_setup": (C.c_int, [E, fp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                     C.c_int, C.c_float]),
        "rtm_b200_migrate": (C.c_int, [E, C.POINTER(Shot), C.c_int, fp, fp]),
        "rtm_b200_migrate_f64": (C.c_int, [E, C.POINTER(Shot), C.c_int, dp, dp]),
        "rtm_b200_model_shots": (C.c_int, [E, C.POINTER(Shot), C.c_int, fp]),
        "rtm_b200_forward": (C.c_int, [E, C.POINTER(Shot), fp, fp]),
        "rtm_b200_backward": (C.c_int, [E, C.POINTER(Shot), fp, fp, fp]),
        "rtm_b200_imaging": (C.c_int, [E, fp, fp, fp, fp]),
        "rtm_b200_num_snapshots": (C.c_int, [E]),
        "rtm_b200_snapshot_bytes": (C.c_longlong, [E]),
        "rtm_b200_get_times": (C.c_int, [E, C.POINTER(Times)]),
        "rtm_b200_reset_times": (C.c_int, [E]),
        "rtm_b200_device_name": (C.c_int, [E, C.c_char_p, C.c_size_t]),
        "rtm_b200_last_error": (C.c_int, [E, C.c_char_p, C.c_size_t]),
        "rtm_b200_autotune_report": (C.c_int, [E, C.c_char_p, C.c_size_t]),
        "rtm_b200_stencil_coefficients": (C.c_int, [C.c_int, fp]),
        "rtm_b200_max_stable_dt": (C.c_float, [C.c_float, C.c_float, C.c_float, C.c_int]),
        "rtm_b200_ricker": (C.c_float, [C.c_float, C.c_float]),
        "rtm_b200_points_per_wavelength": (C.c_float, [C.c_float, C.c_float, C.c_float, C.c_float]),
        "rtm_b200_mute_direct_wave": (None, [C.POINTER(Shot), fp, C.c_float, C.c_float, C.c_float]),
        "rtm_b200_submit": (C.c_int, [E, C.POINTER(Request), C.POINTER(C.c_longlong)]),
        "rtm_b200_serve_step": (C.c_int, [E, C.c_int, C.POINTER(C.c_int)]),
        "rtm_b200_poll": (C.c_int, [E, C.c_longlong, C.POINTER(RequestStatus), fp, fp]),
        "rtm_b200_drain": (C.c_int, [E]),
        "rtm_b200_clock": (C.c_double, [E]),
        "rtm_b200_memory_probe": (C.c_int, [E, C.c_size_t, C.c_int, C.POINTER(C.c_double)]),
        "rtm_b200_postprocess": (C.c_int, [E, C.c_float, C.c_int, vp, vp]),
        "rtm_b200_l2_probe": (C.c_int, [E, C.c_size_t, C.c_int, C.POINTER(C.c_double)]),
        "rtm_b200_model_shot_static": (C.c_int, [C.POINTER(StaticProblem), C.POINTER(Shot), vp, C.c_char_p,
                                                 C.c_size_t]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def header_symbols(path: str = HEADER_PATH):
    """Names of every function declared in include/rtm_b200.h."""
    import re
    text = open(path).read()
    return sorted(set(re.findall(r"RTM_B200_API\s+[\w\s\*]+?\b(rtm_b200_\w+)\s*\(", text)))
