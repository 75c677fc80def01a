"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle_rtm.so`` (built by ``oracle/Makefile`` from
``rtm_oracle.cpp``), a plain-loop CPU restatement of the reference's RTM
(CPUReferenceRTM, reference src/rtm/*.cpp).  Also runs the reference's own
binaries compiled into ``oracle/_ref/`` when they are present.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this module, and only as the checker.  The product library never
touches it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_rtm.so")
REF_DIR = os.path.join(HERE, "_ref")


class OracleParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("dx", C.c_float), ("dz", C.c_float),
                ("ox", C.c_float), ("oz", C.c_float), ("nb", C.c_int), ("order", C.c_int),
                ("sponge_alpha", C.c_float), ("store_interval", C.c_int), ("f0", C.c_float),
                ("nt", C.c_int), ("dt", C.c_float)]


class OracleShot(C.Structure):
    _fields_ = [("sx", C.c_float), ("sz", C.c_float), ("nrec", C.c_int), ("nt", C.c_int),
                ("rx", C.POINTER(C.c_float)), ("rz", C.POINTER(C.c_float)),
                ("traces", C.POINTER(C.c_float))]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
        _lib = C.CDLL(LIB_PATH)
        fp = C.POINTER(C.c_float)
        dp = C.POINTER(C.c_double)
        _lib.oracle_migrate_f32.argtypes = [C.POINTER(OracleParams), fp, C.c_int, C.POINTER(OracleShot), fp, fp]
        _lib.oracle_migrate_f64.argtypes = [C.POINTER(OracleParams), fp, C.c_int, C.POINTER(OracleShot), dp, dp]
        _lib.oracle_migrate_f32_sum64.argtypes = [C.POINTER(OracleParams), fp, C.c_int, C.POINTER(OracleShot), dp,
                                                  dp]
        _lib.oracle_model_shot_f32.argtypes = [C.POINTER(OracleParams), fp, C.POINTER(OracleShot), fp]
        _lib.oracle_model_shot_f64.argtypes = [C.POINTER(OracleParams), fp, C.POINTER(OracleShot), dp]
        _lib.oracle_model_shots_f32.argtypes = [C.POINTER(OracleParams), fp, C.c_int, C.POINTER(OracleShot), fp, C.c_int]
        _lib.oracle_mute_direct_wave.argtypes = [C.c_float, C.c_float, C.c_int, fp, fp, C.c_int, C.c_float, fp,
                                                 C.c_float, C.c_float, C.c_float]
        _lib.oracle_mute_direct_wave.restype = None
        _lib.oracle_ricker.argtypes = [C.c_float, C.c_float]
        _lib.oracle_ricker.restype = C.c_float
        _lib.oracle_max_stable_dt.argtypes = [C.c_float, C.c_float, C.c_float, C.c_int]
        _lib.oracle_max_stable_dt.restype = C.c_float
        _lib.oracle_stencil_coefficients.argtypes = [C.c_int, fp]
    return _lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_params(p) -> OracleParams:
    """``p`` is any object with the RTM parameter attributes (see rtm_b200.Params)."""
    return OracleParams(p.nx, p.nz, p.dx, p.dz, p.ox, p.oz, p.nb, p.order, p.sponge_alpha,
                        p.store_interval, p.f0, p.nt, p.dt)


def _shots(shots, keep):
    arr = (OracleShot * max(1, len(shots)))()
    for i, s in enumerate(shots):
        rx = np.ascontiguousarray(s.rx, np.float32)
        rz = np.ascontiguousarray(s.rz, np.float32)
        tr = None if s.traces is None else np.ascontiguousarray(s.traces, np.float32)
        keep.extend([rx, rz, tr])
        arr[i].sx, arr[i].sz = float(s.sx), float(s.sz)
        arr[i].nrec = rx.size
        arr[i].nt = int(getattr(s, "nt", 0) or 0)
        arr[i].rx, arr[i].rz = _fp(rx), _fp(rz)
        arr[i].traces = _fp(tr) if tr is not None else C.POINTER(C.c_float)()
    return arr


def migrate(params, vel, shots, dtype=np.float32):
    """Reference RTMEngine::migrate restated; returns (image, illum) nx*nz zfast."""
    keep = []
    op = make_params(params)
    v = np.ascontiguousarray(vel, np.float32).ravel()
    n = params.nx * params.nz
    img = np.zeros(n, dtype)
    ill = np.zeros(n, dtype)
    arr = _shots(shots, keep)
    fn = lib().oracle_migrate_f32 if dtype == np.float32 else lib().oracle_migrate_f64
    cv = _fp if dtype == np.float32 else _dp
    rc = fn(C.byref(op), _fp(v), len(shots), arr, cv(img), cv(ill))
    if rc != 0:
        raise ValueError(f"oracle migrate rejected the parameters (code {rc})")
    return img, ill


def migrate_sum64(params, vel, shots):
    """migrate() with FP32 propagation and FP32 products (bit-identical to the
    reference) but FP64 image and illumination sums."""
    keep = []
    op = make_params(params)
    v = np.ascontiguousarray(vel, np.float32).ravel()
    n = params.nx * params.nz
    img = np.zeros(n, np.float64)
    ill = np.zeros(n, np.float64)
    rc = lib().oracle_migrate_f32_sum64(C.byref(op), _fp(v), len(shots), _shots(shots, keep), _dp(img), _dp(ill))
    if rc != 0:
        raise ValueError(f"oracle migrate rejected the parameters (code {rc})")
    return img, ill


def model_shot(params, vel, shot, dtype=np.float32):
    keep = []
    op = make_params(params)
    v = np.ascontiguousarray(vel, np.float32).ravel()
    arr = _shots([shot], keep)
    out = np.zeros(arr[0].nrec * params.nt, dtype)
    if dtype == np.float32:
        rc = lib().oracle_model_shot_f32(C.byref(op), _fp(v), arr, _fp(out))
    else:
        rc = lib().oracle_model_shot_f64(C.byref(op), _fp(v), arr, _dp(out))
    if rc != 0:
        raise ValueError(f"oracle model_shot rejected the parameters (code {rc})")
    return out


def model_shots(params, vel, shots, nthreads=0):
    """Independent shots modelled in parallel on the host; list of nrec*nt arrays."""
    keep = []
    op = make_params(params)
    v = np.ascontiguousarray(vel, np.float32).ravel()
    arr = _shots(shots, keep)
    sizes = [arr[i].nrec * params.nt for i in range(len(shots))]
    out = np.zeros(sum(sizes), np.float32)
    rc = lib().oracle_model_shots_f32(C.byref(op), _fp(v), len(shots), arr, _fp(out), nthreads)
    if rc != 0:
        raise ValueError(f"oracle model_shots rejected the parameters (code {rc})")
    res, off = [], 0
    for n in sizes:
        res.append(out[off:off + n].copy())
        off += n
    return res


def mute_direct_wave(shot, v_surface, t_pad, t_taper, nt, dt):
    tr = np.ascontiguousarray(shot.traces, np.float32).copy()
    rx = np.ascontiguousarray(shot.rx, np.float32)
    rz = np.ascontiguousarray(shot.rz, np.float32)
    lib().oracle_mute_direct_wave(shot.sx, shot.sz, rx.size, _fp(rx), _fp(rz), nt, dt, _fp(tr),
                                  v_surface, t_pad, t_taper)
    return tr


def ricker(t, f0):
    return lib().oracle_ricker(t, f0)


def max_stable_dt(vmax, dx, dz, order):
    return lib().oracle_max_stable_dt(vmax, dx, dz, order)


def stencil_coefficients(order):
    out = np.zeros(7, np.float32)
    h = lib().oracle_stencil_coefficients(order, _fp(out))
    if h < 0:
        raise ValueError("unsupported order")
    return out[:h + 1]


def ref_binary(name):
    """Path of a reference binary built into oracle/_ref/, or None."""
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None
