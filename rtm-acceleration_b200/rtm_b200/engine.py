"""Python mirror of the reference's engine interface over librtm_b200.so.

Names and meanings follow the reference (Marouane-Djabri/RTM-Acceleration):
``RTMParams`` (include/rtm_types.hpp:33-40), ``ShotRecord`` (:49-57), the
``RTMEngine`` methods setup / forward_propagation / backward_propagation /
imaging / migrate / model_shot (include/rtm_engine.hpp:20-83) and
``make_engine`` / ``list_engines`` (include/rtm_factory.hpp:19-23).  Errors
raise :class:`RTMError`, a ``RuntimeError`` like the reference's
``std::runtime_error``.

Every compute call goes through the C ABI to the sm_100a kernels; there is no
CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L


class RTMError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{message} [{L.STATUS_NAMES.get(code, code)}]")
        self.code = code


@dataclass
class RTMParams:
    """Reference RTMParams defaults (include/rtm_types.hpp:33-40)."""
    nb: int = 60
    order: int = 8
    sponge_alpha: float = 0.0053
    store_interval: int = 1
    f0: float = 12.0
    verbose: bool = False


@dataclass
class ShotRecord:
    """One shot gather; traces are trace-major ``traces[ir*nt + it]``."""
    sx: float
    sz: float
    rx: np.ndarray
    rz: np.ndarray
    nt: int = 0
    dt: float = 0.0
    traces: Optional[np.ndarray] = None
    window_x0: int = 0
    window_nx: int = 0
    traces_ptr: int = 0        # raw address (device or page-locked host) used instead of `traces`

    @property
    def nrec(self) -> int:
        return int(np.asarray(self.rx).size)


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def shots_to_c(shots: Sequence[ShotRecord], keep: list):
    """ctypes array of rtm_b200_shot; numpy buffers are appended to ``keep``."""
    arr = (L.Shot * max(1, len(shots)))()
    for i, s in enumerate(shots):
        rx = np.ascontiguousarray(s.rx, np.float32).ravel()
        rz = np.ascontiguousarray(s.rz, np.float32).ravel()
        tr = None if (s.traces is None or s.traces_ptr) else np.ascontiguousarray(s.traces, np.float32).ravel()
        keep.extend([rx, rz, tr])
        c = arr[i]
        c.sx, c.sz, c.nrec, c.nt, c.dt = float(s.sx), float(s.sz), rx.size, int(s.nt), float(s.dt)
        c.rx, c.rz = _fp(rx), _fp(rz)
        if s.traces_ptr:
            c.traces = C.cast(C.c_void_p(s.traces_ptr), C.POINTER(C.c_float))
        else:
            c.traces = _fp(tr) if tr is not None else C.POINTER(C.c_float)()
        c.window_x0, c.window_nx = int(s.window_x0), int(s.window_nx)
    return arr


_MODES = {"plain": L.MODE_PLAIN, "batch": L.MODE_BATCH, "serve": L.MODE_SERVE}
_SNAPS = {"f32": L.SNAP_F32, "bf16": L.SNAP_BF16, "f16": L.SNAP_F16, "recon": L.SNAP_RECON}
_ARITH = {"ieee": L.ARITH_IEEE, "fma": L.ARITH_FMA, "fp64": L.ARITH_FP64, "auto": L.ARITH_AUTO}
_ACC = {"plain": L.ACC_PLAIN, "compensated": L.ACC_COMPENSATED}


class Engine:
    """A B200 RTM engine (one CUDA device, one host thread at a time)."""

    def __init__(self, mode: str = "plain", params: Optional[RTMParams] = None, *, snap: str = "f32",
                 arithmetic: str = "auto", accumulation: str = "compensated", device: int = 0,
                 max_shots_in_flight: int = 0, device_mem_budget: int = 0, tile_cols: int = 0,
                 chunk_steps: int = 0, serve_max_nx: int = 0, serve_max_nz: int = 0):
        self.lib = L.load()
        p = params or RTMParams()
        cfg = L.Config()
        self.lib.rtm_b200_config_init(C.byref(cfg))
        cfg.mode = _MODES[mode]
        cfg.device = device
        cfg.nb, cfg.order, cfg.sponge_alpha = p.nb, p.order, p.sponge_alpha
        cfg.store_interval, cfg.f0, cfg.verbose = p.store_interval, p.f0, int(p.verbose)
        cfg.snap_precision = _SNAPS[snap]
        cfg.arithmetic = _ARITH[arithmetic]
        cfg.accumulation = _ACC[accumulation]
        cfg.max_shots_in_flight = max_shots_in_flight
        cfg.device_mem_budget = int(device_mem_budget)
        cfg.tile_cols = tile_cols
        cfg.chunk_steps = chunk_steps
        cfg.serve_max_nx, cfg.serve_max_nz = serve_max_nx, serve_max_nz
        self.mode, self.params, self.snap, self.arithmetic = mode, p, snap, arithmetic
        h = C.c_void_p()
        rc = self.lib.rtm_b200_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            buf = C.create_string_buffer(512)
            self.lib.rtm_b200_last_error(None, buf, 512)
            raise RTMError(rc, "rtm_b200_create: " + buf.value.decode())
        self.h = h
        self.nx = self.nz = self.nt = 0
        self._keep: list = []

    # -- plumbing ------------------------------------------------------------
    def _check(self, rc: int, what: str):
        if rc != 0:
            buf = C.create_string_buffer(1024)
            self.lib.rtm_b200_last_error(self.h, buf, 1024)
            raise RTMError(rc, f"{what}: {buf.value.decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.rtm_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- RTMEngine -----------------------------------------------------------
    def setup(self, vel: np.ndarray, nx: int, nz: int, dx: float, dz: float, ox: float = 0.0, oz: float = 0.0,
              *, nt: int, dt: float):
        v = np.ascontiguousarray(vel, np.float32).ravel()
        if v.size != nx * nz:
            raise RTMError(L.EINVAL, "velocity model size does not match nx*nz")
        self._check(self.lib.rtm_b200_setup(self.h, _fp(v), nx, nz, dx, dz, ox, oz, nt, dt), "setup")
        self.nx, self.nz, self.nt, self.dt = nx, nz, nt, dt

    def migrate(self, shots: Sequence[ShotRecord]) -> Tuple[np.ndarray, np.ndarray]:
        keep: list = []
        arr = shots_to_c(shots, keep)
        img = np.zeros(self.nx * self.nz, np.float32)
        ill = np.zeros_like(img)
        self._check(self.lib.rtm_b200_migrate(self.h, arr, len(shots), _fp(img), _fp(ill)), "migrate")
        return img, ill

    def migrate_into(self, shots: Sequence[ShotRecord], img_ptr: int, ill_ptr: int):
        """migrate() writing nx*nz float32 results to raw addresses (device or host)."""
        keep: list = []
        arr = shots_to_c(shots, keep)
        fp = C.POINTER(C.c_float)
        self._check(self.lib.rtm_b200_migrate(self.h, arr, len(shots), C.cast(C.c_void_p(img_ptr), fp),
                                              C.cast(C.c_void_p(ill_ptr), fp)), "migrate")

    def migrate_f64_into(self, shots: Sequence[ShotRecord], img_ptr: int, ill_ptr: int):
        """migrate_f64() writing the nx*nz FP64 stacks to raw addresses (device
        memory of the engine's GPU, or host memory)."""
        keep: list = []
        arr = shots_to_c(shots, keep)
        dp = C.POINTER(C.c_double)
        self._check(self.lib.rtm_b200_migrate_f64(self.h, arr, len(shots), C.cast(C.c_void_p(img_ptr), dp),
                                                  C.cast(C.c_void_p(ill_ptr), dp)), "migrate_f64")

    def migrate_f64(self, shots: Sequence[ShotRecord]) -> Tuple[np.ndarray, np.ndarray]:
        keep: list = []
        arr = shots_to_c(shots, keep)
        img = np.zeros(self.nx * self.nz, np.float64)
        ill = np.zeros_like(img)
        self._check(self.lib.rtm_b200_migrate_f64(self.h, arr, len(shots), _dp(img), _dp(ill)), "migrate_f64")
        return img, ill

    def postprocess(self, eps_relative: float = 1e-4, compensate_filtered: bool = True):
        """(illumination-compensated image, Laplacian-filtered image) of the last
        migration, computed on the device (reference imaging.cpp:48-75 as its
        CLI applies them)."""
        ic = np.zeros(self.nx * self.nz, np.float32)
        fl = np.zeros_like(ic)
        self._check(self.lib.rtm_b200_postprocess(self.h, float(eps_relative), 1 if compensate_filtered else 0,
                                                  ic.ctypes.data, fl.ctypes.data), "postprocess")
        return ic, fl

    def model_shots(self, shots: Sequence[ShotRecord]) -> List[np.ndarray]:
        keep: list = []
        arr = shots_to_c(shots, keep)
        sizes = [s.nrec * self.nt for s in shots]
        out = np.zeros(max(1, sum(sizes)), np.float32)
        self._check(self.lib.rtm_b200_model_shots(self.h, arr, len(shots), _fp(out)), "model_shots")
        res, off = [], 0
        for n in sizes:
            res.append(out[off:off + n].copy())
            off += n
        return res

    def model_shot(self, shot: ShotRecord) -> ShotRecord:
        """Reference RTMEngine::model_shot: fills shot.traces/nt/dt."""
        shot.traces = self.model_shots([shot])[0]
        shot.nt, shot.dt = self.nt, self.dt
        return shot

    def forward_propagation(self, shot: ShotRecord, snapshots: bool = True, recorded: bool = False):
        keep: list = []
        arr = shots_to_c([shot], keep)
        sn = np.zeros(self.num_snapshots * self.nx * self.nz, np.float32) if snapshots else None
        rec = np.zeros(shot.nrec * self.nt, np.float32) if recorded else None
        self._check(self.lib.rtm_b200_forward(self.h, arr, _fp(sn) if sn is not None else None,
                                              _fp(rec) if rec is not None else None), "forward_propagation")
        return sn, rec

    def backward_propagation(self, shot: ShotRecord, snapshots: Optional[np.ndarray], image: np.ndarray,
                             illumination: np.ndarray):
        """Accumulates into ``image`` / ``illumination`` (float32 nx*nz) in place."""
        keep: list = []
        arr = shots_to_c([shot], keep)
        sn = None if snapshots is None else np.ascontiguousarray(snapshots, np.float32)
        for a in (image, illumination):
            if a.dtype != np.float32 or not a.flags.c_contiguous:
                raise RTMError(L.EINVAL, "image/illumination must be contiguous float32")
        self._check(self.lib.rtm_b200_backward(self.h, arr, _fp(sn) if sn is not None else None, _fp(image),
                                               _fp(illumination)), "backward_propagation")

    def imaging(self, fwd_snapshot: np.ndarray, bwd_extended: np.ndarray, image: np.ndarray,
                illumination: np.ndarray):
        f = np.ascontiguousarray(fwd_snapshot, np.float32)
        b = np.ascontiguousarray(bwd_extended, np.float32)
        self._check(self.lib.rtm_b200_imaging(self.h, _fp(f), _fp(b), _fp(image), _fp(illumination)), "imaging")

    @property
    def num_snapshots(self) -> int:
        return self.lib.rtm_b200_num_snapshots(self.h)

    @property
    def snapshot_bytes(self) -> int:
        return self.lib.rtm_b200_snapshot_bytes(self.h)

    @property
    def device_name(self) -> str:
        buf = C.create_string_buffer(256)
        self.lib.rtm_b200_device_name(self.h, buf, 256)
        return buf.value.decode()

    def autotune_report(self) -> list:
        """Candidates the autotuner timed per job mix and what it chose."""
        import json
        buf = C.create_string_buffer(1 << 16)
        self._check(self.lib.rtm_b200_autotune_report(self.h, buf, 1 << 16), "autotune_report")
        return json.loads(buf.value.decode())

    def times(self) -> dict:
        t = L.Times()
        self._check(self.lib.rtm_b200_get_times(self.h, C.byref(t)), "get_times")
        return {k: getattr(t, k) for k, _ in L.Times._fields_}

    def reset_times(self):
        self.lib.rtm_b200_reset_times(self.h)

    # -- serving -------------------------------------------------------------
    def submit(self, vel, nx, nz, dx, dz, *, order, f0, nt, dt, store_interval, shots: Sequence[ShotRecord],
               ox=0.0, oz=0.0, arrival_time=0.0) -> int:
        v = np.ascontiguousarray(vel, np.float32).ravel()
        keep: list = [v]
        arr = shots_to_c(shots, keep)
        req = L.Request(_fp(v), nx, nz, dx, dz, ox, oz, order, f0, nt, dt, store_interval, len(shots), arr,
                        arrival_time)
        t = C.c_longlong()
        self._check(self.lib.rtm_b200_submit(self.h, C.byref(req), C.byref(t)), "submit")
        self._keep.append((t.value, keep, arr))   # borrowed until the request completes
        return t.value

    def serve_step(self, max_steps: int = 64) -> int:
        p = C.c_int()
        self._check(self.lib.rtm_b200_serve_step(self.h, max_steps, C.byref(p)), "serve_step")
        return p.value

    def poll(self, ticket: int, nx: int = 0, nz: int = 0):
        st = L.RequestStatus()
        img = np.zeros(nx * nz, np.float32) if nx else None
        ill = np.zeros(nx * nz, np.float32) if nx else None
        self._check(self.lib.rtm_b200_poll(self.h, ticket, C.byref(st), _fp(img) if img is not None else None,
                                           _fp(ill) if ill is not None else None), "poll")
        status = {k: getattr(st, k) for k, _ in L.RequestStatus._fields_}
        if status["state"] == 2:
            self._keep = [k for k in self._keep if k[0] != ticket]
        return status, img, ill

    def drain(self):
        self._check(self.lib.rtm_b200_drain(self.h), "drain")

    def clock(self) -> float:
        return self.lib.rtm_b200_clock(self.h)

    def l2_probe(self, nbytes: int = 24 << 20, reps: int = 40) -> float:
        """L2 read bandwidth (GB/s) of an L2-resident nbytes buffer on the engine's GPU."""
        g = C.c_double()
        self._check(self.lib.rtm_b200_l2_probe(self.h, nbytes, reps, C.byref(g)), "l2_probe")
        return g.value

    def memory_probe(self, nbytes: int, iters: int = 20) -> float:
        """Copy bandwidth (read+write GB/s) over an nbytes buffer on the engine's GPU."""
        g = C.c_double()
        self._check(self.lib.rtm_b200_memory_probe(self.h, nbytes, iters, C.byref(g)), "memory_probe")
        return g.value


ENGINES = ("b200", "b200-batch", "b200-serve")


def list_engines() -> List[str]:
    """Engine names accepted by :func:`make_engine` (reference list_engines)."""
    return list(ENGINES)


def make_engine(name: str, params: Optional[RTMParams] = None, **kw) -> Engine:
    """Reference make_engine: unknown names raise (src/rtm/factory.cpp:36-37)."""
    modes = {"b200": "plain", "b200-batch": "batch", "b200-serve": "serve"}
    if name not in modes:
        raise RTMError(L.EINVAL, f"unknown or unavailable engine: '{name}' (see list_engines())")
    return Engine(modes[name], params, **kw)


# -- host numerics (no GPU) ------------------------------------------------------
def stencil_coefficients(order: int) -> np.ndarray:
    out = np.zeros(7, np.float32)
    h = L.load().rtm_b200_stencil_coefficients(order, _fp(out))
    if h < 0:
        raise RTMError(h, "unsupported spatial order (use 2, 4, 6, 8, 10 or 12)")
    return out[:h + 1]


def max_stable_dt(vmax: float, dx: float, dz: float, order: int) -> float:
    return L.load().rtm_b200_max_stable_dt(vmax, dx, dz, order)


def ricker(t: float, f0: float) -> float:
    return L.load().rtm_b200_ricker(t, f0)


def points_per_wavelength(vmin: float, f0: float, dx: float, dz: float) -> float:
    return L.load().rtm_b200_points_per_wavelength(vmin, f0, dx, dz)


def mute_direct_wave(shot: ShotRecord, v_surface: float, t_pad: float, t_taper: float) -> None:
    """In place on ``shot.traces`` (reference mute_direct_wave)."""
    keep: list = []
    tr = np.ascontiguousarray(shot.traces, np.float32).ravel().copy()
    arr = shots_to_c([shot], keep)
    L.load().rtm_b200_mute_direct_wave(arr, _fp(tr), v_surface, t_pad, t_taper)
    shot.traces = tr
