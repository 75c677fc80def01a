"""Seeded synthetic workloads (velocity models and acquisition geometry).

The reference has no public benchmark suite; its synthetic generator
(src/tools/make_synthetic.cpp:75-137) makes a three-layer model with a dipping
interface and a box diffractor, a split-spread surface line with every receiver
live, and shots at x = xmax*(is+1)/(nshots+1).  The workloads below follow that
recipe and the shapes of the five benchmark configurations:

  config 1  201x151 @10 m, flat layers 1500/2000/2500 (or the reference's
            dipping/box variant), 4 shots, nt 1400, dt 1 ms, f0 12, order 8,
            nb 60, store 2, direct-wave mute 1500 m/s
  config 2  1150x400 @10 m layered-and-faulted 1500-5500 m/s (10 dipping
            interfaces, 3 normal faults), 64 shots, nt 4000, dt 0.8 ms, f0 15,
            order 8, store 2
  config 3  the config-2 family (seed 3), 256 shots on aperture windows of
            uniform random width 400-1150 columns, orders 8 and 12
  config 4  4000x1500 @5 m smooth gradient 1500-4500 m/s with Gaussian lenses
            (+-10%), 16 shots, nt 8000, dt 0.4 ms, f0 20, order 12, store 2
  config 5  Poisson stream of requests on layered models 1500-4000 m/s, grids
            201..2000 x 151..800 @10 m, orders 8/12, nt 1400..6000,
            dt = 0.8 x CFL limit, f0 10..20, 1..32 shots per request

Traces are modelled with the engine itself (the reference does the same:
"inverse crime", make_synthetic.cpp:10-13).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .engine import ShotRecord, max_stable_dt
from .velocity_models import config3_windows, gradient_lenses, layered_faulted, layered_three  # noqa: F401


@dataclass
class Workload:
    name: str
    vel: np.ndarray          # nx*nz zfast float32
    nx: int
    nz: int
    dx: float
    dz: float
    nt: int
    dt: float
    f0: float
    order: int
    nb: int
    store_interval: int
    shots: List[ShotRecord]
    mute_v: float = 0.0
    orders: List[int] = field(default_factory=list)

    def cell_updates(self) -> float:
        """Reference convention: 2*nt*(nx_w+2nb)*(nz+2nb) per shot."""
        tot = 0.0
        for s in self.shots:
            w = s.window_nx or self.nx
            tot += 2.0 * self.nt * (w + 2 * self.nb) * (self.nz + 2 * self.nb)
        return tot


def surface_line(nx, dx, nshots, rec_z=0.0, src_z=0.0, nt=0, dt=0.0) -> List[ShotRecord]:
    """Split-spread surface line: receivers on every column, all live; shots at
    xmax*(is+1)/(nshots+1) (reference make_synthetic.cpp:124-137)."""
    xmax = np.float32((nx - 1) * dx)
    rx = (np.arange(nx, dtype=np.float32) * np.float32(dx)).astype(np.float32)
    rz = np.full(nx, rec_z, np.float32)
    shots = []
    for s in range(nshots):
        sx = float(xmax * np.float32(s + 1) / np.float32(nshots + 1))
        shots.append(ShotRecord(sx, src_z, rx.copy(), rz.copy(), nt=nt, dt=dt))
    return shots


def config1(dipping=False) -> Workload:
    nx, nz, d = 201, 151, 10.0
    v = layered_three(nx, nz, d, d, dipping)
    return Workload("config1", v, nx, nz, d, d, 1400, 0.001, 12.0, 8, 60, 2,
                    surface_line(nx, d, 4, nt=1400, dt=0.001), mute_v=1500.0)


def config2(nshots=64) -> Workload:
    nx, nz, d = 1150, 400, 10.0
    v = layered_faulted(nx, nz, d, d, seed=2)
    dt = 0.0008
    assert dt <= max_stable_dt(float(v.max()), d, d, 8)
    return Workload("config2", v, nx, nz, d, d, 4000, dt, 15.0, 8, 60, 2, surface_line(nx, d, nshots, nt=4000, dt=dt))


def config3(nshots=256, order=8) -> Workload:
    nx, nz, d = 1150, 400, 10.0
    v = layered_faulted(nx, nz, d, d, seed=3)
    dt = 0.0008
    shots = []
    for x0, w in config3_windows(nshots, nx):
        rx = (np.arange(x0, x0 + w, dtype=np.float32) * np.float32(d)).astype(np.float32)
        sx = float(np.float32((x0 + w // 2) * d))
        shots.append(ShotRecord(sx, 0.0, rx, np.zeros(w, np.float32), nt=4000, dt=dt, window_x0=x0, window_nx=w))
    return Workload(f"config3-order{order}", v, nx, nz, d, d, 4000, dt, 15.0, order, 60, 2, shots, orders=[8, 12])


def config4(nshots=16) -> Workload:
    nx, nz, d = 4000, 1500, 5.0
    v = gradient_lenses(nx, nz, d, d, seed=4)
    dt = 0.0004
    return Workload("config4", v, nx, nz, d, d, 8000, dt, 20.0, 12, 60, 2, surface_line(nx, d, nshots, nt=8000, dt=dt))


@dataclass
class ServeRequest:
    arrival: float
    work: Workload


def config5_stream(nreq=24, rate_hz=2.0, seed=5, max_nx=2000, max_nz=800, max_nt=6000, max_shots=32,
                   scale=1.0) -> List[ServeRequest]:
    """Poisson arrivals of requests; ``scale`` < 1 shrinks grids, nt and shot
    counts for quick runs while keeping the mix."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(nreq):
        t += rng.exponential(1.0 / rate_hz)
        nx = int(rng.integers(201, max_nx + 1) * scale) or 201
        nz = int(rng.integers(151, max_nz + 1) * scale) or 151
        nx, nz = max(nx, 41), max(nz, 31)
        order = int(rng.choice([8, 12]))
        nt = max(int(rng.integers(1400, max_nt + 1) * scale), 200)
        f0 = float(rng.uniform(10, 20))
        nshots = max(1, int(rng.integers(1, max_shots + 1) * scale))
        d = 10.0
        v = layered_faulted(nx, nz, d, d, seed=1000 + i, n_interfaces=6, n_faults=1, vmin=1500.0, vmax=4000.0)
        dt = float(np.float32(0.8 * max_stable_dt(float(v.max()), d, d, order)))
        shots = surface_line(nx, d, nshots, nt=nt, dt=dt)
        out.append(ServeRequest(t, Workload(f"req{i}", v, nx, nz, d, d, nt, dt, f0, order, 60, 2, shots)))
    return out


def reference_line(nx, dx, nshots, rec_dx, src_z, rec_z, nt=0, dt=0.0) -> List[ShotRecord]:
    """Acquisition exactly as the reference generator computes it in float:
    nrec = int((nx-1)*dx/rec_dx) + 1, rx = ir*rec_dx, sx = xmax*(is+1)/(nshots+1)
    (reference src/tools/make_synthetic.cpp:124-137)."""
    f = np.float32
    nrec = int(f(f(nx - 1) * f(dx)) / f(rec_dx)) + 1
    xmax = f(f(nx - 1) * f(dx))
    rx = (np.arange(nrec, dtype=np.float32) * f(rec_dx)).astype(np.float32)
    shots = []
    for s in range(nshots):
        sx = float(xmax * f(s + 1) / f(nshots + 1))
        shots.append(ShotRecord(sx, float(f(src_z)), rx.copy(), np.full(nrec, f(rec_z), np.float32), nt=nt, dt=dt))
    return shots


def shots_file_bytes(shots: List[ShotRecord]) -> bytes:
    """RTMS v1 bytes of a shot list (reference src/io/seismic_io.cpp:59-88)."""
    import struct
    nrec, nt, dt = shots[0].nrec, shots[0].nt, shots[0].dt
    parts = [b"RTMS", struct.pack("<4if2i", 1, len(shots), nrec, nt, np.float32(dt), 0, 0)]
    for s in shots:
        parts.append(struct.pack("<2f", s.sx, s.sz))
        parts.append(np.ascontiguousarray(s.rx, "<f4").tobytes())
        parts.append(np.ascontiguousarray(s.rz, "<f4").tobytes())
        parts.append(np.ascontiguousarray(s.traces, "<f4").ravel().tobytes())
    return b"".join(parts)
