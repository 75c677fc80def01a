"""Shared test helpers: small seeded RTM problems and the golden fixtures."""
from __future__ import annotations

import hashlib
import json
import os
from types import SimpleNamespace

import numpy as np

from rtm_b200 import synth
from rtm_b200.engine import ShotRecord

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def params(nx, nz, nt, dt, order=8, nb=20, si=2, f0=15.0, dx=10.0, dz=10.0, ox=0.0, oz=0.0, alpha=0.0053):
    """Attribute bag accepted by both the oracle and the engine set-up."""
    return SimpleNamespace(nx=nx, nz=nz, dx=dx, dz=dz, ox=ox, oz=oz, nb=nb, order=order, sponge_alpha=alpha,
                           store_interval=si, f0=f0, nt=nt, dt=dt)


def small_problem(order=8, nx=61, nz=41, nb=20, nt=300, dt=0.001, f0=15.0, nshots=2, rec_dx=10.0, src_z=0.0,
                  rec_z=0.0, si=2, dipping=True):
    """A small velocity model, acquisition line and oracle-modelled traces."""
    import oracle
    v = synth.layered_three(nx, nz, 10.0, 10.0, dipping)
    shots = synth.reference_line(nx, 10.0, nshots, rec_dx, src_z, rec_z, nt, dt)
    p = params(nx, nz, nt, dt, order=order, nb=nb, si=si, f0=f0)
    traces = oracle.model_shots(params(nx, nz, nt, dt, order=order, nb=nb, si=1, f0=f0), v, shots)
    for s, t in zip(shots, traces):
        s.traces = t
    return p, v, shots


def random_problem(seed, order, nx, nz, nb, nt, si, nrec=None, dt=0.0008, f0=15.0):
    """Random layered model, random (possibly off-grid, duplicated or clamped)
    receiver positions and random traces: exercises every geometry path."""
    rng = np.random.default_rng(seed)
    v = synth.layered_faulted(nx, nz, 10.0, 10.0, seed=seed, n_interfaces=4, n_faults=1, vmin=1500.0,
                              vmax=3000.0)
    nrec = nrec or nx
    rx = rng.uniform(-30.0, (nx + 2) * 10.0, nrec).astype(np.float32)
    rz = rng.uniform(-20.0, (nz + 1) * 10.0, nrec).astype(np.float32)
    rx[: nrec // 4] = rx[nrec // 4: 2 * (nrec // 4)]          # duplicated cells
    shots = []
    for s in range(2):
        tr = rng.standard_normal(nrec * nt).astype(np.float32)
        sx = float(rng.uniform(0, (nx - 1) * 10.0))
        sz = float(rng.uniform(0, (nz - 1) * 10.0))
        shots.append(ShotRecord(sx, sz, rx.copy(), rz.copy(), nt=nt, dt=dt, traces=tr))
    return params(nx, nz, nt, dt, order=order, nb=nb, si=si, f0=f0), v, shots


def make_engine(mode, p, v, **kw):
    from rtm_b200 import Engine, RTMParams
    e = Engine(mode, RTMParams(nb=p.nb, order=p.order, sponge_alpha=p.sponge_alpha, store_interval=p.store_interval,
                               f0=p.f0), **kw)
    e.setup(v, p.nx, p.nz, p.dx, p.dz, p.ox, p.oz, nt=p.nt, dt=p.dt)
    return e


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def rel_l2(ref, test) -> float:
    a = np.asarray(ref, np.float64)
    b = np.asarray(test, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(a), 1e-300))


def sha256(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def golden_cases():
    path = os.path.join(GOLDEN, "cases.json")
    if not os.path.exists(path):
        return []
    with open(path) as f:
        return json.load(f)["cases"]


def golden_arrays(name):
    return (np.load(os.path.join(GOLDEN, name + "_image.npy")),
            np.load(os.path.join(GOLDEN, name + "_illum.npy")))


def golden_inputs(c):
    """Velocity and acquisition of a golden case, as the reference built them."""
    v = synth.layered_three(c["nx"], c["nz"], c["dx"], c["dx"], dipping=(c["model"] == "dipping"))
    shots = synth.reference_line(c["nx"], c["dx"], c["nshots"], c["rec_dx"], c["src_z"], c["rec_z"], c["nt"],
                                 float(np.float32(c["dt"])))
    return v, shots
