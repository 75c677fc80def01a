"""Seeded velocity models and aperture windows of the synthetic workloads.

Plain numpy with no other import from this package, so a process that must not
load the engine library (the reference arm of bench.py, which times the
reference's own CPU engine) can build the very same models by loading this file
on its own.  rtm_b200.synth builds the workloads from these.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np


def layered_three(nx=201, nz=151, dx=10.0, dz=10.0, dipping=False) -> np.ndarray:
    """Three layers 1500/2000/2500 m/s, interfaces at 400 m and 900 m.  With
    ``dipping`` the second interface dips (0.15 slope about the centre) and a
    60x60 m 2800 m/s box sits at (1200, 700) m, like the reference generator."""
    x = (np.arange(nx, dtype=np.float32) * np.float32(dx))[:, None]
    z = (np.arange(nz, dtype=np.float32) * np.float32(dz))[None, :]
    v = np.full((nx, nz), 1500.0, np.float32)
    z2 = (np.float32(900.0) + np.float32(0.15) * (x - np.float32(0.5) * np.float32(nx) * np.float32(dx))
          if dipping else np.full_like(x, 900.0))
    v = np.where(z >= 400.0, np.float32(2000.0), v)
    v = np.where(z >= z2, np.float32(2500.0), v)
    if dipping:
        box = (x >= 1200.0) & (x < 1260.0) & (z >= 700.0) & (z < 760.0)
        v = np.where(box, np.float32(2800.0), v)
    return np.ascontiguousarray(v, np.float32).ravel()


def layered_faulted(nx, nz, dx, dz, seed, n_interfaces=10, n_faults=3, vmin=1500.0, vmax=5500.0) -> np.ndarray:
    """Dipping layers with normal faults; velocity grows with depth/layer."""
    rng = np.random.default_rng(seed)
    X = nx * dx
    Z = nz * dz
    x = np.arange(nx) * dx
    z = np.arange(nz) * dz
    base = np.sort(rng.uniform(0.08 * Z, 0.95 * Z, n_interfaces))
    slopes = rng.uniform(-0.12, 0.12, n_interfaces)
    # normal faults: plane x = xf + (z - z0)*cot(dip); hanging wall dropped by throw
    fx = np.sort(rng.uniform(0.15 * X, 0.85 * X, n_faults))
    dips = rng.uniform(np.deg2rad(55), np.deg2rad(75), n_faults) * rng.choice([-1, 1], n_faults)
    throws = rng.uniform(0.02 * Z, 0.06 * Z, n_faults)
    vel_layers = np.linspace(vmin, vmax, n_interfaces + 1) + rng.uniform(-80, 80, n_interfaces + 1)
    vel_layers[0] = vmin
    vel_layers = np.clip(np.maximum.accumulate(vel_layers), vmin, vmax)
    XX, ZZ = np.meshgrid(x, z, indexing="ij")
    shift = np.zeros_like(XX)
    for xf, dip, thr in zip(fx, dips, throws):
        plane = xf + ZZ / np.tan(dip)
        shift += np.where(XX > plane, thr, 0.0)
    layer = np.zeros_like(XX, dtype=np.int64)
    for k in range(n_interfaces):
        zk = base[k] + slopes[k] * (XX - 0.5 * X) + shift
        layer += (ZZ >= zk).astype(np.int64)
    v = vel_layers[layer]
    return np.ascontiguousarray(v, np.float32).ravel()


def gradient_lenses(nx, nz, dx, dz, seed, vtop=1500.0, vbot=4500.0, nlens=24, amp=0.10) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = np.arange(nx) * dx
    z = np.arange(nz) * dz
    XX, ZZ = np.meshgrid(x, z, indexing="ij")
    v = vtop + (vbot - vtop) * ZZ / max(z[-1], 1.0)
    pert = np.zeros_like(v)
    for _ in range(nlens):
        cx, cz = rng.uniform(0, x[-1]), rng.uniform(0.1 * z[-1], z[-1])
        r = rng.uniform(0.03, 0.1) * min(x[-1], z[-1])
        a = rng.uniform(-amp, amp)
        pert += a * np.exp(-((XX - cx) ** 2 + (ZZ - cz) ** 2) / (2 * r * r))
    v = v * (1.0 + np.clip(pert, -amp, amp))
    return np.ascontiguousarray(np.clip(v, 1400.0, 5000.0), np.float32).ravel()


def config3_windows(nshots: int, nx: int = 1150, seed: int = 3) -> List[Tuple[int, int]]:
    """(first column, width) of each shot's aperture window: widths uniform in
    400..1150 columns, positions uniform inside the model (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nshots):
        w = int(rng.integers(400, 1151))
        x0 = int(rng.integers(0, nx - w + 1))
        out.append((x0, w))
    return out
