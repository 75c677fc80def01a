"""Parity at the configurations' own sizes, against the reference CPU engine.

The reference's own cpu-opt engine (oracle/_ref/rtm, compiled from its sources;
bit-identical to its `cpu` engine, checked in tests/test_oracle_golden.py) and
this library migrate the same files:

  * one whole shot of the 1150 x 400 production model (nt 4000, order 8);
  * one shot of the uneven-aperture survey on its own window (order 12): the
    reference CLI migrates the window's columns as their own model, this
    library migrates the window inside the full model;
  * one shot of the 4000 x 1500 model at order 12 with nt cut to 500;
  * the smallest and largest grids of the serving stream (201 x 151 at nt
    1400, 2000 x 800 at order 12 with nt cut to 1000).

Gates (the reference's own gate is rel-L2 < 1e-5 and correlation > 0.9999,
src/tools/compare_main.cpp:52-53):
  * plain engine, IEEE arithmetic: bit-identical;
  * FMA arithmetic: rel-L2 <= 1e-4 (max-abs in the assertion message);
  * batch and serve engines (FMA, compensated FP32 per shot, FP64 stack):
    rel-L2 <= 1e-4 against the reference and <= 1e-5 against the GPU FP64
    engine (the reference's FP32 image is itself ~5e-6 from FP64);
  * BF16 / FP16 snapshots and source reconstruction: rel-L2 <= 1e-3 against
    the GPU FP64 engine, which tests/test_gpu_parity.py pins to the FP64 oracle.
Traces are modelled by the plain engine (the reference's modelling bit for bit).
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from helpers import bits_equal, rel_l2
from rtm_b200 import Engine, RTMParams, synth
from rtm_b200 import io as rio
from rtm_b200.engine import ShotRecord

pytestmark = pytest.mark.gpu
REF_RTM = oracle.ref_binary("rtm")
needs_ref = pytest.mark.skipif(REF_RTM is None, reason="reference binaries not built into oracle/_ref")


def _model(vel, nx, nz, d, order, nb, nt, dt, f0, shots):
    p = RTMParams(nb=nb, order=order, f0=f0, store_interval=1)
    with Engine("plain", p) as e:
        e.setup(vel, nx, nz, d, d, nt=nt, dt=dt)
        tr = e.model_shots(shots)
    for s, t in zip(shots, tr):
        s.traces = t


def _reference(vel, nx, nz, d, ox, shots, order, nb, f0, si):
    """The reference CLI's image of `shots` on the model `vel` (nx x nz, origin ox)."""
    with tempfile.TemporaryDirectory() as td:
        vp, sp, out = os.path.join(td, "v.bin"), os.path.join(td, "s.bin"), os.path.join(td, "i.bin")
        rio.write_velocity_raw(vp, vel)
        rio.write_header_file(vp + ".hdr", rio.VelocityHeader(nx, nz, d, d, ox, 0.0, "zfast"))
        rio.write_shots_raw(sp, shots)
        env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
        subprocess.run([REF_RTM, "--engine", "cpu-opt", "--velocity", vp, "--shots", sp, "--output", out, "--order",
                        str(order), "--nb", str(nb), "--f0", repr(f0), "--store-interval", str(si), "--quiet"],
                       check=True, capture_output=True, env=env)
        return rio.read_raw_floats(out)


def _migrate(mode, vel, nx, nz, d, nt, dt, order, nb, f0, si, shots, **kw):
    p = RTMParams(nb=nb, order=order, f0=f0, store_interval=si)
    with Engine(mode, p, **kw) as e:
        e.setup(vel, nx, nz, d, d, nt=nt, dt=dt)
        img, _ = e.migrate(shots)
    return img


def _gate(ref, img, tol, what):
    r = rel_l2(ref, img)
    mx = float(np.abs(np.asarray(ref, np.float64) - img).max())
    assert r <= tol, f"{what}: rel-L2 {r:.3e} > {tol:g} (max-abs {mx:.4g}, max|ref| {np.abs(ref).max():.4g})"


@needs_ref
def test_production_model_whole_shot():
    """1150 x 400 @10 m, nt 4000, dt 0.8 ms, order 8, store 2: one whole shot."""
    w = synth.config2(nshots=64)
    shot = w.shots[21]
    _model(w.vel, w.nx, w.nz, w.dx, w.order, w.nb, w.nt, w.dt, w.f0, [shot])
    ref = _reference(w.vel, w.nx, w.nz, w.dx, 0.0, [shot], w.order, w.nb, w.f0, w.store_interval)
    args = (w.vel, w.nx, w.nz, w.dx, w.nt, w.dt, w.order, w.nb, w.f0, w.store_interval, [shot])
    assert bits_equal(_migrate("plain", *args), ref)
    _gate(ref, _migrate("plain", *args, arithmetic="fma"), 1e-4, "plain FMA")
    p = RTMParams(nb=w.nb, order=w.order, f0=w.f0, store_interval=w.store_interval)
    with Engine("batch", p, arithmetic="fp64") as e:
        e.setup(w.vel, w.nx, w.nz, w.dx, w.dx, nt=w.nt, dt=w.dt)
        ref64, _ = e.migrate_f64([shot])
    batch = _migrate("batch", *args)
    _gate(ref, batch, 1e-4, "batch vs reference")
    _gate(ref64, batch, 1e-5, "batch vs FP64")
    _gate(ref64, ref, 1e-4, "reference vs FP64")


@needs_ref
def test_survey_window_order12():
    """A survey shot on its own aperture window, order 12: the window inside the
    full model equals the reference on the window's columns."""
    w = synth.config3(nshots=256, order=12)
    shot = w.shots[5]
    x0, wn = shot.window_x0, shot.window_nx
    v2 = w.vel.reshape(w.nx, w.nz)
    win = np.ascontiguousarray(v2[x0:x0 + wn]).ravel()
    # modelled and migrated on the window, the reference's way
    plain_shot = ShotRecord(shot.sx, shot.sz, shot.rx, shot.rz, nt=shot.nt, dt=shot.dt)
    _model(w.vel, w.nx, w.nz, w.dx, 12, w.nb, w.nt, w.dt, w.f0, [shot])
    plain_shot.traces = shot.traces
    ref = _reference(win, wn, w.nz, w.dx, x0 * w.dx, [plain_shot], 12, w.nb, w.f0, w.store_interval)
    img = _migrate("plain", w.vel, w.nx, w.nz, w.dx, w.nt, w.dt, 12, w.nb, w.f0, w.store_interval, [shot])
    got = img.reshape(w.nx, w.nz)[x0:x0 + wn].ravel()
    assert bits_equal(got, ref)
    assert not np.any(img.reshape(w.nx, w.nz)[:x0]) and not np.any(img.reshape(w.nx, w.nz)[x0 + wn:])


@needs_ref
def test_large_grid_order12_truncated():
    """4000 x 1500 @5 m, order 12, nt cut to 500: plain bit-identical; BF16, FP16
    and source reconstruction within 1e-3 of the GPU FP64 engine."""
    w = synth.config4(nshots=16)
    nt = 500
    shot = w.shots[7]
    shot.nt = nt
    _model(w.vel, w.nx, w.nz, w.dx, w.order, w.nb, nt, w.dt, w.f0, [shot])
    ref = _reference(w.vel, w.nx, w.nz, w.dx, 0.0, [shot], w.order, w.nb, w.f0, w.store_interval)
    args = (w.vel, w.nx, w.nz, w.dx, nt, w.dt, w.order, w.nb, w.f0, w.store_interval, [shot])
    assert bits_equal(_migrate("plain", *args), ref)
    p = RTMParams(nb=w.nb, order=w.order, f0=w.f0, store_interval=w.store_interval)
    with Engine("batch", p, arithmetic="fp64") as e:
        e.setup(w.vel, w.nx, w.nz, w.dx, w.dx, nt=nt, dt=w.dt)
        ref64, _ = e.migrate_f64([shot])
    _gate(ref64, ref, 1e-4, "reference FP32 vs FP64")
    for snap in ("bf16", "f16", "recon"):
        _gate(ref64, _migrate("batch", *args, snap=snap), 1e-3, f"batch {snap}")


@needs_ref
@pytest.mark.parametrize("nx,nz,order,nt", [(201, 151, 8, 1400), (2000, 800, 12, 1000)])
def test_serving_extremes(nx, nz, order, nt):
    """The smallest and largest grids of the serving stream, through the serving
    engine, against the reference."""
    from rtm_b200 import max_stable_dt
    d = 10.0
    v = synth.layered_faulted(nx, nz, d, d, seed=77, n_interfaces=6, n_faults=1, vmin=1500.0, vmax=4000.0)
    dt = float(np.float32(0.8 * max_stable_dt(float(v.max()), d, d, order)))
    shots = synth.surface_line(nx, d, 2, nt=nt, dt=dt)
    _model(v, nx, nz, d, order, 60, nt, dt, 15.0, shots)
    ref = _reference(v, nx, nz, d, 0.0, shots, order, 60, 15.0, 2)
    with Engine("serve", RTMParams(nb=60), serve_max_nx=nx, serve_max_nz=nz, max_shots_in_flight=4) as e:
        t = e.submit(v, nx, nz, d, d, order=order, f0=15.0, nt=nt, dt=dt, store_interval=2, shots=shots,
                     arrival_time=0.0)
        e.drain()
        st, img, _ = e.poll(t, nx, nz)
    assert st["state"] == 2
    _gate(ref, img, 1e-4, "serve vs reference")
