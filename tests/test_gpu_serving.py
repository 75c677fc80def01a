"""Serving (continuous batching) and failure detection on the GPU.

* A request's image is the same whether it runs alone or arrives while other
  requests (other grids, orders and time axes) are already on the device; the
  only difference allowed is the order in which its shots enter the FP64 stack
  (tolerance: rel-L2 <= 1e-6), and both match the FP64 oracle (rel-L2 <= 1e-5).
* Requests are validated at submission (CFL, order, velocity) and rejected with
  EREJECTED; a request whose single shot cannot fit the snapshot budget is
  rejected, while requests that fit are admitted as memory frees up.
* A step whose pipeline stage is never filled makes the kernel's bounded wait
  give up: the call reports ETIMEOUT and the engine stays usable.
"""
import os

import numpy as np
import pytest

import oracle
from helpers import bits_equal, make_engine, params, rel_l2, small_problem
from rtm_b200 import Engine, RTMError, RTMParams, synth
from rtm_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _request(seed, nx, nz, order, nt, nshots, f0=15.0):
    d = 10.0
    v = synth.layered_faulted(nx, nz, d, d, seed=seed, n_interfaces=4, n_faults=1, vmin=1500.0, vmax=3000.0)
    from rtm_b200 import max_stable_dt
    dt = float(np.float32(0.8 * max_stable_dt(float(v.max()), d, d, order)))
    shots = synth.surface_line(nx, d, nshots, nt=nt, dt=dt)
    p = params(nx, nz, nt, dt, order=order, nb=20, si=2, f0=f0)
    traces = oracle.model_shots(params(nx, nz, nt, dt, order=order, nb=20, si=1, f0=f0), v, shots)
    for s, t in zip(shots, traces):
        s.traces = t
    return p, v, shots


def _submit(e, p, v, shots, t=0.0):
    return e.submit(v, p.nx, p.nz, p.dx, p.dz, order=p.order, f0=p.f0, nt=p.nt, dt=p.dt,
                    store_interval=p.store_interval, shots=shots, arrival_time=t)


def _serve_engine(**kw):
    return Engine("serve", RTMParams(nb=20), serve_max_nx=160, serve_max_nz=120, max_shots_in_flight=6, **kw)


def test_request_alone_equals_request_in_the_mix():
    reqs = [_request(1, 90, 60, 8, 240, 3), _request(2, 130, 70, 12, 200, 4), _request(3, 60, 100, 8, 260, 2)]
    alone = []
    for p, v, shots in reqs:
        with _serve_engine() as e:
            t = _submit(e, p, v, shots)
            e.drain()
            st, img, ill = e.poll(t, p.nx, p.nz)
            assert st["state"] == 2 and st["shots_done"] == len(shots)
            alone.append((img, ill))
    with _serve_engine() as e:
        t0 = _submit(e, *reqs[0])
        e.serve_step(64)                        # request 0 is on the device ...
        st, _, _ = e.poll(t0)
        assert st["state"] == 1
        t1 = _submit(e, *reqs[1])               # ... when 1 and 2 arrive
        e.serve_step(32)
        t2 = _submit(e, *reqs[2])
        e.drain()
        mixed = [e.poll(t, p.nx, p.nz)[1:] for t, (p, _, _) in zip((t0, t1, t2), reqs)]
    for (p, v, shots), (ai, asv), (mi, msv) in zip(reqs, alone, mixed):
        assert rel_l2(ai, mi) <= 1e-6 and rel_l2(asv, msv) <= 1e-6
        ref, _ = oracle.migrate(p, v, shots, np.float64)
        assert rel_l2(ref, mi) <= 1e-5


def test_serving_rejects_invalid_requests():
    p, v, shots = _request(4, 60, 50, 8, 120, 2)
    with _serve_engine() as e:
        with pytest.raises(RTMError) as ei:                       # CFL violation
            e.submit(v, p.nx, p.nz, p.dx, p.dz, order=8, f0=15.0, nt=p.nt, dt=p.dt * 3.0, store_interval=2,
                     shots=shots)
        assert ei.value.code == L.EREJECTED
        with pytest.raises(RTMError) as ei:                       # unsupported order
            e.submit(v, p.nx, p.nz, p.dx, p.dz, order=9, f0=15.0, nt=p.nt, dt=p.dt, store_interval=2, shots=shots)
        assert ei.value.code == L.EREJECTED
        bad = v.copy()
        bad[0] = 0.0
        with pytest.raises(RTMError):                             # non-physical velocity
            e.submit(bad, p.nx, p.nz, p.dx, p.dz, order=8, f0=15.0, nt=p.nt, dt=p.dt, store_interval=2, shots=shots)
        with pytest.raises(RTMError) as ei:                       # unknown ticket
            e.poll(12345)
        assert ei.value.code == L.ENOTFOUND
        t = _submit(e, p, v, shots)                               # still serves valid work
        e.drain()
        assert e.poll(t)[0]["state"] == 2


def test_admission_by_snapshot_bytes():
    """With a budget for about two shots' snapshots, a request of several shots
    still completes (shots are admitted as others retire); one whose single
    shot cannot fit is rejected at submission."""
    p, v, shots = _request(5, 120, 80, 8, 2400, 4)
    nsnap = (p.nt - 1) // p.store_interval + 1
    per_shot = nsnap * p.nx * 80 * 4                   # 80 stored rows per column (nb 20, nz 80)
    # what the server keeps aside besides the arena: per-slot tables of its
    # largest grid (160 x 120, 120 stored rows) for 6 slots, plus 2 GiB
    reserve = 6 * (160 * 120 * 16 + 160 * 6000 * 4) + (2 << 30)
    budget = reserve + int(2.5 * per_shot)
    with Engine("serve", RTMParams(nb=20), serve_max_nx=160, serve_max_nz=120, max_shots_in_flight=6,
                device_mem_budget=budget) as e:
        t = _submit(e, p, v, shots)
        e.drain()
        st, img, _ = e.poll(t, p.nx, p.nz)
        assert st["state"] == 2 and st["shots_done"] == 4
        ref, _ = oracle.migrate(p, v, shots, np.float64)
        assert rel_l2(ref, img) <= 1e-5
        # one shot of 15000 snapshots on 150 x 110 cells: far over the budget
        v2 = np.full(150 * 110, 2000.0, np.float32)
        s2 = synth.surface_line(150, 10.0, 1, nt=30000, dt=0.001)
        s2[0].traces = np.zeros(150 * 30000, np.float32)
        p2 = params(150, 110, 30000, 0.001, order=8, nb=20, si=2)
        with pytest.raises(RTMError) as ei:
            _submit(e, p2, v2, s2)
        assert ei.value.code == L.EREJECTED


def test_bounded_wait_gives_up_and_engine_recovers():
    p, v, shots = small_problem(order=8, si=2, nt=120)
    ref_img, _ = oracle.migrate(p, v, shots)
    os.environ["RTM_B200_STALL_TILE"] = "0"
    try:
        e = make_engine("plain", p, v)
    finally:
        del os.environ["RTM_B200_STALL_TILE"]
    with e:
        with pytest.raises(RTMError) as ei:
            e.migrate(shots)
        assert ei.value.code == L.ETIMEOUT
        img, _ = e.migrate(shots)                # the same engine, next call: correct again
        assert bits_equal(img, ref_img)
