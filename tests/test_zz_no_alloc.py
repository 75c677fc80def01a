"""The allocation-free modelling entry point, rtm_b200_model_shot_static.

Some callers cannot call cudaMalloc: plugins whose host application owns all
device memory through its own pool, and loops that cannot afford the
device-wide synchronisation cudaMalloc/cudaFree imply.  For them the library
models one shot using only a fixed scratch array compiled into its device
image.  These tests call that entry point through the C ABI twice in a row and
check that it returns exactly what the ordinary entry point
(rtm_b200_model_shots, which allocates its buffers) returns, that its later
calls leave free device memory unchanged, that two host threads calling it at
the same time both get exact results (the per-device lock serialises them on
the shared array), and that it rejects a problem too large for its scratch
with a clear error.  The free-memory check starts after the first call on
purpose: that call loads the library's device module (which holds the array)
and looks up the array's address, and module loading is not an allocation the
entry point makes.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import bits_equal, make_engine, random_problem
from rtm_b200 import _lib as L
from rtm_b200.engine import shots_to_c

pytestmark = pytest.mark.gpu


def _problem(p, v, device=0):
    vel = np.ascontiguousarray(v, np.float32)
    pr = L.StaticProblem(vel.ctypes.data_as(C.POINTER(C.c_float)), p.nx, p.nz, p.dx, p.dz, p.ox, p.oz, p.nb,
                         p.order, p.sponge_alpha, p.f0, p.nt, p.dt, device)
    return pr, vel


def _call_static(pr, shot_c, out_ptr):
    err = C.create_string_buffer(512)
    rc = L.load().rtm_b200_model_shot_static(C.byref(pr), shot_c, C.c_void_p(out_ptr), err, 512)
    return rc, err.value.decode()


def test_static_modelling_matches_allocating_entry_point_twice():
    import torch
    p, v, shots = random_problem(seed=77, order=8, nx=70, nz=45, nb=12, nt=220, si=1)
    shot = shots[0]
    with make_engine("plain", p, v) as e:          # the ordinary, allocating entry point
        expected = e.model_shots([shot])[0]
    pr, vel = _problem(p, v)
    keep = []
    shot_c = shots_to_c([shot], keep)
    out = np.full(shot.nrec * p.nt, np.nan, np.float32)
    rc, msg = _call_static(pr, shot_c, out.ctypes.data)     # first call: per-device set-up
    assert rc == 0, msg
    assert bits_equal(out, expected)
    free_before = torch.cuda.mem_get_info(0)[0]
    out2 = np.full_like(out, np.nan)
    rc, msg = _call_static(pr, shot_c, out2.ctypes.data)    # second call reuses the scratch
    assert rc == 0, msg
    free_after = torch.cuda.mem_get_info(0)[0]
    assert bits_equal(out2, expected)
    assert abs(free_after - free_before) < (2 << 20)        # nothing was allocated
    # output written straight into caller-owned device memory
    dev = torch.full((shot.nrec * p.nt,), float("nan"), dtype=torch.float32, device="cuda:0")
    rc, msg = _call_static(pr, shot_c, dev.data_ptr())
    assert rc == 0, msg
    assert bits_equal(dev.cpu().numpy(), expected)


def test_static_modelling_from_two_threads_at_once():
    import threading
    p, v, shots = random_problem(seed=78, order=6, nx=64, nz=40, nb=10, nt=180, si=1)
    with make_engine("plain", p, v) as e:
        expected = e.model_shots(shots[:2])
    pr, vel = _problem(p, v)
    keep = []
    shot_cs = [shots_to_c([s], keep) for s in shots[:2]]
    outs = [np.full(s.nrec * p.nt, np.nan, np.float32) for s in shots[:2]]
    rcs = [None, None]

    def work(i):
        for _ in range(3):
            rcs[i] = _call_static(pr, shot_cs[i], outs[i].ctypes.data)
            if rcs[i][0] != 0:
                return

    th = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i in range(2):
        assert rcs[i][0] == 0, rcs[i][1]
        assert bits_equal(outs[i], expected[i])


def test_static_modelling_rejects_problems_beyond_its_scratch():
    p, v, shots = random_problem(seed=3, order=4, nx=16, nz=16, nb=5, nt=10, si=1)
    p.nx, p.nz = 2600, 1300                       # ~3.6 M extended cells: more than the 32 MiB scratch
    big_v = np.full(p.nx * p.nz, 2000.0, np.float32)
    pr, vel = _problem(p, big_v)
    keep = []
    shot_c = shots_to_c([shots[0]], keep)
    out = np.zeros(shots[0].nrec * p.nt, np.float32)
    rc, msg = _call_static(pr, shot_c, out.ctypes.data)
    assert rc == L.EINVAL
    assert "scratch" in msg
