"""The C ABI of librtm_b200.so without a GPU.

* the library loads and exports every function include/rtm_b200.h declares;
* the ctypes mirrors of the ABI structs have the C layout (checked against a
  probe compiled from the header with the system C compiler);
* the host-side numerics behind the ABI (stencil weights, Ricker, CFL limit,
  points per wavelength, direct-wave mute) equal the oracle bit for bit;
* creating an engine where no sm_100 GPU is visible fails loudly with ECUDA and
  a message -- there is no CPU fallback.
"""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from rtm_b200 import RTMError, RTMParams, ShotRecord, make_engine, list_engines
from rtm_b200 import _lib as L
from rtm_b200 import engine as E

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _gpu_visible():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_library_exports_every_declared_symbol():
    lib = L.load()
    declared = L.header_symbols()
    assert len(declared) == open(L.HEADER_PATH).read().count("\nRTM_B200_API ")
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # and nothing else leaks out of the shared object (version script)
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = sorted({ln.split()[-1] for ln in out.splitlines() if " T " in ln})
    assert set(exported) == set(declared), set(exported) ^ set(declared)


def test_ctypes_structs_match_the_c_header():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "rtm_b200.h"
#define P(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  printf("config %zu\nshot %zu\ntimes %zu\nrequest %zu\nstatus %zu\nstatic %zu\n", sizeof(rtm_b200_config),
         sizeof(rtm_b200_shot), sizeof(rtm_b200_times), sizeof(rtm_b200_request),
         sizeof(rtm_b200_request_status), sizeof(rtm_b200_static_problem));
  P(rtm_b200_config, device_mem_budget) P(rtm_b200_config, serve_max_nz) P(rtm_b200_shot, traces)
  P(rtm_b200_shot, window_nx) P(rtm_b200_times, kernel_launches) P(rtm_b200_request, shots)
  P(rtm_b200_request, arrival_time) P(rtm_b200_static_problem, device)
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "probe.c")
        exe = os.path.join(td, "probe")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", exe, c], check=True)
        lines = dict(ln.rsplit(" ", 1) for ln in subprocess.run([exe], capture_output=True, text=True,
                                                                check=True).stdout.splitlines())
    got = {k: int(v) for k, v in lines.items()}
    assert got["config"] == C.sizeof(L.Config)
    assert got["shot"] == C.sizeof(L.Shot)
    assert got["times"] == C.sizeof(L.Times)
    assert got["request"] == C.sizeof(L.Request)
    assert got["status"] == C.sizeof(L.RequestStatus)
    assert got["static"] == C.sizeof(L.StaticProblem)
    assert got["rtm_b200_config.device_mem_budget"] == L.Config.device_mem_budget.offset
    assert got["rtm_b200_config.serve_max_nz"] == L.Config.serve_max_nz.offset
    assert got["rtm_b200_shot.traces"] == L.Shot.traces.offset
    assert got["rtm_b200_shot.window_nx"] == L.Shot.window_nx.offset
    assert got["rtm_b200_times.kernel_launches"] == L.Times.kernel_launches.offset
    assert got["rtm_b200_request.shots"] == L.Request.shots.offset
    assert got["rtm_b200_request.arrival_time"] == L.Request.arrival_time.offset
    assert got["rtm_b200_static_problem.device"] == L.StaticProblem.device.offset


def test_config_defaults_are_the_reference_defaults():
    """RTMParams defaults of the reference (include/rtm_types.hpp:33-40)."""
    cfg = L.Config()
    L.load().rtm_b200_config_init(C.byref(cfg))
    assert cfg.struct_size == C.sizeof(L.Config)
    assert (cfg.nb, cfg.order, cfg.store_interval) == (60, 8, 1)
    assert cfg.sponge_alpha == pytest.approx(0.0053) and cfg.f0 == 12.0
    p = RTMParams()
    assert (p.nb, p.order, p.store_interval, p.f0) == (60, 8, 1, 12.0)


@pytest.mark.parametrize("order", [2, 4, 6, 8, 10, 12])
def test_stencil_coefficients_equal_the_oracle(order):
    a = E.stencil_coefficients(order)
    b = oracle.stencil_coefficients(order)
    assert a.view(np.uint32).tolist() == b.view(np.uint32).tolist()
    assert abs(float(a[0]) + 2 * float(a[1:].sum())) < 1e-5     # a 2nd derivative kills constants


def test_stencil_coefficients_reject_bad_orders():
    for order in (0, 1, 3, 7, 14):
        with pytest.raises(RTMError):
            E.stencil_coefficients(order)


def test_ricker_and_cfl_equal_the_oracle():
    ts = np.linspace(-0.2, 0.5, 997, dtype=np.float32)
    for f0 in (10.0, 12.0, 15.0, 20.0):
        got = np.array([E.ricker(float(t), f0) for t in ts], np.float32)
        ref = np.array([oracle.ricker(float(t), f0) for t in ts], np.float32)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    for order in (2, 4, 6, 8, 10, 12):
        for vmax, d in ((2500.0, 10.0), (5500.0, 10.0), (4500.0, 5.0)):
            a = np.float32(E.max_stable_dt(vmax, d, d, order))
            b = np.float32(oracle.max_stable_dt(vmax, d, d, order))
            assert a.view(np.uint32) == b.view(np.uint32)
    # the CFL limits of the production workloads: 1.008 ms at 5500 m/s, 10 m, order 8
    # (dt 0.8 ms is stable) and ~0.537 ms at 4950 m/s (4500 + 10 % lenses), 5 m, order 12 (dt 0.4 ms is stable)
    assert E.max_stable_dt(5500.0, 10.0, 10.0, 8) == pytest.approx(1.008e-3, rel=2e-3)
    assert E.max_stable_dt(4950.0, 5.0, 5.0, 12) == pytest.approx(0.537e-3, rel=3e-3)
    assert E.points_per_wavelength(1500.0, 15.0, 10.0, 10.0) == pytest.approx(1500.0 / 37.5 / 10.0)


def test_mute_direct_wave_equals_the_oracle():
    rng = np.random.default_rng(4)
    nrec, nt, dt = 37, 300, np.float32(0.001)
    rx = rng.uniform(0, 600, nrec).astype(np.float32)
    rz = rng.uniform(0, 30, nrec).astype(np.float32)
    tr = rng.standard_normal(nrec * nt).astype(np.float32)
    s = ShotRecord(250.0, 5.0, rx, rz, nt=nt, dt=float(dt), traces=tr.copy())
    t_pad = float(np.float32(1.0) / np.float32(12.0))
    E.mute_direct_wave(s, 1500.0, t_pad, t_pad)
    ref = oracle.mute_direct_wave(ShotRecord(250.0, 5.0, rx, rz, nt=nt, dt=float(dt), traces=tr.copy()), 1500.0,
                                  t_pad, t_pad, nt, float(dt))
    assert np.array_equal(np.asarray(s.traces).view(np.uint32), ref.view(np.uint32))
    assert (np.asarray(s.traces).reshape(nrec, nt)[:, 0] == 0).all()


def test_engine_names_and_unknown_engine():
    assert list_engines() == ["b200", "b200-batch", "b200-serve"]
    with pytest.raises(RTMError):
        make_engine("cuda-v9")


@pytest.mark.skipif(_gpu_visible(), reason="checks the behaviour on a host without a GPU")
def test_create_without_gpu_fails_loudly():
    with pytest.raises(RTMError) as ei:
        make_engine("b200")
    assert ei.value.code == L.ECUDA
    assert "device" in str(ei.value).lower() or "cuda" in str(ei.value).lower()


@pytest.mark.skipif(_gpu_visible(), reason="checks the behaviour on a host without a GPU")
def test_static_entry_point_without_gpu_fails_loudly():
    v = np.full(20 * 20, 2000.0, np.float32)
    pr = L.StaticProblem(v.ctypes.data_as(C.POINTER(C.c_float)), 20, 20, 10.0, 10.0, 0.0, 0.0, 8, 8, 0.0053,
                         12.0, 10, 0.001, 0)
    keep = []
    shot = E.shots_to_c([ShotRecord(50.0, 0.0, np.array([10.0], np.float32), np.array([0.0], np.float32))], keep)
    out = np.zeros(10, np.float32)
    err = C.create_string_buffer(256)
    rc = L.load().rtm_b200_model_shot_static(C.byref(pr), shot, C.c_void_p(out.ctypes.data), err, 256)
    assert rc == L.ECUDA and err.value


def test_create_rejects_a_foreign_struct_size():
    cfg = L.Config()
    L.load().rtm_b200_config_init(C.byref(cfg))
    cfg.struct_size = 12
    h = C.c_void_p()
    assert L.load().rtm_b200_create(C.byref(cfg), C.byref(h)) == L.EINVAL
    buf = C.create_string_buffer(256)
    L.load().rtm_b200_last_error(None, buf, 256)
    assert b"struct_size" in buf.value


def test_null_handles_are_rejected():
    lib = L.load()
    assert lib.rtm_b200_destroy(None) == L.EINVAL
    assert lib.rtm_b200_migrate(None, None, 0, None, None) == L.EINVAL
    assert lib.rtm_b200_num_snapshots(None) == 0
    assert lib.rtm_b200_get_times(None, None) == L.EINVAL
