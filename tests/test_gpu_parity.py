"""GPU parity tests: the CUDA engine against the oracle and the reference's own
outputs, through the C ABI.

Tolerances (the reference's gate is L2rel < 1e-5 and corr > 0.9999,
src/tools/compare_main.cpp:52-53):
  * plain engine, IEEE arithmetic: bit-identical to the reference CPU engine;
  * FMA arithmetic: rel-L2 <= 1e-4 against the FP32 reference (north star);
  * batch engine (compensated FP32 per shot + FP64 stack): rel-L2 <= 1e-5
    against the FP32 reference and against the FP64 oracle;
  * FP64 engine: rel-L2 <= 1e-12 against the FP64 oracle;
  * BF16/FP16 snapshots: rel-L2 <= 1e-3 against the FP64 oracle (north star).
"""
import numpy as np
import pytest

import oracle
from helpers import (bits_equal, golden_arrays, golden_cases, golden_inputs, make_engine, random_problem, rel_l2,
                     sha256, small_problem)
from rtm_b200 import RTMError, RTMParams, mute_direct_wave, synth

pytestmark = pytest.mark.gpu


# ---------------------------------------------------------------- reference
@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_reference_golden_bit_exact(case):
    """Regenerate the reference's shot file on the GPU (byte-identical, SHA-256)
    and migrate it into the reference's image, bit for bit."""
    v, shots = golden_inputs(case)
    assert sha256(v.tobytes()) == case["velocity_sha256"]
    pm = RTMParams(nb=case["synth_nb"], order=case["synth_order"], f0=case["f0"], store_interval=1)
    from rtm_b200 import Engine
    dt = float(np.float32(case["dt"]))
    with Engine("plain", pm) as em:
        em.setup(v, case["nx"], case["nz"], case["dx"], case["dx"], nt=case["nt"], dt=dt)
        traces = em.model_shots(shots)
    for s, t in zip(shots, traces):
        s.traces = t
    assert sha256(synth.shots_file_bytes(shots)) == case["shots_sha256"]
    if case["mute"] > 0:
        t_pad = float(np.float32(1.0) / np.float32(case["f0"]))
        for s in shots:
            mute_direct_wave(s, case["mute"], t_pad, t_pad)
    p = RTMParams(nb=case["nb"], order=case["order"], f0=case["f0"], store_interval=case["store"])
    with Engine("plain", p) as e:
        e.setup(v, case["nx"], case["nz"], case["dx"], case["dx"], nt=case["nt"], dt=dt)
        img, ill = e.migrate(shots)
    ref_img, ref_ill = golden_arrays(case["name"])
    assert bits_equal(img, ref_img), rel_l2(ref_img, img)
    assert bits_equal(ill, ref_ill), rel_l2(ref_ill, ill)
    # the batch engine on the same data: within the reference's own gate
    with Engine("batch", p, max_shots_in_flight=4) as eb:
        eb.setup(v, case["nx"], case["nz"], case["dx"], case["dx"], nt=case["nt"], dt=dt)
        bimg, bill = eb.migrate(shots)
    assert rel_l2(ref_img, bimg) <= 1e-5
    assert rel_l2(ref_ill, bill) <= 1e-5


# ------------------------------------------------------------------- oracle
@pytest.mark.parametrize("order", [2, 4, 6, 8, 10, 12])
@pytest.mark.parametrize("si", [1, 2, 3])
def test_plain_bit_exact_vs_oracle(order, si):
    p, v, shots = random_problem(seed=order * 10 + si, order=order, nx=57, nz=43, nb=order // 2 + 3, nt=180, si=si)
    ref_img, ref_ill = oracle.migrate(p, v, shots)
    with make_engine("plain", p, v) as e:
        img, ill = e.migrate(shots)
    assert bits_equal(img, ref_img), rel_l2(ref_img, img)
    assert bits_equal(ill, ref_ill), rel_l2(ref_ill, ill)


@pytest.mark.parametrize("order", [2, 8, 12])
def test_modelling_bit_exact_vs_oracle(order):
    p, v, shots = random_problem(seed=100 + order, order=order, nx=64, nz=50, nb=order // 2 + 2, nt=200, si=1)
    with make_engine("plain", p, v) as e:
        got = e.model_shots(shots)
    with make_engine("batch", p, v) as eb:
        got_b = eb.model_shots(shots)
    for s, g, gb in zip(shots, got, got_b):
        ref = oracle.model_shot(p, v, s)
        assert bits_equal(g, ref)
        assert bits_equal(gb, ref)


def test_tiny_grid_minimum_size():
    """nx = nz = 1 interior cell, nb = half + 1: the smallest legal grid."""
    for order in (2, 8, 12):
        h = order // 2
        p, v, shots = random_problem(seed=7 + order, order=order, nx=1, nz=1, nb=h + 1, nt=40, si=1, nrec=3)
        ref_img, ref_ill = oracle.migrate(p, v, shots)
        with make_engine("plain", p, v) as e:
            img, ill = e.migrate(shots)
        assert bits_equal(img, ref_img) and bits_equal(ill, ref_ill)


def test_ragged_sizes_cross_tile_edges():
    """Grids whose extended size is just off the 128-row / 32-column tiles."""
    for nx, nz, nb in [(97, 9, 6), (33, 129 - 12, 6), (130, 20, 5), (5, 250, 7)]:
        p, v, shots = random_problem(seed=nx + nz, order=8, nx=nx, nz=nz, nb=nb, nt=90, si=2)
        ref_img, ref_ill = oracle.migrate(p, v, shots)
        with make_engine("plain", p, v) as e:
            img, ill = e.migrate(shots)
        assert bits_equal(img, ref_img) and bits_equal(ill, ref_ill), (nx, nz)


def test_window_shot_equals_cropped_model():
    """An aperture-window shot migrates exactly like the reference on the
    cropped model, and lands in those columns of the full image."""
    p, v, shots = random_problem(seed=31, order=8, nx=90, nz=40, nb=10, nt=150, si=2)
    x0, w = 23, 51
    vv = v.reshape(p.nx, p.nz)[x0:x0 + w].copy().ravel()
    pc = type(p)(**{**p.__dict__, "nx": w, "ox": float(np.float32(p.ox) + np.float32(x0) * np.float32(p.dx))})
    ref_img, ref_ill = oracle.migrate(pc, vv, shots)
    for s in shots:
        s.window_x0, s.window_nx = x0, w
    with make_engine("plain", p, v) as e:
        img, ill = e.migrate(shots)
    img = img.reshape(p.nx, p.nz)
    ill = ill.reshape(p.nx, p.nz)
    assert bits_equal(img[x0:x0 + w].ravel(), ref_img)
    assert bits_equal(ill[x0:x0 + w].ravel(), ref_ill)
    assert not img[:x0].any() and not img[x0 + w:].any()


def test_nt_truncation_uses_trace_stride():
    """Shots longer than the time axis (the reference's --nt) are indexed with
    their own trace length."""
    p, v, shots = random_problem(seed=5, order=8, nx=40, nz=30, nb=8, nt=160, si=2)
    p.nt = 120
    ref_img, _ = oracle.migrate(p, v, shots)
    with make_engine("plain", p, v) as e:
        img, _ = e.migrate(shots)
    assert bits_equal(img, ref_img)


def test_fma_arithmetic_within_1e4():
    p, v, shots = small_problem(order=8, si=2)
    ref_img, ref_ill = oracle.migrate(p, v, shots)
    with make_engine("plain", p, v, arithmetic="fma") as e:
        img, ill = e.migrate(shots)
    assert rel_l2(ref_img, img) <= 1e-4 and rel_l2(ref_ill, ill) <= 1e-4


def test_fp64_engine_matches_fp64_oracle():
    p, v, shots = small_problem(order=8, si=2)
    ref_img, ref_ill = oracle.migrate(p, v, shots, np.float64)
    with make_engine("plain", p, v, arithmetic="fp64") as e:
        img, ill = e.migrate_f64(shots)
    assert rel_l2(ref_img, img) <= 1e-12 and rel_l2(ref_ill, ill) <= 1e-12
    with make_engine("batch", p, v, arithmetic="fp64") as e:
        img, ill = e.migrate_f64(shots)
    assert rel_l2(ref_img, img) <= 1e-12


@pytest.mark.parametrize("acc", ["compensated", "plain"])
def test_batch_engine_vs_oracles(acc):
    p, v, shots = small_problem(order=12, nshots=5, si=2)
    ref32, _ = oracle.migrate(p, v, shots)
    ref64, ill64 = oracle.migrate(p, v, shots, np.float64)
    with make_engine("batch", p, v, accumulation=acc, max_shots_in_flight=3) as e:
        img, ill = e.migrate(shots)
        img64, _ = e.migrate_f64(shots)
    assert rel_l2(ref32, img) <= 1e-5
    assert rel_l2(ref64, img64) <= 1e-5
    assert rel_l2(ill64, ill) <= 1e-5


def test_compensated_sums_match_fp64_sums_of_the_fp32_products():
    """Batch engine with IEEE propagation (the reference's FP32 fields and
    products, bit for bit): its per-shot Kahan sums (FP32 sums, BF16
    compensation words) stacked in FP64 against FP64 sums of the same
    products; the uncompensated FP32 sums for scale."""
    p, v, shots = small_problem(order=8, nshots=3, si=1, nt=400)
    ref_img, ref_ill = oracle.migrate_sum64(p, v, shots)
    err = {}
    for acc in ("compensated", "plain"):
        with make_engine("batch", p, v, arithmetic="ieee", accumulation=acc, max_shots_in_flight=3) as e:
            img, ill = e.migrate_f64(shots)
        err[acc] = (rel_l2(ref_img, img), rel_l2(ref_ill, ill))
    assert err["compensated"][0] <= 1e-8 and err["compensated"][1] <= 1e-8, err
    assert err["compensated"][0] <= err["plain"][0] and err["compensated"][1] <= err["plain"][1], err


@pytest.mark.parametrize("snap", ["bf16", "f16"])
def test_reduced_precision_snapshots_within_1e3(snap):
    p, v, shots = small_problem(order=8, nshots=3, si=2)
    ref64, ill64 = oracle.migrate(p, v, shots, np.float64)
    for mode in ("plain", "batch"):
        with make_engine(mode, p, v, snap=snap) as e:
            img, ill = e.migrate(shots)
        err = rel_l2(ref64, img)
        assert err <= 1e-3, (mode, err)
        assert rel_l2(ill64, ill) <= 1e-3


def test_run_to_run_determinism():
    """Bitwise identical on repeat (catches races); batch included."""
    p, v, shots = random_problem(seed=9, order=8, nx=70, nz=50, nb=9, nt=120, si=2)
    for mode in ("plain", "batch"):
        with make_engine(mode, p, v) as e:
            a = e.migrate(shots)
            b = e.migrate(shots)
        assert bits_equal(a[0], b[0]) and bits_equal(a[1], b[1])


# ------------------------------------------------------- method-level API
def test_forward_backward_imaging_methods():
    p, v, shots = small_problem(order=8, si=2, nt=200)
    s = shots[0]
    import oracle as O
    ref_img, ref_ill = O.migrate(p, v, [s])
    with make_engine("plain", p, v) as e:
        snaps, rec = e.forward_propagation(s, snapshots=True, recorded=True)
        assert bits_equal(rec, O.model_shot(p, v, s))
        img = np.zeros(p.nx * p.nz, np.float32)
        ill = np.zeros_like(img)
        e.backward_propagation(s, snaps, img, ill)          # host snapshots
        assert bits_equal(img, ref_img) and bits_equal(ill, ref_ill)
        img2 = np.zeros_like(img)
        ill2 = np.zeros_like(img)
        e.forward_propagation(s, snapshots=False)
        e.backward_propagation(s, None, img2, ill2)          # device-resident snapshots
        assert bits_equal(img2, ref_img)
        # one imaging step on host arrays
        nxe, nze = p.nx + 2 * p.nb, p.nz + 2 * p.nb
        rng = np.random.default_rng(0)
        f = rng.standard_normal(p.nx * p.nz).astype(np.float32)
        b = rng.standard_normal(nxe * nze).astype(np.float32)
        I = rng.standard_normal(p.nx * p.nz).astype(np.float32)
        S = rng.standard_normal(p.nx * p.nz).astype(np.float32)
        bi = b.reshape(nxe, nze)[p.nb:p.nb + p.nx, p.nb:p.nb + p.nz].ravel()
        expI = (I + f * bi).astype(np.float32)
        expS = (S + f * f).astype(np.float32)
        e.imaging(f, b, I, S)
        assert bits_equal(I, expI) and bits_equal(S, expS)


# ------------------------------------------------------------- validation
def test_parameter_validation_errors():
    p, v, shots = small_problem(order=8, si=2, nt=50)
    from rtm_b200 import Engine
    with Engine("plain", RTMParams(order=7)) as e:             # checked at setup, like the reference
        with pytest.raises(RTMError):
            e.setup(v, p.nx, p.nz, 10, 10, nt=50, dt=0.001)
    with Engine("plain", RTMParams(order=8, nb=4)) as e:     # nb < order/2+1
        with pytest.raises(RTMError):
            e.setup(v, p.nx, p.nz, 10, 10, nt=50, dt=0.001)
    with Engine("plain", RTMParams(order=8, nb=20, store_interval=0)) as e:
        with pytest.raises(RTMError):
            e.setup(v, p.nx, p.nz, 10, 10, nt=50, dt=0.001)
    bad = v.copy()
    bad[3] = -1.0
    with Engine("plain", RTMParams(order=8, nb=20)) as e:
        with pytest.raises(RTMError):
            e.setup(bad, p.nx, p.nz, 10, 10, nt=50, dt=0.001)
        with pytest.raises(RTMError):        # migrate before setup
            e.migrate(shots)
        e.setup(v, p.nx, p.nz, 10, 10, nt=50, dt=0.001)
        s = shots[0]
        s.window_x0, s.window_nx = p.nx - 3, 10
        with pytest.raises(RTMError):
            e.migrate([s])
        s.window_x0, s.window_nx = 0, 0
        short = type(s)(s.sx, s.sz, s.rx, s.rz, nt=20, dt=s.dt, traces=s.traces[: s.nrec * 20])
        with pytest.raises(RTMError):        # traces shorter than the time axis
            e.migrate([short])
        img, _ = e.migrate(shots)            # engine still usable after errors
        assert np.isfinite(img).all()


def _post_reference_f32(img, ill, nx, nz, dx, dz, eps_rel=np.float32(1e-4)):
    """The reference's float post-processing (imaging.cpp:48-75, main.cpp:211-223)
    restated with one numpy float32 operation per C operation."""
    f = np.float32
    smax = max(f(0), ill.max())
    eps = f(eps_rel * smax) + f(1e-30)
    comp = (img / (ill + eps)).astype(np.float32)
    a = comp.reshape(nx, nz)
    out = np.zeros_like(a)
    wx, wz = f(1) / f(f(dx) * f(dx)), f(1) / f(f(dz) * f(dz))
    b2 = f(2) * a[1:-1, 1:-1]
    sx = (a[2:, 1:-1] - b2) + a[:-2, 1:-1]
    sz = (a[1:-1, 2:] - b2) + a[1:-1, :-2]
    out[1:-1, 1:-1] = wx * sx + wz * sz
    return comp, out.ravel()


def test_device_postprocess_plain_bit_exact_and_batch_vs_fp64():
    """`_illum` and `_filtered` computed on the device: bit-identical to the
    reference's float formulas from the plain engine's FP32 image, and within
    1e-5 of the FP64 formulas from the batch engine's FP64 stack."""
    p, v, shots = random_problem(seed=44, order=8, nx=72, nz=48, nb=10, nt=160, si=2)
    with make_engine("plain", p, v) as e:
        img, ill = e.migrate(shots)
        comp, filt = e.postprocess(1e-4, True)
    rc, rf = _post_reference_f32(img, ill, p.nx, p.nz, p.dx, p.dz)
    assert bits_equal(comp, rc) and bits_equal(filt, rf)
    with make_engine("batch", p, v) as e:
        i64, s64 = e.migrate_f64(shots)
        comp_b, filt_b = e.postprocess(1e-4, True)
    c64 = i64 / (s64 + (1e-4 * max(0.0, s64.max()) + 1e-30))
    a = c64.reshape(p.nx, p.nz)
    f64 = np.zeros_like(a)
    f64[1:-1, 1:-1] = ((a[2:, 1:-1] - 2 * a[1:-1, 1:-1] + a[:-2, 1:-1]) / p.dx ** 2 +
                       (a[1:-1, 2:] - 2 * a[1:-1, 1:-1] + a[1:-1, :-2]) / p.dz ** 2)
    assert rel_l2(c64, comp_b) < 1e-6 and rel_l2(f64.ravel(), filt_b) < 1e-5
    assert rel_l2(rc, comp_b) < 1e-4
