"""Every FP32 shape of the ring step kernel on one problem, through the C ABI.

The autotuner picks the ring kernel's shape per job mix, so each shape has to
compute the same cells: tile_cols 16 runs 4 consumer warps x 16-column tiles,
tile_cols 32 runs 8 x 32, and tile_cols 16 with RTM_B200_RING_WARPS=8 runs
8 x 16, whose full bands take the per-column path and its general epilogue.
The problem is tall enough for tiles that lie inside the zero ring and hold
neither receivers nor the source (rows 128-255), which in the column-pair
shapes take the lean path of unstored steps.

Tolerances: the plain engine (IEEE arithmetic) is bit-identical to the oracle
in every shape; the batch engine's images are bit-identical across shapes and
within rel-L2 1e-5 (FP32 snapshots) or 1e-3 (BF16) of the FP64 oracle.
"""
import numpy as np
import pytest

import oracle
from helpers import bits_equal, make_engine, rel_l2, small_problem

pytestmark = pytest.mark.gpu

SHAPES = [(16, 4), (16, 8), (32, 8)]   # (tile_cols, consumer warps)


@pytest.fixture
def ring_only(monkeypatch):
    monkeypatch.setenv("RTM_B200_STEP_KERNEL", "ring")
    return monkeypatch


def shape_engine(monkeypatch, mode, p, v, shape, **kw):
    tile_cols, warps = shape
    if warps == 8 and tile_cols == 16:
        monkeypatch.setenv("RTM_B200_RING_WARPS", "8")
    else:
        monkeypatch.delenv("RTM_B200_RING_WARPS", raising=False)
    return make_engine(mode, p, v, tile_cols=tile_cols, **kw)


def tall_problem():
    return small_problem(order=8, nx=150, nz=170, nb=50, nt=260, nshots=3, si=2)


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[1]}x{s[0]}")
def test_plain_every_shape_bit_exact_vs_oracle(ring_only, shape):
    p, v, shots = tall_problem()
    ref_img, ref_ill = oracle.migrate(p, v, shots)
    with shape_engine(ring_only, "plain", p, v, shape) as e:
        img, ill = e.migrate(shots)
    assert bits_equal(img, ref_img), rel_l2(ref_img, img)
    assert bits_equal(ill, ref_ill), rel_l2(ref_ill, ill)


@pytest.mark.parametrize("snap", ["f32", "bf16"])
@pytest.mark.parametrize("acc", ["compensated", "plain"])
def test_batch_shapes_agree_bitwise(ring_only, snap, acc):
    p, v, shots = tall_problem()
    out = []
    for shape in SHAPES:
        with shape_engine(ring_only, "batch", p, v, shape, snap=snap, accumulation=acc, max_shots_in_flight=3) as e:
            out.append(e.migrate(shots))
    for other in out[1:]:
        for a, b in zip(out[0], other):
            assert bits_equal(a, b), rel_l2(a, b)
    ref64, ill64 = oracle.migrate(p, v, shots, np.float64)
    tol = 1e-5 if snap == "f32" else 1e-3
    assert rel_l2(ref64, out[0][0]) <= tol
    assert rel_l2(ill64, out[0][1]) <= tol


@pytest.mark.parametrize("snap", ["f32", "bf16"])
@pytest.mark.parametrize("order", [8, 12])
def test_batch_band_origin_shift_bitwise(monkeypatch, snap, order):
    """nze = 264 = 2 x 128 + 8: the batch (FMA) engine starts its 128-row bands
    at row 4, so two bands cover the live rows (4-259 at order 8, 6-257 at
    order 12, whose first p^n box then starts at row -4) where bands from row 0
    need a third; nxe = 184 = 11 x 16 + 8: its 16-column tiles start at column
    H, so 11 tile columns cover the live columns where 12 start at column 0.
    Same cells, so the images agree bit for bit with RTM_B200_BAND_SHIFT=0, and
    with the FP64 oracle within the tolerances above."""
    p, v, shots = small_problem(order=order, nx=84, nz=164, nb=50, nt=220, nshots=3, si=2)
    out = []
    for shift in ("1", "0"):
        monkeypatch.setenv("RTM_B200_BAND_SHIFT", shift)
        with make_engine("batch", p, v, snap=snap, max_shots_in_flight=3) as e:
            out.append(e.migrate(shots))
    for a, b in zip(out[0], out[1]):
        assert bits_equal(a, b), rel_l2(a, b)
    ref64, ill64 = oracle.migrate(p, v, shots, np.float64)
    tol = 1e-5 if snap == "f32" else 1e-3
    assert rel_l2(ref64, out[0][0]) <= tol
    assert rel_l2(ill64, out[0][1]) <= tol
