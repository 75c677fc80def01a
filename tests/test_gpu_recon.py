"""Snapshot-free source reconstruction on the GPU (snap="recon").

The forward pass stores only the band of order/2 cells around the interior at
every step; the backward pass runs the source field backwards in time inside
the interior (the leapfrog update with its two time levels swapped, the band
taken from the stored strips) and images against it.  The reconstructed field
differs from the forward one by rounding only, so the image is gated like the
reduced-precision snapshots: rel-L2 <= 1e-3 against the FP64 oracle (the same
scheme in double).  It is also compared with the snapshot engine on aperture
windows, checked for run-to-run determinism, for its memory footprint, and for
a serving request.
"""
import numpy as np
import pytest

import oracle
from helpers import bits_equal, make_engine, random_problem, rel_l2, small_problem
from rtm_b200 import Engine, RTMError, RTMParams

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order,si", [(8, 2), (12, 1), (4, 3)])
def test_recon_matches_fp64_oracle(order, si):
    p, v, shots = small_problem(order=order, nx=81, nz=61, nb=order // 2 + 8, nt=420, si=si)
    ref_img, ref_ill = oracle.migrate(p, v, shots, np.float64)
    with make_engine("batch", p, v, snap="recon") as e:
        img, ill = e.migrate(shots)
    assert rel_l2(ref_img, img) <= 1e-3
    assert rel_l2(ref_ill, ill) <= 1e-3
    with make_engine("batch", p, v, snap="f32") as e:
        img32, _ = e.migrate(shots)
    assert rel_l2(ref_img, img32) <= 1e-5      # the snapshot engine, for scale


def test_recon_random_geometry_and_windows_agree_with_snapshots():
    """Off-grid, duplicated and clamped receivers, sources inside the grid, and
    aperture windows: the reconstructing engine against the snapshot engine."""
    p, v, shots = random_problem(seed=61, order=8, nx=96, nz=56, nb=12, nt=300, si=2)
    shots[1].window_x0, shots[1].window_nx = 10, 60
    shots[1].sx = float(np.float32((10 + 25) * 10.0))
    with make_engine("batch", p, v, snap="f32") as e:
        ref, ref_s = e.migrate_f64(shots)
    with make_engine("batch", p, v, snap="recon") as e:
        img, ill = e.migrate_f64(shots)
        img2, ill2 = e.migrate_f64(shots)
    assert rel_l2(ref, img) <= 1e-3 and rel_l2(ref_s, ill) <= 1e-3
    assert np.array_equal(img, img2) and np.array_equal(ill, ill2)   # run to run


def test_recon_footprint_is_the_boundary_strips():
    p, v, shots = small_problem(order=8, nx=200, nz=150, nb=20, nt=400, si=2)
    with make_engine("batch", p, v, snap="f32") as e:
        snap_bytes = e.snapshot_bytes
    with make_engine("batch", p, v, snap="recon") as e:
        strip_bytes = e.snapshot_bytes
    want = (p.nt - 1) * 2 * 4 * (p.nx + p.nz) * 4
    assert want <= strip_bytes < want + 256
    # snapshots / strips ~ (nx nz / si) / (2 H (nx + nz)) = 5.4 here; it grows
    # with the grid (23x on 4000 x 1500 at order 12 against BF16 snapshots)
    assert strip_bytes * 5 < snap_bytes


def test_recon_rejected_by_the_plain_engine():
    p, v, shots = small_problem(order=8, nx=41, nz=31, nb=10, nt=60, si=2)
    with pytest.raises(RTMError):
        make_engine("plain", p, v, snap="recon")


def test_recon_serving_request_matches_fp64():
    p, v, shots = small_problem(order=8, nx=90, nz=60, nb=20, nt=300, si=2, nshots=3)
    ref_img, _ = oracle.migrate(p, v, shots, np.float64)
    with Engine("serve", RTMParams(nb=20), serve_max_nx=160, serve_max_nz=120, max_shots_in_flight=6,
                snap="recon") as e:
        t = e.submit(v, p.nx, p.nz, p.dx, p.dz, order=p.order, f0=p.f0, nt=p.nt, dt=p.dt,
                     store_interval=p.store_interval, shots=shots, arrival_time=0.0)
        e.drain()
        st, img, _ = e.poll(t, p.nx, p.nz)
    assert st["state"] == 2
    assert rel_l2(ref_img, img) <= 1e-3
