"""The oracle pinned against the reference itself (CPU only, no GPU).

The oracle (oracle/rtm_oracle.cpp) is a CPU restatement of the reference's
CPUReferenceRTM.  Before any GPU result is checked against it, it is checked
here against:

  * the golden fixtures in tests/golden/, written by the UNMODIFIED reference
    binaries (tests/golden/make_golden.py): the SHA-256 of every RTMS shot file
    the reference's rtm_synth wrote, and the reference rtm's migrated image and
    illumination -- bit for bit;
  * the reference binaries compiled into oracle/_ref/ (when present) on
    random problems that exercise every order, store interval, duplicated and
    clamped receivers and traces longer than the time axis -- bit for bit.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from helpers import bits_equal, golden_arrays, golden_cases, golden_inputs, params, random_problem, rel_l2, sha256
from rtm_b200 import io as rio
from rtm_b200 import synth


def _model_with_oracle(case, v, shots):
    p = params(case["nx"], case["nz"], case["nt"], float(np.float32(case["dt"])), order=case["synth_order"],
               nb=case["synth_nb"], si=1, f0=case["f0"], dx=case["dx"], dz=case["dx"])
    for s, t in zip(shots, oracle.model_shots(p, v, shots)):
        s.traces = t


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_oracle_reproduces_reference_golden_vectors(case):
    v, shots = golden_inputs(case)
    assert sha256(v.tobytes()) == case["velocity_sha256"]
    _model_with_oracle(case, v, shots)
    # the reference's own shot file, byte for byte
    assert sha256(synth.shots_file_bytes(shots)) == case["shots_sha256"]
    dt = float(np.float32(case["dt"]))
    if case["mute"] > 0:
        t_pad = float(np.float32(1.0) / np.float32(case["f0"]))
        for s in shots:
            s.traces = oracle.mute_direct_wave(s, case["mute"], t_pad, t_pad, case["nt"], dt)
    p = params(case["nx"], case["nz"], case["nt"], dt, order=case["order"], nb=case["nb"], si=case["store"],
               f0=case["f0"], dx=case["dx"], dz=case["dx"])
    img, ill = oracle.migrate(p, v, shots)
    ref_img, ref_ill = golden_arrays(case["name"])
    assert sha256(ref_img.astype("<f4").tobytes()) == case["image_sha256"]
    assert bits_equal(img, ref_img), rel_l2(ref_img, img)
    assert bits_equal(ill, ref_ill), rel_l2(ref_ill, ill)


def test_golden_cases_cover_the_edge_cases():
    """Every order 2..12, store intervals 1..3, duplicated receivers (rec_dx <
    dx), clamped positions (negative depths), the minimum sponge nb = h+1, the
    mute, and both config-1 models."""
    cs = golden_cases()
    assert {c["order"] for c in cs} >= {2, 4, 6, 8, 10, 12}
    assert {c["store"] for c in cs} >= {1, 2, 3}
    assert any(c["rec_dx"] < c["dx"] for c in cs)
    assert any(c["src_z"] < 0 or c["rec_z"] < 0 for c in cs)
    assert any(c["nb"] == c["order"] // 2 + 1 for c in cs)
    assert any(c["mute"] > 0 for c in cs)
    assert {c["name"] for c in cs} >= {"config1_flat", "config1_dipping"}


REF_RTM = oracle.ref_binary("rtm")


def _run_reference(p, v, shots, workdir, engine="cpu"):
    vel = os.path.join(workdir, "v.bin")
    rio.write_velocity_raw(vel, v)
    rio.write_header_file(vel + ".hdr", rio.VelocityHeader(p.nx, p.nz, p.dx, p.dz, p.ox, p.oz, "zfast"))
    sp = os.path.join(workdir, "s.bin")
    rio.write_shots_raw(sp, shots)
    out = os.path.join(workdir, "img.bin")
    cmd = [REF_RTM, "--engine", engine, "--velocity", vel, "--shots", sp, "--output", out, "--order", str(p.order),
           "--nb", str(p.nb), "--f0", repr(float(p.f0)), "--store-interval", str(p.store_interval),
           "--nt", str(p.nt), "--write-illum-map", "--quiet"]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
    return rio.read_raw_floats(out), rio.read_raw_floats(os.path.join(workdir, "img_illummap.bin"))


@pytest.mark.skipif(REF_RTM is None, reason="reference binaries not built into oracle/_ref")
@pytest.mark.parametrize("order,si,nt_trunc", [(2, 1, 0), (6, 3, 0), (8, 2, 30), (12, 2, 0)])
def test_oracle_bit_identical_to_reference_binary(order, si, nt_trunc):
    p, v, shots = random_problem(seed=200 + order, order=order, nx=33, nz=27, nb=order // 2 + 2, nt=90, si=si)
    if nt_trunc:
        p.nt = p.nt - nt_trunc      # the reference's --nt: traces keep their own length
    with tempfile.TemporaryDirectory() as td:
        ref_img, ref_ill = _run_reference(p, v, shots, td)
    img, ill = oracle.migrate(p, v, shots)
    assert bits_equal(img, ref_img), rel_l2(ref_img, img)
    assert bits_equal(ill, ref_ill), rel_l2(ref_ill, ill)


def test_fp64_oracle_is_the_same_scheme():
    """FP64 oracle: same tables, wider arithmetic -> close to the float oracle."""
    p, v, shots = random_problem(seed=11, order=8, nx=40, nz=32, nb=8, nt=120, si=2)
    i32, s32 = oracle.migrate(p, v, shots)
    i64, s64 = oracle.migrate(p, v, shots, np.float64)
    assert 0 < rel_l2(i64, i32) < 1e-4
    assert rel_l2(s64, s32) < 1e-5


def test_fp64_sum_oracle_shares_the_fp32_propagation():
    """migrate_sum64 runs the FP32 scheme and only widens the sums: it sits
    within FP32 rounding of the FP32 oracle, and its sums differ from the
    FP32 ones."""
    p, v, shots = random_problem(seed=5, order=8, nx=37, nz=29, nb=10, nt=120, si=1)
    img32, ill32 = oracle.migrate(p, v, shots)
    img, ill = oracle.migrate_sum64(p, v, shots)
    assert rel_l2(img, img32) <= 1e-6 and rel_l2(ill, ill32) <= 1e-6
    assert not np.array_equal(img.astype(np.float32), img32) or not np.array_equal(ill.astype(np.float32), ill32)


def test_oracle_rejects_what_the_reference_rejects():
    p, v, shots = random_problem(seed=1, order=8, nx=20, nz=20, nb=8, nt=20, si=1)
    for bad in (dict(order=7), dict(nb=4), dict(store_interval=0), dict(nt=0)):
        q = params(**{**{k: getattr(p, k) for k in ("nx", "nz", "nt", "dt", "order", "nb")},
                      "si": p.store_interval, **{("si" if k == "store_interval" else k): x for k, x in bad.items()}})
        with pytest.raises(ValueError):
            oracle.migrate(q, v, shots)


def test_oracle_model_shot_f64_close_to_f32():
    p, v, shots = random_problem(seed=12, order=12, nx=36, nz=30, nb=9, nt=100, si=1)
    a = oracle.model_shot(p, v, shots[0])
    b = oracle.model_shot(p, v, shots[0], np.float64)
    assert rel_l2(b, a) < 1e-4
