"""The C++ command-line tools (rtm, rtm_synth, rtm_compare) and the C++ host
library behind them.

CPU: flag handling, the C++ readers (velocity + .hdr sidecar precedence, RTMS,
SEG-Y) against the Python readers, the comparison tool's metrics and its exit
codes, and the loud failure of the GPU engines on a host without a GPU.
GPU: `rtm --engine b200` writes the same image as the reference's own
`rtm --engine cpu` on the same files (bit for bit), and `rtm_synth` writes the
reference's shot file byte for byte.
"""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from helpers import bits_equal, golden_cases, random_problem, sha256
from rtm_b200 import io as rio
from rtm_b200 import metrics, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "rtm-acceleration_b200", "bin")


def tool(name):
    p = os.path.join(BIN, name)
    if not os.path.exists(p):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "rtm-acceleration_b200"), "tools"])
    return p


def _gpu_visible():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _write_inputs(td, p, v, shots, layout="zfast", header=True):
    vel = os.path.join(td, "v.bin")
    data = v if layout == "zfast" else v.reshape(p.nx, p.nz).T.copy().ravel()
    rio.write_velocity_raw(vel, data)
    if header:
        rio.write_header_file(vel + ".hdr", rio.VelocityHeader(p.nx, p.nz, p.dx, p.dz, p.ox, p.oz, layout))
    sp = os.path.join(td, "s.bin")
    rio.write_shots_raw(sp, shots)
    return vel, sp


def test_list_engines_and_unknown_options():
    out = subprocess.run([tool("rtm"), "--list-engines"], capture_output=True, text=True, check=True).stdout
    assert out.split() == ["b200", "b200-batch", "b200-serve"]
    r = subprocess.run([tool("rtm"), "--bogus"], capture_output=True, text=True)
    assert r.returncode == 1 and "ERROR: unknown option" in r.stderr
    r = subprocess.run([tool("rtm"), "--engine", "cpu", "--velocity", "a", "--shots", "b", "--output", "c"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "unknown or unavailable engine" in r.stderr


@pytest.mark.parametrize("layout", ["zfast", "xfast"])
def test_cpp_readers_match_python(layout):
    p, v, shots = random_problem(seed=61, order=8, nx=37, nz=29, nb=8, nt=70, si=2)
    p.ox, p.oz = 5.0, -2.5
    with tempfile.TemporaryDirectory() as td:
        vel, sp = _write_inputs(td, p, v, shots, layout)
        out = subprocess.run([tool("rtm"), "--velocity", vel, "--shots", sp, "--check-inputs", "--nt", "50"],
                             capture_output=True, text=True, check=True).stdout
        got = json.loads(out)
        # CLI values win over the sidecar
        out2 = json.loads(subprocess.run([tool("rtm"), "--velocity", vel, "--shots", sp, "--check-inputs", "--dx",
                                          "12.5", "--max-shots", "1"], capture_output=True, text=True,
                                         check=True).stdout)
    assert (got["nx"], got["nz"], got["dx"], got["ox"], got["oz"]) == (37, 29, 10.0, 5.0, -2.5)
    assert got["vmin"] == pytest.approx(float(v.min())) and got["vmax"] == pytest.approx(float(v.max()))
    assert got["shots"] == 2 and got["nrec"] == shots[0].nrec and got["nt"] == 50
    assert got["trace_sum"] == pytest.approx(float(sum(np.asarray(s.traces, np.float64).sum() for s in shots)))
    assert out2["dx"] == 12.5 and out2["shots"] == 1


def test_cpp_segy_reader_matches_python(tmp_path):
    import struct
    ns = 5
    bh = bytearray(400)
    struct.pack_into(">h", bh, 16, 2000)
    struct.pack_into(">h", bh, 20, ns)
    struct.pack_into(">h", bh, 24, 5)
    body = bytearray(3200) + bh
    for fldr, sx, gx in ((1, 100, 10), (1, 100, 20), (2, 300, 40)):
        th = bytearray(240)
        struct.pack_into(">i", th, 8, fldr)
        struct.pack_into(">h", th, 70, -10)
        struct.pack_into(">i", th, 72, sx)
        struct.pack_into(">i", th, 80, gx)
        body += th + struct.pack(f">{ns}f", *[0.5 * fldr + k for k in range(ns)])
    sgy = str(tmp_path / "d.sgy")
    open(sgy, "wb").write(bytes(body))
    vel = str(tmp_path / "v.bin")
    rio.write_velocity_raw(vel, np.full(10 * 8, 2000.0, np.float32))
    rio.write_header_file(vel + ".hdr", rio.VelocityHeader(10, 8, 10.0, 10.0))
    got = json.loads(subprocess.run([tool("rtm"), "--velocity", vel, "--shots", sgy, "--check-inputs"],
                                    capture_output=True, text=True, check=True).stdout)
    ref = rio.read_shots(sgy)
    assert got["shots"] == len(ref) == 2 and got["nt"] == ns and got["sx0"] == pytest.approx(ref[0].sx)
    assert got["trace_sum"] == pytest.approx(float(np.concatenate([r.traces for r in ref]).sum()))


def test_velocity_validation_errors(tmp_path):
    vel = str(tmp_path / "v.bin")
    rio.write_velocity_raw(vel, np.full(12, 2000.0, np.float32))
    sp = str(tmp_path / "s.bin")
    rio.write_shots_raw(sp, random_problem(seed=1, order=8, nx=8, nz=8, nb=6, nt=10, si=1)[2])
    for extra in (["--nx", "5", "--nz", "3"], []):
        r = subprocess.run([tool("rtm"), "--velocity", vel, "--shots", sp, "--check-inputs"] + extra,
                           capture_output=True, text=True)
        assert r.returncode == 1 and "ERROR:" in r.stderr


def test_compare_tool_metrics_and_gate(tmp_path):
    rng = np.random.default_rng(5)
    a = rng.standard_normal(1000).astype(np.float32)
    b = (a + 1e-7 * rng.standard_normal(1000)).astype(np.float32)
    c = (a + 1e-2 * rng.standard_normal(1000)).astype(np.float32)
    pa, pb, pc = (str(tmp_path / f"{n}.bin") for n in "abc")
    for path, arr in ((pa, a), (pb, b), (pc, c)):
        rio.write_raw_floats(path, arr)
    csv = str(tmp_path / "cmp.csv")
    r = subprocess.run([tool("rtm_compare"), pa, pb, "--csv", csv, "--engine", "b200"], capture_output=True,
                       text=True)
    assert r.returncode == 0 and "PASS" in r.stdout
    vals = dict(ln.split()[:2] for ln in r.stdout.splitlines() if ln and ln.split()[0] in
                ("l2_relative", "correlation", "max_abs"))
    m = metrics.compare_images(a, b)
    assert float(vals["l2_relative"]) == pytest.approx(m["l2_relative"], rel=1e-6)
    assert float(vals["correlation"]) == pytest.approx(m["correlation"], rel=1e-9)
    r = subprocess.run([tool("rtm_compare"), pa, pc, "--csv", csv], capture_output=True, text=True)
    assert r.returncode == 2 and "FAIL" in r.stdout
    rows = open(csv).read().splitlines()
    assert rows[0].startswith("engine,dataset") and len(rows) == 3 and rows[1].endswith(",1") and rows[2].endswith(",0")


@pytest.mark.skipif(_gpu_visible(), reason="checks the behaviour on a host without a GPU")
def test_rtm_without_gpu_fails_loudly(tmp_path):
    p, v, shots = random_problem(seed=2, order=8, nx=20, nz=16, nb=6, nt=30, si=1)
    vel, sp = _write_inputs(str(tmp_path), p, v, shots)
    r = subprocess.run([tool("rtm"), "--velocity", vel, "--shots", sp, "--output", str(tmp_path / "i.bin"),
                        "--nb", "6"], capture_output=True, text=True)
    assert r.returncode == 1 and "ERROR: rtm_b200_create" in r.stderr


REF_RTM = oracle.ref_binary("rtm")


@pytest.mark.gpu
@pytest.mark.skipif(REF_RTM is None, reason="reference binaries not built into oracle/_ref")
@pytest.mark.parametrize("order,si,mute", [(8, 2, 1500.0), (12, 3, 0.0), (4, 1, 0.0)])
def test_rtm_cli_bit_identical_to_reference_cli(order, si, mute, tmp_path):
    p, v, shots = random_problem(seed=70 + order, order=order, nx=61, nz=45, nb=order // 2 + 4, nt=150, si=si)
    vel, sp = _write_inputs(str(tmp_path), p, v, shots, "xfast")
    args = ["--velocity", vel, "--shots", sp, "--order", str(order), "--nb", str(p.nb), "--f0", "15",
            "--store-interval", str(si), "--mute-direct", str(mute), "--write-illum-map", "--illumination",
            "--filter", "laplacian", "--quiet"]
    ref_out, out = str(tmp_path / "ref.bin"), str(tmp_path / "gpu.bin")
    subprocess.run([REF_RTM, "--engine", "cpu", "--output", ref_out] + args, check=True, capture_output=True)
    subprocess.run([tool("rtm"), "--engine", "b200", "--output", out] + args, check=True, capture_output=True)
    for suffix in ("", "_illummap", "_illum", "_filtered"):
        a = rio.read_raw_floats(ref_out.replace(".bin", suffix + ".bin"))
        b = rio.read_raw_floats(out.replace(".bin", suffix + ".bin"))
        assert bits_equal(a, b), suffix
    r = subprocess.run([tool("rtm_compare"), ref_out, out], capture_output=True, text=True)
    assert r.returncode == 0


@pytest.mark.gpu
def test_rtm_synth_writes_the_reference_shot_file(tmp_path):
    c = next(c for c in golden_cases() if c["name"] == "tiny_o8_s2")
    out = str(tmp_path / "shots.bin")
    subprocess.run([tool("rtm_synth"), "--outdir", str(tmp_path), "--shots-out", out, "--nx", str(c["nx"]), "--nz",
                    str(c["nz"]), "--nt", str(c["nt"]), "--dt", repr(c["dt"]), "--f0", repr(c["f0"]), "--nshots",
                    str(c["nshots"]), "--order", str(c["synth_order"]), "--nb", str(c["synth_nb"]), "--rec-dx",
                    repr(c["rec_dx"]), "--src-z", repr(c["src_z"]), "--rec-z", repr(c["rec_z"])], check=True,
                   capture_output=True)
    assert sha256(open(out, "rb").read()) == c["shots_sha256"]
    assert sha256(open(os.path.join(str(tmp_path), "velocity.bin"), "rb").read()) == c["velocity_sha256"]
