"""The drop-in boundary proven on the reference's own code.

oracle/Makefile (target ref-b200) compiles the reference's unmodified CLI
(src/main.cpp and every reference source except its engine registry) with the
B200 engine bound as a maintainer of the reference would bind it:
rtm-acceleration_b200/integration/b200_engine.cpp, an rtm::RTMEngine subclass
over the C ABI compiled against the reference's include/rtm_engine.hpp, and
integration/factory_b200.cpp, which registers it beside the reference's cpu and
cpu-opt engines.  These tests run that binary: `--engine b200` reproduces the
reference's golden images bit for bit (with the direct-wave mute and the
illumination / Laplacian outputs of the reference's own driver), and the batch
engine passes the reference's own comparison gate against them.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from helpers import bits_equal, golden_arrays, golden_cases, golden_inputs, params, rel_l2
from rtm_b200 import io as rio

pytestmark = pytest.mark.gpu
BOUND = oracle.ref_binary("rtm_b200ref")
REF_RTM = oracle.ref_binary("rtm")
CASES = [c for c in golden_cases() if c["name"] in ("tiny_o8_s2", "tiny_o4_s3", "config1_dipping")]


def _inputs(td, case):
    """The golden case's velocity and shot files; traces modelled by the oracle,
    whose modelling is the reference's bit for bit (tests/test_oracle_golden.py)."""
    v, shots = golden_inputs(case)
    pm = params(case["nx"], case["nz"], case["nt"], float(np.float32(case["dt"])), order=case["synth_order"],
                nb=case["synth_nb"], si=1, f0=case["f0"])
    for s, t in zip(shots, oracle.model_shots(pm, v, shots)):
        s.traces = t
    vp, sp = os.path.join(td, "v.bin"), os.path.join(td, "s.bin")
    rio.write_velocity_raw(vp, v)
    rio.write_header_file(vp + ".hdr", rio.VelocityHeader(case["nx"], case["nz"], case["dx"], case["dx"], 0.0, 0.0,
                                                          "zfast"))
    rio.write_shots_raw(sp, shots)
    return vp, sp


def _run(binary, engine, vp, sp, out, case, extra=()):
    args = [binary, "--engine", engine, "--velocity", vp, "--shots", sp, "--output", out, "--order",
            str(case["order"]), "--nb", str(case["nb"]), "--f0", repr(case["f0"]), "--store-interval",
            str(case["store"]), "--mute-direct", repr(case["mute"]), "--quiet", *extra]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return r


@pytest.mark.skipif(BOUND is None, reason="ref-b200 binary not built into oracle/_ref")
def test_bound_cli_lists_the_b200_engines():
    out = subprocess.run([BOUND, "--list-engines"], capture_output=True, text=True, check=True).stdout.split()
    assert out[:2] == ["cpu", "cpu-opt"] and {"b200", "b200-batch", "b200-serve"} <= set(out)


@pytest.mark.skipif(BOUND is None, reason="ref-b200 binary not built into oracle/_ref")
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_reference_cli_through_rtm_engine_matches_golden(case):
    ref_img, ref_ill = golden_arrays(case["name"])
    with tempfile.TemporaryDirectory() as td:
        vp, sp = _inputs(td, case)
        out = os.path.join(td, "img.bin")
        _run(BOUND, "b200", vp, sp, out, case, ["--write-illum-map", "--illumination", "--filter", "laplacian"])
        img = rio.read_raw_floats(out)
        ill = rio.read_raw_floats(out.replace(".bin", "_illummap.bin"))
        assert bits_equal(img, ref_img) and bits_equal(ill, ref_ill)
        if REF_RTM:
            # the reference's own CPU engine through the same driver writes the
            # same post-processed outputs
            rout = os.path.join(td, "ref.bin")
            _run(REF_RTM, "cpu", vp, sp, rout, case, ["--illumination", "--filter", "laplacian"])
            for suffix in ("_illum", "_filtered"):
                assert bits_equal(rio.read_raw_floats(out.replace(".bin", suffix + ".bin")),
                                  rio.read_raw_floats(rout.replace(".bin", suffix + ".bin"))), suffix
        bout = os.path.join(td, "batch.bin")
        _run(BOUND, "b200-batch", vp, sp, bout, case)
        assert rel_l2(ref_img, rio.read_raw_floats(bout)) < 1e-5
