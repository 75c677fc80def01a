"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the UNMODIFIED reference binaries that ``oracle/Makefile`` compiles from
the reference's own sources into ``oracle/_ref/`` (``rtm_synth`` to model shot
gathers, ``rtm`` to migrate them) and records:

* the SHA-256 of every shot file the reference wrote (RTMS bytes), so a test can
  regenerate the gathers with another engine and prove them byte-identical;
* the reference's migrated image and illumination map (``.npy``);
* the exact parameters of each run (``cases.json``).

Needs the reference tree, named by the REF_ROOT environment variable; the fixtures
it writes are committed, so nothing at test time needs the reference.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rtm-acceleration_b200"))
from rtm_b200 import synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")

# name, model ("dipping" = the reference's built-in model, "flat" = three flat
# layers written to a file), modelling args, migration args
CASES = [
    dict(name="tiny_o8_s2", model="dipping", nx=61, nz=41, dx=10.0, nt=300, dt=0.001, f0=15.0, nshots=2,
         synth_nb=20, synth_order=8, rec_dx=10.0, src_z=0.0, rec_z=0.0,
         order=8, nb=20, store=2, mute=0.0),
    dict(name="tiny_o2_s1", model="dipping", nx=48, nz=37, dx=10.0, nt=250, dt=0.001, f0=15.0, nshots=2,
         synth_nb=12, synth_order=2, rec_dx=10.0, src_z=20.0, rec_z=20.0,
         order=2, nb=12, store=1, mute=0.0),
    dict(name="tiny_o4_s3", model="dipping", nx=53, nz=40, dx=10.0, nt=260, dt=0.001, f0=14.0, nshots=3,
         synth_nb=15, synth_order=4, rec_dx=10.0, src_z=0.0, rec_z=10.0,
         order=4, nb=15, store=3, mute=1500.0),
    dict(name="tiny_o6_dup", model="dipping", nx=45, nz=33, dx=10.0, nt=240, dt=0.001, f0=15.0, nshots=2,
         synth_nb=10, synth_order=6, rec_dx=5.0, src_z=0.0, rec_z=0.0,
         order=6, nb=10, store=2, mute=0.0),
    dict(name="tiny_o10_clamp", model="dipping", nx=50, nz=36, dx=10.0, nt=240, dt=0.0008, f0=15.0, nshots=2,
         synth_nb=14, synth_order=10, rec_dx=10.0, src_z=-15.0, rec_z=-25.0,
         order=10, nb=14, store=2, mute=0.0),
    dict(name="tiny_o12_nb7", model="dipping", nx=40, nz=30, dx=10.0, nt=220, dt=0.0008, f0=15.0, nshots=2,
         synth_nb=7, synth_order=12, rec_dx=10.0, src_z=0.0, rec_z=0.0,
         order=12, nb=7, store=2, mute=0.0),
    dict(name="config1_dipping", model="dipping", nx=201, nz=151, dx=10.0, nt=1400, dt=0.001, f0=12.0,
         nshots=4, synth_nb=60, synth_order=8, rec_dx=10.0, src_z=0.0, rec_z=0.0,
         order=8, nb=60, store=2, mute=1500.0),
    dict(name="config1_flat", model="flat", nx=201, nz=151, dx=10.0, nt=1400, dt=0.001, f0=12.0,
         nshots=4, synth_nb=60, synth_order=8, rec_dx=10.0, src_z=0.0, rec_z=0.0,
         order=8, nb=60, store=2, mute=1500.0),
]


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 20), b""):
            h.update(blk)
    return h.hexdigest()


def run(cmd, cwd):
    subprocess.run(cmd, cwd=cwd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)


def make_case(c, tmp):
    d = os.path.join(tmp, c["name"])
    os.makedirs(d, exist_ok=True)
    fmt = lambda v: repr(float(v)) if isinstance(v, float) else str(v)  # noqa: E731
    synth_cmd = [os.path.join(REF, "rtm_synth"), "--outdir", d, "--nx", str(c["nx"]), "--nz", str(c["nz"]),
                 "--dx", fmt(c["dx"]), "--dz", fmt(c["dx"]), "--nt", str(c["nt"]), "--dt", fmt(c["dt"]),
                 "--f0", fmt(c["f0"]), "--nshots", str(c["nshots"]), "--order", str(c["synth_order"]),
                 "--nb", str(c["synth_nb"]), "--rec-dx", fmt(c["rec_dx"]), "--src-z", fmt(c["src_z"]),
                 "--rec-z", fmt(c["rec_z"])]
    vel_path = os.path.join(d, "velocity.bin")
    if c["model"] == "flat":
        v = synth.layered_three(c["nx"], c["nz"], c["dx"], c["dx"], dipping=False)
        v.astype("<f4").tofile(vel_path)
        with open(vel_path + ".hdr", "w") as f:
            f.write(f"nx = {c['nx']}\nnz = {c['nz']}\ndx = {c['dx']}\ndz = {c['dx']}\nox = 0\noz = 0\n"
                    "layout = zfast\n")
        synth_cmd += ["--velocity", vel_path, "--shots-out", os.path.join(d, "shots.bin")]
    run(synth_cmd, d)
    v = np.fromfile(vel_path, "<f4")
    img_path = os.path.join(d, "image.bin")
    mig_cmd = [os.path.join(REF, "rtm"), "--velocity", vel_path, "--shots", os.path.join(d, "shots.bin"),
               "--output", img_path, "--order", str(c["order"]), "--nb", str(c["nb"]), "--f0", fmt(c["f0"]),
               "--store-interval", str(c["store"]), "--write-illum-map", "--quiet"]
    if c["mute"] > 0:
        mig_cmd += ["--mute-direct", fmt(c["mute"])]
    run(mig_cmd, d)
    img = np.fromfile(img_path, "<f4")
    ill = np.fromfile(os.path.join(d, "image_illummap.bin"), "<f4")
    out = dict(c)
    out["velocity_sha256"] = hashlib.sha256(v.tobytes()).hexdigest()
    out["shots_sha256"] = sha256(os.path.join(d, "shots.bin"))
    out["image_sha256"] = hashlib.sha256(img.tobytes()).hexdigest()
    out["illum_sha256"] = hashlib.sha256(ill.tobytes()).hexdigest()
    np.save(os.path.join(HERE, c["name"] + "_image.npy"), img)
    np.save(os.path.join(HERE, c["name"] + "_illum.npy"), ill)
    return out


def main():
    ref_root = os.environ.get("REF_ROOT")
    if not ref_root:
        sys.exit("set REF_ROOT to the reference checkout")
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF_ROOT={ref_root}"])
    if not os.path.exists(os.path.join(REF, "rtm")):
        sys.exit("reference binaries are not built (oracle/_ref); is the reference tree present?")
    cases = []
    with tempfile.TemporaryDirectory() as tmp:
        for c in CASES:
            print("case", c["name"], flush=True)
            cases.append(make_case(c, tmp))
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump({"generated_by": "tests/golden/make_golden.py (reference binaries in oracle/_ref)",
                   "cases": cases}, f, indent=1)


if __name__ == "__main__":
    main()
