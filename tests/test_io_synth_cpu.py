"""Readers, writers, synthetic workloads and the comparison metrics (CPU only).

The formats are the reference's (src/io/velocity_io.cpp, src/io/seismic_io.cpp):
raw float32 velocity with a ``key = value`` .hdr sidecar in zfast or xfast
layout, RTMS v1 shot files and a minimal SEG-Y rev 0/1 reader.  Where the
reference binaries are built (oracle/_ref) the files written here are also
read back by the reference itself.
"""
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from helpers import bits_equal
from rtm_b200 import RTMError, ShotRecord, metrics, synth
from rtm_b200 import io as rio


def _shots(n=3, nrec=5, nt=17, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append(ShotRecord(float(10 * i + 0.5), 2.0, rng.uniform(0, 100, nrec).astype(np.float32),
                              np.full(nrec, 3.0, np.float32), nt=nt, dt=0.002,
                              traces=rng.standard_normal(nrec * nt).astype(np.float32)))
    return out


def test_velocity_header_and_raw_round_trip_both_layouts(tmp_path):
    v = np.random.default_rng(1).uniform(1500, 4000, 7 * 5).astype(np.float32)
    p = str(tmp_path / "v.bin")
    rio.write_velocity_raw(p, v)
    h = rio.VelocityHeader(7, 5, 12.5, 10.0, 1.0, 2.0, "zfast")
    rio.write_header_file(p + ".hdr", h)
    h2 = rio.read_header_file(p + ".hdr")
    assert (h2.nx, h2.nz, h2.dx, h2.dz, h2.ox, h2.oz, h2.layout) == (7, 5, 12.5, 10.0, 1.0, 2.0, "zfast")
    assert bits_equal(rio.read_velocity_raw(p, h2), v)
    # xfast file: v[iz*nx+ix] on disk, returned transposed to zfast
    vx = v.reshape(7, 5).T.copy().ravel()
    rio.write_velocity_raw(p, vx)
    h2.layout = "xfast"
    assert bits_equal(rio.read_velocity_raw(p, h2), v)
    assert rio.read_header_file(str(tmp_path / "missing.hdr")) is None


def test_header_comments_and_unknown_keys(tmp_path):
    p = tmp_path / "a.hdr"
    p.write_text("# comment\nnx = 11   # trailing\n\nnz=9\nfoo = bar\ndx = 2.5\nlayout = xfast\n")
    h = rio.read_header_file(str(p))
    assert (h.nx, h.nz, h.dx, h.layout) == (11, 9, 2.5, "xfast")


def test_velocity_validation(tmp_path):
    p = str(tmp_path / "v.bin")
    rio.write_velocity_raw(p, np.full(12, 2000.0, np.float32))
    with pytest.raises(RTMError):                      # size mismatch
        rio.read_velocity_raw(p, rio.VelocityHeader(5, 3))
    with pytest.raises(RTMError):                      # nx/nz unset
        rio.read_velocity_raw(p, rio.VelocityHeader(0, 0))
    bad = np.full(12, 2000.0, np.float32)
    bad[4] = 25000.0
    rio.write_velocity_raw(p, bad)
    with pytest.raises(RTMError):                      # outside (0, 20000]
        rio.read_velocity_raw(p, rio.VelocityHeader(4, 3))


def test_rtms_round_trip_and_bytes(tmp_path):
    shots = _shots()
    p = str(tmp_path / "s.bin")
    rio.write_shots_raw(p, shots)
    assert open(p, "rb").read() == synth.shots_file_bytes(shots)
    back = rio.read_shots_raw(p)
    assert len(back) == 3
    for a, b in zip(shots, back):
        assert (a.sx, a.sz, a.nt) == (b.sx, b.sz, b.nt)
        assert bits_equal(a.rx, b.rx) and bits_equal(a.traces, b.traces)
    assert rio.read_shots(p)[0].nrec == 5


def test_rtms_rejects_bad_files(tmp_path):
    p = str(tmp_path / "s.bin")
    rio.write_shots_raw(p, _shots())
    data = open(p, "rb").read()
    for bad in (b"XXXX" + data[4:], data[:20], data[:-4], data[:4] + struct.pack("<i", 2) + data[8:]):
        open(p, "wb").write(bad)
        with pytest.raises(RTMError):
            rio.read_shots_raw(p)
    ragged = _shots()
    ragged[1] = _shots(1, nrec=4)[0]
    with pytest.raises(RTMError):
        rio.write_shots_raw(p, ragged)


def _ibm(x: float) -> int:
    """IEEE value -> IBM System/360 single (test helper, exact for the values used)."""
    if x == 0:
        return 0
    sign = 0x80000000 if x < 0 else 0
    x = abs(x)
    e = 0
    while x >= 1.0:
        x /= 16.0
        e += 1
    while x < 1.0 / 16.0:
        x *= 16.0
        e -= 1
    return sign | ((e + 64) << 24) | int(round(x * (1 << 24)))


@pytest.mark.parametrize("fmt", [1, 2, 3, 5])
def test_segy_reader_groups_by_field_record(tmp_path, fmt):
    ns, dt_us = 6, 2000
    traces = [(1, 100, 10, [0.5, -1.25, 2.0, 0.0, 3.0, -0.75]), (1, 100, 20, [1, 2, 3, 4, 5, 6]),
              (2, 300, 40, [-1, 0, 1, 0, -1, 0])]
    if fmt in (2, 3):
        traces = [(f, s, g, [float(int(x)) for x in t]) for f, s, g, t in traces]
    bh = bytearray(400)
    struct.pack_into(">h", bh, 16, dt_us)
    struct.pack_into(">h", bh, 20, ns)
    struct.pack_into(">h", bh, 24, fmt)
    body = bytearray(b" " * 3200) + bh
    for fldr, sx, gx, t in traces:
        th = bytearray(240)
        struct.pack_into(">i", th, 8, fldr)
        struct.pack_into(">h", th, 70, -10)          # scalco: divide by 10
        struct.pack_into(">i", th, 72, sx)
        struct.pack_into(">i", th, 80, gx)
        body += th
        if fmt == 1:
            body += b"".join(struct.pack(">I", _ibm(x)) for x in t)
        elif fmt == 5:
            body += struct.pack(f">{ns}f", *t)
        elif fmt == 2:
            body += struct.pack(f">{ns}i", *[int(x) for x in t])
        else:
            body += struct.pack(f">{ns}h", *[int(x) for x in t])
    p = str(tmp_path / "d.sgy")
    open(p, "wb").write(bytes(body))
    shots = rio.read_shots(p, src_depth=7.0, rec_depth=9.0)
    assert len(shots) == 2
    assert shots[0].sx == pytest.approx(10.0) and shots[1].sx == pytest.approx(30.0)
    assert shots[0].nrec == 2 and shots[1].nrec == 1
    assert shots[0].rx.tolist() == pytest.approx([1.0, 2.0]) and shots[0].rz.tolist() == [9.0, 9.0]
    assert shots[0].sz == 7.0 and shots[0].nt == ns and shots[0].dt == pytest.approx(0.002)
    assert np.allclose(shots[0].traces.reshape(2, ns)[0], traces[0][3])
    assert np.allclose(shots[1].traces, traces[2][3])


def test_segy_rejects_unsupported_format(tmp_path):
    bh = bytearray(400)
    struct.pack_into(">h", bh, 16, 1000)
    struct.pack_into(">h", bh, 20, 4)
    struct.pack_into(">h", bh, 24, 8)
    p = str(tmp_path / "d.segy")
    open(p, "wb").write(bytes(3200) + bytes(bh) + bytes(240 + 16))
    with pytest.raises(RTMError):
        rio.read_shots(p)


REF_RTM = oracle.ref_binary("rtm")


@pytest.mark.skipif(REF_RTM is None, reason="reference binaries not built into oracle/_ref")
def test_reference_reads_our_files(tmp_path):
    """Velocity, header and RTMS files written here migrate in the reference
    exactly like the same data handed to the oracle in memory."""
    from helpers import random_problem
    p, v, shots = random_problem(seed=41, order=4, nx=25, nz=20, nb=5, nt=60, si=1)
    vel = str(tmp_path / "v.bin")
    rio.write_velocity_raw(vel, v.reshape(p.nx, p.nz).T.copy().ravel())     # xfast on disk
    rio.write_header_file(vel + ".hdr", rio.VelocityHeader(p.nx, p.nz, p.dx, p.dz, 0.0, 0.0, "xfast"))
    sp = str(tmp_path / "s.bin")
    rio.write_shots_raw(sp, shots)
    out = str(tmp_path / "i.bin")
    subprocess.run([REF_RTM, "--engine", "cpu", "--velocity", vel, "--shots", sp, "--output", out, "--order", "4",
                    "--nb", "5", "--f0", repr(float(p.f0)), "--store-interval", "1", "--quiet"], check=True,
                   stdout=subprocess.DEVNULL)
    img, _ = oracle.migrate(p, v, shots)
    assert bits_equal(rio.read_raw_floats(out), img)


def test_workloads_have_the_configured_shapes():
    c1 = synth.config1()
    assert (c1.nx, c1.nz, c1.nt, c1.dt, c1.f0, c1.order, c1.nb, c1.store_interval) == \
        (201, 151, 1400, 0.001, 12.0, 8, 60, 2)
    assert len(c1.shots) == 4 and c1.shots[0].nrec == 201 and set(np.unique(c1.vel)) == {1500, 2000, 2500}
    assert c1.cell_updates() == pytest.approx(0.974e9, rel=1e-3)
    c2 = synth.config2(nshots=64)
    assert (c2.nx, c2.nz, c2.nt, c2.order, c2.store_interval) == (1150, 400, 4000, 8, 2)
    assert 1500 <= c2.vel.min() and c2.vel.max() <= 5500 and c2.dt <= E_cfl(c2)
    assert len(c2.shots) == 64 and all(s.nrec == 1150 for s in c2.shots)
    c3 = synth.config3()
    assert len(c3.shots) == 256
    ws = [s.window_nx for s in c3.shots]
    assert min(ws) >= 400 and max(ws) <= 1150
    assert all(0 <= s.window_x0 and s.window_x0 + s.window_nx <= c3.nx for s in c3.shots)
    # seeded: the same workload every time
    assert [s.window_x0 for s in synth.config3().shots] == [s.window_x0 for s in c3.shots]


def E_cfl(w):
    from rtm_b200 import max_stable_dt
    return max_stable_dt(float(w.vel.max()), w.dx, w.dz, w.order)


def test_serving_stream_is_cfl_valid_and_seeded():
    reqs = synth.config5_stream(nreq=6, scale=0.2)
    assert [r.arrival for r in reqs] == sorted(r.arrival for r in reqs)
    for r in reqs:
        w = r.work
        assert w.order in (8, 12) and w.dt <= E_cfl(w) and 1 <= len(w.shots) <= 32
    assert [r.arrival for r in synth.config5_stream(nreq=6, scale=0.2)] == [r.arrival for r in reqs]


def test_compare_images_formulas():
    a = np.array([1.0, -2.0, 3.0, 0.0], np.float32)
    b = np.array([1.0, -2.0, 3.5, 0.0], np.float32)
    m = metrics.compare_images(a, b)
    assert m["max_abs"] == 0.5 and m["argmax"] == 2
    assert m["l2_relative"] == pytest.approx(0.5 / np.sqrt(14.0))
    assert m["correlation"] == pytest.approx(np.dot(a, b) / np.linalg.norm(a) / np.linalg.norm(b))
    assert metrics.gate_pass(metrics.compare_images(a, a))
    assert not metrics.gate_pass(m)
    with pytest.raises(ValueError):
        metrics.compare_images(a, b[:3])
