"""Readers and writers of the reference's file formats (numpy, host only).

* velocity: raw float32 little-endian, ``.hdr`` sidecar ``key = value`` with
  ``#`` comments, layouts zfast (v[ix*nz+iz]) / xfast (v[iz*nx+ix]), sanity
  range 0 < v <= 20000 (reference src/io/velocity_io.cpp:11-113);
* shots: RTMS v1 (32-byte header, then per shot sx, sz, rx[nrec], rz[nrec],
  traces[nrec*nt] trace-major; reference src/io/seismic_io.cpp:39-124) and a
  minimal SEG-Y rev 0/1 reader (formats 1/2/3/5, shots grouped by field record
  number, scalco applied; seismic_io.cpp:126-249);
* images: raw float32 (reference write_raw_floats / read_raw_floats).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass
from typing import List

import numpy as np

from .engine import RTMError, ShotRecord
from . import _lib as L

RTMS_MAGIC = b"RTMS"


@dataclass
class VelocityHeader:
    nx: int = 0
    nz: int = 0
    dx: float = 10.0
    dz: float = 10.0
    ox: float = 0.0
    oz: float = 0.0
    layout: str = "zfast"


def read_header_file(path: str, h: VelocityHeader | None = None) -> VelocityHeader | None:
    """Returns None when the file does not exist (reference returns false)."""
    if not os.path.exists(path):
        return None
    h = h or VelocityHeader()
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0]
            if "=" not in line:
                continue
            key, val = (t.strip() for t in line.split("=", 1))
            if key == "nx":
                h.nx = int(val)
            elif key == "nz":
                h.nz = int(val)
            elif key in ("dx", "dz", "ox", "oz"):
                setattr(h, key, float(np.float32(val)))
            elif key == "layout":
                h.layout = val
    return h


def write_header_file(path: str, h: VelocityHeader) -> None:
    with open(path, "w") as f:
        f.write("# RTM velocity model header\n# data file: float32, little-endian, no header\n")
        for k in ("nx", "nz", "dx", "dz", "ox", "oz"):
            v = getattr(h, k)
            f.write(f"{k} = {v:g}\n" if isinstance(v, float) else f"{k} = {v}\n")
        f.write(f"layout = {h.layout}   # zfast: v[ix*nz+iz]  |  xfast: v[iz*nx+ix]\n")


def read_velocity_raw(path: str, h: VelocityHeader) -> np.ndarray:
    """Returns v as a zfast float32 array of nx*nz."""
    if h.nx <= 0 or h.nz <= 0:
        raise RTMError(L.EINVAL, "velocity nx/nz not set (use a .hdr file or --nx/--nz)")
    if not os.path.exists(path):
        raise RTMError(L.EINVAL, f"cannot open velocity file: {path}")
    n = h.nx * h.nz
    size = os.path.getsize(path)
    if size != n * 4:
        raise RTMError(L.EINVAL, f"velocity file size mismatch: {size} bytes, expected {n * 4} "
                                 f"(nx={h.nx}, nz={h.nz}, float32)")
    raw = np.fromfile(path, dtype="<f4")
    v = raw.reshape(h.nz, h.nx).T.copy().ravel() if h.layout == "xfast" else raw.copy()
    if not np.all((v > 0) & (v <= 20000)):
        raise RTMError(L.EINVAL, "velocity model contains a non-physical value")
    return v.astype(np.float32)


def write_velocity_raw(path: str, v: np.ndarray) -> None:
    np.ascontiguousarray(v, "<f4").tofile(path)


def write_shots_raw(path: str, shots: List[ShotRecord]) -> None:
    if not shots:
        raise RTMError(L.EINVAL, "no shots to write")
    nrec, nt, dt = shots[0].nrec, shots[0].nt, shots[0].dt
    for s in shots:
        if s.nrec != nrec or s.nt != nt:
            raise RTMError(L.EINVAL, "RAW format requires constant nrec and nt")
    with open(path, "wb") as f:
        f.write(RTMS_MAGIC + struct.pack("<4if2i", 1, len(shots), nrec, nt, dt, 0, 0))
        for s in shots:
            f.write(struct.pack("<2f", s.sx, s.sz))
            f.write(np.ascontiguousarray(s.rx, "<f4").tobytes())
            f.write(np.ascontiguousarray(s.rz, "<f4").tobytes())
            f.write(np.ascontiguousarray(s.traces, "<f4").ravel().tobytes())


def read_shots_raw(path: str) -> List[ShotRecord]:
    with open(path, "rb") as f:
        data = f.read()
    if data[:4] != RTMS_MAGIC:
        raise RTMError(L.EINVAL, f"{path}: not an RTMS file (bad magic)")
    if len(data) < 32:
        raise RTMError(L.EINVAL, f"RTMS file truncated: {path}")
    version, nshots, nrec, nt = struct.unpack_from("<4i", data, 4)
    (dt,) = struct.unpack_from("<f", data, 20)
    if version != 1:
        raise RTMError(L.EINVAL, "unsupported RTMS version")
    if nshots <= 0 or nrec <= 0 or nt <= 0 or not dt > 0:
        raise RTMError(L.EINVAL, "RTMS header contains invalid values")
    per = 8 + 8 * nrec + 4 * nrec * nt
    shots, off = [], 32
    for _ in range(nshots):
        if off + per > len(data):
            raise RTMError(L.EINVAL, f"RTMS file truncated: {path}")
        sx, sz = struct.unpack_from("<2f", data, off)
        rx = np.frombuffer(data, "<f4", nrec, off + 8).astype(np.float32)
        rz = np.frombuffer(data, "<f4", nrec, off + 8 + 4 * nrec).astype(np.float32)
        tr = np.frombuffer(data, "<f4", nrec * nt, off + 8 + 8 * nrec).astype(np.float32)
        shots.append(ShotRecord(sx, sz, rx, rz, nt=nt, dt=dt, traces=tr))
        off += per
    return shots


def _ibm_to_ieee(words: np.ndarray) -> np.ndarray:
    """IBM hex float (big-endian words already decoded) -> float32, computed in
    double and rounded like the reference (seismic_io.cpp:153-161)."""
    w = words.astype(np.uint64)
    sign = (w >> 31) & 1
    expo = ((w >> 24) & 0x7F).astype(np.int64) - 64
    frac = (w & 0x00FFFFFF).astype(np.float64) / 16777216.0
    x = frac * np.power(16.0, expo.astype(np.float64))
    x = np.where(sign == 1, -x, x)
    x = np.where(w == 0, 0.0, x)
    return x.astype(np.float32)


def _scalco(coord: int, scalco: int) -> float:
    if scalco > 0:
        return float(np.float32(coord) * np.float32(scalco))
    if scalco < 0:
        return float(np.float32(coord) / np.float32(-scalco))
    return float(np.float32(coord))


def read_shots_segy(path: str, src_depth: float, rec_depth: float) -> List[ShotRecord]:
    size = os.path.getsize(path)
    if size < 3600:
        raise RTMError(L.EINVAL, f"SEG-Y too short: {path}")
    with open(path, "rb") as f:
        data = f.read()
    bh = data[3200:3600]
    dt_us, = struct.unpack_from(">h", bh, 16)
    ns, = struct.unpack_from(">h", bh, 20)
    fmt, = struct.unpack_from(">h", bh, 24)
    if ns <= 0:
        raise RTMError(L.EINVAL, "SEG-Y: invalid samples per trace")
    if dt_us <= 0:
        raise RTMError(L.EINVAL, "SEG-Y: invalid sample interval")
    if fmt in (1, 2, 5):
        bps = 4
    elif fmt == 3:
        bps = 2
    else:
        raise RTMError(L.EINVAL, f"SEG-Y sample format {fmt} is not supported (use 1, 2, 3 or 5)")
    tb = 240 + ns * bps
    ntr = (size - 3600) // tb
    if ntr <= 0:
        raise RTMError(L.EINVAL, "SEG-Y contains no traces")
    dt = float(np.float32(dt_us) * np.float32(1e-6))
    shots: List[ShotRecord] = []
    cur = None
    rxs, tr_list = [], []

    def close():
        if cur is not None:
            s = cur
            s.rx = np.array(rxs, np.float32)
            s.rz = np.full(len(rxs), rec_depth, np.float32)
            s.traces = np.concatenate(tr_list).astype(np.float32)
            shots.append(s)

    cur_fldr, cur_sx = 0, 0.0
    for i in range(ntr):
        off = 3600 + i * tb
        th = data[off:off + 240]
        fldr, = struct.unpack_from(">i", th, 8)
        scalco, = struct.unpack_from(">h", th, 70)
        sx = _scalco(struct.unpack_from(">i", th, 72)[0], scalco)
        gx = _scalco(struct.unpack_from(">i", th, 80)[0], scalco)
        new = cur is None or fldr != cur_fldr or (fldr == 0 and sx != cur_sx)
        if new:
            close()
            cur = ShotRecord(sx, src_depth, np.zeros(0, np.float32), np.zeros(0, np.float32), nt=ns, dt=dt)
            rxs, tr_list = [], []
            cur_fldr, cur_sx = fldr, sx
        rxs.append(gx)
        body = data[off + 240:off + tb]
        if fmt == 1:
            tr = _ibm_to_ieee(np.frombuffer(body, ">u4"))
        elif fmt == 5:
            tr = np.frombuffer(body, ">f4").astype(np.float32)
        elif fmt == 2:
            tr = np.frombuffer(body, ">i4").astype(np.float32)
        else:
            tr = np.frombuffer(body, ">i2").astype(np.float32)
        tr_list.append(tr)
    close()
    if not shots:
        raise RTMError(L.EINVAL, "SEG-Y: no shots decoded")
    return shots


def read_shots(path: str, src_depth: float = 10.0, rec_depth: float = 10.0) -> List[ShotRecord]:
    ext = os.path.splitext(path)[1].lower()
    if ext in (".sgy", ".segy"):
        return read_shots_segy(path, src_depth, rec_depth)
    return read_shots_raw(path)


def write_raw_floats(path: str, v: np.ndarray) -> None:
    np.ascontiguousarray(v, "<f4").tofile(path)


def read_raw_floats(path: str) -> np.ndarray:
    size = os.path.getsize(path)
    if size % 4:
        raise RTMError(L.EINVAL, f"file is not a float32 array: {path}")
    return np.fromfile(path, "<f4").astype(np.float32)
