#!/usr/bin/env python
"""Benchmark of the B200 RTM engine (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (default): 1150 x 400 cells at 10 m, layered-and-faulted velocity
1500-5500 m/s (10 dipping interfaces, 3 normal faults, seed 2), 64 shots with a
split-spread line of receivers on every column, nt 4000, dt 0.8 ms, Ricker 15
Hz, order 8, nb 60, store interval 2.  Traces are modelled on the GPU with the
same scheme before timing (synthetic data; the reference's own synthetic data is
made the same way).  One step = one full migration of the shot set.

value      shots/s with the shot gathers already resident in HBM (device time,
           CUDA events on the engine's stream, max over ranks);
e2e        shots/s through the C ABI with page-locked HOST traces and host
           outputs, the host->device copies inside the timed region;
roofline   algorithmic bytes of the step kernel (16 B per cell update, snapshot
           stores and reloads, image/illumination read+write, traces) per
           second of device time, against the measured HBM copy bandwidth;
cpu_baseline  the reference's own CPU engine (oracle/_ref/rtm, engine cpu-opt,
           all host cores) on one shot with a truncated time axis, extrapolated
           per cell update.

--impl reference runs only that reference CPU engine (rank 0), one bounded
sample per step.  Multi-GPU (torchrun): shots are sharded across ranks (each
rank migrates a fixed 64-shot share: weak scaling) and the FP64 image stacks are
summed with one NCCL all-reduce at the end of each step.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rtm-acceleration_b200"))

import numpy as np  # noqa: E402

SHOTS_PER_GPU = 64
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
TRAFFIC_PATH = os.path.join(ROOT, "profiles", "roofline_traffic.json")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--shots", type=int, default=SHOTS_PER_GPU, help="shots per GPU")
    ap.add_argument("--nt", type=int, default=0, help="override nt (0 = 4000)")
    ap.add_argument("--mode", default="batch", choices=["batch", "plain"])
    ap.add_argument("--max-in-flight", type=int, default=0, help="0 = the engine's default (16)")
    ap.add_argument("--tile-cols", type=int, default=0, help="0 = autotuned")
    ap.add_argument("--snap", default="f32", choices=["f32", "bf16", "f16"])
    ap.add_argument("--arith", default="auto", choices=["auto", "ieee", "fma"])
    ap.add_argument("--no-fp64-check", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="config2", choices=["config1", "config2", "config3", "config4", "config5"],
                    help="config2 is the contract line; the others print one extra JSON line each")
    ap.add_argument("--plain-shots", type=int, default=64, help="config3: shots timed on the plain engine")
    ap.add_argument("--requests", type=int, default=24, help="config5: requests in the stream")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                      "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                     stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        rows = [r.split(", ") for r in self.lines if r and r[0].isdigit()]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        load = [r for r in rows if r[4].strip().isdigit() and int(r[4]) >= 50] or rows
        sm = [float(r[1]) for r in load]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load for i in range(4) if r[6 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(load[0][2]), "reasons": reasons,
                "samples": len(load)}


# ---------------------------------------------------------------- workload
def make_workload(nshots_total, nt_override):
    from rtm_b200 import synth
    w = synth.config2(nshots=nshots_total)
    if nt_override:
        w.nt = nt_override
        for s in w.shots:
            s.nt = nt_override
    return w


def model_traces(w, device):
    from rtm_b200 import Engine, RTMParams
    p = RTMParams(nb=w.nb, order=w.order, f0=w.f0, store_interval=1)
    with Engine("batch", p, device=device, max_shots_in_flight=16) as e:
        e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
        tr = e.model_shots(w.shots)
    for s, t in zip(w.shots, tr):
        s.traces = t


def algorithmic_bytes_per_shot(w, snap_bytes):
    """16 B per cell update + snapshot store/reload + image/illum RMW + traces."""
    nsnap = (w.nt - 1) // w.store_interval + 1
    nint = w.nx * w.nz
    upd = 2.0 * w.nt * (w.nx + 2 * w.nb) * (w.nz + 2 * w.nb)
    return 16.0 * upd + nsnap * nint * snap_bytes + nsnap * nint * (snap_bytes + 16.0) + w.nx * w.nt * 4.0


def read_peak():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def read_traffic():
    try:
        with open(TRAFFIC_PATH) as f:
            return json.load(f)
    except Exception:
        return None


# ------------------------------------------------------------ reference CPU
def reference_sample(w, workdir, nt_sample, threads):
    """Time the reference's cpu-opt engine on one config shot with a truncated
    time axis; returns (cell_updates_per_s, seconds, description)."""
    ref = os.path.join(ROOT, "oracle", "_ref", "rtm")
    if not os.path.exists(ref):
        return None
    from rtm_b200 import io as rio
    vel = os.path.join(workdir, "velocity.bin")
    rio.write_velocity_raw(vel, w.vel)
    rio.write_header_file(vel + ".hdr", rio.VelocityHeader(w.nx, w.nz, w.dx, w.dz, 0.0, 0.0, "zfast"))
    s0 = w.shots[len(w.shots) // 2]
    rng = np.random.default_rng(7)
    from rtm_b200.engine import ShotRecord
    sh = ShotRecord(s0.sx, s0.sz, s0.rx, s0.rz, nt=nt_sample, dt=w.dt,
                    traces=(rng.standard_normal(s0.nrec * nt_sample) * 1e-3).astype(np.float32))
    shots_path = os.path.join(workdir, "shots.bin")
    rio.write_shots_raw(shots_path, [sh])
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    cmd = [ref, "--engine", "cpu-opt", "--velocity", vel, "--shots", shots_path, "--output",
           os.path.join(workdir, "img.bin"), "--order", str(w.order), "--nb", str(w.nb), "--f0", str(w.f0),
           "--store-interval", str(w.store_interval), "--quiet"]
    t0 = time.perf_counter()
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, env=env)
    dt = time.perf_counter() - t0
    upd = 2.0 * nt_sample * (w.nx + 2 * w.nb) * (w.nz + 2 * w.nb)
    desc = (f"reference cpu-opt, 1 shot of the workload with nt truncated to {nt_sample} "
            f"({upd / 1e9:.2f} G cell updates), {threads} threads, wall time of the rtm process")
    return upd / dt, dt, desc


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    w = make_workload(SHOTS_PER_GPU, args.nt)
    upd_shot = 2.0 * w.nt * (w.nx + 2 * w.nb) * (w.nz + 2 * w.nb)
    nt_sample = 300
    ref = os.path.join(ROOT, "oracle", "_ref", "rtm")
    if not os.path.exists(ref):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU engine not built (oracle/_ref/rtm)"}))
        return
    rates = []
    desc = ""
    with tempfile.TemporaryDirectory() as td:
        for i in range(args.warmup + args.steps):
            r = reference_sample(w, td, nt_sample, threads)
            if i >= args.warmup:
                rates.append(r[0])
                desc = r[2]
    rate = statistics.median(rates)
    value = rate / upd_shot
    line = {"impl": "reference", "metric": "shots/s", "value": value, "unit": "shots/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * SHOTS_PER_GPU / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "gcell_updates_per_s": rate / 1e9,
            "config": {"workload": "config2: 1150x400 @10 m, 64 shots, nt 4000, order 8, store 2",
                       "inputs": "random traces, one shot per sample (timing only)"},
            "cpu_baseline": {"value": value, "unit": "shots/s", "cores": threads, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": value, "unit": "shots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ----------------------------------------------------------------- B200 arm
def run_b200_arm(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    from rtm_b200 import Engine, RTMParams, metrics
    from rtm_b200.engine import ShotRecord

    # The survey has SHOTS_PER_GPU * world shots; each rank takes a cost-balanced
    # share (rtm_b200.shard: every rank computes the same assignment).
    from rtm_b200 import shard
    w_all = make_workload(args.shots * world, args.nt)
    all_shots = w_all.shots
    w = w_all
    w.shots = shard.rank_shots(all_shots, rank, world, w.nx, w.nz, w.nb, w.nt)
    model_traces(w, local)
    nsh = len(w.shots)
    n_img = w.nx * w.nz

    p = RTMParams(nb=w.nb, order=w.order, f0=w.f0, store_interval=w.store_interval)
    eng = Engine(args.mode, p, device=local, snap=args.snap, arithmetic=args.arith,
                 max_shots_in_flight=args.max_in_flight, tile_cols=args.tile_cols)
    eng.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)

    # device-resident inputs and outputs for `value`
    dev_tr = [torch.from_numpy(s.traces).to(f"cuda:{local}") for s in w.shots]
    dev_shots = [ShotRecord(s.sx, s.sz, s.rx, s.rz, nt=s.nt, dt=s.dt, traces_ptr=t.data_ptr())
                 for s, t in zip(w.shots, dev_tr)]
    img = torch.zeros(n_img, dtype=torch.float32, device=f"cuda:{local}")
    ill = torch.zeros_like(img)
    stack = torch.zeros(2 * n_img, dtype=torch.float64, device=f"cuda:{local}")

    def one_step(shots, img_ptr, ill_ptr):
        eng.migrate_into(shots, img_ptr, ill_ptr)
        if dist is not None:   # the one exchange of the path: sum the ranks' stacks
            stack[:n_img].copy_(img)
            stack[n_img:].copy_(ill)
            shard.allreduce_stack(stack[:n_img], stack[n_img:])

    for _ in range(args.warmup):
        one_step(dev_shots, img.data_ptr(), ill.data_ptr())
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    eng.reset_times()
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        one_step(dev_shots, img.data_ptr(), ill.data_ptr())
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    tm = eng.times()
    dev_time = tm["kernel"]
    if dist is not None:
        t = torch.tensor([dev_time, wall], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_time, wall = float(t[0]), float(t[1])
        dist.barrier()
    if sampler:
        sampler.stop()
    total_shots = nsh * world * args.steps
    value = total_shots / dev_time
    gcell = w.cell_updates() * world * args.steps / dev_time / 1e9
    launches = tm["kernel_launches"]

    # e2e through the C ABI with page-locked host traces and host outputs
    pin_tr = [torch.from_numpy(s.traces).pin_memory() for s in w.shots]
    host_shots = [ShotRecord(s.sx, s.sz, s.rx, s.rz, nt=s.nt, dt=s.dt, traces_ptr=t.data_ptr())
                  for s, t in zip(w.shots, pin_tr)]
    himg = torch.zeros(n_img, dtype=torch.float32).pin_memory()
    hill = torch.zeros_like(himg).pin_memory()
    one_step(host_shots, himg.data_ptr(), hill.data_ptr())   # warm
    eng.reset_times()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        one_step(host_shots, himg.data_ptr(), hill.data_ptr())
    e1.record()
    torch.cuda.synchronize()
    e2e_time = e0.elapsed_time(e1) * 1e-3
    te = eng.times()
    if dist is not None:
        t = torch.tensor([e2e_time], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_time = float(t[0])
    e2e = total_shots / e2e_time
    h2d = te["h2d_bytes"] / args.steps
    d2h = te["d2h_bytes"] / args.steps

    # accuracy of the timed image against an FP64 run of the same scheme
    rel64 = None
    if not args.no_fp64_check:
        img_h = himg.numpy().copy()
        with Engine("batch", p, device=local, arithmetic="fp64") as e64:
            e64.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
            ref64, _ = e64.migrate_f64(w.shots)
        rel64 = metrics.compare_images(ref64, img_h)["l2_relative"]

    l2_gbs = eng.memory_probe(48 << 20, 50)
    tune = [r["pick"] for r in eng.autotune_report()]
    eng.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return

    snap_b = {"f32": 4, "bf16": 2, "f16": 2}[args.snap]
    algo_bytes = algorithmic_bytes_per_shot(w, snap_b) * nsh * args.steps
    step_launches = max(1, launches)
    achieved = algo_bytes / dev_time / 1e9          # this GPU's step-kernel bytes per device second
    peak, peak_kind = read_peak()
    traffic = read_traffic()
    cpu = None
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        with tempfile.TemporaryDirectory() as td:
            r = reference_sample(w_all if world == 1 else w, td, 300, threads)
        if r:
            upd_shot = 2.0 * w.nt * (w.nx + 2 * w.nb) * (w.nz + 2 * w.nb)
            cpu = {"value": r[0] / upd_shot, "unit": "shots/s", "cores": threads, "kind": "reference",
                   "sample": r[2]}
    clocks = sampler.summary() if sampler else None
    line = {
        "metric": "shots/s", "value": value, "unit": "shots/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_time / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.arith == "fma" and "f32-fma" or "f32",
        "data": "synthetic (seeded model, GPU-modelled traces)",
        "config": {"workload": f"config2: {w.nx}x{w.nz} @{w.dx:g} m, {nsh} shots/GPU, nt {w.nt}, "
                               f"order {w.order}, store {w.store_interval}",
                   "engine": args.mode, "max_shots_in_flight": args.max_in_flight, "tile_cols": args.tile_cols,
                   "snapshots": args.snap, "arithmetic": args.arith, "accumulation": "compensated FP32 + FP64 stack",
                   "l2": "inputs and snapshots larger than L2 (126 MB)", "autotuned_step_kernel": tune},
        "gcell_updates_per_s": gcell,
        "rel_l2_vs_fp64": rel64,
        "gpu_launches": launches,
        "wall_s_timed": wall,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic.get("bytes_per_launch") if traffic else None,
                     "peak_source": peak_kind, "l2_copy_probe_gbs": l2_gbs,
                     "algorithmic_bytes_per_step_launch": algo_bytes / step_launches},
        "e2e": {"value": e2e, "unit": "shots/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    print(json.dumps(line))


# ------------------------------------------------------ other workloads
def _timed_migrate(eng, shots, f64=False):
    """One migration timed with the engine's CUDA events (device seconds)."""
    eng.reset_times()
    out = eng.migrate_f64(shots) if f64 else eng.migrate(shots)
    return out, eng.times()


def _model(w, device, shots=None):
    from rtm_b200 import Engine, RTMParams
    shots = shots if shots is not None else w.shots
    p = RTMParams(nb=w.nb, order=w.order, f0=w.f0, store_interval=1)
    with Engine("batch", p, device=device, max_shots_in_flight=16) as e:
        e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
        tr = e.model_shots(shots)
    for s, t in zip(shots, tr):
        s.traces = t


def run_config1(args):
    """The reference's CPU-runnable case (201 x 151, 3 flat layers, 4 shots,
    nt 1400, order 8, store 2, direct-wave mute 1500 m/s): the plain engine
    (bit-identical to the reference) and the batched engine against the
    reference's own cpu and cpu-opt engines on this host, same files."""
    import torch
    from rtm_b200 import Engine, RTMParams, metrics, mute_direct_wave, synth
    from rtm_b200 import io as rio
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    w = synth.config1(dipping=False)
    _model(w, dev)
    t_pad = float(np.float32(1.0) / np.float32(w.f0))
    for sh in w.shots:
        mute_direct_wave(sh, w.mute_v, t_pad, t_pad)
    p = RTMParams(nb=w.nb, order=w.order, f0=w.f0, store_interval=w.store_interval)
    res, imgs = {}, {}
    for name, mode in (("plain", "plain"), ("batch", "batch")):
        with Engine(mode, p, device=dev) as e:
            e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
            _timed_migrate(e, w.shots)
            (img, _), t = _timed_migrate(e, w.shots)
            res[name] = {"shots_per_s": len(w.shots) / t["kernel"], "gcell_updates_per_s":
                         t["cell_updates"] / t["kernel"] / 1e9, "seconds": t["kernel"]}
            imgs[name] = img
    cpu = {}
    ref = os.path.join(ROOT, "oracle", "_ref", "rtm")
    if os.path.exists(ref):
        with tempfile.TemporaryDirectory() as td:
            vel = os.path.join(td, "v.bin")
            rio.write_velocity_raw(vel, w.vel)
            rio.write_header_file(vel + ".hdr", rio.VelocityHeader(w.nx, w.nz, w.dx, w.dz, 0.0, 0.0, "zfast"))
            shp = os.path.join(td, "s.bin")
            # the unmuted traces: the reference applies the mute itself
            raw = synth.config1(dipping=False)
            _model(raw, dev)
            rio.write_shots_raw(shp, raw.shots)
            for eng, threads in (("cpu", 1), ("cpu-opt", os.cpu_count() or 1)):
                out = os.path.join(td, f"{eng}.bin")
                t0 = time.perf_counter()
                subprocess.run([ref, "--engine", eng, "--velocity", vel, "--shots", shp, "--output", out,
                                "--order", "8", "--nb", "60", "--f0", "12", "--store-interval", "2",
                                "--mute-direct", "1500", "--quiet"], check=True, stdout=subprocess.DEVNULL,
                               env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
                sec = time.perf_counter() - t0
                ref_img = rio.read_raw_floats(out)
                cpu[eng] = {"shots_per_s": len(w.shots) / sec, "seconds_wall": sec, "threads": threads,
                            "plain_bit_identical": bool(np.array_equal(ref_img.view(np.uint32),
                                                                       imgs["plain"].view(np.uint32))),
                            "batch_rel_l2": metrics.compare_images(ref_img, imgs["batch"])["l2_relative"]}
    print(json.dumps({"workload": "config1", "metric": "shots/s", "unit": "shots/s", "higher_is_better": True,
                      "value": res["plain"]["shots_per_s"], "b200": res, "reference_cpu": cpu,
                      "data": "synthetic (the reference's generator recipe, GPU-modelled traces)",
                      "config": {"grid": "201x151 @10 m", "shots": 4, "nt": 1400, "order": 8, "store": 2,
                                 "mute": 1500}}))


def run_config3(args):
    """256 shots on uneven aperture windows (400-1150 columns of the
    1150 x 400 model), orders 8 and 12: the batched engine (FP32 and BF16
    snapshots, autotuned) against the plain one-shot-at-a-time engine."""
    import torch
    from rtm_b200 import Engine, RTMParams, metrics, synth
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    nshots = args.shots if args.shots != SHOTS_PER_GPU else 256
    for order in (8, 12):
        w = synth.config3(nshots=nshots, order=order)
        _model(w, dev)
        p = RTMParams(nb=w.nb, order=order, f0=w.f0, store_interval=w.store_interval)
        res, times, images = {}, {}, {}
        for name, mode, snap in (("batch_f32", "batch", "f32"), ("batch_bf16", "batch", "bf16")):
            with Engine(mode, p, device=dev, snap=snap) as e:
                e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
                _timed_migrate(e, w.shots[:16])                 # warm-up: autotune, graphs
                (img, _), t = _timed_migrate(e, w.shots)
                res[name] = len(w.shots) / t["kernel"]
                times[name] = t
                images[name] = img
                tune = e.autotune_report()
        sub = w.shots[:args.plain_shots]
        with Engine("plain", p, device=dev) as e:
            e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
            _timed_migrate(e, sub[:2])
            _, t = _timed_migrate(e, sub)
            res["plain_f32"] = len(sub) / t["kernel"]
            times["plain_f32"] = t
        # accuracy on a 16-shot subset against an FP64 run of the same scheme
        acc = {}
        chk = w.shots[:16]
        with Engine("batch", p, device=dev, arithmetic="fp64") as e:
            e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
            ref64, _ = e.migrate_f64(chk)
        for name, mode, snap in (("batch_f32", "batch", "f32"), ("batch_bf16", "batch", "bf16"),
                                 ("plain_f32", "plain", "f32")):
            with Engine(mode, p, device=dev, snap=snap) as e:
                e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
                img, _ = e.migrate(chk)
            acc[name] = metrics.compare_images(ref64, img)["l2_relative"]
        print(json.dumps({
            "workload": f"config3-order{order}", "metric": "shots/s", "unit": "shots/s", "higher_is_better": True,
            "value": res["batch_bf16"], "batch_f32": res["batch_f32"], "batch_bf16": res["batch_bf16"],
            "plain_f32": res["plain_f32"], "speedup_batch_bf16_vs_plain_f32": res["batch_bf16"] / res["plain_f32"],
            "speedup_batch_f32_vs_plain_f32": res["batch_f32"] / res["plain_f32"],
            "gcell_updates_per_s": {k: v["cell_updates"] / v["kernel"] / 1e9 for k, v in times.items()},
            "rel_l2_vs_fp64": acc, "autotune": tune, "data": "synthetic (seeded model, GPU-modelled traces)",
            "config": {"shots": len(w.shots), "plain_shots_timed": len(sub), "windows": "400-1150 columns, seed 3",
                       "grid": f"{w.nx}x{w.nz} @{w.dx:g} m", "nt": w.nt, "order": order, "store": w.store_interval,
                       "accuracy_subset": f"first {len(chk)} shots, FP64 GPU run of the same scheme"}}))
        sys.stdout.flush()


def run_config4(args):
    """4000 x 1500 cells at 5 m, order 12, 16 shots, nt 8000: BF16 and FP16
    snapshots with a power-of-two scale per column segment, Kahan FP32 per
    shot, FP64 stack."""
    import torch
    from rtm_b200 import Engine, RTMParams, metrics, synth
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    nshots = args.shots if args.shots != SHOTS_PER_GPU else 16
    w = synth.config4(nshots=nshots)
    _model(w, dev)
    p = RTMParams(nb=w.nb, order=w.order, f0=w.f0, store_interval=w.store_interval)
    res, gc, mem = {}, {}, {}
    for snap in ("bf16", "f16"):
        with Engine("batch", p, device=dev, snap=snap) as e:
            e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
            mem[snap] = e.snapshot_bytes
            (_, _), t = _timed_migrate(e, w.shots)
            res[snap] = len(w.shots) / t["kernel"]
            gc[snap] = t["cell_updates"] / t["kernel"] / 1e9
    # error against FP64: FP64 snapshots of the full time axis would need
    # 195 GB per shot, so the comparison runs 2 shots on the first 2000 steps
    nt_chk = 2000
    chk = w.shots[:2]
    acc = {}
    with Engine("batch", p, device=dev, arithmetic="fp64") as e:
        e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=nt_chk, dt=w.dt)
        ref64, _ = e.migrate_f64(chk)
    for snap in ("f32", "bf16", "f16"):
        with Engine("batch", p, device=dev, snap=snap) as e:
            e.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=nt_chk, dt=w.dt)
            img, _ = e.migrate(chk)
        acc[snap] = metrics.compare_images(ref64, img)["l2_relative"]
    print(json.dumps({
        "workload": "config4", "metric": "shots/s", "unit": "shots/s", "higher_is_better": True,
        "value": res["bf16"], "bf16": res["bf16"], "f16": res["f16"], "gcell_updates_per_s": gc,
        "snapshot_bytes_per_shot": mem, "rel_l2_vs_fp64": acc,
        "accuracy_run": f"{len(chk)} shots, nt truncated to {nt_chk} (FP64 snapshots of the full axis: 195 GB/shot)",
        "data": "synthetic (seeded model, GPU-modelled traces)",
        "config": {"grid": f"{w.nx}x{w.nz} @{w.dx:g} m", "shots": len(w.shots), "nt": w.nt, "order": w.order,
                   "store": w.store_interval}}))


def run_config5(args):
    """Serving stream: Poisson arrivals of migration requests with their own
    grids (201-2000 x 151-800), orders (8/12), time axes (1400-6000) and
    1-32 shots, admitted by snapshot memory, continuously batched."""
    import torch
    from rtm_b200 import Engine, RTMParams, metrics, synth
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    reqs = synth.config5_stream(nreq=args.requests, rate_hz=1.0, seed=5)
    for r in reqs:
        _model(r.work, dev)
    work = sum(r.work.cell_updates() for r in reqs)
    # arrival rate chosen so that the stream keeps the GPU about 90% busy at the
    # throughput of the batched engine (~150 G cell updates/s)
    busy = work / 150e9
    gaps = np.diff([0.0] + [r.arrival for r in reqs])
    scale = (0.9 * busy) / max(sum(gaps), 1e-9)
    arrivals = np.cumsum(gaps * scale)
    with Engine("serve", RTMParams(nb=60), device=dev, serve_max_nx=2000, serve_max_nz=800,
                max_shots_in_flight=16) as e:
        t0 = e.clock()
        tickets, nxt, done = {}, 0, {}
        while len(done) < len(reqs):
            now = e.clock() - t0
            while nxt < len(reqs) and arrivals[nxt] <= now:
                w = reqs[nxt].work
                tk = e.submit(w.vel, w.nx, w.nz, w.dx, w.dz, order=w.order, f0=w.f0, nt=w.nt, dt=w.dt,
                              store_interval=w.store_interval, shots=w.shots, arrival_time=t0 + arrivals[nxt])
                tickets[tk] = nxt
                nxt += 1
            e.serve_step(64)
            for tk, i in tickets.items():
                if i in done:
                    continue
                st, _, _ = e.poll(tk)
                if st["state"] == 2:
                    w = reqs[i].work
                    _, img, _ = e.poll(tk, w.nx, w.nz)
                    done[i] = (st, img)
            if nxt < len(reqs) and not any(i not in done for i in tickets.values()):
                time.sleep(max(0.0, min(0.05, arrivals[nxt] - (e.clock() - t0))))
        lat = sorted(done[i][0]["finish_time"] - (t0 + arrivals[i]) for i in done)
        span = max(done[i][0]["finish_time"] for i in done) - (t0 + arrivals[0])
        shots = sum(len(r.work.shots) for r in reqs)
    # accuracy of the three smallest requests against FP64 runs of the same scheme
    acc = []
    for i in sorted(range(len(reqs)), key=lambda k: reqs[k].work.cell_updates())[:3]:
        w = reqs[i].work
        with Engine("batch", RTMParams(nb=60, order=w.order, f0=w.f0, store_interval=w.store_interval), device=dev,
                    arithmetic="fp64") as e64:
            e64.setup(w.vel, w.nx, w.nz, w.dx, w.dz, nt=w.nt, dt=w.dt)
            ref64, _ = e64.migrate_f64(w.shots)
        acc.append(metrics.compare_images(ref64, done[i][1])["l2_relative"])
    q = lambda f: lat[min(len(lat) - 1, int(f * len(lat)))]
    print(json.dumps({
        "workload": "config5", "metric": "shots/s", "unit": "shots/s", "higher_is_better": True,
        "value": shots / span, "latency_s": {"p50": q(0.5), "p99": q(0.99), "max": lat[-1], "min": lat[0]},
        "gcell_updates_per_s": work / span / 1e9, "requests": len(reqs), "shots": shots,
        "offered_load": "arrivals scaled to keep the GPU ~90% busy at 150 G cell updates/s",
        "rel_l2_vs_fp64_smallest3": acc, "data": "synthetic (seeded models, GPU-modelled traces)",
        "config": {"grids": "201-2000 x 151-800 @10 m", "orders": [8, 12], "nt": "1400-6000",
                   "shots_per_request": "1-32", "seed": 5}}))


def main():
    args = parse_args()
    if args.impl != "reference" and args.workload != "config2":
        {"config1": run_config1, "config3": run_config3, "config4": run_config4,
         "config5": run_config5}[args.workload](args)
        return
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_b200_arm(args)


if __name__ == "__main__":
    main()
