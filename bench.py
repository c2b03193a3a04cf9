#!/usr/bin/env python
"""Throughput of the OpenLPT IPR hot path (detection -> stereo matching -> shake ->
residual, looped) on B200, against the reference CPU implementation.

Metric: particles/s (IPR+shake) = 3D particles reconstructed per second of
IPR::runIPR on one synthetic frame.  One step = one full IPR run (all outer loops,
all shake iterations) over the frame's camera images.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica of the workload on
its own GPU ("replicas only": the frame loop has no cross-GPU exchange); value is
the particles of all ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from pyopenlpt_b200 import synth  # noqa: E402

METRIC = "particles/s (IPR+shake)"

WORKLOADS = {
    # The single-frame IPR scene: 4 pinhole cameras (f = 5000 px, 45 deg ring, 30 deg
    # tilt), 1024^2 uint8, 10,000 particles in 40x40x20 mm, a=200, b=c=0.5, sigma=2;
    # 4 IPR loops x 4 shake iterations, shake width 0.25 mm, threshold 30, tol_2d 1 px.
    "ipr_1024_u8_10k": dict(scene=dict(n_particles=10000, n_cam=4, size=1024, focal=5000.0,
                                       a=200.0, b=0.5, c=0.5, noise=2.0, bits=8),
                            settings=dict()),
}
DEFAULT_WORKLOAD = "ipr_1024_u8_10k"


def build_scene(name: str, seed: int):
    w = WORKLOADS[name]
    sc = synth.make_scene(seed=seed, **w["scene"])
    s = synth.IPRSettings(**w["settings"])
    s.match_cam_count = min(s.match_cam_count, sc.n_cam)
    return sc, s


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = []
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        max_mhz = None
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                max_mhz = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max_mhz,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ----------------------------------------------------------------------------- reference arm
class _MuteStdout:
    """Silence C/C++ writes to fd 1 (the reference logs progress on std::cout)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)
        return False


def reference_ipr_time(sc, s, threads: int):
    """Wall time of the reference IPR::runIPR on this host (compiled from source)."""
    from oracle.ref import RefOracle
    ref = RefOracle(sc, s, threads=threads)
    imgs = [im.astype(np.float64) for im in sc.images]
    with _MuteStdout():
        t = time.perf_counter()
        out = ref.ipr(imgs)
        dt = time.perf_counter() - t
    ref.close()
    return len(out["xyz"]), dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sc, s = build_scene(args.workload, 1234)
    threads = os.cpu_count() or 1
    times, counts = [], []
    for i in range(args.warmup + args.steps):
        n, dt = reference_ipr_time(sc, s, threads)
        if i >= args.warmup:
            times.append(dt)
            counts.append(n)
    value = sum(counts) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particles/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload, sc, s),
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": threads,
                         "kind": "reference",
                         "sample": "whole frame per step (IPR::runIPR, OpenMP, all host threads)"},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(name, sc, s):
    H, W = sc.images[0].shape
    return {"workload": name, "particles": int(len(sc.xyz)), "cameras": sc.n_cam,
            "image": f"{H}x{W} {sc.images[0].dtype}", "ipr_loops": s.n_loop_ipr,
            "shake_loops": s.n_shake_loop, "shake_width_mm": s.shake_width,
            "tol_2d_px": s.tol_2d_px, "tol_3d_mm": s.tol_3d_mm, "parallelism": "replicas",
            "l2": "flushed (256 MiB write) between timed steps"}


# ----------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import torch.distributed as dist
    from pyopenlpt_b200 import _ffi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    sc, s = build_scene(args.workload, 1234 + rank)
    prec = 1 if args.precision == "fp64" else 0
    ctx = _ffi.Context(local)
    ctx.upload_cameras([_ffi.camera_desc_from_pinhole(c) for c in sc.cams])
    from pyopenlpt_b200.synth import otf_table_array
    ctx.upload_otf(2, 2, 2, sc.volume, otf_table_array(sc.n_cam, sc.otf_abc))
    params = _ffi.ipr_params(s, sc.volume, prec)
    H, W = sc.images[0].shape
    dtype = _ffi._DTYPES[sc.images[0].dtype]
    dev_imgs = [torch.from_numpy(im).cuda() for im in sc.images]
    host_imgs = [torch.from_numpy(im).pin_memory() for im in sc.images]
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    def step_device():
        ctx.upload_images_device([t.data_ptr() for t in dev_imgs], dtype, [H] * sc.n_cam,
                                 [W] * sc.n_cam)
        return ctx.ipr_run(params)

    def step_e2e():
        ctx.upload_images([t.numpy() for t in host_imgs])
        n = ctx.ipr_run(params)
        xyz, uv = ctx.ipr_result(n)
        return n, xyz, uv

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()

    # ---- device-resident timed region
    clocks = ClockSampler(local)
    clocks.start()
    ctx.profile(True)
    barrier()
    torch.cuda.synchronize()
    launches0 = _ffi.launch_count()
    t_wall = time.perf_counter()
    dev_ms = 0.0
    parts = 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        n = step_device()
        e1.record(stream)
        e1.synchronize()
        dev_ms += e0.elapsed_time(e1)
        parts += n
    torch.cuda.synchronize()
    barrier()
    wall = time.perf_counter() - t_wall
    launches = _ffi.launch_count() - launches0
    prof = {k: ctx.profile_read(k) for k in range(4)}
    ctx.profile(False)
    clk = clocks.stop()

    # ---- end-to-end through the C ABI with host buffers
    barrier()
    torch.cuda.synchronize()
    e2e_t = 0.0
    e2e_parts = 0
    bo = 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n, xyz, uv = step_e2e()
        e2e_t += time.perf_counter() - t0
        e2e_parts += n
        bo += xyz.nbytes + uv.nbytes
    barrier()
    bi = sum(im.nbytes for im in sc.images)

    # ---- max over ranks
    vals = torch.tensor([dev_ms, float(parts), e2e_t, float(e2e_parts)], dtype=torch.float64,
                        device="cuda")
    if world > 1:
        tmax = vals.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        tsum = vals.clone()
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        dev_ms_max, e2e_max = tmax[0].item(), tmax[2].item()
        parts_all, e2e_parts_all = tsum[1].item(), tsum[3].item()
    else:
        dev_ms_max, e2e_max = dev_ms, e2e_t
        parts_all, e2e_parts_all = float(parts), float(e2e_parts)

    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        names = {0: "peak detection", 1: "stereo level expansion", 2: "residual image",
                 3: "shake (warp per particle)"}
        # dominant HBM-bound kernel: the one with the largest share of device time
        cand = {k: prof[k] for k in (0, 2, 3) if prof[k][1] > 0}
        dom = max(cand, key=lambda k: cand[k][0]) if cand else 2
        ms, nl, by = prof[dom]
        achieved = (by / nl) / ((ms / nl) * 1e-3) / 1e9 if nl and ms > 0 else 0.0
        kernel_ms = {names[k]: round(prof[k][0] / args.steps, 4) for k in range(4)}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            ncpu, tcpu = reference_ipr_time(sc, s, threads)
            cpu = {"value": ncpu / tcpu, "unit": "particles/s", "cores": threads,
                   "kind": "reference",
                   "sample": "one whole frame of the same workload (IPR::runIPR compiled "
                             "from the reference sources, OpenMP)"}
        line = {
            "metric": METRIC, "value": parts_all / (dev_ms_max * 1e-3), "unit": "particles/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == 0 else "f64", "data": "synthetic",
            "config": dict(workload_config(args.workload, sc, s),
                           precision="fp32 residual/shake, fp64 geometry" if prec == 0 else "fp64"),
            "frames_per_s": world * args.steps / (dev_ms_max * 1e-3),
            "wall_s": wall,
            "e2e": {"value": e2e_parts_all / e2e_max, "unit": "particles/s",
                    "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo // max(1, args.steps)},
            "gpu_launches": int(launches),
            "kernel_ms_per_step": kernel_ms,
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "traffic": None},
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
