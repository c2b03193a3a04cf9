#!/usr/bin/env python
"""Throughput of the OpenLPT hot path on B200 against the reference CPU implementation.

Metric: particles/s (IPR+shake).

* stb_2048_u16_6cam_poly_419k (default): the high-density Shake-the-Box sequence --
  6 cubic polynomial cameras (seeded, up to 2 px of distortion at the corners) on a
  45 deg ring of radius 500 mm tilted 30 deg, 2048^2 12-bit images (uint16), 0.1 ppp
  = 419,430 particles in 80x80x40 mm advected by ABC flow (A = B = C = 1, wavelength
  40 mm, at most 4 px/frame), a seeded 5x5x5 OTF grid (a in [2400, 3600], b and c in
  [0.3, 0.9]), noise sigma 20.  After the 4-frame initial phase, one step = one
  convergence-phase STB::processFrame.  The line compares the plain GPU form with the
  learned form on the same frames, at their recall and ghost rate against the
  generator's ground truth, and reports the FP32 path's position error against the
  FP64 mode.  The reference's CPU path cannot finish this workload in a bench run
  (its initial phase alone is hours of CPU time); its arm times the same generator
  at 256^2 (stb_256_u16_6cam_poly_6.5k: same rig, ppp, flow, OTF and settings in
  pixels, 1/64 of the particles, epipolar strips 1/8 as long).
* stb_1280x800_u16_51k: the Shake-the-Box sequence -- 4 pinhole cameras
  (f = 5000 px, 45 deg ring of radius 500 mm, 30 deg tilt), 1280x800 12-bit images,
  51,000 particles in 60x40x30 mm advected by a Burgers vortex plus drift.  After the
  4-frame initial phase, one step = one convergence-phase STB::processFrame (predict,
  shake the predictions, IPR on the residual, repeat check, link, linear-fit prune).
  Particles per step = track points the frame adds over the four track lists.
* ipr_1024_u8_10k: one step = IPR::runIPR on one 4 x 1024^2 uint8 frame of 10,000
  particles; particles per step = reconstructed objects.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica of the workload on its
own GPU ("replicas only": the frame loop has no cross-GPU exchange); value is the
particles of all ranks divided by the slowest rank's time.
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
N_INIT = 4  # STB initial-phase frames

WORKLOADS = {
    # 4 x 1280x800 12-bit (a=3000, b=c=0.5, noise 20), 51,000 particles, Burgers vortex
    # (circulation 2e4 mm^2/s, core 8 mm, strain 2/s) + 20 mm/s drift, <= 3 px/frame.
    # IPR: threshold 300, shake width 0.025 mm (0.25 px), 4 loops x 4 shakes, tol_2d 1 px,
    # tol_3d 0.06 mm; STB: 4 initial frames, link radii 1 mm, field 11x11x6, r 3 mm.
    "stb_1280x800_u16_51k": dict(kind="stb", seq=dict(), settings=dict(min_obj_int=300,
                                                                       shake_width=0.025),
                                 stb=dict()),
    # 4 x 1024^2 uint8 (a=200, b=c=0.5, noise 2), 10,000 particles in 40x40x20 mm;
    # 4 IPR loops x 4 shake iterations, shake width 0.25 mm, threshold 30, tol_2d 1 px.
    "ipr_1024_u8_10k": dict(kind="ipr", scene=dict(n_particles=10000, n_cam=4, size=1024,
                                                   focal=5000.0, a=200.0, b=0.5, c=0.5,
                                                   noise=2.0, bits=8),
                            settings=dict()),
}
# High-density polynomial-camera STB: settings in pixels of the rig (shake width
# 0.25 px, tol_3d 0.6 px, link radii 10 px, field radius 30 px, threshold 300 on the
# 12-bit images); every camera in the build (match_cam_count = 6: with check
# cameras the reference's StereoMatch aborts, StereoMatch.cpp:120-127).
POLY_PX = dict(shake_width=0.25, tol_3d=0.6, link=10.0, pf_r=30.0)
# The reference's default cap of 200,000 detections per camera (limit2DObjectNumber,
# IPR.cpp:19-38) drops each camera's detections independently at random; at 0.1 ppp on
# 2048^2 (about 420,000 detections per camera) a particle would keep all six views
# with probability 0.48^6 (about 1%), so these workloads raise the cap above the
# detection count.  Six convergence-phase frames run untimed after the initial phase
# (and before the warm-up frames) so that the timed frames see a converging tracker.
WORKLOADS["stb_2048_u16_6cam_poly_419k"] = dict(
    kind="stb", gen="poly", seq=dict(ppp=0.1, n_cam=6, size=2048,
                                     volume=(-40.0, 40.0, -40.0, 40.0, -20.0, 20.0), bits=12),
    settings=dict(min_obj_int=300, n_obj2d_process_max=1_000_000),
    stb=dict(pf_nx=11, pf_ny=11, pf_nz=6), converge=6)
WORKLOADS["stb_256_u16_6cam_poly_6.5k"] = dict(
    kind="stb", gen="poly", seq=dict(ppp=0.1, n_cam=6, size=256,
                                     volume=(-5.0, 5.0, -5.0, 5.0, -2.5, 2.5), bits=12),
    settings=dict(min_obj_int=300, n_obj2d_process_max=1_000_000),
    stb=dict(pf_nx=11, pf_ny=11, pf_nz=6), converge=6)
# Many independent sequences on one GPU: 64 seeded sequences (synth.batch_plan:
# particles log-uniform in [2,000, 80,000], 4-6 pinhole cameras, 512/1024/2048^2 uint8
# (a = 200, b = c = 0.5, noise 2), 20 frames of Taylor-Green flow with wavelength in
# [20, 60] mm at <= 3 px/frame); settings in pixels of each rig as above, threshold 30.
# One step = one convergence-phase frame of every sequence (olpt_stb_process_frame_batch).
WORKLOADS["stb_batch64_tg_u8"] = dict(
    kind="batch", n_seq=64, n_frames=20,
    settings=dict(min_obj_int=30, n_obj2d_process_max=1_000_000),
    stb=dict(pf_nx=11, pf_ny=11, pf_nz=6))
# one sequence of the batch's shapes that the CPU path finishes (its reference sample)
WORKLOADS["stb_tg_512_u8_4cam_2k"] = dict(
    kind="stb", gen="tg", seq=dict(n_particles=2000, n_cam=4, size=512, wavelength=40.0),
    settings=dict(min_obj_int=30, n_obj2d_process_max=1_000_000),
    stb=dict(pf_nx=11, pf_ny=11, pf_nz=6))
# the reference arm's sample of each workload (a workload the CPU path finishes)
REFERENCE_SAMPLE = {"stb_2048_u16_6cam_poly_419k": "stb_256_u16_6cam_poly_6.5k",
                    "stb_batch64_tg_u8": "stb_tg_512_u8_4cam_2k"}
DEFAULT_WORKLOAD = "stb_2048_u16_6cam_poly_419k"


def pre_frames(name: str) -> int:
    """Frames processed before the warm-up frames: the initial phase plus the
    workload's untimed convergence-phase frames."""
    return N_INIT + WORKLOADS[name].get("converge", 0)


def ipr_settings(name: str, n_cam: int):
    s = synth.IPRSettings(**WORKLOADS[name]["settings"])
    s.match_cam_count = min(s.match_cam_count, n_cam)
    return s


def build_scene(name: str, seed: int):
    sc = synth.make_scene(seed=seed, **WORKLOADS[name]["scene"])
    return sc, ipr_settings(name, sc.n_cam)


def px_settings(seq, w):
    """IPR / STB knobs of a workload whose lengths are given in pixels of the rig
    (POLY_PX), every camera in the build."""
    mm_px = 1.0 / max(synth.px_per_mm(c, np.zeros(3)) for c in seq.cams)
    s = synth.IPRSettings(**w["settings"])
    s.match_cam_count = seq.n_cam
    s.shake_width = POLY_PX["shake_width"] * mm_px
    s.tol_3d_mm = POLY_PX["tol_3d"] * mm_px
    st = synth.STBSettings(radius_search_obj=POLY_PX["link"] * mm_px,
                           radius_search_track=POLY_PX["link"] * mm_px,
                           pf_r=POLY_PX["pf_r"] * mm_px, **w["stb"])
    return s, st


def build_sequence(name: str, seed: int, n_frames: int, device="cpu", with_images=True):
    w = WORKLOADS[name]
    if w.get("gen") == "poly":
        seq = synth.make_poly_sequence(n_frames=n_frames, seed=seed, device=device,
                                       with_images=with_images, **w["seq"])
        return (seq, *px_settings(seq, w))
    if w.get("gen") == "tg":
        seq = synth.make_tg_sequence(n_frames=n_frames, seed=seed, device=device, **w["seq"])
        return (seq, *px_settings(seq, w))
    seq = synth.make_sequence(n_frames=n_frames, seed=seed, with_images=with_images, **w["seq"])
    return seq, ipr_settings(name, seq.n_cam), synth.STBSettings(**w["stb"])


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


def reference_ipr_time(sc, s, threads: int, images=None):
    """Wall time of the reference IPR::runIPR on this host (compiled from source)."""
    from oracle.ref import RefOracle
    ref = RefOracle(sc, s, threads=threads)
    imgs = [im.astype(np.float64) for im in (images if images is not None else sc.images)]
    with _MuteStdout():
        t = time.perf_counter()
        out = ref.ipr(imgs)
        dt = time.perf_counter() - t
    ref.close()
    return len(out["xyz"]), dt


REF_STB_BUDGET_S = 420.0  # convergence frames of the reference arm stop after this


def reference_stb(name, threads, warmup, steps, budget_s, converge=None):
    """The reference STB (compiled from its sources) on the workload's CPU sample:
    N_INIT initial-phase and ``warmup`` convergence-phase frames untimed, then up to
    ``steps`` convergence frames timed (wall clock), stopping once ``budget_s`` has
    passed.  Particles per frame = track points the frame adds over the four lists."""
    from oracle.ref import RefSTB
    sample_name = REFERENCE_SAMPLE.get(name, name)
    pre = pre_frames(name) if converge is None else N_INIT + converge
    nf = pre + warmup + steps
    seq, s, st = build_sequence(sample_name, 1234, nf)
    times, counts = [], []
    with _MuteStdout():
        ref = RefSTB(seq, s, st, threads=threads, match_cam_count=s.match_cam_count)
        t_start = time.perf_counter()
        for t in range(nf):
            a = time.perf_counter()
            ref.frame(t)
            dt = time.perf_counter() - a
            if t >= pre + warmup:
                rows = ref.tracks()
                times.append(dt)
                counts.append(sum(int(np.count_nonzero(v[:, 1] == t)) for v in rows.values()
                                  if len(v)))
                if time.perf_counter() - t_start > budget_s:
                    break
        ref.close()
    return times, counts, seq, s, st, sample_name


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    kind = WORKLOADS[args.workload]["kind"]
    times, counts = [], []
    if kind == "ipr":
        sc, s = build_scene(args.workload, 1234)
        for i in range(args.warmup + args.steps):
            n, dt = reference_ipr_time(sc, s, threads)
            if i >= args.warmup:
                times.append(dt)
                counts.append(n)
        cfg = workload_config(args.workload, s, sc=sc)
        sample = "whole frame per step (IPR::runIPR, OpenMP, all host threads)"
    else:
        times, counts, seq, s, st, sample_name = reference_stb(
            args.workload, threads, args.warmup, args.steps, REF_STB_BUDGET_S)
        if kind == "batch":
            cfg = {"workload": args.workload, "sequences": WORKLOADS[args.workload]["n_seq"],
                   "reference_sample": workload_config(sample_name, s, seq=seq, st=st)}
        elif sample_name != args.workload:
            main = build_sequence(args.workload, 1234, 1, with_images=False)
            cfg = workload_config(args.workload, main[1], seq=main[0], st=main[2])
            cfg["reference_sample"] = workload_config(sample_name, s, seq=seq, st=st)
        else:
            cfg = workload_config(args.workload, s, seq=seq, st=st)
        sample = (f"STB::processFrame on {sample_name}: {N_INIT} initial-phase and "
                  f"{pre_frames(args.workload) - N_INIT + args.warmup} convergence-phase "
                  f"frames untimed, then {len(times)} "
                  f"convergence-phase frames timed (the same frame indices as the GPU arm; "
                  f"stops after {REF_STB_BUDGET_S:.0f} s); OpenMP, all host threads")
    value = sum(counts) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particles/s",
        "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(name, s, sc=None, seq=None, st=None):
    base = {"workload": name, "ipr_loops": s.n_loop_ipr, "shake_loops": s.n_shake_loop,
            "shake_width_mm": s.shake_width, "threshold": s.min_obj_int,
            "tol_2d_px": s.tol_2d_px, "tol_3d_mm": s.tol_3d_mm, "parallelism": "replicas",
            "l2": "flushed (256 MiB write) before every timed step"}
    if sc is not None:
        H, W = sc.images[0].shape
        base.update(particles=int(len(sc.xyz)), cameras=sc.n_cam,
                    image=f"{H}x{W} {sc.images[0].dtype}")
    else:
        H, W = seq.cams[0].n_row, seq.cams[0].n_col
        dt = "uint8" if seq.max_val <= 255 else "uint16"
        base.update(particles=int(len(seq.truth[0])), cameras=seq.n_cam,
                    image=f"{H}x{W} {dt} ({int(seq.max_val).bit_length()}-bit)",
                    ppp=round(len(seq.truth[0]) / (H * W), 4),
                    initial_frames=N_INIT,
                    untimed_convergence_frames=WORKLOADS[name].get("converge", 0),
                    link_radius_mm=st.radius_search_track,
                    pred_field=f"{st.pf_nx}x{st.pf_ny}x{st.pf_nz} r {st.pf_r} mm",
                    match_cam_count=s.match_cam_count,
                    detection_cap=s.n_obj2d_process_max,
                    step="one convergence-phase frame")
        if WORKLOADS[name].get("gen") == "tg":
            base.update(camera_model="pinhole ring rig", otf="uniform (a, b, c) = "
                        f"{tuple(float(x) for x in seq.otf_table[:3, 0, 0])}",
                        flow="Taylor-Green cells (random phase), <= 3 px/frame")
        elif isinstance(seq, synth.PolySequence):
            base.update(camera_model="cubic polynomial (20 terms), <= 2 px corner distortion",
                        otf=f"{'x'.join(map(str, seq.otf_n))} grid, a in [2400, 3600], "
                            "b, c in [0.3, 0.9]",
                        flow="ABC (A = B = C = 1, wavelength 40 mm), <= 4 px/frame")
    return base


# ----------------------------------------------------------------------------- our arm
PROF_NAMES = {0: "peak detection", 1: "stereo level expansion", 2: "residual image",
              3: "shake (warp per particle)", 4: "predictive field"}
PHASE_NAMES = {5: "detection", 6: "stereo matching (all)", 7: "candidate sort + prune + greedy",
               8: "shake (all)", 9: "output + residual", 10: "STB track work",
               11: "sequential greedy (replacement fallback)", 12: "track work: prediction",
               13: "track work: extension", 14: "track work: linking and new tracks",
               15: "track work: linear-fit pruning"}


# Per camera count: DRAM bytes per shaken object measured with ncu, and the kernel's
# algorithmic bytes per object in FP32 (C x 64 ROI pixels x 4 B + 2 x (24 + C x 16 + 8) B
# of state + C x 5 x 4 B of OTF).  4 cameras: dram__bytes_read.sum + dram__bytes_write.sum
# of three shake_kernel launches of the 1280x800 STB convergence frames (16-19 k objects
# each) over their objects.  6 cameras: two launches of the first IPR of a 2048^2 headline
# frame (14,840 objects each), dram__bytes.sum.per_second x duration over the objects.
SHAKE_TRAFFIC = {4: (7_300.0, 1_296.0), 6: (22_440.0, 1_912.0)}


def shake_traffic(args, prec, dom, bytes_per_launch, cams):
    """DRAM traffic of an average shake launch of the STB workload, scaled from the
    per-object figure by the objects the launch processes; None elsewhere."""
    if dom != 3 or prec != 0 or WORKLOADS[args.workload]["kind"] != "stb":
        return None
    if cams not in SHAKE_TRAFFIC:
        return None
    dram, algo = SHAKE_TRAFFIC[cams]
    return bytes_per_launch / algo * dram


def reduce_replicas(dist, values, device):
    """Whole-job numbers over the replicas (one per rank): the slowest rank's times
    (values[0] device ms, values[2] end-to-end s) and the sum of the particles
    (values[1], values[3])."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = t.clone()
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return tmax[0].item(), tsum[1].item(), tmax[2].item(), tsum[3].item()


class Ours:
    """One rank of our arm: device set-up, rank reduction and the JSON line."""

    def __init__(self, args):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.args = torch, dist, args
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(self.local)
        if self.world > 1:
            import datetime
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", self.local))
        self.prec = 1 if args.precision == "fp64" else 0
        self.flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def context(self, sc):
        """A context with the rig of a scene or sequence: its cameras (pinhole or
        polynomial) and its OTF (uniform 2x2x2, or the sequence's grid)."""
        from pyopenlpt_b200 import _ffi
        ctx = _ffi.Context(self.local)
        ctx.upload_cameras([_ffi.camera_desc(c) for c in sc.cams])
        if getattr(sc, "otf_table", None) is not None:
            ctx.upload_otf(*sc.otf_n, sc.volume, sc.otf_table)
        else:
            ctx.upload_otf(2, 2, 2, sc.volume, synth.otf_table_array(len(sc.cams), sc.otf_abc))
        return ctx

    def reduce(self, dev_ms, parts, e2e_s, e2e_parts):
        if self.world == 1:
            return dev_ms, float(parts), e2e_s, float(e2e_parts)
        return reduce_replicas(self.dist, [dev_ms, parts, e2e_s, e2e_parts], "cuda")

    def line(self, prof, dev_ms, parts, e2e_s, e2e_parts, bi, bo, launches, clk, cfg, cpu,
             extra):
        args = self.args
        peak, peak_kind = measured_peak_hbm()
        # dominant HBM-bound kernel: the largest share of device time among the
        # streaming kernels (detection, residual, shake)
        cand = {k: prof[k] for k in (0, 2, 3) if prof[k][1] > 0}
        dom = max(cand, key=lambda k: cand[k][0]) if cand else 2
        ms, nl, by = prof[dom]
        achieved = (by / nl) / ((ms / nl) * 1e-3) / 1e9 if nl and ms > 0 else 0.0
        kernel_ms = {PROF_NAMES[k]: round(prof[k][0] / args.steps, 4) for k in PROF_NAMES}
        phase_ms = {PHASE_NAMES[k]: round(prof[k][0] / args.steps, 3) for k in PHASE_NAMES}
        line = {
            "metric": METRIC, "value": parts / (dev_ms * 1e-3), "unit": "particles/s",
            "n_gpus": self.world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if self.prec == 0 else "f64", "data": "synthetic",
            "config": dict(cfg, precision="fp32 residual/shake, fp64 geometry"
                           if self.prec == 0 else "fp64"),
            "frames_per_s": self.world * args.steps / (dev_ms * 1e-3),
            "e2e": {"value": e2e_parts / e2e_s, "unit": "particles/s",
                    "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo},
            "gpu_launches": int(launches),
            "kernel_ms_per_step": kernel_ms,
            "host_phase_ms_per_step": phase_ms,
            "roofline": {"bound": "hbm", "kernel": PROF_NAMES[dom], "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind,
                         "bytes_per_launch": by / nl if nl else 0.0,
                         "launch_ms": ms / nl if nl else 0.0,
                         "traffic": shake_traffic(args, self.prec, dom, by / nl if nl else 0.0,
                                                  cfg.get("cameras"))},
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)


def run_ours_ipr(args, o: Ours, pre):
    from pyopenlpt_b200 import _ffi
    torch = o.torch
    sc, s = build_scene(args.workload, 1234 + o.rank)
    ctx = o.context(sc)
    params = _ffi.ipr_params(s, sc.volume, o.prec)
    H, W = sc.images[0].shape
    dtype = _ffi._DTYPES[sc.images[0].dtype]
    dev_imgs = [torch.from_numpy(im).cuda() for im in sc.images]
    host_imgs = [torch.from_numpy(im).pin_memory() for im in sc.images]
    stream = torch.cuda.ExternalStream(ctx.stream())
    torch.cuda.synchronize()

    def step_device():
        ctx.upload_images_device([t.data_ptr() for t in dev_imgs], dtype, [H] * sc.n_cam,
                                 [W] * sc.n_cam)
        return ctx.ipr_run(params)

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    clocks = ClockSampler(o.local)
    clocks.start()
    ctx.profile(True)
    o.barrier()
    torch.cuda.synchronize()
    launches0 = _ffi.launch_count()
    dev_ms, parts = 0.0, 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            o.flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        n = step_device()
        e1.record(stream)
        e1.synchronize()
        dev_ms += e0.elapsed_time(e1)
        parts += n
    torch.cuda.synchronize()
    o.barrier()
    launches = _ffi.launch_count() - launches0
    prof = {k: ctx.profile_read(k) for k in list(PROF_NAMES) + list(PHASE_NAMES)}
    ctx.profile(False)
    clk = clocks.stop()

    # end to end through the C ABI with host buffers
    o.barrier()
    e2e_s, e2e_parts, bo = 0.0, 0, 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            o.flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.upload_images([t.numpy() for t in host_imgs])
        n = ctx.ipr_run(params)
        xyz, uv = ctx.ipr_result(n)
        e2e_s += time.perf_counter() - t0
        e2e_parts += n
        bo += xyz.nbytes + uv.nbytes
    o.barrier()
    bi = sum(im.nbytes for im in sc.images)
    dev_ms, parts, e2e_s, e2e_parts = o.reduce(dev_ms, parts, e2e_s, e2e_parts)
    if o.rank == 0:
        cpu = None
        if o.world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            ncpu, tcpu = reference_ipr_time(sc, s, threads)
            cpu = {"value": ncpu / tcpu, "unit": "particles/s", "cores": threads,
                   "kind": "reference",
                   "sample": "one whole frame of the same workload (IPR::runIPR compiled "
                             "from the reference sources, OpenMP)"}
        o.line(prof, dev_ms, parts, e2e_s, e2e_parts, bi, bo // max(1, args.steps), launches,
               clk, workload_config(args.workload, s, sc=sc), cpu, dict(pre))
    ctx.close()


def recall_ghost(found, truth, radius):
    """Fraction of true particles with an output within radius, and fraction of
    outputs with no true particle within radius."""
    from scipy.spatial import cKDTree
    if len(found) == 0:
        return 0.0, 0.0
    d_gt, _ = cKDTree(found).query(truth)
    d_f, _ = cKDTree(truth).query(found)
    return float(np.mean(d_gt <= radius)), float(np.mean(d_f > radius))


def frame_quality(xyz, truth):
    r05, g05 = recall_ghost(xyz, truth, 0.05)
    r10, g10 = recall_ghost(xyz, truth, 0.1)
    return {"n": int(len(xyz)), "recall_05": r05, "ghost_05": g05, "recall_10": r10,
            "ghost_10": g10}


def mean_quality(qs):
    keys = ("recall_05", "ghost_05", "recall_10", "ghost_10")
    out = {k: round(float(np.mean([q[k] for q in qs])), 5) for k in keys}
    if qs and "ms" in qs[0]:
        ms = float(np.sum([q["ms"] for q in qs]))
        out.update(ms_per_frame=round(ms / len(qs), 3),
                   particles_per_s=round(float(np.sum([q["parts"] for q in qs])) / (ms * 1e-3), 1))
    return out


def meets(m, plain, slack=0.005):
    """Recall within slack of the plain form's and no higher ghost rate, at 0.05 and
    0.1 mm."""
    return all(m["recall_" + k] >= plain["recall_" + k] - slack and
               m["ghost_" + k] <= plain["ghost_" + k] + 1e-9 for k in ("05", "10"))


def timed_frame(o, stream, fn):
    """Event-timed call on the library stream (L2 flushed first); milliseconds."""
    torch = o.torch
    with torch.cuda.stream(stream):
        o.flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_ours_stb(args, o: Ours, pre_lines):
    from pyopenlpt_b200 import _ffi
    from pyopenlpt_b200 import learned as L
    torch = o.torch
    n_pre = pre_frames(args.workload)
    nf = n_pre + args.warmup + args.steps
    t_gen = time.perf_counter()
    seq, s, st = build_sequence(args.workload, 1234 + o.rank, nf, device=f"cuda:{o.local}")
    t_gen = time.perf_counter() - t_gen
    H, W = seq.cams[0].n_row, seq.cams[0].n_col
    C = seq.n_cam
    frames = [np.ascontiguousarray(np.stack(f)) for f in seq.frames]
    dtype = _ffi._DTYPES[frames[0].dtype]
    dev_frames = [torch.from_numpy(f).cuda() for f in frames]
    host_frames = [torch.from_numpy(f).pin_memory() for f in frames]
    params = _ffi.stb_params(s, st, seq.volume, 0, nf - 1, o.prec)
    t0_frame = n_pre + args.warmup

    def new_ctx(prec=o.prec, sk=None):
        ctx = o.context(seq)
        ctx.stb_configure(_ffi.stb_params(sk or s, st, seq.volume, 0, nf - 1, prec))
        return ctx

    def frame_device(ctx, t):
        ctx.upload_images_device([dev_frames[t][c].data_ptr() for c in range(C)], dtype,
                                 [H] * C, [W] * C)
        ctx.stb_process_frame(t)

    ctx = new_ctx()
    stream = torch.cuda.ExternalStream(ctx.stream())
    torch.cuda.synchronize()
    init_ms = []
    for t in range(N_INIT):
        a = time.perf_counter()
        frame_device(ctx, t)
        init_ms.append(1e3 * (time.perf_counter() - a))
    conv_ms = []
    for t in range(N_INIT, n_pre):
        a = time.perf_counter()
        frame_device(ctx, t)
        conv_ms.append(1e3 * (time.perf_counter() - a))
    want_learned = (o.world == 1 and args.learn_frames > 0
                    and WORKLOADS[args.workload].get("gen") == "poly")
    state_init = L.stb_state(ctx) if want_learned else None
    plain_warm = []
    for t in range(n_pre, t0_frame):
        ms = timed_frame(o, stream, lambda: frame_device(ctx, t))
        plain_warm.append(dict(frame_quality(ctx.stb_frame_objects(), seq.truth[t]), ms=ms,
                               parts=ctx.stb_frame_points(t)))
    state_t0 = L.stb_state(ctx) if want_learned else None
    torch.cuda.synchronize()

    clocks = ClockSampler(o.local)
    clocks.start()
    ctx.profile(True)
    o.barrier()
    torch.cuda.synchronize()
    launches0 = _ffi.launch_count()
    dev_ms, parts, ext_new = 0.0, 0, 0
    quality, plain_objs = [], {}
    for t in range(t0_frame, nf):
        with torch.cuda.stream(stream):
            o.flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        frame_device(ctx, t)
        e1.record(stream)
        e1.synchronize()
        dev_ms += e0.elapsed_time(e1)
        parts += ctx.stb_frame_points(t)
        _, ne, nn = ctx.stb_counts()
        ext_new += ne + nn
        # outside the events: the frame's particles against the ground truth
        launches_q = _ffi.launch_count()
        xyz = ctx.stb_frame_objects()
        plain_objs[t] = xyz
        quality.append(dict(frame_quality(xyz, seq.truth[t]), ms=e0.elapsed_time(e1),
                            parts=ctx.stb_frame_points(t)))
        launches0 += _ffi.launch_count() - launches_q
    torch.cuda.synchronize()
    o.barrier()
    launches = _ffi.launch_count() - launches0
    prof = {k: ctx.profile_read(k) for k in list(PROF_NAMES) + list(PHASE_NAMES)}
    ctx.profile(False)
    clk = clocks.stop()
    lists, _, _ = ctx.stb_counts()
    ctx.close()

    # end to end through the C ABI with host (pinned) images: a second tracker over the
    # same frames; each timed step uploads the frame, processes it and reads back the
    # frame's particles
    ctx = new_ctx()
    stream = torch.cuda.ExternalStream(ctx.stream())
    for t in range(t0_frame):
        ctx.upload_images(list(host_frames[t].numpy()))
        ctx.stb_process_frame(t)
    o.barrier()
    e2e_s, e2e_parts, bo = 0.0, 0, 0
    for t in range(t0_frame, nf):
        with torch.cuda.stream(stream):
            o.flush.zero_()
        torch.cuda.synchronize()
        a = time.perf_counter()
        ctx.upload_images(list(host_frames[t].numpy()))
        ctx.stb_process_frame(t)
        xyz = ctx.stb_frame_objects()
        e2e_s += time.perf_counter() - a
        e2e_parts += ctx.stb_frame_points(t)
        bo += xyz.nbytes
    o.barrier()
    ctx.close()
    bi = C * H * W * frames[0].itemsize
    dev_ms, parts, e2e_s, e2e_parts = o.reduce(dev_ms, parts, e2e_s, e2e_parts)
    if o.rank == 0:
        cpu = None
        extra = {"initial_phase_ms_per_frame": [round(x, 1) for x in init_ms],
                 "untimed_convergence_ms_per_frame": [round(x, 1) for x in conv_ms],
                 "extended_plus_new_per_step": ext_new / args.steps,
                 "track_lists_after": dict(zip(_ffi.TRACK_LISTS, lists)),
                 "quality_vs_truth": mean_quality(quality),
                 "generation_s": round(t_gen, 1)}
        # the secondary measurements: a failure is recorded in the line, not fatal
        def guarded(key, fn):
            try:
                extra[key] = fn()
            except Exception as e:  # noqa: BLE001
                extra[key] = {"error": f"{type(e).__name__}: {e}"}

        if want_learned:
            guarded("learned", lambda: learned_stb(args, o, seq, s, st, nf, t0_frame, new_ctx,
                                                   frame_device, state_init, state_t0,
                                                   plain_warm, quality))
        if o.world == 1 and o.prec == 0 and not args.no_fp64_check:
            guarded("fp64_check", lambda: fp64_check(o, seq, s, nf - 1, plain_objs[nf - 1]))
        if o.world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            times, counts, rseq, _, _, sname = reference_stb(args.workload, threads, 0, 2, 60.0,
                                                             converge=0)
            cpu = {"value": sum(counts) / sum(times), "unit": "particles/s", "cores": threads,
                   "kind": "reference",
                   "sample": f"STB::processFrame compiled from the reference sources (OpenMP) "
                             f"on {sname}: {N_INIT} initial-phase frames untimed, then "
                             f"{len(times)} convergence-phase frames timed"}
        extra.update(pre_lines)
        o.line(prof, dev_ms, parts, e2e_s, e2e_parts, bi, bo // max(1, args.steps), launches,
               clk, workload_config(args.workload, s, seq=seq, st=st), cpu, extra)


def run_ours_batch(args, o: Ours, pre_lines):
    """Many independent sequences at once: every sequence's frame t in one
    olpt_stb_process_frame_batch call (one step).  `value`: frames resident in HBM;
    `e2e`: a second pass whose steps upload every sequence's frame from pinned host
    memory and read back its particles.  The same sequences run one at a time on one
    context each give the batching gain and the per-sequence equality check (track
    lists identical to the batched run's after the last frame)."""
    from pyopenlpt_b200 import _ffi
    torch = o.torch
    w = WORKLOADS[args.workload]
    plan = synth.batch_plan(w["n_seq"], seed=2024 + 1000 * o.rank)
    nf = max(w["n_frames"], N_INIT + args.warmup + args.steps)
    t0_frame = N_INIT + args.warmup
    t_gen = time.perf_counter()
    seqs, sets = [], []
    for p in plan:
        seq = synth.make_tg_sequence(n_frames=nf, device=f"cuda:{o.local}", **p)
        seqs.append(seq)
        sets.append(px_settings(seq, w))
    t_gen = time.perf_counter() - t_gen
    dev = [[torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in q.frames] for q in seqs]
    host = [[torch.from_numpy(np.ascontiguousarray(f)).pin_memory() for f in q.frames]
            for q in seqs]

    def make(i):
        q = seqs[i]
        s, st = sets[i]
        ctx = o.context(q)
        ctx.stb_configure(_ffi.stb_params(s, st, q.volume, 0, nf - 1, o.prec))
        return ctx

    def put_device(ctx, i, t):
        q = seqs[i]
        H, W = q.cams[0].n_row, q.cams[0].n_col
        d = dev[i][t]
        ctx.upload_images_device([d[c].data_ptr() for c in range(q.n_cam)], _ffi.OLPT_U8,
                                 [H] * q.n_cam, [W] * q.n_cam)

    def lists(ctx):
        return [ctx.stb_tracks(k) for k in range(4)]

    # batched pass, device-resident frames
    ctxs = [make(i) for i in range(len(seqs))]
    for t in range(t0_frame):
        for i, c in enumerate(ctxs):
            put_device(c, i, t)
        _ffi.stb_process_frame_batch(ctxs, [t] * len(ctxs))
    for c in ctxs:
        c.profile(True)
    clocks = ClockSampler(o.local)
    clocks.start()
    torch.cuda.synchronize()
    launches0 = _ffi.launch_count()
    step_ms, parts = [], 0
    for t in range(t0_frame, t0_frame + args.steps):
        o.flush.zero_()
        torch.cuda.synchronize()
        a = time.perf_counter()
        for i, c in enumerate(ctxs):
            put_device(c, i, t)
        _ffi.stb_process_frame_batch(ctxs, [t] * len(ctxs))
        torch.cuda.synchronize()
        step_ms.append(1e3 * (time.perf_counter() - a))
        parts += sum(c.stb_frame_points(t) for c in ctxs)
    launches = _ffi.launch_count() - launches0
    clk = clocks.stop()
    prof = {}
    for k in list(PROF_NAMES) + list(PHASE_NAMES):
        vals = [c.profile_read(k) for c in ctxs]
        prof[k] = (sum(v[0] for v in vals), sum(v[1] for v in vals), sum(v[2] for v in vals))
    batched_lists = [lists(c) for c in ctxs]
    for c in ctxs:
        c.close()

    # end to end: pinned host frames uploaded through the C ABI, particles read back
    ctxs = [make(i) for i in range(len(seqs))]
    for t in range(t0_frame):
        for i, c in enumerate(ctxs):
            c.upload_images(list(host[i][t].numpy()))
        _ffi.stb_process_frame_batch(ctxs, [t] * len(ctxs))
    e2e_s, e2e_parts, bi, bo = 0.0, 0, 0, 0
    for t in range(t0_frame, t0_frame + args.steps):
        o.flush.zero_()
        torch.cuda.synchronize()
        a = time.perf_counter()
        for i, c in enumerate(ctxs):
            c.upload_images(list(host[i][t].numpy()))
        _ffi.stb_process_frame_batch(ctxs, [t] * len(ctxs))
        outs = [c.stb_frame_objects() for c in ctxs]
        e2e_s += time.perf_counter() - a
        e2e_parts += sum(c.stb_frame_points(t) for c in ctxs)
        bo += sum(x.nbytes for x in outs)
    bi = sum(q.n_cam * q.cams[0].n_row * q.cams[0].n_col for q in seqs)
    for c in ctxs:
        c.close()

    # one sequence at a time, same frames: the batching gain and the equality check
    solo_ms, equal = 0.0, 0
    mism = []
    for i in range(len(seqs)):
        ctx = make(i)
        stream = torch.cuda.ExternalStream(ctx.stream())
        for t in range(t0_frame + args.steps):
            put_device(ctx, i, t)
            if t < t0_frame:
                ctx.stb_process_frame(t)
            else:
                solo_ms += timed_frame(o, stream, lambda: ctx.stb_process_frame(t))
        same = all(all(np.array_equal(x, y) for x, y in zip(a_, b_))
                   for a_, b_ in zip(lists(ctx), batched_lists[i]))
        equal += int(same)
        if not same:
            mism.append(i)
        ctx.close()

    dev_ms = sum(step_ms)
    dev_ms, parts, e2e_s, e2e_parts = o.reduce(dev_ms, parts, e2e_s, e2e_parts)
    if o.rank != 0:
        return
    cpu = None
    if o.world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        times, counts, _, _, _, sname = reference_stb(args.workload, threads, 0, 2, 60.0,
                                                      converge=0)
        cpu = {"value": sum(counts) / sum(times), "unit": "particles/s", "cores": threads,
               "kind": "reference",
               "sample": f"STB::processFrame compiled from the reference sources (OpenMP) on "
                         f"{sname} (one sequence of the batch's shapes): {N_INIT} initial-phase "
                         f"frames untimed, then {len(times)} convergence-phase frames timed"}
    sizes = {}
    for p in plan:
        key = f"{p['n_cam']}cam_{p['size']}"
        sizes[key] = sizes.get(key, 0) + 1
    cfg = {"workload": args.workload, "sequences": len(plan),
           "particles_total": int(sum(p["n_particles"] for p in plan)),
           "particles_range": [min(p["n_particles"] for p in plan),
                               max(p["n_particles"] for p in plan)],
           "rigs": sizes, "frames": nf, "initial_frames": N_INIT,
           "step": "one convergence-phase frame of every sequence",
           "settings": "threshold 30, shake width 0.25 px, tol_2d 1 px, tol_3d 0.6 px, "
                       "link radii 10 px, field 11x11x6 r 30 px, 4 IPR loops x 4 shakes, "
                       "match_cam_count = cameras",
           "parallelism": "one context per sequence, persistent host workers, one stream each",
           "timing": "wall clock around each batched step with device synchronisation on both "
                     "sides (the step spans one stream per sequence)",
           "l2": "flushed (256 MiB write) before every timed step; the step's frames "
                 f"({bi / 2**20:.0f} MiB) exceed L2"}
    extra = {"generation_s": round(t_gen, 1),
             "one_at_a_time": {"value": parts / (solo_ms * 1e-3) if solo_ms else None,
                               "unit": "particles/s", "ms_per_step": solo_ms / args.steps,
                               "batching_gain": solo_ms / dev_ms if dev_ms else None},
             "per_sequence_equal_to_one_at_a_time": f"{equal}/{len(seqs)}",
             "mismatched_sequences": mism}
    extra.update(pre_lines)
    o.line(prof, dev_ms, parts, e2e_s, e2e_parts, bi, bo // max(1, args.steps), launches, clk,
           cfg, cpu, extra)


def learned_stb(args, o, seq, s, st, nf, t0_frame, new_ctx, frame_device, state_init, state_t0,
                plain_warm, plain_timed):
    """The learned form on the same frames as the plain form.

    1. Tuples from the plain GPU shake on a separate seeded sequence of the same
       workload: prediction-like starts (true particles displaced by 0.3 and 1 px,
       plus 10% uniform points) and the candidates of the first IPR loop.
    2. Training on the device (olpt_mlp_train).
    3. Calibration on the warm-up frames, from the plain tracker's tracks before them:
       the fastest settings whose recall is within 0.5% of the plain
       form's and whose ghost rate is not higher, at 0.05 and 0.1 mm.
    4. Evaluation on the timed frames, from the plain tracker's tracks at the first
       timed frame, device-timed like the plain form."""
    import dataclasses
    from pyopenlpt_b200 import learned as L
    torch = o.torch
    mm_px = 1.0 / max(synth.px_per_mm(c, np.zeros(3)) for c in seq.cams)
    ls0 = L.LearnedSettings(out_scale_mm=0.5 * mm_px, ghost_tol_mm=1.5 * mm_px,
                            refine_width_mm=0.4 * s.shake_width, ghost_logit=5.0,
                            refine_loops=1, fallback_residual=1e9)
    # 1. tuples
    t_c = time.perf_counter()
    tseq, _, _ = build_sequence(args.workload, 4321 + o.rank, args.learn_frames,
                                device=f"cuda:{o.local}")
    ctx = new_ctx()
    xs, ts = [], []
    per_frame = max(1, args.learn_tuples // max(1, args.learn_frames))
    for f in range(args.learn_frames):
        ctx.upload_images(list(tseq.frames[f]))
        x, t = L.collect_predictions(ctx, tseq.truth[f], s, ls0, (0.3 * mm_px, 1.0 * mm_px),
                                     tseq.volume, n_max=int(0.8 * per_frame), seed=f)
        xs.append(x)
        ts.append(t)
        ctx.upload_images(list(tseq.frames[f]))
        x, t = L.collect_ipr(ctx, tseq.truth[f], s, tseq.volume, ls0, loops=1)
        room = max(0, per_frame - len(xs[-1]))
        if len(x) > room:
            keep = np.random.default_rng(f).choice(len(x), room, replace=False)
            x, t = x[keep], t[keep]
        xs.append(x)
        ts.append(t)
    x = np.concatenate(xs)
    t = np.concatenate(ts)
    del xs, ts, tseq
    t_collect = time.perf_counter() - t_c
    # 2. training
    ctx.mlp_init(1)
    t_t = time.perf_counter()
    losses = L.train(ctx, x, t, steps=args.learn_steps, batch=8192, lr=2e-3)
    t_train = time.perf_counter() - t_t
    n_tuples, ghost_share = len(x), float(np.mean(t[:, 3]))
    del x, t
    params = ctx.mlp_get_params()
    ctx.close()

    def run(ls, loops, state, frames):
        c = new_ctx(sk=dataclasses.replace(s, n_loop_ipr=loops))
        c.mlp_set_params(params)
        c.learned_configure(ls.params(enable=True))
        L.set_stb_state(c, state)
        st_ = torch.cuda.ExternalStream(c.stream())
        a0, b0 = c.learned_stats()
        out = []
        for f in frames:
            ms = timed_frame(o, st_, lambda: frame_device(c, f))
            out.append(dict(frame_quality(c.stb_frame_objects(), seq.truth[f]), ms=ms,
                            parts=c.stb_frame_points(f)))
        a1, b1 = c.learned_stats()
        c.close()
        return out, (b1 - b0) / max(1, a1 - a0)

    # 3. calibration on the warm-up frames
    warm = list(range(t0_frame - len(plain_warm), t0_frame))
    pw = mean_quality(plain_warm)
    sweep, chosen = [], None
    # (IPR loops per frame, settings): the network's proposals let the IPR on the
    # residual run fewer loops; the fallback re-runs the plain shake for hard objects
    grid = [(1, dict(refine_loops=1, ghost_logit=5.0, fallback_residual=1e9)),
            (1, dict(refine_loops=1, ghost_logit=5.0, fallback_residual=0.3)),
            (2, dict(refine_loops=1, ghost_logit=5.0, fallback_residual=1e9)),
            (2, dict(refine_loops=1, ghost_logit=5.0, fallback_residual=0.3)),
            (s.n_loop_ipr, dict(refine_loops=1, ghost_logit=5.0, fallback_residual=1e9)),
            (s.n_loop_ipr, dict(refine_loops=2, ghost_logit=8.0, fallback_residual=0.1))]
    for loops, g in grid:
        ls = dataclasses.replace(ls0, **g)
        res, fb = run(ls, loops, state_init, warm)
        m = mean_quality(res)
        ok = meets(m, pw)
        sweep.append(dict(g, ipr_loops=loops, **m, fallback_fraction=round(fb, 4), meets=ok))
        if ok and (chosen is None or m["ms_per_frame"] < chosen[2]["ms_per_frame"]):
            chosen = (ls, loops, m)
    if chosen is not None:
        ls, loops = chosen[0], chosen[1]
    else:
        loops, ls = grid[-1][0], dataclasses.replace(ls0, **grid[-1][1])
    # 4. evaluation on the timed frames
    res, fb = run(ls, loops, state_t0, list(range(t0_frame, nf)))
    lm, pm = mean_quality(res), mean_quality(plain_timed)
    return {
        "form": "MLP proposal on every prediction and IPR candidate (ghosts dropped), "
                "refine_loops plain shake iterations, plain-shake fallback above the "
                "residual threshold",
        "train": {"frames": args.learn_frames, "tuples": n_tuples,
                  "ghost_share": round(ghost_share, 4), "steps": len(losses),
                  "collect_s": round(t_collect, 1), "train_s": round(t_train, 1),
                  "loss_first": round(losses[0], 4),
                  "loss_last50": round(float(np.mean(losses[-50:])), 4)},
        "calibration": {"frames": warm, "plain": pw, "sweep": sweep,
                        "chosen": {"ipr_loops": loops, "refine_loops": ls.refine_loops,
                                   "ghost_logit": ls.ghost_logit,
                                   "fallback_residual": ls.fallback_residual,
                                   "refine_width_mm": ls.refine_width_mm,
                                   "out_scale_mm": ls.out_scale_mm},
                        "met": chosen is not None},
        "eval": {"frames": list(range(t0_frame, nf)), "plain": pm, "learned": lm,
                 "fallback_fraction": round(fb, 4),
                 "speedup_particles_per_s": round(lm["particles_per_s"] / pm["particles_per_s"], 3),
                 "speedup_time": round(pm["ms_per_frame"] / lm["ms_per_frame"], 3),
                 "meets_recall_and_ghost": meets(lm, pm)},
    }


def fp64_check(o, seq, s, t, xyz):
    """The FP32 production shake against the library's FP64 mode (the reference's
    arithmetic) on the same input: frame t's images and the plain tracker's particles
    of that frame as starting positions, one runShake in each precision.  Reports the
    position differences, the reprojection differences on every camera, and the
    residual image of camera 0 (FP32 plane against the FP64 one)."""
    from pyopenlpt_b200 import _ffi, learned as L
    ctx = _ffi.Context(o.local)
    L.bind_rig(ctx, seq)
    H, W = seq.cams[0].n_row, seq.cams[0].n_col
    out, res = {}, {}
    for prec in (0, 1):
        ctx.upload_images(list(seq.frames[t]))
        ctx.upload_objects(xyz)
        sp = _ffi.shake_params(s, prec)
        ctx.shake(sp)
        out[prec] = ctx.objects()
        ctx.residual(sp)
        res[prec] = ctx.residual_image(0, (H, W), np.float64)
    d = np.max(np.abs(out[0]["xyz"] - out[1]["xyz"]), axis=1)
    r = np.max(np.abs(out[0]["uv"] - out[1]["uv"]), axis=(1, 2))
    ok = np.isfinite(d)
    ctx.close()
    return {"frame": t, "objects": int(len(xyz)),
            "position_mm": {"median": float(np.median(d[ok])), "p99": float(np.quantile(d[ok], 0.99)),
                            "max": float(d[ok].max()), "frac_le_1e-4": float(np.mean(d[ok] <= 1e-4))},
            "reprojection_px": {"median": float(np.median(r[ok])), "max": float(r[ok].max())},
            "flags_differ": int(np.sum(out[0]["flags"] != out[1]["flags"])),
            "residual_cam0_max_abs": float(np.max(np.abs(res[0] - res[1])))}


# ----------------------------------------------------------------------------- learned
LEARN_PPP = (0.01, 0.02, 0.03, 0.05, 0.08, 0.1)


def learned_comparison(args, o: Ours):
    """The learned proposal against the plain GPU form on its own workload (4 cameras,
    1024^2 uint8, the 40 x 40 x 20 mm volume filling the images so that ppp counts the
    illuminated area, OTF b, c uniform in [0.3, 0.8], settings in pixels of the rig:
    shake width 0.25 px): tuples from the plain pipeline on
    seeded frames at 0.01-0.1 ppp, training on the device, calibration on a validation
    frame (fewest IPR loops whose recall is within 0.5% of the plain 4-loop IPR and
    whose ghost rate is not higher, at 0.05 and 0.1 mm), then device-timed IPR of both
    forms on held-out frames at 0.02 and 0.08 ppp."""
    from pyopenlpt_b200 import _ffi, learned as L
    import dataclasses
    torch = o.torch
    s, ls = L.rig_settings(L.scene(0, 0.01))
    ctx = _ffi.Context(o.local)
    t0 = time.perf_counter()
    xs, ts = [], []
    for i in range(args.learn_ipr_frames):
        x, t = L.collect(ctx, L.scene(i, LEARN_PPP[i % len(LEARN_PPP)]), s, ls)
        xs.append(x)
        ts.append(t)
    x, t = np.concatenate(xs), np.concatenate(ts)
    del xs, ts
    t_collect = time.perf_counter() - t0
    ctx.mlp_init(1)
    t0 = time.perf_counter()
    losses = L.train(ctx, x, t, steps=args.learn_steps, batch=8192, lr=2e-3)
    t_train = time.perf_counter() - t0
    n_tuples = len(x)
    del x, t
    k, cfg, plain_val, _ = L.calibrate(ctx, L.scene(900, 0.02), s, ls)
    stream = torch.cuda.ExternalStream(ctx.stream())

    def timed(sc, sk, lsx, reps):
        L.bind(ctx, sc)
        ctx.learned_configure((lsx or L.LearnedSettings()).params(enable=lsx is not None))
        p = _ffi.ipr_params(sk, sc.volume)
        ctx.ipr_run(p)  # warm-up
        ms = []
        for _ in range(reps):
            ctx.upload_images(sc.images)
            with torch.cuda.stream(stream):
                o.flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            n = ctx.ipr_run(p)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        xyz, _ = ctx.ipr_result(n)
        m = L.metrics(xyz, sc.xyz)
        m["ms"] = float(np.median(ms))
        m["particles_per_s"] = m["n"] / (m["ms"] * 1e-3)
        m["true_particles_per_s"] = m["recall_10"] * len(sc.xyz) / (m["ms"] * 1e-3)
        return {kk: round(v, 5) for kk, v in m.items()}

    evals = {}
    for i, ppp in enumerate((0.02, 0.08)):
        sc = L.scene(901 + i, ppp)
        plain = timed(sc, s, None, args.learn_reps)
        a0, b0 = ctx.learned_stats()
        learned = timed(sc, dataclasses.replace(s, n_loop_ipr=k), cfg, args.learn_reps)
        a1, b1 = ctx.learned_stats()
        learned["fallback_fraction"] = round((b1 - b0) / max(1, a1 - a0), 4)
        evals[f"ppp_{ppp}"] = {
            "n_true": len(sc.xyz), "plain": plain, "learned": learned,
            "speedup_particles_per_s": round(learned["particles_per_s"] / plain["particles_per_s"], 3),
            "speedup_time": round(plain["ms"] / learned["ms"], 3),
            "meets_recall_and_ghost": L.meets(learned, plain)}
    # batched: B independent frames at once (olpt_ipr_run_batch: one context, host thread
    # and stream per frame), wall time of the whole batch, against the same frames one
    # at a time through the plain form
    params = ctx.mlp_get_params()
    ctx.close()
    B = args.learn_batch
    ctxs = [_ffi.Context(o.local) for _ in range(B)]
    for c in ctxs:
        c.mlp_set_params(params)
    scenes = [L.scene(950 + i, 0.02) for i in range(B)]
    sk = dataclasses.replace(s, n_loop_ipr=k)

    def batch_ms(sub, sset, lsx):
        L.run_ipr_batch(sub, scenes[:len(sub)], sset, lsx)  # warm-up
        runs = [L.run_ipr_batch(sub, scenes[:len(sub)], sset, lsx) for _ in range(args.learn_reps)]
        best = sorted(runs, key=lambda m: m["ms"])[len(runs) // 2]
        return {kk: round(v, 5) for kk, v in best.items()}

    plain_one = [batch_ms([ctxs[i]], s, None) for i in range(B)]
    plain_one_ms = sum(m["ms"] for m in plain_one)
    plain_one_n = sum(m["n"] for m in plain_one)
    plain_one_true = sum(m["true_particles_per_s"] * m["ms"] * 1e-3 for m in plain_one)
    plain_b = batch_ms(ctxs, s, None)
    learned_b = batch_ms(ctxs, sk, cfg)
    for c in ctxs:
        c.close()
    batched = {
        "frames": B, "ppp": 0.02,
        "plain_one_at_a_time": {"ms_per_frame": round(plain_one_ms / B, 3),
                                "particles_per_s": round(plain_one_n / (plain_one_ms * 1e-3)),
                                "true_particles_per_s": round(plain_one_true / (plain_one_ms * 1e-3))},
        "plain_batched": dict(plain_b, ms_per_frame=round(plain_b["ms"] / B, 3)),
        "learned_batched": dict(learned_b, ms_per_frame=round(learned_b["ms"] / B, 3)),
        "learned_batched_vs_plain": {
            "frames_per_s": round(plain_one_ms / learned_b["ms"], 3),
            "particles_per_s": round(learned_b["particles_per_s"] / (plain_one_n / (plain_one_ms * 1e-3)), 3),
            "true_particles_per_s": round(learned_b["true_particles_per_s"] / (plain_one_true / (plain_one_ms * 1e-3)), 3)},
    }
    return {
        "workload": "4 pinhole cams, 1024^2 uint8, a=200, OTF b,c ~ U[0.3,0.8], noise 2; "
                    "plain = olpt_ipr_run 4 loops x 4 shakes; learned = MLP proposal + 1 "
                    "refine shake, calibrated loop count; eval: device time per IPR, L2 "
                    "flushed; batched: wall time, frames on concurrent contexts/streams",
        "batched": batched,
        "train": {"frames": args.learn_ipr_frames, "tuples": n_tuples, "steps": len(losses),
                  "collect_s": round(t_collect, 1), "train_s": round(t_train, 1),
                  "loss_first": round(losses[0], 4),
                  "loss_last50": round(float(np.mean(losses[-50:])), 4)},
        "calibrated": {"n_loop_ipr": k, "ghost_logit": cfg.ghost_logit,
                       "fallback_residual": cfg.fallback_residual,
                       "refine_loops": cfg.refine_loops, "refine_width_mm": cfg.refine_width_mm},
        "eval": evals,
    }


# ----------------------------------------------------------------------------- detection
DET_SIZE, DET_CAMS, DET_PPP = 2048, 6, 0.1


def render_spots(rng, H, W, n, amp=3000.0, noise=20.0, bits=12):
    """n Gaussian spots (a exp(-0.5 (dx^2 + dy^2)), 7 x 7 window, fused by max) on
    Gaussian noise, rounded and clipped to `bits` bits, uint16."""
    im = np.zeros((H, W))
    ys, xs = rng.uniform(-3, H + 3, n), rng.uniform(-3, W + 3, n)
    for dy in range(-3, 4):
        for dx in range(-3, 4):
            r = np.floor(ys).astype(np.int64) + dy
            c = np.floor(xs).astype(np.int64) + dx
            ok = (r >= 0) & (r < H) & (c >= 0) & (c < W)
            v = amp * np.exp(-0.5 * ((r - ys) ** 2 + (c - xs) ** 2))
            np.maximum.at(im, (r[ok], c[ok]), v[ok])
    im += rng.normal(0, noise, im.shape)
    return np.clip(np.round(im), 0, 2 ** bits - 1).astype(np.uint16)


def detection_roofline(args, o: Ours):
    """The detection kernel alone at the image size of the 6-camera 2048^2 uint16
    configuration (0.1 ppp of seeded spots per image): device time per launch with the
    L2 flushed before each launch (the flush is queued on the library stream just
    before the launch, so the events time the device work only), against HBM."""
    from pyopenlpt_b200 import _ffi
    torch = o.torch
    rng = np.random.default_rng(2024)
    n_spots = int(DET_PPP * DET_SIZE * DET_SIZE)
    imgs = [render_spots(rng, DET_SIZE, DET_SIZE, n_spots) for _ in range(DET_CAMS)]
    sc = synth.make_scene(n_particles=10, size=512, focal=2500.0, seed=1)
    ctx = _ffi.Context(o.local)
    ctx.upload_cameras([_ffi.camera_desc_from_pinhole(sc.cams[0])] * DET_CAMS)
    ctx.upload_images(imgs)
    stream = torch.cuda.ExternalStream(ctx.stream())
    for _ in range(args.warmup):
        counts = ctx.find_peaks(300)
    ctx.profile(True)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            o.flush.zero_()
        counts = ctx.find_peaks(300)
    ms, n, img_bytes = ctx.profile_read(_ffi.PROF_PEAKS)
    ctx.profile(False)
    ctx.close()
    peak, peak_kind = measured_peak_hbm()
    dets = int(counts.sum())
    # algorithmic bytes: the image read once + 8 B per detection (an FP32 x, y pair);
    # the kernel writes FP64 x, y and the int32 peak pixel (24 B per detection), which
    # is stated beside it
    algo = img_bytes / n + 8.0 * dets
    written = img_bytes / n + 24.0 * dets
    sec = ms / n * 1e-3
    achieved = algo / sec / 1e9
    return {"kernel": "detect_kernel<uint16_t> (staged single read)",
            "images": f"{DET_CAMS} x {DET_SIZE}x{DET_SIZE} uint16 (12-bit), {n_spots} spots "
                      f"each (0.1 ppp), noise sigma 20, threshold 300",
            "detections_per_launch": dets, "launch_us": round(ms / n * 1e3, 2),
            "bytes_per_launch": algo,
            "bytes_per_launch_note": "image + 8 B per detection (FP32 x, y)",
            "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "launches": n,
            "bytes_moved_per_launch": written,
            "bytes_moved_note": "image + 24 B per detection as written (FP64 x, y, int32 "
                                "row/col)",
            "achieved_moved": written / sec / 1e9,
            "timing": "CUDA events on the library stream, L2 flushed before each launch"}


def run_ours(args):
    o = Ours(args)
    learned = None
    if o.world == 1 and args.learn_ipr_frames > 0:
        learned = learned_comparison(args, o)
        o.torch.cuda.synchronize()
    pre = {} if learned is None else {"learned_ipr_1024_u8": learned}
    if o.world == 1 and not args.no_detection_roofline:
        pre["detection_roofline"] = detection_roofline(args, o)
        o.torch.cuda.synchronize()
    kind = WORKLOADS[args.workload]["kind"]
    if kind == "ipr":
        run_ours_ipr(args, o, pre)
    elif kind == "batch":
        run_ours_batch(args, o, pre)
    else:
        run_ours_stb(args, o, pre)
    if o.world > 1:
        o.dist.destroy_process_group()
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
    ap.add_argument("--no-fp64-check", action="store_true",
                    help="skip the FP32-vs-FP64 comparison of the STB workload")
    ap.add_argument("--no-detection-roofline", action="store_true",
                    help="skip the detection kernel's roofline measurement")
    ap.add_argument("--learn-frames", type=int, default=3,
                    help="frames of training tuples for the learned form of the STB "
                         "workload (0 = skip)")
    ap.add_argument("--learn-ipr-frames", type=int, default=24,
                    help="frames of training tuples for the learned single-frame IPR "
                         "comparison at 1024^2 (0 = skip)")
    ap.add_argument("--learn-steps", type=int, default=3000)
    ap.add_argument("--learn-tuples", type=int, default=2_000_000,
                    help="training tuples of the learned form on the STB workloads")
    ap.add_argument("--learn-reps", type=int, default=5)
    ap.add_argument("--learn-batch", type=int, default=4,
                    help="frames processed at once in the batched learned comparison")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
