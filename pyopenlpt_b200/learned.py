"""The learned proposal end to end: training tuples generated by the plain GPU
pipeline, training on the device kernels, calibration of the fallback threshold,
and evaluation against the generator's ground truth.

Tuples come from IPR loops run step by step through the C ABI exactly as
``olpt_ipr_run`` runs them (detection, stereo matching, shake, residual): for every
candidate of a loop, the features against the residual with all candidates
(``olpt_mlp_features``, the input the learned shake sees), the converged plain-shake
correction in units of ``out_scale_mm``, and a ghost label from the ground truth (no
particle within ``ghost_tol_mm`` of the converged position).
"""
from __future__ import annotations

import dataclasses
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
from scipy.spatial import cKDTree

from . import _ffi, synth


@dataclasses.dataclass
class LearnedSettings:
    out_scale_mm: float = 0.05
    ghost_tol_mm: float = 0.1
    ghost_logit: float = 5.0
    refine_loops: int = 1
    refine_width_mm: float = 0.02
    fallback_residual: float = 1e9

    def params(self, enable: bool = True) -> _ffi.LearnedParams:
        return _ffi.LearnedParams(enable=int(enable), out_scale_mm=self.out_scale_mm,
                                  ghost_logit=self.ghost_logit, refine_loops=self.refine_loops,
                                  refine_width_mm=self.refine_width_mm,
                                  fallback_residual=self.fallback_residual)


VOLUME = (-20.0, 20.0, -20.0, 20.0, -10.0, 10.0)


def scene(seed: int, ppp: float, size: int = 1024, n_cam: int = 4,
          bc: Optional[Tuple[float, float]] = None) -> synth.Scene:
    """A learned-proposal frame: 4 cameras, size^2 uint8, ppp * size^2 particles in the
    40 x 40 x 20 mm volume, the focal length chosen so that the volume fills the
    images (ppp then counts the illuminated area), OTF b, c uniform in [0.3, 0.8]
    unless given."""
    rng = np.random.default_rng(10_000 + seed)
    b, c = bc if bc is not None else rng.uniform(0.3, 0.8, 2)
    focal = min(synth.focal_for_volume(n_cam, size, VOLUME))
    return synth.make_scene(n_particles=int(ppp * size * size), n_cam=n_cam, size=size,
                            focal=focal, volume=VOLUME, b=float(b), c=float(c), seed=seed)


def rig_settings(rig, **over) -> Tuple[synth.IPRSettings, LearnedSettings]:
    """IPR and learned-shake knobs in pixels of the rig: shake width 0.25 px, tol_3d
    0.6 px, network output unit 0.5 px, ghost label beyond 1.5 px, refinement width
    0.1 px (mm per px from the largest image motion per mm at the volume's centre)."""
    c0 = 0.5 * (np.array(rig.volume[0::2]) + np.array(rig.volume[1::2]))
    mm_px = 1.0 / max(synth.px_per_mm(cm, c0) for cm in rig.cams)
    s = synth.IPRSettings(shake_width=0.25 * mm_px, tol_3d_mm=0.6 * mm_px, **over)
    s.match_cam_count = min(s.match_cam_count, len(rig.cams))
    ls = LearnedSettings(out_scale_mm=0.5 * mm_px, ghost_tol_mm=1.5 * mm_px,
                         refine_width_mm=0.1 * mm_px)
    return s, ls


def bind(ctx: _ffi.Context, sc: synth.Scene):
    """Cameras, OTF table and images of a frame into the context."""
    ctx.upload_cameras([_ffi.camera_desc_from_pinhole(c) for c in sc.cams])
    ctx.upload_otf(2, 2, 2, sc.volume, synth.otf_table_array(sc.n_cam, sc.otf_abc))
    ctx.upload_images(sc.images)


def collect(ctx: _ffi.Context, sc: synth.Scene, s: synth.IPRSettings,
            ls: LearnedSettings) -> Tuple[np.ndarray, np.ndarray]:
    """Training tuples of one frame: features (n x 493) and targets (n x 4)."""
    bind(ctx, sc)
    ctx.learned_configure(ls.params(enable=False))
    sm = _ffi.sm_params(s, sc.volume)
    sp = _ffi.shake_params(s, 0)
    tree = cKDTree(sc.xyz)
    tol0 = sm.tol_2d_px
    xs: List[np.ndarray] = []
    ts: List[np.ndarray] = []
    for loop in range(s.n_loop_ipr):
        sm.tol_2d_px = tol0 * 1.5 ** loop
        ctx.find_peaks(s.min_obj_int)
        _, nm = ctx.stereo_match(sm)
        if nm == 0:
            break
        x = ctx.mlp_features(sp)
        x0 = ctx.objects()["xyz"]
        ctx.shake(sp)
        o = ctx.objects()
        d, _ = tree.query(o["xyz"])
        t = np.zeros((nm, 4), np.float32)
        t[:, :3] = (o["xyz"] - x0) / ls.out_scale_mm
        t[:, 3] = (d > ls.ghost_tol_mm).astype(np.float32)
        xs.append(x)
        ts.append(t)
        ctx.residual(sp, use_flags=True, make_current=True)
    return np.concatenate(xs), np.concatenate(ts)


def train(ctx: _ffi.Context, x: np.ndarray, t: np.ndarray, steps: int, batch: int = 8192,
          lr: float = 2e-3, ghost_weight: float = 1.0, seed: int = 0) -> List[float]:
    """Adam on uniform mini-batches of the tuples held on the device (olpt_mlp_train),
    learning rate decayed by a cosine to 5% of lr; the step losses."""
    return [float(v) for v in ctx.mlp_train(x, t, steps, batch=batch, lr=lr,
                                            ghost_weight=ghost_weight, seed=seed)]


def train_from_host(ctx: _ffi.Context, x: np.ndarray, t: np.ndarray, steps: int,
                    batch: int = 8192, lr: float = 2e-3, ghost_weight: float = 1.0,
                    seed: int = 0, time_budget_s: Optional[float] = None) -> List[float]:
    """The same schedule with each mini-batch drawn on the host and copied
    (olpt_mlp_train_step per step)."""
    rng = np.random.default_rng(seed)
    losses = []
    t0 = time.perf_counter()
    n = len(x)
    for it in range(steps):
        idx = rng.integers(0, n, min(batch, n))
        a = lr * (0.05 + 0.95 * 0.5 * (1 + np.cos(np.pi * it / max(steps, 1))))
        losses.append(ctx.mlp_train_step(x[idx], t[idx], lr=a, ghost_weight=ghost_weight))
        if time_budget_s is not None and time.perf_counter() - t0 > time_budget_s:
            break
    return losses


def run_ipr_batch(ctxs: Sequence[_ffi.Context], scenes: Sequence[synth.Scene],
                  s: synth.IPRSettings, ls: Optional[LearnedSettings]) -> Dict[str, float]:
    """The frames at once (olpt_ipr_run_batch, one context each): metrics summed over
    the frames and the wall time of the whole batch."""
    for ctx, sc in zip(ctxs, scenes):
        bind(ctx, sc)
        ctx.learned_configure((ls or LearnedSettings()).params(enable=ls is not None))
    p = _ffi.ipr_params(s, scenes[0].volume)
    t0 = time.perf_counter()
    counts = _ffi.ipr_run_batch(ctxs, p)
    ms = 1e3 * (time.perf_counter() - t0)
    found = n_true = n_out = 0.0
    for ctx, sc, n in zip(ctxs, scenes, counts):
        xyz, _ = ctx.ipr_result(int(n))
        m = metrics(xyz, sc.xyz)
        found += m["recall_10"] * len(sc.xyz)
        n_true += len(sc.xyz)
        n_out += m["n"]
    return {"frames": float(len(ctxs)), "n": n_out, "recall_10": found / max(n_true, 1.0),
            "ms": ms, "particles_per_s": n_out / (ms * 1e-3),
            "true_particles_per_s": found / (ms * 1e-3)}


def metrics(xyz: np.ndarray, truth: np.ndarray) -> Dict[str, float]:
    """Recall and ghost rate at 0.05 and 0.1 mm, RMSE of the matched positions."""
    out: Dict[str, float] = {"n": float(len(xyz))}
    if len(xyz) == 0:
        return {**out, "recall_05": 0.0, "recall_10": 0.0, "ghost_05": 0.0, "ghost_10": 0.0,
                "rmse_mm": float("nan")}
    rt = cKDTree(xyz)
    gt = cKDTree(truth)
    d_truth, _ = rt.query(truth)
    d_rec, _ = gt.query(xyz)
    for tol, key in ((0.05, "05"), (0.1, "10")):
        out["recall_" + key] = float(np.mean(d_truth <= tol))
        out["ghost_" + key] = float(np.mean(d_rec > tol))
    ok = d_rec <= 0.1
    out["rmse_mm"] = float(np.sqrt(np.mean(d_rec[ok] ** 2))) if ok.any() else float("nan")
    return out


def run_ipr(ctx: _ffi.Context, sc: synth.Scene, s: synth.IPRSettings,
            ls: Optional[LearnedSettings]) -> Dict[str, float]:
    """One olpt_ipr_run on the frame, plain (ls None) or learned; metrics + wall ms."""
    bind(ctx, sc)
    ctx.learned_configure((ls or LearnedSettings()).params(enable=ls is not None))
    p = _ffi.ipr_params(s, sc.volume)
    t0 = time.perf_counter()
    n = ctx.ipr_run(p)
    ms = 1e3 * (time.perf_counter() - t0)
    xyz, _ = ctx.ipr_result(n)
    m = metrics(xyz, sc.xyz)
    m["ms"] = ms
    return m


def meets(m: Dict[str, float], plain: Dict[str, float], slack: float = 0.005) -> bool:
    """Recall within slack of the plain method's and no higher ghost rate, at both
    0.05 and 0.1 mm."""
    return all(m["recall_" + k] >= plain["recall_" + k] - slack and
               m["ghost_" + k] <= plain["ghost_" + k] for k in ("05", "10"))


def calibrate(ctx: _ffi.Context, sc: synth.Scene, s: synth.IPRSettings, ls: LearnedSettings,
              loops: Sequence[int] = (1, 2, 3, 4), logits: Sequence[float] = (5.0, 3.0),
              fallback_grid: Sequence[float] = (3.0, 1.0, 0.3, 0.1, 0.03, 0.0),
              slack: float = 0.005):
    """The fastest learned form that meets the plain method (s.n_loop_ipr loops) on a
    validation frame: fewest IPR loops first, then the ghost logit; if none does, the
    largest fallback threshold at the full loop count.  Returns (n_loop_ipr,
    settings, plain metrics, sweep)."""
    plain = run_ipr(ctx, sc, s, None)
    sweep = []
    for k in loops:
        sk = dataclasses.replace(s, n_loop_ipr=k)
        for g in logits:
            cand = dataclasses.replace(ls, ghost_logit=float(g), fallback_residual=1e9)
            m = run_ipr(ctx, sc, sk, cand)
            sweep.append(((k, g, 1e9), m))
            if meets(m, plain, slack):
                return k, cand, plain, sweep
    for thr in fallback_grid:
        cand = dataclasses.replace(ls, ghost_logit=float(logits[0]), fallback_residual=float(thr))
        m = run_ipr(ctx, sc, s, cand)
        sweep.append(((s.n_loop_ipr, logits[0], thr), m))
        if meets(m, plain, slack):
            return s.n_loop_ipr, cand, plain, sweep
    return s.n_loop_ipr, dataclasses.replace(ls, fallback_residual=0.0), plain, sweep


# ----------------------------------------------------------------------------- STB rigs
def bind_rig(ctx: _ffi.Context, rig) -> None:
    """Cameras (pinhole or polynomial) and OTF (uniform or a grid) of a scene or
    sequence into the context."""
    ctx.upload_cameras([_ffi.camera_desc(c) for c in rig.cams])
    if getattr(rig, "otf_table", None) is not None:
        ctx.upload_otf(*rig.otf_n, rig.volume, rig.otf_table)
    else:
        ctx.upload_otf(2, 2, 2, rig.volume, synth.otf_table_array(len(rig.cams), rig.otf_abc))


def collect_predictions(ctx: _ffi.Context, truth: np.ndarray, s: synth.IPRSettings,
                        ls: LearnedSettings, sigma_mm: Sequence[float], volume,
                        frac_random: float = 0.1, n_max: Optional[int] = None,
                        seed: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """Tuples at the starting points the STB frame loop shakes: true particles
    displaced by Gaussian noise (the predictions of live tracks; the sigmas are used
    in equal shares), plus ``frac_random`` of uniform points in the volume (the
    predictions of lost tracks).  Features against the residual with all of them,
    the converged plain-shake correction, and a ghost label (no true particle within
    ghost_tol_mm of the converged position).  The context holds the frame's images."""
    rng = np.random.default_rng(seed)
    base = truth if n_max is None or n_max >= len(truth) else truth[
        rng.choice(len(truth), n_max, replace=False)]
    parts = np.array_split(base, len(sigma_mm))
    starts = [p + rng.normal(0.0, sg, p.shape) for p, sg in zip(parts, sigma_mm)]
    lo = np.array(volume[0::2], dtype=np.float64)
    hi = np.array(volume[1::2], dtype=np.float64)
    n_rand = int(frac_random * len(base))
    starts.append(lo + (hi - lo) * rng.random((n_rand, 3)))
    x0 = np.concatenate(starts)
    sp = _ffi.shake_params(s, 0)
    ctx.upload_objects(x0)
    x = ctx.mlp_features(sp)
    ctx.shake(sp)
    o = ctx.objects()
    d, _ = cKDTree(truth).query(o["xyz"])
    t = np.zeros((len(x0), 4), np.float32)
    t[:, :3] = (o["xyz"] - x0) / ls.out_scale_mm
    t[:, 3] = (d > ls.ghost_tol_mm).astype(np.float32)
    return x, t


def collect_ipr(ctx: _ffi.Context, truth: np.ndarray, s: synth.IPRSettings, volume,
                ls: LearnedSettings, loops: int = 1) -> Tuple[np.ndarray, np.ndarray]:
    """IPR-candidate tuples of the frame in the context (the first ``loops`` IPR loops
    run step by step, as ``collect`` does for a scene)."""
    ctx.learned_configure(ls.params(enable=False))
    sm = _ffi.sm_params(s, volume)
    sp = _ffi.shake_params(s, 0)
    tree = cKDTree(truth)
    tol0 = sm.tol_2d_px
    xs: List[np.ndarray] = []
    ts: List[np.ndarray] = []
    for loop in range(loops):
        sm.tol_2d_px = tol0 * 1.5 ** loop
        ctx.find_peaks(s.min_obj_int)
        _, nm = ctx.stereo_match(sm)
        if nm == 0:
            break
        x = ctx.mlp_features(sp)
        x0 = ctx.objects()["xyz"]
        ctx.shake(sp)
        o = ctx.objects()
        d, _ = tree.query(o["xyz"])
        t = np.zeros((nm, 4), np.float32)
        t[:, :3] = (o["xyz"] - x0) / ls.out_scale_mm
        t[:, 3] = (d > ls.ghost_tol_mm).astype(np.float32)
        xs.append(x)
        ts.append(t)
        ctx.residual(sp, use_flags=True, make_current=True)
    if not xs:
        return np.zeros((0, ctx.mlp_dims()[0]), np.float32), np.zeros((0, 4), np.float32)
    return np.concatenate(xs), np.concatenate(ts)


def stb_state(ctx: _ffi.Context):
    """The four track lists of a tracker (rows of track id, frame, xyz)."""
    return [ctx.stb_tracks(w) for w in range(4)]


def set_stb_state(ctx: _ffi.Context, state) -> None:
    for w, (tid, fr, xyz) in enumerate(state):
        ctx.stb_set_tracks(w, tid, fr, xyz)
