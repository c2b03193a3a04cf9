"""Seeded synthetic LPT scenes: pinhole camera rigs, particle clouds and rendered
camera images, written in the reference's own file formats.

Camera files follow the PINHOLE layout read by ``Camera::loadParameters``
(src/srcMath/Camera.cpp:19-98 of OpenLPT); OTF files follow ``OTF::loadParam``
(src/srcSTB/OTF.cpp:195-243).  Rendering follows the reference fixture generator
(test/inputs/test_IPR/getTiffImg.py: per-particle Gaussian, max fusion), plus
additive Gaussian noise, clipping and rounding to the integer image type.

Everything here is plain numpy on the host: it produces *inputs* only.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional, Sequence

import numpy as np


@dataclasses.dataclass
class PinholeCam:
    n_row: int
    n_col: int
    fx: float
    fy: float
    cx: float
    cy: float
    R: np.ndarray          # 3x3 world -> camera
    T: np.ndarray          # 3
    dist: Sequence[float] = (0.0, 0.0, 0.0, 0.0, 0.0)

    @property
    def Rinv(self) -> np.ndarray:
        return self.R.T.copy()

    @property
    def Tinv(self) -> np.ndarray:
        return -(self.R.T @ self.T)

    def to_text(self) -> str:
        def row(v):
            return ",".join(repr(float(x)) for x in v)
        K = [[self.fx, 0.0, self.cx], [0.0, self.fy, self.cy], [0.0, 0.0, 1.0]]
        lines = [
            "# Camera Model: (PINHOLE/POLYNOMIAL)", "PINHOLE",
            "# Camera Calibration Error: ", "None",
            "# Pose Calibration Error: ", "None",
            "# Image Size: (n_row,n_col)", f"{self.n_row},{self.n_col}",
            "# Camera Matrix: ", row(K[0]), row(K[1]), row(K[2]),
            "# Distortion Coefficients: ", row(self.dist),
            "# Rotation Vector: ", "0.0,0.0,0.0",
            "# Rotation Matrix: ", row(self.R[0]), row(self.R[1]), row(self.R[2]),
            "# Inverse of Rotation Matrix: ", row(self.Rinv[0]), row(self.Rinv[1]), row(self.Rinv[2]),
            "# Translation Vector: ", row(self.T),
            "# Inverse of Translation Vector: ", row(self.Tinv),
        ]
        return "\n".join(lines) + "\n"

    def project(self, xyz: np.ndarray) -> np.ndarray:
        """Undistorted pinhole projection (numpy, float64) -> (N,2) [col,row]."""
        pc = xyz @ self.R.T + self.T
        u = pc[:, 0] / pc[:, 2] * self.fx + self.cx
        v = pc[:, 1] / pc[:, 2] * self.fy + self.cy
        return np.stack([u, v], axis=1)


def ring_rig(n_cam: int, n_row: int, n_col: int, focal: float, radius: float = 500.0,
             elevation_deg: float = 30.0, az_step_deg: float = 45.0) -> List[PinholeCam]:
    """Cameras on a horizontal ring, tilted down by ``elevation_deg``, all aimed at
    the origin (the BASELINE rig: R=500 mm, 45 deg spacing, 30 deg tilt)."""
    cams = []
    el = math.radians(elevation_deg)
    for i in range(n_cam):
        az = math.radians(az_step_deg * i)
        C = radius * np.array([math.cos(el) * math.cos(az), math.cos(el) * math.sin(az), math.sin(el)])
        fwd = -C / np.linalg.norm(C)
        up = np.array([0.0, 0.0, 1.0])
        right = np.cross(fwd, up)
        right /= np.linalg.norm(right)
        down = np.cross(fwd, right)
        R = np.stack([right, down, fwd])
        T = -R @ C
        cams.append(PinholeCam(n_row, n_col, focal, focal, (n_col - 1) / 2.0, (n_row - 1) / 2.0, R, T))
    return cams


def render(cam: PinholeCam, xyz: np.ndarray, a: float, b: float, c: float, noise_sigma: float,
           max_val: int, dtype, rng: np.random.Generator, half: int = 3) -> np.ndarray:
    """Max-fused Gaussian particle images, + N(0, sigma^2), clipped and rounded."""
    H, W = cam.n_row, cam.n_col
    img = np.zeros((H, W), dtype=np.float64)
    uv = cam.project(xyz)
    cu = np.rint(uv[:, 0]).astype(np.int64)
    cv = np.rint(uv[:, 1]).astype(np.int64)
    for dy in range(-half, half + 1):
        for dx in range(-half, half + 1):
            x = cu + dx
            y = cv + dy
            ok = (x >= 0) & (x < W) & (y >= 0) & (y < H)
            ddx = x[ok] - uv[ok, 0]
            ddy = y[ok] - uv[ok, 1]
            val = a * np.exp(-b * ddx * ddx - c * ddy * ddy)
            np.maximum.at(img, (y[ok], x[ok]), val)
    if noise_sigma > 0:
        img += rng.normal(0.0, noise_sigma, size=img.shape)
    img = np.clip(np.rint(img), 0, max_val)
    return img.astype(dtype)


@dataclasses.dataclass
class Scene:
    cams: List[PinholeCam]
    xyz: np.ndarray                  # ground truth (N,3)
    images: List[np.ndarray]         # per camera, native integer dtype
    volume: tuple                    # (xmin,xmax,ymin,ymax,zmin,zmax)
    otf_abc: tuple                   # (a, b, c)
    max_val: int

    @property
    def n_cam(self) -> int:
        return len(self.cams)


def make_scene(n_particles: int = 10000, n_cam: int = 4, size: int = 1024, focal: float = 5000.0,
               volume=(-20.0, 20.0, -20.0, 20.0, -10.0, 10.0), a: float = 200.0, b: float = 0.5,
               c: float = 0.5, noise: float = 2.0, bits: int = 8, seed: int = 1234,
               n_row: Optional[int] = None, n_col: Optional[int] = None,
               require_all_views: bool = True) -> Scene:
    """A single frame: uniform particles in ``volume`` seen by a ring rig.

    Defaults are the BASELINE single-frame IPR scene: 4 cams, 1024^2 uint8,
    f = 5000 px, 10,000 particles in a 40x40x20 mm box, a=200, b=c=0.5, sigma=2.
    """
    rng = np.random.default_rng(seed)
    n_row = n_row or size
    n_col = n_col or size
    cams = ring_rig(n_cam, n_row, n_col, focal)
    lo = np.array(volume[0::2])
    hi = np.array(volume[1::2])
    xyz = lo + (hi - lo) * rng.random((n_particles, 3))
    if require_all_views:
        keep = np.ones(len(xyz), dtype=bool)
        for cm in cams:
            uv = cm.project(xyz)
            keep &= (uv[:, 0] > 4) & (uv[:, 0] < n_col - 5) & (uv[:, 1] > 4) & (uv[:, 1] < n_row - 5)
        xyz = xyz[keep]
    max_val = (1 << bits) - 1
    dtype = np.uint8 if bits <= 8 else np.uint16
    images = [render(cm, xyz, a, b, c, noise, max_val, dtype, rng) for cm in cams]
    return Scene(cams, xyz, images, tuple(volume), (a, b, c), max_val)


def burgers_velocity(xyz: np.ndarray, center, gamma: float = 2e4, r_core: float = 8.0,
                     strain: float = 2.0, drift=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Burgers vortex along z through `center` (circulation gamma mm^2/s, core radius
    r_core mm, axial strain 1/s) plus a uniform drift; mm/s."""
    d = xyz - np.asarray(center)
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    r2 = x * x + y * y
    r2s = np.maximum(r2, 1e-12)
    ut_over_r = gamma / (2 * np.pi * r2s) * (1.0 - np.exp(-r2s / (r_core * r_core)))
    u = -ut_over_r * y - 0.5 * strain * x + drift[0]
    v = ut_over_r * x - 0.5 * strain * y + drift[1]
    w = strain * z + drift[2]
    return np.stack([u, v, w], axis=1)


def rk4(f, xyz: np.ndarray, dt: float) -> np.ndarray:
    k1 = f(xyz)
    k2 = f(xyz + 0.5 * dt * k1)
    k3 = f(xyz + 0.5 * dt * k2)
    k4 = f(xyz + dt * k3)
    return xyz + dt / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)


@dataclasses.dataclass
class Sequence_:
    cams: List[PinholeCam]
    frames: List[List[np.ndarray]]   # frames[t][cam] images
    truth: List[np.ndarray]          # truth[t] (N,3) positions
    ids: List[np.ndarray]            # truth[t] particle ids (re-seeded particles get new ids)
    volume: tuple
    otf_abc: tuple
    max_val: int
    dt: float

    @property
    def n_cam(self) -> int:
        return len(self.cams)


def make_sequence(n_particles: int = 51000, n_frames: int = 50, n_cam: int = 4,
                  n_row: int = 800, n_col: int = 1280, focal: float = 5000.0,
                  volume=(-30.0, 30.0, -20.0, 20.0, -15.0, 15.0), a: float = 3000.0,
                  b: float = 0.5, c: float = 0.5, noise: float = 20.0, bits: int = 12,
                  max_px_per_frame: float = 3.0, gamma: float = 2e4, r_core: float = 8.0,
                  strain: float = 2.0, drift=(20.0, 0.0, 0.0), seed: int = 1234,
                  with_images: bool = True) -> Sequence_:
    """Particles advected by a Burgers vortex plus drift (RK4, FP64); the time step
    gives at most `max_px_per_frame` pixels of image motion per frame; particles that
    leave the volume are re-seeded uniformly.  Defaults: the BASELINE STB sequence
    (51,000 particles, 4 x 1280x800 12-bit, 60x40x30 mm, 50 frames)."""
    rng = np.random.default_rng(seed)
    cams = ring_rig(n_cam, n_row, n_col, focal)
    lo = np.array(volume[0::2])
    hi = np.array(volume[1::2])
    center = 0.5 * (lo + hi)
    vel = lambda p: burgers_velocity(p, center, gamma, r_core, strain, drift)  # noqa: E731
    xyz = lo + (hi - lo) * rng.random((n_particles, 3))
    ids = np.arange(n_particles)
    next_id = n_particles
    # time step from the fastest image motion over a probe cloud
    probe = lo + (hi - lo) * rng.random((200000, 3))
    vmax = float(np.max(np.linalg.norm(vel(probe), axis=1)))
    mm_per_px = 500.0 / focal
    dt = max_px_per_frame * mm_per_px / max(vmax, 1e-9)
    max_val = (1 << bits) - 1
    dtype = np.uint8 if bits <= 8 else np.uint16
    frames, truth, idl = [], [], []
    for t in range(n_frames):
        truth.append(xyz.copy())
        idl.append(ids.copy())
        if with_images:
            frames.append([render(cm, xyz, a, b, c, noise, max_val, dtype, rng) for cm in cams])
        xyz = rk4(vel, xyz, dt)
        out = np.any((xyz < lo) | (xyz > hi), axis=1)
        k = int(out.sum())
        if k:
            xyz[out] = lo + (hi - lo) * rng.random((k, 3))
            ids[out] = np.arange(next_id, next_id + k)
            next_id += k
    return Sequence_(cams, frames, truth, idl, tuple(volume), (a, b, c), max_val, dt)


def otf_table_array(n_cam: int, abc, alpha: float = 0.0, n=(2, 2, 2)) -> np.ndarray:
    """Uniform OTF table [4][n_cam][nx*ny*nz] (a, b, c, alpha planes)."""
    ng = n[0] * n[1] * n[2]
    t = np.empty((4, n_cam, ng), dtype=np.float64)
    t[0], t[1], t[2], t[3] = abc[0], abc[1], abc[2], alpha
    return t


def otf_text(n_cam: int, volume, a: float, b: float, c: float, alpha: float = 0.0,
             nx: int = 2, ny: int = 2, nz: int = 2) -> str:
    """Uniform OTF table in the reference's OTF file layout."""
    ng = nx * ny * nz
    def block(v):
        return "\n".join(",".join(repr(float(v)) for _ in range(ng)) for _ in range(n_cam))
    return "\n".join([
        "# Size: (n_cam,nx,ny,nz,n_grid)", f"{n_cam},{nx},{ny},{nz},{ng}",
        "# Boundary: (xmin,xmax,ymin,ymax,zmin,zmax)", ",".join(repr(float(v)) for v in volume),
        "# a: (n_cam,n_grid)", block(a), "# b: (n_cam,n_grid)", block(b),
        "# c: (n_cam,n_grid)", block(c), "# alpha: (n_cam,n_grid)", block(alpha),
    ]) + "\n"


@dataclasses.dataclass
class IPRSettings:
    """Tracer/IPR knobs of the reference's object config (src/srcSTB/Config.cpp:199-253)."""
    min_obj_int: int = 30
    radius_obj: float = 2.0
    shake_width: float = 0.25
    n_shake_loop: int = 4
    thred_ghost: float = 0.1
    ratio_augimg: int = 2
    match_cam_count: int = 4
    idmap_cell_px: int = 4
    tol_2d_px: float = 1.0
    tol_3d_mm: float = 0.06
    n_cam_reduced: int = 0
    n_loop_ipr: int = 4
    n_loop_ipr_reduced: int = 2
    n_obj2d_process_max: int = 200000

    @property
    def shakewidth_min(self) -> float:
        return self.shake_width / 20


@dataclasses.dataclass
class STBSettings:
    """STB / predictive-field knobs of the reference's object config
    (src/srcSTB/Config.cpp:199-214); lengths in mm (voxel_to_mm = 1)."""
    radius_search_obj: float = 1.0
    n_initial_frames: int = 4
    radius_search_track: float = 1.0
    pf_nx: int = 11
    pf_ny: int = 11
    pf_nz: int = 6
    pf_r: float = 3.0


def write_raw_frame(path: str, img: np.ndarray):
    """The oracle's raw frame format: b"ORIM", int32 rows, int32 cols, int32 dtype."""
    code = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.float64): 3}[img.dtype]
    with open(path, "wb") as f:
        f.write(b"ORIM")
        f.write(np.array([img.shape[0], img.shape[1], code], dtype=np.int32).tobytes())
        f.write(np.ascontiguousarray(img).tobytes())


def write_tiff_frame(path: str, img: np.ndarray):
    """Uncompressed baseline TIFF (one strip, 8 or 16 bits, little-endian)."""
    img = np.ascontiguousarray(img)
    bits = {np.dtype(np.uint8): 8, np.dtype(np.uint16): 16}[img.dtype]
    rows, cols = img.shape
    data = img.astype("<u2" if bits == 16 else "u1").tobytes()
    entries = [(256, 3, 1, cols), (257, 3, 1, rows), (258, 3, 1, bits), (259, 3, 1, 1),
               (262, 3, 1, 1), (273, 4, 1, 8), (277, 3, 1, 1), (278, 3, 1, rows),
               (279, 4, 1, len(data)), (284, 3, 1, 1)]
    ifd = bytearray(np.array([len(entries)], "<u2").tobytes())
    for tag, typ, cnt, val in entries:
        ifd += np.array([tag, typ], "<u2").tobytes() + np.array([cnt], "<u4").tobytes()
        ifd += (np.array([val, 0], "<u2").tobytes() if typ == 3
                else np.array([val], "<u4").tobytes())
    ifd += bytes(4)
    with open(path, "wb") as f:
        f.write(b"II" + np.array([42], "<u2").tobytes() + np.array([8 + len(data)], "<u4").tobytes())
        f.write(data)
        f.write(bytes(ifd))


def write_stb_config(seq, folder: str, ipr: "IPRSettings", stb: STBSettings,
                     n_frames: Optional[int] = None, image_format: str = "raw") -> str:
    """Reference-format main config (BasicSetting::readConfig, Config.cpp:49-135), tracer
    config (readCommonConfig + TracerConfig::readConfig, Config.cpp:163-286), camera
    files, image lists with the frames ("raw": the oracle's raw format; "tif": TIFF),
    and the OTF file.  Returns the main config path."""
    os.makedirs(folder, exist_ok=True)
    n_frames = n_frames or len(seq.frames)
    cam_paths = []
    for i, cm in enumerate(seq.cams):
        p = os.path.join(folder, f"cam{i + 1}.txt")
        with open(p, "w") as f:
            f.write(cm.to_text())
        cam_paths.append(p)
    lists = []
    for i in range(seq.n_cam):
        names = []
        for t in range(n_frames):
            ext = "tif" if image_format == "tif" else "raw"
            nm = f"cam{i + 1}_{t:05d}.{ext}"
            if ext == "tif":
                write_tiff_frame(os.path.join(folder, nm), seq.frames[t][i])
            else:
                write_raw_frame(os.path.join(folder, nm), seq.frames[t][i])
            names.append(os.path.join(folder, nm))
        lp = f"cam{i + 1}ImageNames.txt"
        with open(os.path.join(folder, lp), "w") as f:
            f.write("\n".join(names) + "\n")
        lists.append(os.path.join(folder, lp))
    with open(os.path.join(folder, "otf.txt"), "w") as f:
        f.write(otf_text(seq.n_cam, seq.volume, *seq.otf_abc))
    tracer = os.path.join(folder, "tracerConfig.txt")
    with open(tracer, "w") as f:
        f.write("\n".join(str(v) for v in [
            stb.radius_search_obj, stb.n_initial_frames, stb.radius_search_track, ipr.shake_width,
            stb.pf_nx, stb.pf_ny, stb.pf_nz, stb.pf_r, ipr.n_loop_ipr, ipr.n_shake_loop,
            ipr.thred_ghost, ipr.tol_2d_px, ipr.tol_3d_mm, ipr.n_cam_reduced,
            ipr.n_loop_ipr_reduced, ipr.min_obj_int, ipr.radius_obj]) + "\n")
    main = os.path.join(folder, "config.txt")
    out_dir = os.path.join(folder, "out") + "/"
    lines = [f"0,{n_frames - 1}", "1", "0", str(seq.n_cam)]
    lines += [f"{p},{seq.max_val}" for p in cam_paths]
    lines += lists
    lines += [",".join(repr(float(v)) for v in seq.volume), "1.0", out_dir, "Tracer", tracer, "0"]
    with open(main, "w") as f:
        f.write("\n".join(lines) + "\n")
    return main


def write_scene_files(scene: Scene, folder: str) -> List[str]:
    """Write camera files (cam{i}.txt) and the OTF file; return camera paths."""
    os.makedirs(folder, exist_ok=True)
    paths = []
    for i, cm in enumerate(scene.cams):
        p = os.path.join(folder, f"cam{i + 1}.txt")
        with open(p, "w") as f:
            f.write(cm.to_text())
        paths.append(p)
    with open(os.path.join(folder, "otf.txt"), "w") as f:
        f.write(otf_text(scene.n_cam, scene.volume, *scene.otf_abc))
    return paths
