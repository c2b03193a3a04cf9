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
