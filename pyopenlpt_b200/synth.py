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
    the origin (default: R=500 mm, 45 deg spacing, 30 deg tilt)."""
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
    otf_table: Optional[np.ndarray] = None   # [4][n_cam][nx*ny*nz] when not uniform
    otf_n: tuple = (2, 2, 2)

    @property
    def n_cam(self) -> int:
        return len(self.cams)


def make_scene(n_particles: int = 10000, n_cam: int = 4, size: int = 1024, focal: float = 5000.0,
               volume=(-20.0, 20.0, -20.0, 20.0, -10.0, 10.0), a: float = 200.0, b: float = 0.5,
               c: float = 0.5, noise: float = 2.0, bits: int = 8, seed: int = 1234,
               n_row: Optional[int] = None, n_col: Optional[int] = None,
               require_all_views: bool = True) -> Scene:
    """A single frame: uniform particles in ``volume`` seen by a ring rig.

    Defaults are the single-frame IPR scene of 4 cams, 1024^2 uint8, f = 5000 px,
    10,000 particles in a 40x40x20 mm box, a=200, b=c=0.5, sigma=2 (0.01 ppp).
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
    leave the volume are re-seeded uniformly.  Defaults: the STB sequence of 51,000
    particles (0.05 ppp), 4 x 1280x800 12-bit, 60x40x30 mm, 50 frames."""
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
        if getattr(seq, "otf_table", None) is not None:
            f.write(otf_text_table(seq.otf_table, seq.otf_n, seq.volume))
        else:
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
        if scene.otf_table is not None:
            f.write(otf_text_table(scene.otf_table, scene.otf_n, scene.volume))
        else:
            f.write(otf_text(scene.n_cam, scene.volume, *scene.otf_abc))
    return paths


# ----------------------------------------------------------------------------- polynomial rigs
# Exponent rows (px, py, pz) of a full cubic in (X, Y, Z): 20 monomials, constant first.
CUBIC_TERMS = [(i, j, k) for d in range(4) for i in range(d, -1, -1) for j in range(d - i, -1, -1)
               for k in [d - i - j]]


@dataclasses.dataclass
class PolyCam:
    """Camera of the reference's POLYNOMIAL model (Camera::polyProject,
    src/srcMath/Camera.cpp:969-990): u = sum_i cu_i X^pu_i Y^qu_i Z^ru_i, same for v;
    lines of sight by Newton inversion on the two reference planes (REF_Z here)."""
    n_row: int
    n_col: int
    u_coeffs: np.ndarray           # (n, 4): coefficient, x power, y power, z power
    v_coeffs: np.ndarray
    plane: tuple                   # the two REF_Z planes (z values, mm)
    ref_plane: int = 3

    def project(self, xyz: np.ndarray) -> np.ndarray:
        xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
        out = np.zeros((len(xyz), 2))
        for k, co in enumerate((self.u_coeffs, self.v_coeffs)):
            for c, px, py, pz in co:
                out[:, k] += c * xyz[:, 0] ** px * xyz[:, 1] ** py * xyz[:, 2] ** pz
        return out

    def to_text(self) -> str:
        """The POLYNOMIAL camera file (Camera::loadParameters, Camera.cpp:99-158)."""
        ref = {1: "REF_X", 2: "REF_Y", 3: "REF_Z"}[self.ref_plane]

        def rows(co):
            return [",".join(repr(float(v)) for v in r) for r in co]
        lines = ["# Camera Model: (PINHOLE/POLYNOMIAL)", "POLYNOMIAL",
                 "# Camera Calibration Error: ", "None",
                 "# Image Size: (n_row,n_col)", f"{self.n_row},{self.n_col}",
                 "# Reference Plane: (REF_X/REF_Y/REF_Z,coordinate,coordinate)",
                 f"{ref},{float(self.plane[0])!r},{float(self.plane[1])!r}",
                 "# Number of Coefficients: ", str(len(self.u_coeffs)),
                 "# U_Coeff (coefficient, x power, y power, z power)"] + rows(self.u_coeffs) + [
                 "# V_Coeff (coefficient, x power, y power, z power)"] + rows(self.v_coeffs)
        return "\n".join(lines) + "\n"


def focal_for_volume(n_cam: int, size: int, volume, fill: float = 0.92, **rig) -> List[float]:
    """Per camera of a ring rig, the focal length (px) at which the volume's corners
    project inside ``fill`` of the image, so the particles cover as much of every
    image as the box's outline allows."""
    lo = np.array(volume[0::2], dtype=np.float64)
    hi = np.array(volume[1::2], dtype=np.float64)
    corners = np.array([[lo[0] if i & 1 else hi[0], lo[1] if i & 2 else hi[1],
                         lo[2] if i & 4 else hi[2]] for i in range(8)])
    out = []
    for cm in ring_rig(n_cam, size, size, 1.0, **rig):
        uv = cm.project(corners) - np.array([cm.cx, cm.cy])
        out.append(fill * 0.5 * (size - 1) / float(np.max(np.abs(uv))))
    return out


def poly_rig(n_cam: int, size: int, volume, max_distortion_px: float = 2.0, seed: int = 0,
             **rig) -> List[PolyCam]:
    """Seeded cubic polynomial cameras: a ring rig of pinholes (focal sized to the
    volume) plus a radial and decentring distortion of at most ``max_distortion_px``
    at the image corners, fitted by least squares with the 20 monomials of a full cubic
    in (X, Y, Z) over the slab of the viewing frustum between the two reference planes
    (z = zmin and z = zmax of the volume), as a calibration with targets filling the
    view on both planes would.  The fitted polynomials are the cameras: images are
    rendered with them."""
    rng = np.random.default_rng(seed)
    focals = focal_for_volume(n_cam, size, volume, **rig)
    pins = [ring_rig(n_cam, size, size, f, **rig)[i] for i, f in enumerate(focals)]
    z0, z1 = float(volume[4]), float(volume[5])
    g = np.linspace(-0.02 * size, 1.02 * size, 33)
    pu, pv = [a.ravel() for a in np.meshgrid(g, g, indexing="ij")]
    A_terms = np.array(CUBIC_TERMS, dtype=np.float64)
    cams = []
    for pc in pins:
        # rays of the pixel grid, cut by 9 planes between the reference planes
        d_cam = np.stack([(pu - pc.cx) / pc.fx, (pv - pc.cy) / pc.fy, np.ones_like(pu)], axis=1)
        d_w = d_cam @ pc.R          # R^T d: directions in world coordinates
        o_w = pc.Tinv
        P = []
        for z in np.linspace(z0, z1, 9):
            s_ = (z - o_w[2]) / d_w[:, 2]
            P.append(o_w + s_[:, None] * d_w)
        P = np.concatenate(P)
        A = np.stack([P[:, 0] ** i * P[:, 1] ** j * P[:, 2] ** k for i, j, k in CUBIC_TERMS],
                     axis=1)
        uv = pc.project(P)
        d = uv - np.array([pc.cx, pc.cy])
        r_corner = math.hypot(pc.cx, pc.cy)
        r2 = (d * d).sum(axis=1) / (r_corner * r_corner)
        k_rad = rng.uniform(0.5, 1.0) * max_distortion_px / r_corner * rng.choice([-1.0, 1.0])
        t = rng.normal(0.0, 0.25 * max_distortion_px / r_corner, size=2)
        uvd = uv + d * (k_rad * r2)[:, None] + np.outer(r2, t) * r_corner
        cu, *_ = np.linalg.lstsq(A, uvd[:, 0], rcond=None)
        cv, *_ = np.linalg.lstsq(A, uvd[:, 1], rcond=None)
        cams.append(PolyCam(size, size, np.column_stack([cu, A_terms]),
                            np.column_stack([cv, A_terms]), (z0, z1)))
    return cams


# ----------------------------------------------------------------------------- OTF grids
def otf_grid(n_cam: int, n=(5, 5, 5), a_range=(2400.0, 3600.0), bc_range=(0.3, 0.9),
             seed: int = 0) -> np.ndarray:
    """Seeded spatially varying OTF table [4][n_cam][nx*ny*nz] (a, b, c, alpha = 0):
    a, b and c drawn uniformly per grid node, interpolated trilinearly in between."""
    rng = np.random.default_rng(seed)
    ng = n[0] * n[1] * n[2]
    t = np.zeros((4, n_cam, ng))
    t[0] = rng.uniform(*a_range, size=(n_cam, ng))
    t[1] = rng.uniform(*bc_range, size=(n_cam, ng))
    t[2] = rng.uniform(*bc_range, size=(n_cam, ng))
    return t


def otf_eval(table: np.ndarray, n, volume, cam: int, xyz: np.ndarray) -> np.ndarray:
    """(a, b, c) at each point: OTF::getOTFParam (src/srcSTB/OTF.cpp:273-338) --
    clamp to the box, trilinear interpolation in the grid cell (index x*ny*nz+y*nz+z)."""
    nx, ny, nz = n
    lo = np.array(volume[0::2], dtype=np.float64)
    hi = np.array(volume[1::2], dtype=np.float64)
    p = np.clip(np.asarray(xyz, dtype=np.float64).reshape(-1, 3), lo, hi)
    cells = np.array([nx, ny, nz]) - 1
    f = (p - lo) / (hi - lo) * cells
    i0 = np.clip(np.floor(f).astype(np.int64), 0, cells - 1)
    w = f - i0
    out = np.zeros((len(p), 3))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                idx = (i0[:, 0] + dx) * ny * nz + (i0[:, 1] + dy) * nz + (i0[:, 2] + dz)
                wt = ((w[:, 0] if dx else 1 - w[:, 0]) * (w[:, 1] if dy else 1 - w[:, 1])
                      * (w[:, 2] if dz else 1 - w[:, 2]))
                out += wt[:, None] * table[:3, cam, idx].T
    return out


def otf_text_table(table: np.ndarray, n, volume) -> str:
    """An OTF table [4][n_cam][n_grid] in the reference's OTF file layout
    (OTF::loadParam, src/srcSTB/OTF.cpp:195-243)."""
    n_cam, ng = table.shape[1], table.shape[2]

    def block(q):
        return "\n".join(",".join(repr(float(v)) for v in table[q, c]) for c in range(n_cam))
    return "\n".join([
        "# Size: (n_cam,nx,ny,nz,n_grid)", f"{n_cam},{n[0]},{n[1]},{n[2]},{ng}",
        "# Boundary: (xmin,xmax,ymin,ymax,zmin,zmax)", ",".join(repr(float(v)) for v in volume),
        "# a: (n_cam,n_grid)", block(0), "# b: (n_cam,n_grid)", block(1),
        "# c: (n_cam,n_grid)", block(2), "# alpha: (n_cam,n_grid)", block(3),
    ]) + "\n"


# ----------------------------------------------------------------------------- flows
def abc_velocity(xyz: np.ndarray, A: float = 1.0, B: float = 1.0, C_: float = 1.0,
                 wavelength: float = 40.0) -> np.ndarray:
    """Arnold-Beltrami-Childress flow, k = 2 pi / wavelength:
    u = A sin kz + C cos ky, v = B sin kx + A cos kz, w = C sin ky + B cos kx."""
    k = 2.0 * math.pi / wavelength
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    return np.stack([A * np.sin(k * z) + C_ * np.cos(k * y),
                     B * np.sin(k * x) + A * np.cos(k * z),
                     C_ * np.sin(k * y) + B * np.cos(k * x)], axis=1)


# ----------------------------------------------------------------------------- torch rendering
def _project_torch(cm, P):
    """The camera's projection of torch points P (n, 3) float64 (pinhole without
    distortion, or the cubic polynomial)."""
    import torch
    if isinstance(cm, PolyCam):
        out = []
        for co in (cm.u_coeffs, cm.v_coeffs):
            acc = torch.zeros(len(P), dtype=torch.float64, device=P.device)
            for c, px, py, pz in co:
                acc = acc + float(c) * P[:, 0] ** int(px) * P[:, 1] ** int(py) * P[:, 2] ** int(pz)
            out.append(acc)
        return torch.stack(out, dim=1)
    R = torch.as_tensor(cm.R, dtype=torch.float64, device=P.device)
    T = torch.as_tensor(cm.T, dtype=torch.float64, device=P.device)
    pc = P @ R.T + T
    return torch.stack([pc[:, 0] / pc[:, 2] * cm.fx + cm.cx, pc[:, 1] / pc[:, 2] * cm.fy + cm.cy],
                       dim=1)


def _otf_torch(table, n, volume, cam, P):
    """otf_eval on torch points."""
    import torch
    nx, ny, nz = n
    lo = torch.tensor(volume[0::2], dtype=torch.float64, device=P.device)
    hi = torch.tensor(volume[1::2], dtype=torch.float64, device=P.device)
    p = torch.minimum(torch.maximum(P, lo), hi)
    cells = torch.tensor([nx - 1, ny - 1, nz - 1], device=P.device)
    f = (p - lo) / (hi - lo) * cells
    i0 = torch.minimum(torch.clamp(torch.floor(f).long(), min=0), cells - 1)
    w = f - i0
    tab = torch.as_tensor(table[:3, cam], dtype=torch.float64, device=P.device)  # (3, ng)
    out = torch.zeros((len(P), 3), dtype=torch.float64, device=P.device)
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                idx = (i0[:, 0] + dx) * ny * nz + (i0[:, 1] + dy) * nz + (i0[:, 2] + dz)
                wt = ((w[:, 0] if dx else 1 - w[:, 0]) * (w[:, 1] if dy else 1 - w[:, 1])
                      * (w[:, 2] if dz else 1 - w[:, 2]))
                out += wt[:, None] * tab[:, idx].T
    return out


def render_frame(cams, xyz: np.ndarray, otf_table: np.ndarray, otf_n, volume,
                 noise: np.ndarray, max_val: int, dtype, device="cpu", half: int = 3):
    """Render one frame of every camera with torch on ``device``: per particle its
    projection by the camera's own model and its (a, b, c) from the OTF table,
    a exp(-b dx^2 - c dy^2) over a (2 half + 1)^2 window, fused by max, plus the given
    noise planes (n_cam, H, W), rounded and clipped.  Returns numpy (n_cam, H, W)
    ``dtype``."""
    import torch
    P = torch.from_numpy(np.ascontiguousarray(xyz, dtype=np.float64)).to(device)
    out = []
    for ci, cm in enumerate(cams):
        H, W = cm.n_row, cm.n_col
        uv = _project_torch(cm, P)
        abc = _otf_torch(otf_table, otf_n, volume, ci, P)
        img = torch.zeros(H * W, dtype=torch.float64, device=device)
        cu = torch.round(uv[:, 0]).long()
        cv = torch.round(uv[:, 1]).long()
        for dy in range(-half, half + 1):
            for dx in range(-half, half + 1):
                x = cu + dx
                y = cv + dy
                ok = (x >= 0) & (x < W) & (y >= 0) & (y < H)
                ddx = x[ok].double() - uv[ok, 0]
                ddy = y[ok].double() - uv[ok, 1]
                val = abc[ok, 0] * torch.exp(-abc[ok, 1] * ddx * ddx - abc[ok, 2] * ddy * ddy)
                img.scatter_reduce_(0, y[ok] * W + x[ok], val, reduce="amax")
        img = img.view(H, W) + torch.from_numpy(noise[ci]).to(device, torch.float64)
        img = torch.clamp(torch.round(img), 0, max_val)
        out.append(img.to(torch.int32).cpu().numpy().astype(dtype))
    return np.stack(out)


@dataclasses.dataclass
class PolySequence:
    """A particle sequence seen by polynomial cameras with a spatially varying OTF."""
    cams: List[PolyCam]
    frames: List[np.ndarray]         # frames[t]: (n_cam, H, W) images
    truth: List[np.ndarray]          # truth[t]: (N, 3) positions
    ids: List[np.ndarray]
    volume: tuple
    otf_table: np.ndarray            # [4][n_cam][nx*ny*nz]
    otf_n: tuple
    max_val: int
    dt: float

    @property
    def n_cam(self) -> int:
        return len(self.cams)


def px_per_mm(cam, at) -> float:
    """Largest image motion (px) per mm of world motion at point ``at`` (the spectral
    norm of the projection's Jacobian, central differences)."""
    at = np.asarray(at, dtype=np.float64).reshape(1, 3)
    J = np.stack([(cam.project(at + e) - cam.project(at - e))[0] / 2e-3
                  for e in np.eye(3) * 1e-3], axis=1)
    return float(np.linalg.norm(J, 2))


def make_poly_sequence(ppp: float = 0.1, n_frames: int = 100, n_cam: int = 6, size: int = 2048,
                       volume=(-40.0, 40.0, -40.0, 40.0, -20.0, 20.0), bits: int = 16,
                       noise_sigma: float = 20.0, otf_n=(5, 5, 5), a_range=(2400.0, 3600.0),
                       bc_range=(0.3, 0.9), max_px_per_frame: float = 4.0,
                       wavelength: float = 40.0, max_distortion_px: float = 2.0,
                       seed: int = 1234, device="cpu", with_images: bool = True) -> PolySequence:
    """Particles advected by ABC flow (A = B = C = 1, RK4 in FP64) seen by ``n_cam``
    cubic polynomial cameras (seeded, at most ``max_distortion_px`` of distortion at
    the corners), images of size^2 pixels with ppp * size^2 particles in ``volume``
    (whose projection fills the images), a seeded 5x5x5 OTF grid (a in a_range, b and
    c in bc_range), Gaussian noise, ``bits``-bit integer images.  The time step gives
    at most ``max_px_per_frame`` of image motion; particles leaving the volume are
    re-seeded uniformly.  Defaults: 6 cameras, 2048^2 uint16, 0.1 ppp (419,430
    particles), 80x80x40 mm, 100 frames."""
    rng = np.random.default_rng(seed)
    cams = poly_rig(n_cam, size, volume, max_distortion_px, seed=seed + 1)
    table = otf_grid(n_cam, otf_n, a_range, bc_range, seed=seed + 2)
    n = int(round(ppp * size * size))
    lo = np.array(volume[0::2], dtype=np.float64)
    hi = np.array(volume[1::2], dtype=np.float64)
    xyz = lo + (hi - lo) * rng.random((n, 3))
    ids = np.arange(n)
    next_id = n
    vel = lambda p: abc_velocity(p, wavelength=wavelength)  # noqa: E731
    probe = lo + (hi - lo) * rng.random((100000, 3))
    vmax = float(np.max(np.linalg.norm(vel(probe), axis=1)))
    # image motion per mm: the largest over the cameras at the volume's centre
    c0 = 0.5 * (lo + hi)
    ppm = max(px_per_mm(cm, c0) for cm in cams)
    dt = max_px_per_frame / (ppm * max(vmax, 1e-9))
    max_val = (1 << bits) - 1 if bits < 16 else 65535
    dtype = np.uint8 if bits <= 8 else np.uint16
    frames, truth, idl = [], [], []
    for t in range(n_frames):
        truth.append(xyz.copy())
        idl.append(ids.copy())
        if with_images:
            nz = rng.standard_normal((n_cam, size, size), dtype=np.float32) * noise_sigma
            frames.append(render_frame(cams, xyz, table, otf_n, volume, nz, max_val, dtype,
                                       device))
        xyz = rk4(vel, xyz, dt)
        out = np.any((xyz < lo) | (xyz > hi), axis=1)
        k = int(out.sum())
        if k:
            xyz[out] = lo + (hi - lo) * rng.random((k, 3))
            ids[out] = np.arange(next_id, next_id + k)
            next_id += k
    return PolySequence(cams, frames, truth, idl, tuple(volume), table, tuple(otf_n), max_val, dt)


def make_poly_scene(ppp: float = 0.02, size: int = 512, n_cam: int = 6,
                    volume=(-10.0, 10.0, -10.0, 10.0, -5.0, 5.0), bits: int = 12,
                    noise_sigma: float = 20.0, seed: int = 7, **kw) -> Scene:
    """One frame of make_poly_sequence as a Scene (polynomial cameras, 5x5x5 OTF)."""
    seq = make_poly_sequence(ppp=ppp, n_frames=1, n_cam=n_cam, size=size, volume=volume,
                             bits=bits, noise_sigma=noise_sigma, seed=seed, **kw)
    a_mid = float(np.mean(seq.otf_table[0]))
    return Scene(seq.cams, seq.truth[0], list(seq.frames[0]), seq.volume,
                 (a_mid, float(np.mean(seq.otf_table[1])), float(np.mean(seq.otf_table[2]))),
                 seq.max_val, otf_table=seq.otf_table, otf_n=seq.otf_n)


# ----------------------------------------------------------------------------- many sequences
def taylor_green_velocity(xyz: np.ndarray, wavelength: float, phase=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Taylor-Green cells (u = sin kx cos ky cos kz, v = -cos kx sin ky cos kz, w = 0,
    k = 2 pi / wavelength, shifted by ``phase`` in mm): divergence-free, unit peak speed."""
    k = 2.0 * math.pi / wavelength
    x = k * (xyz[:, 0] + phase[0])
    y = k * (xyz[:, 1] + phase[1])
    z = k * (xyz[:, 2] + phase[2])
    return np.stack([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z),
                     np.zeros_like(x)], axis=1)


def make_tg_sequence(n_particles: int, n_cam: int, size: int, n_frames: int = 20,
                     wavelength: float = 40.0, volume=(-20.0, 20.0, -20.0, 20.0, -10.0, 10.0),
                     a: float = 200.0, b: float = 0.5, c: float = 0.5, noise: float = 2.0,
                     max_px_per_frame: float = 3.0, seed: int = 0,
                     device="cpu") -> PolySequence:
    """One sequence of the many-sequence batch: ``n_cam`` pinhole cameras on the ring
    rig (focal sized so the volume fills the size^2 images), 8-bit images with a uniform
    Gaussian OTF (a, b, c) and noise, particles advected by Taylor-Green cells of the
    given wavelength (random phase; RK4 in FP64; at most ``max_px_per_frame`` of image
    motion), re-seeded uniformly when they leave the volume."""
    rng = np.random.default_rng(seed)
    focal = min(focal_for_volume(n_cam, size, volume))
    cams = ring_rig(n_cam, size, size, focal)
    table = otf_table_array(n_cam, (a, b, c))
    lo = np.array(volume[0::2], dtype=np.float64)
    hi = np.array(volume[1::2], dtype=np.float64)
    phase = tuple(rng.uniform(0.0, wavelength, 3))
    vel = lambda p: taylor_green_velocity(p, wavelength, phase)  # noqa: E731
    ppm = max(px_per_mm(cm, 0.5 * (lo + hi)) for cm in cams)
    dt = max_px_per_frame / ppm  # unit peak speed
    xyz = lo + (hi - lo) * rng.random((n_particles, 3))
    ids = np.arange(n_particles)
    next_id = n_particles
    frames, truth, idl = [], [], []
    for t in range(n_frames):
        truth.append(xyz.copy())
        idl.append(ids.copy())
        nz = rng.standard_normal((n_cam, size, size), dtype=np.float32) * noise
        frames.append(render_frame(cams, xyz, table, (2, 2, 2), volume, nz, 255, np.uint8, device))
        xyz = rk4(vel, xyz, dt)
        out = np.any((xyz < lo) | (xyz > hi), axis=1)
        k = int(out.sum())
        if k:
            xyz[out] = lo + (hi - lo) * rng.random((k, 3))
            ids[out] = np.arange(next_id, next_id + k)
            next_id += k
    return PolySequence(cams, frames, truth, idl, tuple(volume), table, (2, 2, 2), 255, dt)


def batch_plan(n_seq: int = 64, seed: int = 2024, n_min: int = 2000, n_max: int = 80000):
    """Seeded shapes of the many-sequence batch: per sequence (particles log-uniform in
    [n_min, n_max], cameras in 4..6, image size in {512, 1024, 2048}, wavelength
    uniform in [20, 60] mm, seed)."""
    rng = np.random.default_rng(seed)
    plan = []
    for i in range(n_seq):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        plan.append(dict(n_particles=n, n_cam=int(rng.integers(4, 7)),
                         size=int(rng.choice([512, 1024, 2048])),
                         wavelength=float(rng.uniform(20.0, 60.0)), seed=seed + 1 + i))
    return plan
