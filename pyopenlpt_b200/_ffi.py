"""ctypes binding of the C ABI in include/olpt.h (libolpt_cuda.so).

This is the thin Python view of the boundary: plain pointers and sizes, no torch
types.  It fails loudly when the CUDA library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libolpt_cuda.so")

OLPT_U8, OLPT_U16, OLPT_F32, OLPT_F64 = 0, 1, 2, 3
_DTYPES = {np.dtype(np.uint8): OLPT_U8, np.dtype(np.uint16): OLPT_U16,
           np.dtype(np.float32): OLPT_F32, np.dtype(np.float64): OLPT_F64}

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_u16p = C.POINTER(C.c_uint16)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)

MLP_IN, MLP_OUT, MLP_PARAMS = 493, 4, 259076   # the network of a 4-camera rig

# olpt_near_record: one near-tolerance 2D test of stereo matching
NEAR_RECORD = np.dtype([("kind", "<i4"), ("n_chosen", "<i4"), ("cam", "<i4"), ("id", "<i4"),
                        ("other_cam", "<i4"), ("other_id", "<i4"), ("margin_px", "<f8")])


class LearnedParams(C.Structure):
    """olpt_learned_params: the learned shake used inside IPR when enable != 0."""
    _fields_ = [("enable", C.c_int), ("out_scale_mm", C.c_double), ("ghost_logit", C.c_double),
                ("refine_loops", C.c_int), ("refine_width_mm", C.c_double),
                ("fallback_residual", C.c_double)]


class CameraDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int), ("n_row", C.c_int), ("n_col", C.c_int), ("is_active", C.c_int),
        ("cam_mtx", C.c_double * 9), ("n_dist", C.c_int), ("dist", C.c_double * 12),
        ("r_mtx", C.c_double * 9), ("t_vec", C.c_double * 3), ("r_inv", C.c_double * 9),
        ("t_inv", C.c_double * 3), ("ref_plane", C.c_int), ("plane", C.c_double * 2),
        ("n_coeff", C.c_int), ("u_coeffs", _dp), ("v_coeffs", _dp),
    ]


class Tuning(C.Structure):
    _fields_ = [("shake_warps_per_block", C.c_int), ("residual_threads", C.c_int),
                ("shake_regs", C.c_int)]


class SmParams(C.Structure):
    _fields_ = [("match_cam_count", C.c_int), ("idmap_cell_px", C.c_int),
                ("tol_2d_px", C.c_double), ("tol_3d_mm", C.c_double), ("limit", C.c_double * 6)]


def sm_params(settings, limit) -> SmParams:
    p = SmParams(match_cam_count=settings.match_cam_count, idmap_cell_px=settings.idmap_cell_px,
                 tol_2d_px=settings.tol_2d_px, tol_3d_mm=settings.tol_3d_mm)
    for i in range(6):
        p.limit[i] = limit[i]
    return p


class ShakeParams(C.Structure):
    _fields_ = [("shake_width", C.c_double), ("shakewidth_min", C.c_double),
                ("n_shake_loop", C.c_int), ("thred_ghost", C.c_double), ("ratio_augimg", C.c_int),
                ("radius_obj", C.c_double), ("tol_3d_mm", C.c_double), ("precision", C.c_int)]


def shake_params(settings, precision: int = 0) -> ShakeParams:
    return ShakeParams(shake_width=settings.shake_width, shakewidth_min=settings.shakewidth_min,
                       n_shake_loop=settings.n_shake_loop, thred_ghost=settings.thred_ghost,
                       ratio_augimg=settings.ratio_augimg, radius_obj=settings.radius_obj,
                       tol_3d_mm=settings.tol_3d_mm, precision=precision)


class OlptError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"olpt status {code}: {msg}")
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() "
                              "(the CUDA extension is required; there is no CPU path)")
        L = C.CDLL(LIB_PATH)
        L.olpt_last_error.restype = C.c_char_p
        L.olpt_last_error.argtypes = [C.c_void_p]
        L.olpt_ctx_destroy.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def mlp_dims(n_cam: int):
    """(n_in, n_params) of the learned proposal's network for a rig of n_cam cameras."""
    n_in = C.c_int()
    n_p = C.c_int64()
    rc = lib().olpt_mlp_dims(int(n_cam), C.byref(n_in), C.byref(n_p))
    if rc:
        raise OlptError(rc, f"mlp_dims: unsupported camera count {n_cam}")
    return n_in.value, n_p.value


def launch_count() -> int:
    """Kernel launches issued by libolpt_cuda.so in this process."""
    L = lib()
    L.olpt_launch_count.restype = C.c_int64
    return int(L.olpt_launch_count())


def _p(a: Optional[np.ndarray], t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def camera_desc_from_pinhole(cam, active: bool = True) -> CameraDesc:
    d = CameraDesc()
    d.type = 0
    d.n_row, d.n_col, d.is_active = cam.n_row, cam.n_col, int(active)
    K = [cam.fx, 0.0, cam.cx, 0.0, cam.fy, cam.cy, 0.0, 0.0, 1.0]
    for i in range(9):
        d.cam_mtx[i] = K[i]
    dist = list(cam.dist)
    d.n_dist = len(dist)
    for i, v in enumerate(dist):
        d.dist[i] = v
    R, Ri, T, Ti = cam.R.ravel(), cam.Rinv.ravel(), cam.T, cam.Tinv
    for i in range(9):
        d.r_mtx[i] = R[i]
        d.r_inv[i] = Ri[i]
    for i in range(3):
        d.t_vec[i] = T[i]
        d.t_inv[i] = Ti[i]
    return d


def camera_desc_from_poly(cam, active: bool = True) -> CameraDesc:
    """A POLYNOMIAL camera (n_coeff x 4 tables of coefficient, x, y, z powers); the
    descriptor keeps its coefficient arrays alive."""
    d = CameraDesc()
    d.type = 1
    d.n_row, d.n_col, d.is_active = cam.n_row, cam.n_col, int(active)
    d.ref_plane = int(cam.ref_plane)
    d.plane[0], d.plane[1] = float(cam.plane[0]), float(cam.plane[1])
    u = np.ascontiguousarray(cam.u_coeffs, dtype=np.float64)
    v = np.ascontiguousarray(cam.v_coeffs, dtype=np.float64)
    d.n_coeff = len(u)
    d.u_coeffs, d.v_coeffs = _p(u), _p(v)
    d._keep = (u, v)
    return d


def camera_desc(cam, active: bool = True) -> CameraDesc:
    """Descriptor of a synth camera of either model."""
    if hasattr(cam, "u_coeffs"):
        return camera_desc_from_poly(cam, active)
    return camera_desc_from_pinhole(cam, active)


class Context:
    """One olpt_ctx (one CUDA stream + device-resident rig state)."""

    def __init__(self, device: int = 0):
        self.L = lib()
        h = C.c_void_p()
        self._check(self.L.olpt_ctx_create(C.byref(h), device), None)
        self.h = h
        self.n_cam = 0

    def _check(self, rc: int, h=None):
        if rc != 0:
            msg = self.L.olpt_last_error(h if h is not None else self.h).decode() \
                if (h is not None or getattr(self, "h", None)) else ""
            raise OlptError(rc, msg)

    def close(self):
        if getattr(self, "h", None):
            self.L.olpt_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- rig
    def upload_cameras(self, descs: Sequence[CameraDesc]):
        arr = (CameraDesc * len(descs))(*descs)
        self._keep = descs
        self._check(self.L.olpt_cameras_upload(self.h, arr, len(descs)))
        self.n_cam = len(descs)

    def set_active(self, active: Sequence[int]):
        a = (C.c_int * self.n_cam)(*[int(x) for x in active])
        self._check(self.L.olpt_cameras_set_active(self.h, a))

    def upload_otf(self, nx: int, ny: int, nz: int, bound6, abca: np.ndarray):
        b = np.ascontiguousarray(bound6, dtype=np.float64)
        t = np.ascontiguousarray(abca, dtype=np.float64)
        self._check(self.L.olpt_otf_upload(self.h, nx, ny, nz, _p(b), _p(t)))

    def project(self, cam: int, xyz: np.ndarray) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        uv = np.empty((len(xyz), 2))
        self._check(self.L.olpt_camera_project(self.h, cam, C.c_int64(len(xyz)), _p(xyz), _p(uv)))
        return uv

    def los(self, cam: int, uv: np.ndarray) -> np.ndarray:
        uv = np.ascontiguousarray(uv, dtype=np.float64).reshape(-1, 2)
        out = np.empty((len(uv), 6))
        self._check(self.L.olpt_camera_los(self.h, cam, C.c_int64(len(uv)), _p(uv), _p(out)))
        return out

    def triangulate(self, lines: np.ndarray):
        """lines: (n_sets, k, 6) -> (out (n_sets, 4), ok (n_sets,))"""
        lines = np.ascontiguousarray(lines, dtype=np.float64)
        n, k = lines.shape[0], lines.shape[1]
        out = np.empty((n, 4))
        ok = np.empty(n, dtype=np.int32)
        self._check(self.L.olpt_triangulate(self.h, C.c_int64(n), k, _p(lines), _p(out), _p(ok, _i32p)))
        return out, ok.astype(bool)

    def otf_param(self, cam: int, xyz: np.ndarray) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        out = np.empty((len(xyz), 5))
        self._check(self.L.olpt_otf_param(self.h, cam, C.c_int64(len(xyz)), _p(xyz), _p(out)))
        return out

    # ---------------------------------------------------------------- images
    def upload_images(self, imgs: Sequence[np.ndarray]):
        imgs = [np.ascontiguousarray(im) for im in imgs]
        dt = _DTYPES[imgs[0].dtype]
        ptrs = (C.c_void_p * len(imgs))(*[im.ctypes.data for im in imgs])
        H = (C.c_int * len(imgs))(*[im.shape[0] for im in imgs])
        W = (C.c_int * len(imgs))(*[im.shape[1] for im in imgs])
        self._check(self.L.olpt_images_upload(self.h, len(imgs), dt, ptrs, H, W, None, 0))
        self._imgs_keep = imgs

    def upload_images_device(self, ptrs: Sequence[int], dtype: int, H, W, pitch=None):
        n = len(ptrs)
        p = (C.c_void_p * n)(*ptrs)
        h = (C.c_int * n)(*H)
        w = (C.c_int * n)(*W)
        pt = None if pitch is None else (C.c_int64 * n)(*pitch)
        self._check(self.L.olpt_images_upload(self.h, n, dtype, p, h, w, pt, 1))

    def image(self, cam: int, dtype=np.float64) -> np.ndarray:
        H, W = self._shape(cam)
        out = np.empty((H, W), dtype=dtype)
        self._check(self.L.olpt_image_download(self.h, cam, _DTYPES[np.dtype(dtype)],
                                               out.ctypes.data_as(C.c_void_p)))
        return out

    def _shape(self, cam: int):
        return self._imgs_keep[cam].shape

    # ---------------------------------------------------------------- detections
    def find_peaks(self, min_int: float):
        counts = np.zeros(self.n_cam, dtype=np.int64)
        self._check(self.L.olpt_find_peaks(self.h, C.c_double(min_int), _p(counts, _i64p)))
        return counts

    def otf_estimate(self, min_int: float, radius_obj: float, max_per_image: int = 1000):
        """olpt_otf_estimate on the context's planes: (a, b, c), or None when an image
        has no detection; and the number of window samples used."""
        abc = np.zeros(3)
        n = C.c_int64()
        self._check(self.L.olpt_otf_estimate(self.h, C.c_double(min_int), C.c_double(radius_obj),
                                             int(max_per_image), _p(abc), C.byref(n)))
        return (abc if n.value > 0 else None), n.value

    def get_peaks(self, cam: int, n: int):
        xy = np.empty((n, 2))
        rc = np.empty((n, 2), dtype=np.int32)
        self._check(self.L.olpt_get_peaks(self.h, cam, _p(xy), _p(rc, _i32p), C.c_int64(n)))
        return xy, rc

    def upload_detections(self, dets: Sequence[np.ndarray]):
        d = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 2) for x in dets]
        counts = np.array([len(x) for x in d], dtype=np.int64)
        ptrs = (_dp * len(d))(*[_p(x) for x in d])
        self._check(self.L.olpt_detections_upload(self.h, len(d), _p(counts, _i64p), ptrs))

    # ---------------------------------------------------------------- stereo
    def stereo_match(self, params: SmParams):
        nc = C.c_int64()
        nm = C.c_int64()
        self._check(self.L.olpt_stereo_match(self.h, C.byref(params), C.byref(nc), C.byref(nm)))
        return nc.value, nm.value

    def near_log_enable(self, band_px: float, capacity: int = 1 << 20):
        """Log every stereo 2D test whose distance is within band_px of tol_2d_px."""
        self._check(self.L.olpt_stereo_near_log_enable(self.h, C.c_double(band_px),
                                                       C.c_int64(capacity)))

    def near_log(self, cap: int = 1 << 20):
        """(records, total): the logged near-tolerance tests (NEAR_RECORD array) and how
        many were seen since the last enable / reset."""
        out = np.zeros(cap, dtype=NEAR_RECORD)
        n = C.c_int64()
        self._check(self.L.olpt_stereo_near_log_read(self.h, out.ctypes.data_as(C.c_void_p),
                                                     C.c_int64(cap), C.byref(n)))
        return out[:min(cap, n.value)], n.value

    def near_log_reset(self):
        self._check(self.L.olpt_stereo_near_log_reset(self.h))

    def candidates(self, n: int):
        ids = np.empty((n, self.n_cam), dtype=np.int32)
        e = np.empty(n)
        x = np.empty((n, 3))
        self._check(self.L.olpt_get_candidates(self.h, _p(ids, _i32p), _p(e), _p(x)))
        return ids, e, x

    def matches(self, n: int):
        ids = np.empty((n, self.n_cam), dtype=np.int32)
        x = np.empty((n, 3))
        self._check(self.L.olpt_get_matches(self.h, _p(ids, _i32p), _p(x)))
        return ids, x

    def prune_matches(self, ids: np.ndarray, e_check: np.ndarray, det_counts, active=None):
        """StereoMatch::pruneMatch on a candidate list (reference order) on the device;
        returns the kept flags."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        M, n = ids.shape
        e = np.ascontiguousarray(e_check, dtype=np.float64)
        cnt = np.ascontiguousarray(det_counts, dtype=np.int64)
        act = (C.c_int * n)(*([1] * n if active is None else [int(a) for a in active]))
        sel = np.zeros(M, dtype=np.uint8)
        self._check(self.L.olpt_prune_matches_device(
            self.h, n, C.c_int64(M), _p(ids, _i32p), _p(e), _p(cnt, _i64p), act,
            sel.ctypes.data_as(C.POINTER(C.c_uint8))))
        return sel.astype(bool)

    # ---------------------------------------------------------------- objects / shake
    def upload_objects(self, xyz: np.ndarray):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self._check(self.L.olpt_objects_upload(self.h, C.c_int64(len(xyz)), _p(xyz)))

    def n_objects(self) -> int:
        n = C.c_int64()
        self._check(self.L.olpt_objects_count(self.h, C.byref(n)))
        return n.value

    def objects(self):
        n = self.n_objects()
        xyz = np.empty((n, 3))
        uv = np.empty((n, self.n_cam, 2))
        fl = np.empty(n, dtype=np.uint8)
        sc = np.empty(n)
        self._check(self.L.olpt_objects_download(self.h, _p(xyz), _p(uv),
                                                 fl.ctypes.data_as(C.POINTER(C.c_uint8)), _p(sc)))
        return {"xyz": xyz, "uv": uv, "flags": fl.astype(np.int64), "score": sc}

    def shake(self, params: ShakeParams):
        self._check(self.L.olpt_shake(self.h, C.byref(params)))

    def residual(self, params: ShakeParams, use_flags: bool = False, make_current: bool = False):
        self._check(self.L.olpt_residual(self.h, C.byref(params), int(use_flags), int(make_current)))

    def residual_image(self, cam: int, shape, dtype=np.float64) -> np.ndarray:
        out = np.empty(shape, dtype=dtype)
        self._check(self.L.olpt_residual_download(self.h, cam, _DTYPES[np.dtype(dtype)],
                                                  out.ctypes.data_as(C.c_void_p)))
        return out

    # ---------------------------------------------------------------- IPR
    def ipr_run(self, params: "IprParams") -> int:
        n = C.c_int64()
        self._check(self.L.olpt_ipr_run(self.h, C.byref(params), C.byref(n)))
        return n.value

    def tuning(self):
        """(shake warps per block, residual threads per block, shake registers a thread)."""
        t = Tuning()
        self._check(self.L.olpt_tuning_get(self.h, C.byref(t)))
        return t.shake_warps_per_block, t.residual_threads, t.shake_regs

    def set_tuning(self, shake_warps: int, residual_threads: int, shake_regs: int = 64):
        self._check(self.L.olpt_tuning_set(
            self.h, C.byref(Tuning(shake_warps, residual_threads, shake_regs))))

    def autotune_ipr(self, params: "IprParams", reps: int = 2):
        """olpt_autotune_ipr on the current images: the fastest launch shapes (kept in the
        context) and their mean IPR time in ms."""
        t = Tuning()
        ms = C.c_double()
        cand = np.zeros(8)
        self._check(self.L.olpt_autotune_ipr(self.h, C.byref(params), int(reps), C.byref(t),
                                             C.byref(ms), _p(cand)))
        self.autotune_trials = dict(zip(tuning_candidates(), cand.tolist()))
        return (t.shake_warps_per_block, t.residual_threads, t.shake_regs), ms.value

    def ipr_result(self, n: int):
        xyz = np.empty((n, 3))
        uv = np.empty((n, self.n_cam, 2))
        self._check(self.L.olpt_ipr_result(self.h, _p(xyz), _p(uv)))
        return xyz, uv

    # ---------------------------------------------------------------- STB
    def stb_configure(self, params: "StbParams"):
        self._stb_params = params  # keeps output_path alive
        self._check(self.L.olpt_stb_configure(self.h, C.byref(params)))

    def stb_process_frame(self, frame: int):
        self._check(self.L.olpt_stb_process_frame(self.h, int(frame)))

    def stb_counts(self):
        """(sizes of long_active, short_active, long_inactive, exit), n_extended, n_new"""
        c = (C.c_int64 * 4)()
        ne = C.c_int64()
        nn = C.c_int64()
        self._check(self.L.olpt_stb_counts(self.h, c, C.byref(ne), C.byref(nn)))
        return tuple(c), ne.value, nn.value

    def stb_frame_image(self, cam: int, H: int, W: int) -> np.ndarray:
        """The image of one camera as processFrame leaves it (FP64)."""
        out = np.empty((H, W))
        self._check(self.L.olpt_stb_frame_image(self.h, cam, 3, _p(out)))
        return out

    def stb_frame_points(self, frame: int) -> int:
        """Track points with this frame id over the four lists."""
        n = C.c_int64(0)
        self._check(self.L.olpt_stb_frame_points(self.h, int(frame), C.byref(n)))
        return n.value

    def stb_frame_objects(self) -> np.ndarray:
        """Particles of the last frame (extended predictions, then new objects)."""
        n = C.c_int64(0)
        self._check(self.L.olpt_stb_frame_objects(self.h, C.byref(n), None))
        xyz = np.empty((n.value, 3))
        self._check(self.L.olpt_stb_frame_objects(self.h, C.byref(n), _p(xyz)))
        return xyz

    def stb_tracks(self, which: int):
        """Rows of one track list: (track_id int32, frame int32, xyz (n, 3))."""
        nt = C.c_int64()
        nr = C.c_int64()
        self._check(self.L.olpt_stb_track_rows(self.h, which, C.byref(nt), C.byref(nr)))
        n = nr.value
        tid = np.empty(n, np.int32)
        fr = np.empty(n, np.int32)
        xyz = np.empty((n, 3))
        self._check(self.L.olpt_stb_get_tracks(self.h, which, tid.ctypes.data_as(C.c_void_p),
                                               fr.ctypes.data_as(C.c_void_p), _p(xyz), C.c_int64(n)))
        return tid, fr, xyz

    def stb_set_tracks(self, which: int, tid, frame, xyz):
        tid = np.ascontiguousarray(tid, dtype=np.int32)
        frame = np.ascontiguousarray(frame, dtype=np.int32)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self._check(self.L.olpt_stb_set_tracks(self.h, which, tid.ctypes.data_as(C.c_void_p),
                                               frame.ctypes.data_as(C.c_void_p), _p(xyz),
                                               C.c_int64(len(tid))))

    def stb_save_tracks(self, which: int, path: str):
        self._check(self.L.olpt_stb_save_tracks(self.h, which, str(path).encode()))

    def stb_load_tracks(self, which: int, path: str):
        self._check(self.L.olpt_stb_load_tracks(self.h, which, str(path).encode()))

    def track_files_async(self, enable: bool = True):
        """Track files written by the context's writer thread while later calls run."""
        self._check(self.L.olpt_track_files_async(self.h, int(bool(enable))))

    def flush_track_files(self):
        self._check(self.L.olpt_track_files_flush(self.h))

    def format_fixed6(self, values) -> str:
        """The device formatter: '%.6f' of each value, one per line."""
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        n = C.c_int64()
        self._check(self.L.olpt_format_fixed6(self.h, _p(v), C.c_int64(v.size), None,
                                              C.c_int64(0), C.byref(n)))
        buf = C.create_string_buffer(max(n.value, 1))
        self._check(self.L.olpt_format_fixed6(self.h, _p(v), C.c_int64(v.size), buf,
                                              C.c_int64(n.value), C.byref(n)))
        return buf.raw[:n.value].decode()

    # ---------------------------------------------------------------- profiling
    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self.L.olpt_stream(self.h, C.byref(s)))
        return s.value or 0

    # ---------------------------------------------------------------- learned proposal
    def mlp_dims(self):
        """(n_in, n_params) of the network for this context's camera count."""
        cams = getattr(self, "n_cam", 0)
        return mlp_dims(cams if cams >= 2 else 4)

    def mlp_init(self, seed: int = 0):
        self._check(self.L.olpt_mlp_init(self.h, C.c_uint64(seed)))

    def mlp_set_params(self, flat: np.ndarray):
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        assert flat.size == self.mlp_dims()[1]
        self._check(self.L.olpt_mlp_set_params(self.h, _p(flat, _fp)))

    def mlp_get_params(self) -> np.ndarray:
        out = np.empty(self.mlp_dims()[1], np.float32)
        self._check(self.L.olpt_mlp_get_params(self.h, _p(out, _fp)))
        return out

    def mlp_forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.mlp_dims()[0])
        out = np.empty((len(x), MLP_OUT), np.float32)
        self._check(self.L.olpt_mlp_forward(self.h, C.c_int64(len(x)), _p(x, _fp), _p(out, _fp), 0))
        return out

    def mlp_forward_device(self, x_ptr: int, n: int, out_ptr: int):
        """Device pointers (e.g. torch tensors' data_ptr())."""
        self._check(self.L.olpt_mlp_forward(self.h, C.c_int64(n), C.c_void_p(x_ptr),
                                            C.c_void_p(out_ptr), 1))

    def mlp_train_step(self, x: np.ndarray, t: np.ndarray, lr: float = 1e-3,
                       ghost_weight: float = 1.0, update: bool = True, want_grad: bool = False):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.mlp_dims()[0])
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, MLP_OUT)
        loss = C.c_double()
        g = np.empty(self.mlp_dims()[1], np.float32) if want_grad else None
        self._check(self.L.olpt_mlp_train_step(self.h, C.c_int64(len(x)), _p(x, _fp), _p(t, _fp), 0,
                                               C.c_double(lr), C.c_double(ghost_weight),
                                               int(update), C.byref(loss), _p(g, _fp)))
        return (loss.value, g) if want_grad else loss.value

    def mlp_train(self, x: np.ndarray, t: np.ndarray, steps: int, batch: int = 8192,
                  lr: float = 2e-3, ghost_weight: float = 1.0, seed: int = 0) -> np.ndarray:
        """olpt_mlp_train: the dataset goes to the device once; returns the step losses."""
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.mlp_dims()[0])
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, MLP_OUT)
        losses = np.zeros(max(steps, 1), np.float32)
        self._check(self.L.olpt_mlp_train(self.h, C.c_int64(len(x)), _p(x, _fp), _p(t, _fp), 0,
                                          int(batch), int(steps), C.c_double(lr),
                                          C.c_double(ghost_weight), C.c_uint64(seed),
                                          _p(losses, _fp)))
        return losses[:steps]

    def mlp_train_step_device(self, x_ptr: int, t_ptr: int, n: int, lr: float,
                              ghost_weight: float = 1.0) -> float:
        loss = C.c_double()
        self._check(self.L.olpt_mlp_train_step(self.h, C.c_int64(n), C.c_void_p(x_ptr),
                                               C.c_void_p(t_ptr), 1, C.c_double(lr),
                                               C.c_double(ghost_weight), 1, C.byref(loss), None))
        return loss.value

    def mlp_features(self, params: ShakeParams) -> np.ndarray:
        n = self.n_objects()
        x = np.zeros((n, self.mlp_dims()[0]), np.float32)
        if n:
            self._check(self.L.olpt_mlp_features(self.h, C.byref(params), _p(x, _fp), 0))
        return x

    def learned_configure(self, p: LearnedParams):
        self._check(self.L.olpt_learned_configure(self.h, C.byref(p)))

    def shake_learned(self, params: ShakeParams):
        self._check(self.L.olpt_shake_learned(self.h, C.byref(params)))

    def learned_stats(self):
        a, b = C.c_int64(), C.c_int64()
        self._check(self.L.olpt_learned_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def bf16_gemm(self, a_bits: np.ndarray, b_bits: np.ndarray, bias=None, gelu=False):
        a = np.ascontiguousarray(a_bits, dtype=np.uint16)
        b = np.ascontiguousarray(b_bits, dtype=np.uint16)
        M, K = a.shape
        N = b.shape[0]
        bias = None if bias is None else np.ascontiguousarray(bias, dtype=np.float32)
        out = np.empty((M, N), np.float32)
        self._check(self.L.olpt_bf16_gemm(self.h, M, N, K, _p(a, _u16p), _p(b, _u16p),
                                          _p(bias, _fp), int(gelu), _p(out, _fp)))
        return out

    def profile(self, enable: bool):
        self._check(self.L.olpt_profile(self.h, int(enable)))

    def profile_read(self, kernel: int):
        ms = C.c_double()
        n = C.c_int64()
        b = C.c_double()
        self._check(self.L.olpt_profile_read(self.h, kernel, C.byref(ms), C.byref(n), C.byref(b)))
        return ms.value, n.value, b.value


PROF_PEAKS, PROF_STEREO, PROF_RESIDUAL, PROF_SHAKE, PROF_PF = 0, 1, 2, 3, 4
# host phases (wall clock): id = PROF_N + phase
PROF_N = 5
PH_DETECT, PH_STEREO, PH_PRUNE, PH_SHAKE, PH_OUTPUT, PH_TRACK, PH_GREEDY_HOST = range(
    PROF_N, PROF_N + 7)


class IprParams(C.Structure):
    _fields_ = [("min_obj_int", C.c_double), ("sm", SmParams), ("shake", ShakeParams),
                ("n_cam_reduced", C.c_int), ("n_loop_ipr", C.c_int),
                ("n_loop_ipr_reduced", C.c_int), ("n_obj2d_process_max", C.c_int64)]


def ipr_params(settings, limit, precision: int = 0) -> IprParams:
    return IprParams(min_obj_int=float(settings.min_obj_int), sm=sm_params(settings, limit),
                     shake=shake_params(settings, precision), n_cam_reduced=settings.n_cam_reduced,
                     n_loop_ipr=settings.n_loop_ipr, n_loop_ipr_reduced=settings.n_loop_ipr_reduced,
                     n_obj2d_process_max=settings.n_obj2d_process_max)


def tuning_candidates():
    """The autotuner's launch-shape candidates in trial order."""
    L = lib()
    n = C.c_int()
    arr = (Tuning * 8)()
    rc = L.olpt_tuning_candidates(arr, C.byref(n))
    if rc != 0:
        raise OlptError(rc, "olpt_tuning_candidates")
    return [(t.shake_warps_per_block, t.residual_threads, t.shake_regs) for t in arr[:n.value]]


def stb_process_frame_batch(ctxs: Sequence["Context"], frames: Sequence[int]):
    """olpt_stb_process_frame_batch: frame frames[i] of every context's sequence at once
    (persistent host workers, one stream per context)."""
    L = lib()
    arr = (C.c_void_p * len(ctxs))(*[c.h for c in ctxs])
    fr = (C.c_int * len(ctxs))(*[int(f) for f in frames])
    rc = L.olpt_stb_process_frame_batch(arr, len(ctxs), fr)
    if rc != 0:
        for c in ctxs:
            msg = L.olpt_last_error(c.h)
            if msg:
                raise OlptError(rc, msg.decode())
        raise OlptError(rc, "olpt_stb_process_frame_batch failed")


def ipr_run_batch(ctxs: Sequence["Context"], params: IprParams):
    """olpt_ipr_run_batch: every context's IPR at once (one host thread and stream each);
    returns the per-context object counts."""
    L = lib()
    arr = (C.c_void_p * len(ctxs))(*[c.h for c in ctxs])
    out = np.zeros(len(ctxs), dtype=np.int64)
    rc = L.olpt_ipr_run_batch(arr, len(ctxs), C.byref(params), _p(out, _i64p))
    if rc != 0:
        for c in ctxs:
            msg = L.olpt_last_error(c.h)
            if msg:
                raise OlptError(rc, msg.decode())
        raise OlptError(rc, "olpt_ipr_run_batch failed")
    return out


TRACK_LONG_ACTIVE, TRACK_SHORT_ACTIVE, TRACK_LONG_INACTIVE, TRACK_EXIT = 0, 1, 2, 3
TRACK_LISTS = ("long_active", "short_active", "long_inactive", "exit")


class StbParams(C.Structure):
    _fields_ = [("ipr", IprParams), ("frame_start", C.c_int), ("frame_end", C.c_int),
                ("n_initial_frames", C.c_int), ("radius_search_obj_mm", C.c_double),
                ("radius_search_track_mm", C.c_double), ("limit", C.c_double * 6),
                ("pf_n", C.c_int * 3), ("pf_r_mm", C.c_double), ("pf_nbin", C.c_int * 3),
                ("pf_smooth", C.c_int), ("pf_sigma", C.c_double * 3),
                ("output_path", C.c_char_p)]


def stb_params(ipr_settings, stb_settings, limit, frame_start: int, frame_end: int,
               precision: int = 0, output_path: Optional[str] = None) -> StbParams:
    """STB parameters from IPR/STB knobs in mm (voxel_to_mm already applied)."""
    p = StbParams(ipr=ipr_params(ipr_settings, limit, precision), frame_start=frame_start,
                  frame_end=frame_end, n_initial_frames=stb_settings.n_initial_frames,
                  radius_search_obj_mm=stb_settings.radius_search_obj,
                  radius_search_track_mm=stb_settings.radius_search_track,
                  pf_r_mm=stb_settings.pf_r, pf_smooth=1,
                  output_path=None if output_path is None else str(output_path).encode())
    for i in range(6):
        p.limit[i] = limit[i]
    p.pf_n[0], p.pf_n[1], p.pf_n[2] = stb_settings.pf_nx, stb_settings.pf_ny, stb_settings.pf_nz
    for i in range(3):
        p.pf_nbin[i] = 11
        p.pf_sigma[i] = 1.0
    return p
