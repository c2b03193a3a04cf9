"""Test infrastructure only: ctypes access to the two CPU oracles.

* ``RefOracle``  -- the reference OpenLPT C++ core compiled from its own sources
  (oracle/_ref/liboref.so, see oracle/Makefile), driven through ref_driver.cpp.
* ``Restated``   -- this directory's C restatement (oracle/_ref/libolpt_oracle.so).

Nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "liboref.so")
ORACLE_SO = os.path.join(HERE, "_ref", "libolpt_oracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Cfg(C.Structure):
    _fields_ = [
        ("n_cam", C.c_int), ("min_obj_int", C.c_int), ("radius_obj", C.c_double),
        ("shake_width", C.c_double), ("n_shake_loop", C.c_int), ("thred_ghost", C.c_double),
        ("shakewidth_min", C.c_double), ("ratio_augimg", C.c_int),
        ("match_cam_count", C.c_int), ("idmap_cell_px", C.c_int), ("tol_2d_px", C.c_double),
        ("tol_3d_mm", C.c_double), ("limit", C.c_double * 6),
        ("n_cam_reduced", C.c_int), ("n_loop_ipr", C.c_int), ("n_loop_ipr_reduced", C.c_int),
        ("n_obj2d_process_max", C.c_int),
        ("radius_search_obj", C.c_double), ("n_initial_frames", C.c_int),
        ("radius_search_track", C.c_double),
        ("pf_nx", C.c_int), ("pf_ny", C.c_int), ("pf_nz", C.c_int), ("pf_r", C.c_double),
        ("otf_nx", C.c_int), ("otf_ny", C.c_int), ("otf_nz", C.c_int),
        ("otf_bound", C.c_double * 6), ("otf_abca", _dp),
    ]


def _as_dp(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _ptr_array(arrs: Sequence[np.ndarray]):
    t = (_dp * len(arrs))()
    for i, a in enumerate(arrs):
        t[i] = _as_dp(a)
    return t


def otf_table(n_cam: int, abc, alpha: float = 0.0, n=(2, 2, 2)) -> np.ndarray:
    ng = n[0] * n[1] * n[2]
    t = np.empty((4, n_cam, ng), dtype=np.float64)
    t[0], t[1], t[2], t[3] = abc[0], abc[1], abc[2], alpha
    return t


class RefOracle:
    """The reference implementation, loaded from oracle/_ref/liboref.so."""

    def __init__(self, scene, settings, limit=None, otf=None, otf_n=(2, 2, 2),
                 workdir: Optional[str] = None, threads: int = 0):
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} missing: run `make -C oracle`")
        self.lib = lib = C.CDLL(REF_SO)
        for name in ("oref_find_peaks", "oref_stereo", "oref_shake", "oref_residual", "oref_ipr",
                     "oref_cams_new", "oref_cfg_new"):
            getattr(lib, name).restype = C.c_void_p
        lib.oref_res_len.restype = C.c_longlong
        lib.oref_res_len.argtypes = [C.c_void_p, C.c_char_p]
        lib.oref_res_copy.argtypes = [C.c_void_p, C.c_char_p, _dp]
        lib.oref_res_free.argtypes = [C.c_void_p]
        lib.oref_last_error.restype = C.c_char_p
        lib.oref_set_threads(int(threads))
        self.scene = scene
        self.n_cam = scene.n_cam
        self._tmp = workdir or tempfile.mkdtemp(prefix="oref_")
        from pyopenlpt_b200.synth import write_scene_files
        paths = write_scene_files(scene, self._tmp)
        arr = (C.c_char_p * len(paths))(*[p.encode() for p in paths])
        self.cams = lib.oref_cams_new(len(paths), arr)
        if not self.cams:
            raise RuntimeError(lib.oref_last_error().decode())
        s = settings
        lim = limit if limit is not None else scene.volume
        if otf is None and getattr(scene, "otf_table", None) is not None:
            otf, otf_n = scene.otf_table, scene.otf_n
        self.otf = otf if otf is not None else otf_table(self.n_cam, scene.otf_abc, n=otf_n)
        self.otf = np.ascontiguousarray(self.otf, dtype=np.float64)
        cfg = _Cfg(n_cam=self.n_cam, min_obj_int=s.min_obj_int, radius_obj=s.radius_obj,
                   shake_width=s.shake_width, n_shake_loop=s.n_shake_loop,
                   thred_ghost=s.thred_ghost, shakewidth_min=s.shakewidth_min,
                   ratio_augimg=s.ratio_augimg, match_cam_count=s.match_cam_count,
                   idmap_cell_px=s.idmap_cell_px, tol_2d_px=s.tol_2d_px, tol_3d_mm=s.tol_3d_mm,
                   n_cam_reduced=s.n_cam_reduced, n_loop_ipr=s.n_loop_ipr,
                   n_loop_ipr_reduced=s.n_loop_ipr_reduced,
                   n_obj2d_process_max=s.n_obj2d_process_max,
                   radius_search_obj=1.0, n_initial_frames=4, radius_search_track=1.0,
                   pf_nx=2, pf_ny=2, pf_nz=2, pf_r=1.0,
                   otf_nx=otf_n[0], otf_ny=otf_n[1], otf_nz=otf_n[2],
                   otf_abca=_as_dp(self.otf))
        for i in range(6):
            cfg.limit[i] = lim[i]
            cfg.otf_bound[i] = scene.volume[i]
        self._cfg_struct = cfg
        self.cfg = lib.oref_cfg_new(C.byref(cfg), C.c_void_p(self.cams))

    # ------------------------------------------------------------ helpers
    def _take(self, h, names: List[str]):
        if not h:
            raise RuntimeError("reference call failed: " + self.lib.oref_last_error().decode())
        h = C.c_void_p(h)
        out = {}
        for n in names:
            ln = self.lib.oref_res_len(h, n.encode())
            if ln < 0:
                continue
            a = np.empty(ln, dtype=np.float64)
            if ln:
                self.lib.oref_res_copy(h, n.encode(), _as_dp(a))
            out[n] = a
        self.lib.oref_res_free(h)
        return out

    def _imgs(self, imgs):
        d = [np.ascontiguousarray(im, dtype=np.float64) for im in imgs]
        H = (C.c_int * len(d))(*[im.shape[0] for im in d])
        W = (C.c_int * len(d))(*[im.shape[1] for im in d])
        return d, _ptr_array(d), H, W

    def srand(self, seed: int):
        """Seed the C library's rand() (the polynomial camera's Newton start points)."""
        self.lib.oref_srand(C.c_uint(seed))

    def set_active(self, active: Sequence[int]):
        a = (C.c_int * self.n_cam)(*[int(x) for x in active])
        self.lib.oref_cams_set_active(C.c_void_p(self.cams), a)

    # ------------------------------------------------------------ stages
    def project(self, cam: int, xyz: np.ndarray) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        uv = np.empty((len(xyz), 2))
        rc = self.lib.oref_project(C.c_void_p(self.cams), cam, C.c_longlong(len(xyz)), _as_dp(xyz), _as_dp(uv))
        assert rc == 0
        return uv

    def los(self, cam: int, uv: np.ndarray) -> np.ndarray:
        uv = np.ascontiguousarray(uv, dtype=np.float64).reshape(-1, 2)
        out = np.empty((len(uv), 6))
        rc = self.lib.oref_los(C.c_void_p(self.cams), cam, C.c_longlong(len(uv)), _as_dp(uv), _as_dp(out))
        assert rc == 0
        return out

    def triangulate(self, lines6: np.ndarray):
        lines6 = np.ascontiguousarray(lines6, dtype=np.float64).reshape(-1, 6)
        out = np.empty(4)
        rc = self.lib.oref_triangulate(len(lines6), _as_dp(lines6), _as_dp(out))
        return (None if rc != 0 else out)

    def otf_param(self, cam: int, xyz: np.ndarray) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        out = np.empty((len(xyz), 5))
        self.lib.oref_otf_param(C.c_void_p(self.cfg), cam, C.c_longlong(len(xyz)), _as_dp(xyz), _as_dp(out))
        return out

    def find_peaks(self, img: np.ndarray) -> np.ndarray:
        d = np.ascontiguousarray(img, dtype=np.float64)
        h = self.lib.oref_find_peaks(C.c_void_p(self.cfg), _as_dp(d), d.shape[0], d.shape[1])
        return self._take(h, ["xy"])["xy"].reshape(-1, 2)

    def stereo(self, dets: Sequence[np.ndarray]):
        d = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 2) for x in dets]
        counts = (C.c_longlong * len(d))(*[len(x) for x in d])
        h = self.lib.oref_stereo(C.c_void_p(self.cams), C.c_void_p(self.cfg), len(d), counts, _ptr_array(d))
        r = self._take(h, ["cand", "e_check", "sel", "kept", "xyz", "uv", "ref_cam"])
        n = self.n_cam
        return {
            "cand": r["cand"].reshape(-1, n).astype(np.int64),
            "e_check": r["e_check"],
            "sel": r["sel"].reshape(-1, n).astype(np.int64),
            "kept": r["kept"].astype(bool),
            "xyz": r["xyz"].reshape(-1, 3),
            "ref_cam": int(r["ref_cam"][0]),
        }

    def shake(self, xyz: np.ndarray, imgs):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        d, p, H, W = self._imgs(imgs)
        h = self.lib.oref_shake(C.c_void_p(self.cams), C.c_void_p(self.cfg), C.c_longlong(len(xyz)),
                                _as_dp(xyz), self.n_cam, p, H, W)
        r = self._take(h, ["xyz", "flags", "score", "uv"])
        return {"xyz": r["xyz"].reshape(-1, 3), "flags": r["flags"].astype(np.int64),
                "score": r["score"], "uv": r["uv"].reshape(len(xyz), self.n_cam, 2)}

    def residual(self, xyz: np.ndarray, imgs, flags=None):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        d, p, H, W = self._imgs(imgs)
        fl = None
        if flags is not None:
            fl = np.ascontiguousarray(flags, dtype=np.int32)
        h = self.lib.oref_residual(C.c_void_p(self.cams), C.c_void_p(self.cfg), C.c_longlong(len(xyz)),
                                   _as_dp(xyz), fl.ctypes.data_as(_ip) if fl is not None else None,
                                   self.n_cam, p, H, W)
        r = self._take(h, [f"img{c}" for c in range(self.n_cam)])
        return [r[f"img{c}"].reshape(d[c].shape) for c in range(self.n_cam)]

    def otf_estimate(self, cam: int, imgs):
        """OTF::estimateUniformOTFFromImage of camera `cam` on its images: (a, b, c, alpha)
        of the estimate, or None when the reference skipped it."""
        d, p, H, W = self._imgs(imgs)
        out = np.zeros(4)
        rc = self.lib.oref_otf_estimate(C.c_void_p(self.cfg), cam, len(d), p, H, W, _as_dp(out))
        if rc < 0:
            raise RuntimeError(self.lib.oref_last_error().decode())
        return None if rc == 1 else out

    def ipr(self, imgs):
        d, p, H, W = self._imgs(imgs)
        h = self.lib.oref_ipr(C.c_void_p(self.cams), C.c_void_p(self.cfg), self.n_cam, p, H, W)
        r = self._take(h, ["xyz", "uv"])
        return {"xyz": r["xyz"].reshape(-1, 3), "uv": r["uv"].reshape(-1, self.n_cam, 2)}

    def close(self):
        if getattr(self, "cfg", None):
            self.lib.oref_cfg_free(C.c_void_p(self.cfg))
            self.cfg = None
        if getattr(self, "cams", None):
            self.lib.oref_cams_free(C.c_void_p(self.cams))
            self.cams = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefSTB:
    """The reference STB (processFrame) on a synthetic sequence, built from
    reference-format config files written by synth.write_stb_config."""

    def __init__(self, seq, ipr_settings, stb_settings, workdir: Optional[str] = None,
                 threads: int = 0, n_frames: Optional[int] = None, otf_override: bool = True,
                 match_cam_count: Optional[int] = None):
        from pyopenlpt_b200.synth import write_stb_config
        self.lib = lib = C.CDLL(REF_SO)
        lib.oref_stb_new.restype = C.c_void_p
        lib.oref_stb_tracks.restype = C.c_void_p
        lib.oref_res_len.restype = C.c_longlong
        lib.oref_res_len.argtypes = [C.c_void_p, C.c_char_p]
        lib.oref_res_copy.argtypes = [C.c_void_p, C.c_char_p, _dp]
        lib.oref_res_free.argtypes = [C.c_void_p]
        lib.oref_last_error.restype = C.c_char_p
        lib.oref_set_threads(int(threads))
        self.seq = seq
        self._tmp = workdir or tempfile.mkdtemp(prefix="oref_stb_")
        main = write_stb_config(seq, self._tmp, ipr_settings, stb_settings, n_frames=n_frames)
        self.main_config = main
        otf = os.path.join(self._tmp, "otf.txt") if otf_override else ""
        self.h = lib.oref_stb_new(main.encode(), otf.encode())
        if not self.h:
            raise RuntimeError(lib.oref_last_error().decode())
        if match_cam_count is not None:
            lib.oref_stb_set_match_cam_count(C.c_void_p(self.h), int(match_cam_count))

    def frame(self, t: int, imgs=None):
        imgs = imgs if imgs is not None else self.seq.frames[t]
        d = [np.ascontiguousarray(im, dtype=np.float64) for im in imgs]
        H = (C.c_int * len(d))(*[im.shape[0] for im in d])
        W = (C.c_int * len(d))(*[im.shape[1] for im in d])
        rc = self.lib.oref_stb_frame(C.c_void_p(self.h), t, len(d), _ptr_array(d), H, W)
        if rc != 0:
            raise RuntimeError(self.lib.oref_last_error().decode())

    def tracks(self):
        h = C.c_void_p(self.lib.oref_stb_tracks(C.c_void_p(self.h)))
        out = {}
        for name in ("long_active", "short_active", "long_inactive", "exit"):
            n = self.lib.oref_res_len(h, name.encode())
            a = np.empty(max(n, 0))
            if n > 0:
                self.lib.oref_res_copy(h, name.encode(), _as_dp(a))
            out[name] = a.reshape(-1, 5)
        self.lib.oref_res_free(h)
        return out

    def otf(self) -> np.ndarray:
        """The OTF table the reference tracks with, [4][n_cam][n_grid]."""
        self.lib.oref_stb_otf.restype = C.c_int
        ng = self.lib.oref_stb_otf(C.c_void_p(self.h), None)
        out = np.empty((4, self.seq.n_cam, ng))
        self.lib.oref_stb_otf(C.c_void_p(self.h), _as_dp(out))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.oref_stb_free(C.c_void_p(self.h))
            self.h = None
