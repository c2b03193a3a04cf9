"""Test infrastructure only: ctypes view of the C restatement (libolpt_oracle.so)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_ref", "libolpt_oracle.so")
_dp = C.POINTER(C.c_double)


class Pinhole(C.Structure):
    _fields_ = [("fx", C.c_double), ("fy", C.c_double), ("cx", C.c_double), ("cy", C.c_double),
                ("n_dist", C.c_int), ("dist", C.c_double * 12), ("R", C.c_double * 9),
                ("T", C.c_double * 3), ("Rinv", C.c_double * 9), ("Tinv", C.c_double * 3)]


class Poly(C.Structure):
    _fields_ = [("n_coeff", C.c_int), ("ref_plane", C.c_int), ("plane", C.c_double * 2),
                ("u", _dp), ("v", _dp)]


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Restated:
    def __init__(self):
        if not os.path.exists(SO):
            raise FileNotFoundError(f"{SO} missing: run `make -C oracle oracle-only`")
        self.L = L = C.CDLL(SO)
        L.oo_find_peaks.restype = C.c_int64
        L.oo_find_peaks.argtypes = [_dp, C.c_int, C.c_int, C.c_double, _dp, C.c_int64]
        L.oo_triangulate.argtypes = [_dp, C.c_int, _dp]
        L.oo_residual.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int64, _dp, _dp, C.c_double, C.c_int]
        L.oo_otf_param.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_int, C.c_int, _dp, _dp]
        self._keep = []

    @staticmethod
    def pinhole(p) -> Pinhole:
        """p: pyopenlpt_b200.camfile.CameraParams (PINHOLE) or synth.PinholeCam"""
        c = Pinhole()
        if hasattr(p, "cam_mtx") and p.cam_mtx is not None:
            K = p.cam_mtx
            c.fx, c.fy, c.cx, c.cy = K[0, 0], K[1, 1], K[0, 2], K[1, 2]
            dist = list(p.dist)
        else:
            c.fx, c.fy, c.cx, c.cy = p.fx, p.fy, p.cx, p.cy
            dist = list(p.dist)
        c.n_dist = len(dist)
        for i, v in enumerate(dist):
            c.dist[i] = v
        for i, v in enumerate(np.ravel(p.R)):
            c.R[i] = v
        for i, v in enumerate(np.ravel(p.Rinv)):
            c.Rinv[i] = v
        for i, v in enumerate(np.ravel(p.T)):
            c.T[i] = v
        for i, v in enumerate(np.ravel(p.Tinv)):
            c.Tinv[i] = v
        return c

    def poly(self, p) -> Poly:
        u, v = _d(p.u_coeffs), _d(p.v_coeffs)
        self._keep += [u, v]
        c = Poly(n_coeff=len(u), ref_plane=p.ref_plane, u=u.ctypes.data_as(_dp), v=v.ctypes.data_as(_dp))
        c.plane[0], c.plane[1] = p.plane
        return c

    def _vec_call(self, fn, cam, pts, n_in, n_out):
        pts = _d(pts).reshape(-1, n_in)
        out = np.empty((len(pts), n_out))
        for i in range(len(pts)):
            fn(C.byref(cam), pts[i].ctypes.data_as(_dp), out[i].ctypes.data_as(_dp))
        return out

    def project(self, cam, xyz):
        return self._vec_call(self.L.oo_pinhole_project, cam, xyz, 3, 2)

    def world_to_undist(self, cam, xyz):
        return self._vec_call(self.L.oo_pinhole_world_to_undist, cam, xyz, 3, 2)

    def distort(self, cam, xy):
        return self._vec_call(self.L.oo_pinhole_distort, cam, xy, 2, 2)

    def undistort(self, cam, uv):
        return self._vec_call(self.L.oo_pinhole_undistort, cam, uv, 2, 2)

    def los(self, cam, uv):
        return self._vec_call(self.L.oo_pinhole_los, cam, uv, 2, 6)

    def poly_project(self, cam, xyz):
        return self._vec_call(self.L.oo_poly_project, cam, xyz, 3, 2)

    def find_peaks(self, img, min_int):
        img = _d(img)
        H, W = img.shape
        cap = H * W // 2 + 1
        out = np.empty((cap, 2))
        n = self.L.oo_find_peaks(img.ctypes.data_as(_dp), H, W, float(min_int), out.ctypes.data_as(_dp), cap)
        return out[:n].copy()

    def triangulate(self, lines6):
        lines6 = _d(lines6).reshape(-1, 6)
        out = np.empty(4)
        rc = self.L.oo_triangulate(lines6.ctypes.data_as(_dp), len(lines6), out.ctypes.data_as(_dp))
        return None if rc != 0 else out

    def otf_param(self, n, bound, table, n_cam, cam, xyz):
        b, t = _d(bound), _d(table)
        xyz = _d(xyz).reshape(-1, 3)
        out = np.empty((len(xyz), 5))
        for i in range(len(xyz)):
            self.L.oo_otf_param(n[0], n[1], n[2], b.ctypes.data_as(_dp), t.ctypes.data_as(_dp),
                                n_cam, cam, xyz[i].ctypes.data_as(_dp), out[i].ctypes.data_as(_dp))
        return out

    def residual(self, orig, uv, otf5, r_px, clamp):
        orig = _d(orig)
        H, W = orig.shape
        res = np.empty_like(orig)
        uv, otf5 = _d(uv).reshape(-1, 2), _d(otf5).reshape(-1, 5)
        self.L.oo_residual(res.ctypes.data_as(_dp), orig.ctypes.data_as(_dp), H, W, len(uv),
                           uv.ctypes.data_as(_dp), otf5.ctypes.data_as(_dp), float(r_px), int(clamp))
        return res
