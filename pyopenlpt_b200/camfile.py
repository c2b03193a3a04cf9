"""Camera parameter files in the reference's text format.

Camera::loadParameters(file) (src/srcMath/Camera.cpp:19-158, 311-338 of OpenLPT):
lines whose first character is '#' are dropped, text after a later '#' is cut,
the remaining lines are joined by tabs and read as a stream -- whitespace-delimited
tokens, matrices read number by number with one optional ',' after each.
PINHOLE and POLYNOMIAL models are supported (PINPLATE is not on this path).
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np


class _Stream:
    def __init__(self, text: str):
        self.s = text
        self.i = 0

    def _skip_ws(self):
        while self.i < len(self.s) and self.s[self.i].isspace():
            self.i += 1

    def token(self) -> str:
        self._skip_ws()
        j = self.i
        while j < len(self.s) and not self.s[j].isspace():
            j += 1
        t = self.s[self.i:j]
        self.i = j
        if not t:
            raise ValueError("unexpected end of camera file")
        return t

    def number(self) -> float:
        """`is >> double` then skip one ',' (Matrix(rows, cols, istream), Matrix.hpp:102-116)."""
        self._skip_ws()
        j = self.i
        while j < len(self.s) and (self.s[j].isdigit() or self.s[j] in "+-.eE"):
            j += 1
        v = float(self.s[self.i:j])
        self.i = j
        if self.i < len(self.s) and self.s[self.i] == ",":
            self.i += 1
        return v

    def integer(self) -> int:
        self._skip_ws()
        j = self.i
        while j < len(self.s) and (self.s[j].isdigit() or self.s[j] in "+-"):
            j += 1
        v = int(self.s[self.i:j])
        self.i = j
        return v

    def matrix(self, n: int) -> List[float]:
        return [self.number() for _ in range(n)]


def _strip(text: str) -> str:
    out = []
    for line in text.splitlines():
        pos = line.find("#")
        if pos == 0:
            continue
        if pos > 0:
            line = line[:pos]
        out.append(line)
    return "\t".join(out) + "\t"


@dataclasses.dataclass
class CameraParams:
    type: int                      # 0 PINHOLE, 1 POLYNOMIAL
    n_row: int
    n_col: int
    cam_mtx: Optional[np.ndarray] = None
    dist: Optional[np.ndarray] = None
    R: Optional[np.ndarray] = None
    Rinv: Optional[np.ndarray] = None
    T: Optional[np.ndarray] = None
    Tinv: Optional[np.ndarray] = None
    ref_plane: int = 3
    plane: tuple = (0.0, 0.0)
    u_coeffs: Optional[np.ndarray] = None
    v_coeffs: Optional[np.ndarray] = None
    max_intensity: float = 255.0
    is_active: bool = True

    @property
    def is_distorted(self) -> bool:
        return self.dist is not None and bool(np.any(self.dist > 1e-8))


def parse(text: str) -> CameraParams:
    st = _Stream(_strip(text))
    kind = st.token()
    if kind == "PINHOLE":
        st.token()
        st.token()
        r, c = st.token().split(",")[:2]
        K = np.array(st.matrix(9)).reshape(3, 3)
        dtok = st.token()
        dist = [float(x) for x in dtok.split(",") if x.strip() != ""]
        nd = len(dist)
        if any(d > 1e-8 for d in dist) and nd not in (4, 5, 8, 12):
            raise ValueError(f"number of distortion coefficients is wrong: {nd}")
        st.token()  # rotation vector
        R = np.array(st.matrix(9)).reshape(3, 3)
        Rinv = np.array(st.matrix(9)).reshape(3, 3)
        T = np.array(st.matrix(3))
        Tinv = np.array(st.matrix(3))
        return CameraParams(0, int(r), int(c), cam_mtx=K, dist=np.array(dist), R=R, Rinv=Rinv,
                            T=T, Tinv=Tinv)
    if kind == "POLYNOMIAL":
        st.token()
        r, c = st.token().split(",")[:2]
        ptok = st.token().split(",")
        ref = {"REF_X": 1, "REF_Y": 2, "REF_Z": 3}.get(ptok[0])
        if ref is None:
            raise ValueError(f"reference plane is wrong: {ptok[0]}")
        plane = (float(ptok[1]), float(ptok[2]))
        n = st.integer()
        u = np.array(st.matrix(4 * n)).reshape(n, 4)
        v = np.array(st.matrix(4 * n)).reshape(n, 4)
        return CameraParams(1, int(r), int(c), ref_plane=ref, plane=plane, u_coeffs=u, v_coeffs=v)
    raise ValueError(f"unsupported camera type: {kind}")


def load(path: str) -> CameraParams:
    with open(path) as f:
        return parse(f.read())
