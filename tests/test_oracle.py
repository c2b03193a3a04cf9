"""CPU tests of the oracle: the C restatement against the reference's golden
vectors (test_Camera.cpp solutions) and against the reference compiled from its
own sources (bit-exact)."""
import json
import os

import numpy as np
import pytest

from oracle.restated import Restated
from pyopenlpt_b200 import camfile, synth
from tests import _scenes

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "camera_golden.json")))
REF_SO = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "liboref.so")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference oracle not built")


@pytest.fixture(scope="module")
def oo():
    return Restated()


def _cam(name):
    return camfile.parse(GOLD["cameras"][name])


def test_golden_pinhole_projection(oo):
    """test_Camera.cpp test_function_2: worldToUndistImg exact to the 8 printed
    digits, distort and project within 1e-3 px."""
    f2 = np.array(GOLD["f2"]).reshape(3, 5, 2)
    X = np.array(GOLD["f2_world"])
    for i in range(5):
        c = oo.pinhole(_cam(f"cam{i + 1}"))
        und = oo.world_to_undist(c, X)[0]
        assert np.allclose(und, f2[0, i], rtol=1e-7, atol=1e-12)
        assert np.max(np.abs(oo.distort(c, und)[0] - f2[1, i])) <= 1e-3
        assert np.max(np.abs(oo.project(c, X)[0] - f2[2, i])) <= 1e-3


def test_golden_line_of_sight(oo):
    """test_function_3: undistort, pinholeLine and lineOfSight within 1e-5."""
    f3 = np.array(GOLD["f3"])
    und = f3[:10].reshape(5, 2)
    pl = f3[10:40].reshape(5, 6)
    los = f3[40:70].reshape(5, 6)
    uv = np.array(GOLD["f3_pixel"])
    for i in range(5):
        c = oo.pinhole(_cam(f"cam{i + 1}"))
        assert np.max(np.abs(oo.undistort(c, uv)[0] - und[i])) <= 1e-5
        L = oo.los(c, uv)[0]
        assert np.max(np.abs(L - los[i])) <= 1e-5
        assert np.max(np.abs(L - pl[i])) <= 1e-5


def test_golden_polynomial_projection(oo):
    """test_function_5: polyProject of (1, 0, 3)."""
    f5 = np.array(GOLD["f5"]).reshape(2, 2, 2)
    X = np.array(GOLD["f5_world"])
    for i, name in enumerate(["cam1_poly", "cam2_poly"]):
        c = oo.poly(_cam(name))
        assert np.allclose(oo.poly_project(c, X)[0], f5[0, i], rtol=1e-8)


def test_camfile_roundtrip():
    sc = _scenes.scene("small")
    for cm in sc.cams:
        p = camfile.parse(cm.to_text())
        assert p.type == 0 and (p.n_row, p.n_col) == (cm.n_row, cm.n_col)
        assert np.array_equal(p.R, cm.R) and np.array_equal(p.Rinv, cm.Rinv)
        assert np.array_equal(p.T, cm.T) and np.array_equal(p.Tinv, cm.Tinv)
        assert p.cam_mtx[0, 0] == cm.fx and p.cam_mtx[1, 2] == cm.cy


@needs_ref
def test_restatement_matches_reference_bit_exact(oo):
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    rng = np.random.default_rng(2)
    lo, hi = np.array(sc.volume[0::2]), np.array(sc.volume[1::2])
    X = lo + (hi - lo) * rng.random((300, 3))
    for ci, cm in enumerate(sc.cams):
        c = oo.pinhole(cm)
        uv = oo.project(c, X)
        assert np.array_equal(uv, ref.project(ci, X))
        assert np.array_equal(oo.los(c, uv), ref.los(ci, uv))
    d0 = oo.find_peaks(sc.images[0], 30)
    assert np.array_equal(d0, ref.find_peaks(sc.images[0]))
    lines = np.stack([ref.los(ci, ref.project(ci, X) + rng.normal(0, .3, (len(X), 2)))
                      for ci in range(sc.n_cam)], axis=1)
    for i in range(0, len(X), 10):
        a, b = oo.triangulate(lines[i]), ref.triangulate(lines[i])
        assert (a is None) == (b is None)
        if a is not None:
            assert np.array_equal(a, b)
    tab = synth.otf_table_array(sc.n_cam, sc.otf_abc)
    for ci in range(sc.n_cam):
        assert np.array_equal(oo.otf_param((2, 2, 2), sc.volume, tab, sc.n_cam, ci, X * 1.2),
                              ref.otf_param(ci, X * 1.2))


@needs_ref
def test_restated_residual_matches_reference(oo):
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    X = sc.xyz[:400]
    want = ref.residual(X, sc.images)
    tab = synth.otf_table_array(sc.n_cam, sc.otf_abc)
    for ci, cm in enumerate(sc.cams):
        uv = ref.project(ci, X)
        o5 = ref.otf_param(ci, X)
        got = oo.residual(sc.images[ci], uv, o5, 2.0, 1)
        assert np.array_equal(got, want[ci])
