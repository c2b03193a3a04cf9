"""Kernel family (b) parity: the checked candidate set (ids, e_check), the prune
selection and the triangulated matches against the reference's StereoMatch,
given identical 2D detections.  All bit-exact."""
import numpy as np
import pytest

from pyopenlpt_b200 import _ffi, synth
from tests import _scenes

pytestmark = pytest.mark.gpu


def _run(kind, dets=None, tol_2d=None, active=None):
    sc = _scenes.scene(kind)
    ref = _scenes.ref_oracle(kind)
    s = _scenes.settings(kind)
    if tol_2d is not None:
        s.tol_2d_px = tol_2d
    ctx = _scenes.gpu_context(sc)
    if active is not None:
        ctx.set_active(active)
        ref.set_active(active)
        s.match_cam_count = int(sum(active))
    if dets is None:
        dets = [ref.find_peaks(im) for im in sc.images]
    ctx.upload_detections(dets)
    prm = _ffi.sm_params(s, sc.volume)
    n_cand, n_match = ctx.stereo_match(prm)
    ids, e, x = ctx.candidates(n_cand)
    mids, mx = ctx.matches(n_match)
    # the reference with the same knobs
    from oracle.ref import RefOracle
    r = RefOracle(sc, s, threads=8) if (tol_2d is not None or active is not None) else ref
    if active is not None:
        r.set_active(active)
    want = r.stereo(dets)
    if active is not None:
        ref.set_active([1] * sc.n_cam)
    return (ids, e, x, mids, mx), want


@pytest.mark.parametrize("kind", ["small", "cfg1", "u16"])
def test_candidate_set_and_matches_bit_exact(kind):
    (ids, e, x, mids, mx), want = _run(kind)
    assert len(ids) == len(want["cand"]), (len(ids), len(want["cand"]))
    assert np.array_equal(ids, want["cand"])
    assert np.array_equal(e, want["e_check"])
    assert np.array_equal(mids, want["sel"])
    assert np.array_equal(mx, want["xyz"])


def test_wider_tolerance_and_camera_subset():
    (ids, e, x, mids, mx), want = _run("small", tol_2d=2.25)
    assert np.array_equal(ids, want["cand"]) and np.array_equal(e, want["e_check"])
    assert np.array_equal(mids, want["sel"]) and np.array_equal(mx, want["xyz"])
    (ids, e, x, mids, mx), want = _run("small", active=[1, 0, 1, 1])
    assert np.array_equal(ids, want["cand"]) and np.array_equal(e, want["e_check"])
    assert np.array_equal(mids, want["sel"]) and np.array_equal(mx, want["xyz"])


def test_empty_and_tiny_inputs():
    sc = _scenes.scene("small")
    ctx = _scenes.gpu_context(sc)
    prm = _ffi.sm_params(synth.IPRSettings(), sc.volume)
    ctx.upload_detections([np.zeros((0, 2))] * sc.n_cam)
    assert ctx.stereo_match(prm) == (0, 0)
    ctx.upload_detections([np.array([[100.0, 100.0]])] * sc.n_cam)
    n_cand, n_match = ctx.stereo_match(prm)
    assert n_match <= 1
