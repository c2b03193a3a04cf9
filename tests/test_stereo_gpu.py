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


@pytest.mark.parametrize("kind", ["small", "cfg1", "u16", "poly"])
def test_candidate_set_and_matches_bit_exact(kind):
    """Also 6 polynomial cameras, whose candidate id keys (6 x 12 bits) need the
    two-word device sort."""
    (ids, e, x, mids, mx), want = _run(kind)
    assert len(ids) == len(want["cand"]), (len(ids), len(want["cand"]))
    assert np.array_equal(ids, want["cand"])
    assert np.array_equal(mids, want["sel"])
    if kind == "poly":
        # the reference's polynomial lines of sight start their Newton solve at rand()
        # draws, so e_check and positions agree to rounding, not bit for bit; e_check
        # (an RMS distance from a difference of squares) to 1e-9 mm absolute
        print(f"poly: {len(ids)} candidates, {len(mids)} matches; max |de| "
              f"{np.max(np.abs(e - want['e_check'])):.3g}, max |dxyz| "
              f"{np.max(np.abs(mx - want['xyz'])):.3g} mm")
        assert np.max(np.abs(e - want["e_check"])) <= 1e-9
        assert np.max(np.abs(mx - want["xyz"])) <= 1e-9
    else:
        assert np.array_equal(e, want["e_check"])
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


def _near_margin(ctx, dets, rec, tol):
    """|distance| - tol of one logged test, recomputed on the host from the device's
    camera model: the image line of one detection's line of sight on the other camera
    (two projected points, normalised twice as IDMap does) and the point's distance to
    it."""
    if rec["kind"] == 0:  # target detection vs the chosen detection's image line
        src_cam, src, pt_cam, pt = rec["other_cam"], rec["other_id"], rec["cam"], rec["id"]
    else:                 # chosen point vs the target detection's image line
        src_cam, src, pt_cam, pt = rec["cam"], rec["id"], rec["other_cam"], rec["other_id"]
    L = ctx.los(int(src_cam), dets[src_cam][src:src + 1])[0]
    a = ctx.project(int(pt_cam), L[None, :3])[0]
    b = ctx.project(int(pt_cam), (L[:3] + L[3:])[None, :])[0]
    d = b - a
    u = d / np.sqrt(d[0] * d[0] + d[1] * d[1])
    u = u / np.sqrt(u[0] * u[0] + u[1] * u[1])
    q = dets[pt_cam][pt]
    z = (q[1] - a[1]) * u[0] - (q[0] - a[0]) * u[1]
    return abs(z) - tol


@pytest.mark.parametrize("kind", ["small", "cfg1", "u16", "poly"])
def test_near_tolerance_log(kind):
    """Every 2D stereo test within 1e-6 px of tol_2d_px is logged (the decisions that
    rounding could flip); the candidate sets still equal the reference's."""
    sc = _scenes.scene(kind)
    ref = _scenes.ref_oracle(kind)
    s = _scenes.settings(kind)
    ctx = _scenes.gpu_context(sc)
    dets = [ref.find_peaks(im) for im in sc.images]
    ctx.upload_detections(dets)
    ctx.near_log_enable(1e-6)
    n_cand, _ = ctx.stereo_match(_ffi.sm_params(s, sc.volume))
    rec, total = ctx.near_log()
    print(f"{kind}: {n_cand} candidates, {total} stereo tests within 1e-6 px of tol_2d "
          f"{s.tol_2d_px} px")
    for r in rec:
        print(f"  kind {r['kind']} k {r['n_chosen']} cam {r['cam']} id {r['id']} vs cam "
              f"{r['other_cam']} id {r['other_id']}: margin {r['margin_px']:.3e} px")
    assert len(rec) == total and np.all(np.abs(rec["margin_px"]) < 1e-6)


def test_near_tolerance_log_records():
    """With a wide band (0.05 px) the log holds many tests; each record's margin is
    recomputed on the host and agrees, and logging changes no candidate."""
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    s = _scenes.settings("small")
    ctx = _scenes.gpu_context(sc)
    dets = [ref.find_peaks(im) for im in sc.images]
    ctx.upload_detections(dets)
    prm = _ffi.sm_params(s, sc.volume)
    n0, _ = ctx.stereo_match(prm)
    ids0, e0, _ = ctx.candidates(n0)
    ctx.near_log_enable(0.05)
    n1, _ = ctx.stereo_match(prm)
    ids1, e1, _ = ctx.candidates(n1)
    assert np.array_equal(ids0, ids1) and np.array_equal(e0, e1)
    rec, total = ctx.near_log()
    print(f"{total} tests within 0.05 px of the tolerance "
          f"({np.sum(rec['kind'] == 0)} strip, {np.sum(rec['kind'] == 1)} back-projection)")
    assert total > 50 and len(rec) == total
    assert np.all(np.abs(rec["margin_px"]) < 0.05)
    for r in rec[:: max(1, len(rec) // 200)]:
        m = _near_margin(ctx, dets, r, s.tol_2d_px)
        assert abs(m - r["margin_px"]) <= 1e-12, (r, m)
    ctx.near_log_reset()
    assert ctx.near_log()[1] == 0
    ctx.near_log_enable(0.0)
    ctx.stereo_match(prm)
    assert ctx.near_log()[1] == 0
