"""The device prune (percentile scores, greedy order and the greedy itself on the
GPU) against the reference's own selection and against the host restatement of
StereoMatch::pruneMatch (src/srcSTB/StereoMatch.cpp:631-980) on random candidate
lists with ties, non-finite checks and shared points."""
import os

import numpy as np
import pytest

from pyopenlpt_b200 import _ffi
from tests import _scenes
from tests.test_prune import REF_SO, _prune

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = _ffi.Context(0)
    yield c
    c.close()


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference oracle not built")
@pytest.mark.parametrize("kind", ["small", "cfg1"])
def test_device_prune_selects_reference_matches(ctx, kind):
    sc = _scenes.scene(kind)
    ref = _scenes.ref_oracle(kind)
    dets = [ref.find_peaks(im) for im in sc.images]
    w = ref.stereo(dets)
    ctx.profile(True)
    sel = ctx.prune_matches(w["cand"], w["e_check"], [len(d) for d in dets])
    _, n_host_greedy, _ = ctx.profile_read(_ffi.PH_GREEDY_HOST)
    ctx.profile(False)
    assert np.array_equal(w["cand"][sel], w["sel"])
    assert n_host_greedy == 0  # the greedy ran on the device


def test_device_prune_edge_cases(ctx):
    assert ctx.prune_matches(np.zeros((0, 3), np.int32), np.zeros(0), [5, 5, 5]).size == 0
    assert ctx.prune_matches(np.array([[0, 1, 2]]), np.array([0.01]), [5, 5, 5]).tolist() == [True]
    s = ctx.prune_matches(np.array([[0, 1, 2], [0, 3, 4]]), np.array([0.02, 0.01]), [5, 5, 5])
    assert s.tolist() == [False, True]
    s = ctx.prune_matches(np.array([[0, 1, 2], [1, 2, 3]]), np.array([np.nan, 0.01]), [5, 5, 5])
    assert s.tolist() == [False, True]
    # an inactive camera's ids are ignored
    s = ctx.prune_matches(np.array([[0, 1, -1], [0, 2, -1]]), np.array([0.02, 0.01]), [5, 5, 0],
                          active=[1, 1, 0])
    assert s.tolist() == [False, True]
    with pytest.raises(_ffi.OlptError):
        ctx.prune_matches(np.array([[0, 9, 2]]), np.array([0.01]), [5, 5, 5])


def _random_list(rng, n_cam, n_pts, M, n_levels, p_missing, p_nan):
    ids = rng.integers(0, n_pts, size=(M, n_cam)).astype(np.int32)
    if n_cam > 3:  # some candidates on n_cam - 1 cameras
        drop = rng.random(M) < p_missing
        ids[drop, rng.integers(0, n_cam, size=drop.sum())] = -1
    ids = np.unique(ids, axis=0)  # the reference's candidate list is sorted by ids
    e = rng.integers(0, n_levels, size=len(ids)) * 1e-3 + 1e-3  # many exact ties
    e[rng.random(len(ids)) < p_nan] = np.nan
    return ids, e


@pytest.mark.parametrize("seed", range(6))
def test_device_prune_matches_host_on_random_lists(ctx, seed):
    rng = np.random.default_rng(seed)
    n_cam = 3 + seed % 2
    n_pts = [40, 200, 1000][seed % 3]
    M = [300, 3000, 20000][seed % 3]
    ids, e = _random_list(rng, n_cam, n_pts, M, n_levels=[3, 50, 10**6][seed // 2],
                          p_missing=0.3, p_nan=0.02)
    counts = [n_pts] * n_cam
    want = _prune(ids, e, counts, [1] * n_cam)
    got = ctx.prune_matches(ids, e, counts)
    assert np.array_equal(got, want)
    # no two kept candidates share a point
    kept = ids[got]
    for c in range(n_cam):
        col = kept[:, c][kept[:, c] >= 0]
        assert len(np.unique(col)) == len(col)
