"""The host prune (StereoMatch::pruneMatch restated with the same libstdc++
stable_sort) selects exactly the reference's matches from the reference's own
candidate list.  CPU only."""
import ctypes as C
import os

import numpy as np
import pytest

from tests import _scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "pyopenlpt_b200", "libolpt_cuda.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "liboref.so")


def _prune(cand, e, counts, active):
    L = C.CDLL(LIB)
    M, n = cand.shape
    ids = np.ascontiguousarray(cand, dtype=np.int32)
    e = np.ascontiguousarray(e, dtype=np.float64)
    cnt = np.ascontiguousarray(counts, dtype=np.int64)
    act = (C.c_int * n)(*active)
    sel = np.zeros(M, dtype=np.uint8)
    rc = L.olpt_prune_matches(n, C.c_int64(M), ids.ctypes.data_as(C.c_void_p),
                              e.ctypes.data_as(C.c_void_p), cnt.ctypes.data_as(C.c_void_p), act,
                              sel.ctypes.data_as(C.c_void_p))
    assert rc == 0
    return sel.astype(bool)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference oracle not built")
@pytest.mark.parametrize("kind", ["small", "cfg1"])
def test_prune_selects_reference_matches(kind):
    sc = _scenes.scene(kind)
    ref = _scenes.ref_oracle(kind)
    dets = [ref.find_peaks(im) for im in sc.images]
    w = ref.stereo(dets)
    sel = _prune(w["cand"], w["e_check"], [len(d) for d in dets], [1] * sc.n_cam)
    assert np.array_equal(w["cand"][sel], w["sel"])


def test_prune_edge_cases():
    # empty list; a single candidate; two candidates sharing a point (better one wins)
    assert _prune(np.zeros((0, 3), np.int32), np.zeros(0), [5, 5, 5], [1, 1, 1]).size == 0
    s = _prune(np.array([[0, 1, 2]]), np.array([0.01]), [5, 5, 5], [1, 1, 1])
    assert s.tolist() == [True]
    s = _prune(np.array([[0, 1, 2], [0, 3, 4]]), np.array([0.02, 0.01]), [5, 5, 5], [1, 1, 1])
    assert s.tolist() == [False, True]
    # non-finite e_check is never selected
    s = _prune(np.array([[0, 1, 2], [1, 2, 3]]), np.array([np.nan, 0.01]), [5, 5, 5], [1, 1, 1])
    assert s.tolist() == [False, True]
