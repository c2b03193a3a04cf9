"""The allocation-free detector (olpt_find_peaks_noalloc) gives the same detections
as the context-based olpt_find_peaks, on two calls in a row.

It is meant for callers that cannot allocate device memory themselves (code inside
another framework's allocator or a host that budgets device memory), so this test
allocates every input and output on their behalf and only checks the results.  It
lives in its own file, collected last, and passes both alone in a fresh process and
after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from pyopenlpt_b200 import _ffi, synth

pytestmark = pytest.mark.gpu


def _noalloc(L, img, min_int, stream_ptr):
    import torch
    H, W = img.shape
    d_img = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    cap = (H * W + 1) // 2
    d_x = torch.empty(cap, dtype=torch.float64, device="cuda")
    d_y = torch.empty(cap, dtype=torch.float64, device="cuda")
    d_rc = torch.empty((cap, 2), dtype=torch.int32, device="cuda")
    d_n = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = L.olpt_find_peaks_noalloc(
        C.c_void_p(d_img.data_ptr()), _ffi._DTYPES[img.dtype], H, W,
        C.c_int64(W * img.dtype.itemsize), C.c_double(min_int), C.c_void_p(d_x.data_ptr()),
        C.c_void_p(d_y.data_ptr()), C.c_void_p(d_rc.data_ptr()), C.c_int64(cap),
        C.c_void_p(d_n.data_ptr()), C.c_void_p(stream_ptr))
    assert rc == 0, L.olpt_find_peaks_noalloc_error()
    torch.cuda.synchronize()
    n = int(d_n.item())
    return np.stack([d_x[:n].cpu().numpy(), d_y[:n].cpu().numpy()], axis=1)


def test_noalloc_matches_context_detector_twice():
    import torch
    L = _ffi.lib()
    L.olpt_find_peaks_noalloc_error.restype = C.c_char_p
    sc = synth.make_scene(n_particles=1500, size=512, focal=2500.0, seed=21)
    ctx = _ffi.Context(0)
    ctx.upload_cameras([_ffi.camera_desc_from_pinhole(c) for c in sc.cams])
    ctx.upload_images(sc.images)
    counts = ctx.find_peaks(30)
    stream = torch.cuda.current_stream().cuda_stream
    for c in (0, 1):  # two calls in a row on different images
        want, _ = ctx.get_peaks(c, int(counts[c]))
        got = _noalloc(L, sc.images[c], 30, stream)
        assert got.shape == want.shape and np.array_equal(got, want)
    ctx.close()


def test_noalloc_rejects_oversize_and_misaligned():
    L = _ffi.lib()
    dummy = C.c_void_p(16)
    rc = L.olpt_find_peaks_noalloc(dummy, 0, 20000, 64, C.c_int64(64), C.c_double(30), dummy,
                                   dummy, dummy, C.c_int64(10 ** 9), dummy, None)
    assert rc == 1  # OLPT_ERR_INVALID_ARG, before touching any memory
    rc = L.olpt_find_peaks_noalloc(dummy, 0, 64, 64, C.c_int64(65), C.c_double(30), dummy, dummy,
                                   dummy, C.c_int64(10 ** 6), dummy, None)
    assert rc == 1
