"""The allocation-free detector (olpt_find_peaks_noalloc) gives the same detections
as the context-based olpt_find_peaks, on two calls in a row.

It is meant for callers that cannot allocate device memory themselves (code inside
another framework's allocator or a host that budgets device memory), so this test
allocates every input and output on their behalf and only checks the results:
sub-pixel positions and integer peak pixels, bit for bit, for 8-bit, 12-bit (2048^2)
and float images and for a ragged width whose rows end in a partial 16-byte chunk.
It lives in its own file, collected last, and passes both alone in a fresh process
and after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from pyopenlpt_b200 import _ffi, synth

pytestmark = pytest.mark.gpu


def _noalloc(L, img, min_int, stream_ptr):
    """Run the allocation-free detector on a pitched device copy of ``img``."""
    import torch
    H, W = img.shape
    esz = img.dtype.itemsize
    pitch_elems = ((W * esz + 15) // 16 * 16) // esz
    tdt = {np.uint8: torch.uint8, np.uint16: torch.int16, np.float32: torch.float32,
           np.float64: torch.float64}[img.dtype.type]
    host = np.zeros((H, pitch_elems), dtype=img.dtype)
    host[:, :W] = img
    d_img = torch.from_numpy(host.view(np.int16) if img.dtype == np.uint16 else host).to(
        "cuda", dtype=tdt)
    cap = (H * W + 1) // 2
    d_x = torch.full((cap,), float("nan"), dtype=torch.float64, device="cuda")
    d_y = torch.full((cap,), float("nan"), dtype=torch.float64, device="cuda")
    d_rc = torch.full((cap, 2), -7, dtype=torch.int32, device="cuda")
    d_n = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = L.olpt_find_peaks_noalloc(
        C.c_void_p(d_img.data_ptr()), _ffi._DTYPES[img.dtype], H, W,
        C.c_int64(pitch_elems * esz), C.c_double(min_int), C.c_void_p(d_x.data_ptr()),
        C.c_void_p(d_y.data_ptr()), C.c_void_p(d_rc.data_ptr()), C.c_int64(cap),
        C.c_void_p(d_n.data_ptr()), C.c_void_p(stream_ptr))
    assert rc == 0, L.olpt_find_peaks_noalloc_error()
    torch.cuda.synchronize()
    n = int(d_n.item())
    xy = np.stack([d_x[:n].cpu().numpy(), d_y[:n].cpu().numpy()], axis=1)
    return xy, d_rc[:n].cpu().numpy()


def _images(kind):
    if kind == "u8_512":
        sc = synth.make_scene(n_particles=1500, size=512, focal=2500.0, seed=21)
        return sc.images[:2], 30.0
    if kind == "u16_2048":
        sc = synth.make_scene(n_particles=40000, n_cam=2, size=2048, focal=10000.0, a=3000.0,
                              noise=20.0, bits=12, seed=22)
        return sc.images, 300.0
    if kind == "f32_ragged":
        sc = synth.make_scene(n_particles=1200, n_cam=2, n_row=300, n_col=1021, focal=2500.0,
                              seed=23)
        rng = np.random.default_rng(5)
        return [(im + rng.random(im.shape)).astype(np.float32) for im in sc.images], 30.5
    if kind == "u8_ragged":
        sc = synth.make_scene(n_particles=1200, n_cam=2, n_row=301, n_col=1021, focal=2500.0,
                              seed=24)
        return sc.images, 30.0
    raise KeyError(kind)


@pytest.mark.parametrize("kind", ["u8_512", "u16_2048", "f32_ragged", "u8_ragged"])
def test_noalloc_matches_context_detector_twice(kind):
    import torch
    L = _ffi.lib()
    L.olpt_find_peaks_noalloc_error.restype = C.c_char_p
    imgs, thr = _images(kind)
    H, W = imgs[0].shape
    ctx = _ffi.Context(0)
    ctx.upload_cameras([_ffi.camera_desc_from_pinhole(c)
                        for c in synth.ring_rig(len(imgs), H, W, 2500.0)])
    ctx.upload_images(imgs)
    counts = ctx.find_peaks(thr)
    stream = torch.cuda.current_stream().cuda_stream
    for c in range(len(imgs)):  # two calls in a row, on different images
        want_xy, want_rc = ctx.get_peaks(c, int(counts[c]))
        got_xy, got_rc = _noalloc(L, imgs[c], thr, stream)
        print(f"{kind} camera {c}: {len(want_xy)} detections")
        assert len(want_xy) > 0
        assert got_xy.shape == want_xy.shape and np.array_equal(got_xy, want_xy)
        assert np.array_equal(got_rc, want_rc)
    ctx.close()


def test_noalloc_rejects_oversize_and_misaligned():
    L = _ffi.lib()
    dummy = C.c_void_p(16)
    rc = L.olpt_find_peaks_noalloc(dummy, 0, 20000, 64, C.c_int64(64), C.c_double(30), dummy,
                                   dummy, dummy, C.c_int64(10 ** 9), dummy, None)
    assert rc == 1  # OLPT_ERR_INVALID_ARG, before touching any memory
    rc = L.olpt_find_peaks_noalloc(dummy, 0, 64, 20000, C.c_int64(20000), C.c_double(30), dummy,
                                   dummy, dummy, C.c_int64(10 ** 9), dummy, None)
    assert rc == 1  # too many columns
    rc = L.olpt_find_peaks_noalloc(dummy, 0, 64, 64, C.c_int64(65), C.c_double(30), dummy, dummy,
                                   dummy, C.c_int64(10 ** 6), dummy, None)
    assert rc == 1  # pitch not a multiple of 16 bytes
    rc = L.olpt_find_peaks_noalloc(dummy, 0, 64, 64, C.c_int64(64), C.c_double(30), dummy, dummy,
                                   dummy, C.c_int64(10), dummy, None)
    assert rc == 1  # capacity below (H * W + 1) / 2
