"""Kernel family (a) parity: detections (integer peak pixels, raster order and the
sub-pixel centres) against ObjectFinder2D::findObject2D of the reference."""
import dataclasses

import numpy as np
import pytest

from pyopenlpt_b200 import _ffi
from tests import _scenes

pytestmark = pytest.mark.gpu


def _check(ctx, ref, imgs, min_int):
    counts = ctx.find_peaks(min_int)
    for c, im in enumerate(imgs):
        want = ref.find_peaks(im)
        assert counts[c] == len(want), (c, counts[c], len(want))
        xy, rc = ctx.get_peaks(c, counts[c])
        # integer peak pixels and order: bit-exact
        assert np.array_equal(xy, want), f"camera {c}: sub-pixel centres differ"


@pytest.mark.parametrize("kind", ["small", "cfg1", "u16"])
def test_peaks_integer_images_bit_exact(kind):
    sc = _scenes.scene(kind)
    ref = _scenes.ref_oracle(kind)
    ctx = _scenes.gpu_context(sc)
    ctx.upload_images(sc.images)
    _check(ctx, ref, sc.images, 30)


def test_peaks_float_image_pixels_exact():
    """Residual-like float images: peak pixels exact; sub-pixel within 1e-9 px
    (CUDA log vs libm log)."""
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    ctx = _scenes.gpu_context(sc)
    rng = np.random.default_rng(1)
    imgs = [im.astype(np.float64) - rng.random(im.shape) * 3.0 for im in sc.images]
    imgs = [np.maximum(im, 0.0) for im in imgs]
    ctx.upload_images(imgs)
    counts = ctx.find_peaks(30)
    for c, im in enumerate(imgs):
        want = ref.find_peaks(im)
        assert counts[c] == len(want)
        xy, _ = ctx.get_peaks(c, counts[c])
        assert np.allclose(xy, want, rtol=0, atol=1e-9)


def test_peaks_edge_cases():
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    ctx = _scenes.gpu_context(sc)
    H, W = sc.images[0].shape
    empty = [np.zeros((H, W), np.uint8) for _ in sc.cams]
    ctx.upload_images(empty)
    assert list(ctx.find_peaks(30)) == [0] * sc.n_cam
    # plateaus and ties: tie rule keeps the top-left pixel only
    im = np.zeros((H, W), np.uint8)
    im[10, 10:12] = 200
    im[20:22, 30] = 150
    im[40:42, 40:42] = 99
    im[0, 5] = 255          # border rows/cols are never peaks
    im[7, W - 1] = 255
    imgs = [im.copy() for _ in sc.cams]
    ctx.upload_images(imgs)
    counts = ctx.find_peaks(30)
    want = ref.find_peaks(im)
    assert counts[0] == len(want)
    xy, rc = ctx.get_peaks(0, counts[0])
    assert np.array_equal(xy, want)


def _spot_image(rng, H, W, n, dtype, amp):
    """n Gaussian spots (max-fused, 7 x 7) on a noisy background."""
    im = rng.random((H, W)) * amp * 0.05
    ys, xs = rng.uniform(-3, H + 3, n), rng.uniform(-3, W + 3, n)
    for dy in range(-3, 4):
        for dx in range(-3, 4):
            r = np.floor(ys).astype(int) + dy
            c = np.floor(xs).astype(int) + dx
            ok = (r >= 0) & (r < H) & (c >= 0) & (c < W)
            v = amp * np.exp(-0.5 * ((r - ys) ** 2 + (c - xs) ** 2))
            np.maximum.at(im, (r[ok], c[ok]), v[ok])
    if np.issubdtype(dtype, np.integer):
        im = np.clip(np.round(im), 0, np.iinfo(dtype).max)
    return im.astype(dtype)


def _check_any(ctx, ref, imgs, min_int):
    counts = ctx.find_peaks(min_int)
    for c, im in enumerate(imgs):
        want = ref.find_peaks(im)
        assert counts[c] == len(want), (c, counts[c], len(want))
        xy, rc = ctx.get_peaks(c, counts[c])
        if np.issubdtype(im.dtype, np.integer):
            assert np.array_equal(xy, want), f"camera {c}: sub-pixel centres differ"
        else:  # CUDA log vs libm log on float levels
            assert np.allclose(xy, want, rtol=0, atol=1e-9), f"camera {c}"
        # the integer peak pixel is the centre's pixel to within the fit's half-pixel
        assert np.all(np.abs(rc[:, 0] - xy[:, 1]) <= 0.5 + 1e-9)
        assert np.all(np.abs(rc[:, 1] - xy[:, 0]) <= 0.5 + 1e-9)


@pytest.mark.parametrize("dtype,shape", [
    (np.uint8, (301, 517)),    # ragged rows and columns, two boxes per row
    (np.uint16, (257, 1000)),  # 4 boxes, last one partial
    (np.float32, (190, 771)),
    (np.float64, (65, 300)),
    (np.uint8, (3, 40)),       # one interior row, one box narrower than 256
    (np.uint16, (2, 7)),       # no interior row at all
])
def test_peaks_ragged_shapes(dtype, shape):
    """Band and box edges of the staged detector at every image type against the
    reference (each camera a different image)."""
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    ctx = _scenes.gpu_context(sc)
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    H, W = shape
    amp = 200.0 if dtype == np.uint8 else 3000.0
    imgs = [_spot_image(rng, H, W, max(1, H * W // 150), dtype, amp) for _ in range(sc.n_cam)]
    ctx.upload_images(imgs)
    _check_any(ctx, ref, imgs, 30)


def test_peaks_dense_detections():
    """Noise with threshold 0: about a fifth of all pixels are peaks, so every band's
    look-back carries large counts."""
    from oracle.ref import RefOracle
    sc = _scenes.scene("small")
    ref = RefOracle(sc, dataclasses.replace(_scenes.settings("small"), min_obj_int=0))
    ctx = _scenes.gpu_context(sc)
    rng = np.random.default_rng(5)
    imgs = [rng.integers(0, 256, (512, 512)).astype(np.uint8) for _ in range(sc.n_cam)]
    ctx.upload_images(imgs)
    counts = ctx.find_peaks(0)
    assert counts.min() > 20000
    _check_any(ctx, ref, imgs, 0)


def test_peaks_wide_rows_two_pass():
    """Rows too wide to stage three of in shared memory (f64, 9000 columns) take the
    two-pass detector; same results."""
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    ctx = _scenes.gpu_context(sc)
    rng = np.random.default_rng(9)
    imgs = [_spot_image(rng, 9, 9000, 400, np.float64, 200.0) for _ in range(sc.n_cam)]
    ctx.upload_images(imgs)
    _check_any(ctx, ref, imgs, 30)


def test_peaks_inactive_camera():
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    ctx = _scenes.gpu_context(sc)
    ctx.upload_images(sc.images)
    ctx.set_active([1, 0, 1, 1])
    counts = ctx.find_peaks(30)
    assert counts[1] == 0
    for c in (0, 2, 3):
        want = ref.find_peaks(sc.images[c])
        assert counts[c] == len(want)
        xy, _ = ctx.get_peaks(c, counts[c])
        assert np.array_equal(xy, want)


def test_lookback_timeout_reports_and_context_recovers():
    """A band that never publishes its count (the failure-detection hook) makes the
    bands after it give up their bounded look-back wait (1 ms here): olpt_find_peaks
    returns OLPT_ERR_TIMEOUT, and the same context then detects normally again."""
    import ctypes as C
    sc = _scenes.scene("small")
    ctx = _scenes.gpu_context(sc)
    ctx.upload_images(sc.images)
    want = ctx.find_peaks(30)
    L = _ffi.lib()
    for ticket in (0, 3):
        assert L.olpt_test_hold_detection_band(ctx.h, ticket, C.c_int64(1_000_000)) == 0
        with pytest.raises(_ffi.OlptError) as e:
            ctx.find_peaks(30)
        assert e.value.code == 4  # OLPT_ERR_TIMEOUT
        assert np.array_equal(ctx.find_peaks(30), want)
    assert L.olpt_test_hold_detection_band(ctx.h, -1, C.c_int64(1000)) == 1
    ctx.close()
