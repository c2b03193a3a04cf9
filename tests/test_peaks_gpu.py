"""Kernel family (a) parity: detections (integer peak pixels, raster order and the
sub-pixel centres) against ObjectFinder2D::findObject2D of the reference."""
import numpy as np
import pytest

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
