"""Kernel family (c) parity: residual image and Shake::runShake against the
reference.  FP64 mode must agree to rounding of exp(); the FP32 production path
is held to the 1e-4 mm position tolerance for the bulk of the particles."""
import numpy as np
import pytest

from pyopenlpt_b200 import _ffi
from tests import _scenes

pytestmark = pytest.mark.gpu


def _objs(kind):
    """Particles as stereo matching delivers them (the reference's own output)."""
    sc = _scenes.scene(kind)
    ref = _scenes.ref_oracle(kind)
    dets = [ref.find_peaks(im) for im in sc.images]
    return ref.stereo(dets)["xyz"]


@pytest.mark.parametrize("precision,atol", [(1, 1e-9), (0, 2e-3)])
def test_residual_image(precision, atol):
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    xyz = _objs("small")
    ctx = _scenes.gpu_context(sc)
    ctx.upload_images(sc.images)
    ctx.upload_objects(xyz)
    ctx.residual(_ffi.shake_params(_scenes.settings("small"), precision))
    want = ref.residual(xyz, sc.images)
    for c in range(sc.n_cam):
        got = ctx.residual_image(c, sc.images[c].shape)
        assert np.max(np.abs(got - want[c])) <= atol, (c, np.max(np.abs(got - want[c])))


def _shake_cmp(kind, precision):
    sc = _scenes.scene(kind)
    ref = _scenes.ref_oracle(kind)
    xyz = _objs(kind)
    ctx = _scenes.gpu_context(sc)
    ctx.upload_images(sc.images)
    ctx.upload_objects(xyz)
    ctx.shake(_ffi.shake_params(_scenes.settings(kind), precision))
    got = ctx.objects()
    want = ref.shake(xyz, sc.images)
    d = np.max(np.abs(got["xyz"] - want["xyz"]), axis=1)
    return got, want, d


def test_shake_fp64_matches_reference():
    got, want, d = _shake_cmp("small", 1)
    n = len(d)
    frac_exact = np.mean(d <= 1e-9)
    frac_tol = np.mean(d <= 1e-4)
    print(f"fp64 shake: n={n} <=1e-9mm {frac_exact:.4f} <=1e-4mm {frac_tol:.4f} max {d.max():.3g}")
    assert frac_tol >= 0.995
    assert np.mean(got["flags"] == want["flags"]) >= 0.995
    ok = d <= 1e-9
    assert np.allclose(got["score"][ok], want["score"][ok], rtol=1e-9)


def test_shake_fp32_position_tolerance():
    got, want, d = _shake_cmp("small", 0)
    frac = np.mean(d <= 1e-4)
    print(f"fp32 shake: <=1e-4mm {frac:.4f} median {np.median(d):.3g} p99 {np.quantile(d, .99):.3g}")
    assert frac >= 0.95
