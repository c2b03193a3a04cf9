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


@pytest.mark.parametrize("precision,atol", [(1, 1e-9), (0, 5e-3)])
def test_residual_image(precision, atol):
    """FP64 mode to 1e-9; FP32 mode within 5e-3 intensity units of a = 200: the FP32
    Gaussian (exp in single precision, relative error ~1e-7) and the FP32 residual
    plane (an FP32 ulp of the 8-bit levels is ~1.5e-5) bound it well below that."""
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


@pytest.mark.parametrize("kind", ["small", "cfg1"])
def test_shake_fp64_matches_reference(kind):
    """FP64 mode against Shake::runShake: every object's position, flag and score.
    exp() is the only operation whose rounding differs from glibc's, so a line-search
    decision can flip only where two residues tie to rounding; each object beyond
    1e-9 mm is printed, and at most 0.2% may differ beyond 1e-4 mm."""
    got, want, d = _shake_cmp(kind, 1)
    n = len(d)
    n9, n4 = int(np.sum(d > 1e-9)), int(np.sum(d > 1e-4))
    flags_diff = int(np.sum(got["flags"] != want["flags"]))
    print(f"fp64 shake {kind}: {n} objects, beyond 1e-9 mm {n9}, beyond 1e-4 mm {n4}, "
          f"flags differ {flags_diff}, max {d.max():.3g} mm")
    for i in np.flatnonzero(d > 1e-9)[:10]:
        print(f"  object {i}: |dxyz| {d[i]:.3e} mm, score {got['score'][i]:.9g} vs "
              f"{want['score'][i]:.9g}, flag {got['flags'][i]} vs {want['flags'][i]}")
    assert n4 <= max(1, int(0.002 * n))
    assert flags_diff <= max(1, int(0.002 * n))
    ok = d <= 1e-9
    assert np.allclose(got["score"][ok], want["score"][ok], rtol=1e-9)


@pytest.mark.parametrize("kind", ["small", "cfg1"])
def test_shake_fp32_against_fp64_reference(kind):
    """FP32 production shake (residual, OTF Gaussian and sums in FP32) against the
    reference: the distribution of position errors and the count of objects beyond
    1e-4 mm (decisions that FP32 rounding flips), printed; at most 2% beyond 1e-4 mm."""
    got, want, d = _shake_cmp(kind, 0)
    n = len(d)
    n4 = int(np.sum(d > 1e-4))
    print(f"fp32 shake {kind}: {n} objects, median {np.median(d):.3g} mm, p99 "
          f"{np.quantile(d, .99):.3g} mm, max {d.max():.3g} mm, beyond 1e-4 mm {n4} "
          f"({n4 / max(n, 1):.4f}), flags differ {int(np.sum(got['flags'] != want['flags']))}")
    assert n4 <= max(2, int(0.02 * n))
