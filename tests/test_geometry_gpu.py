"""GPU parity of the FP64 geometry (camera model, line of sight, triangulation,
OTF lookup) against the reference compiled from source: bit-exact."""
import numpy as np
import pytest

from tests import _scenes

pytestmark = pytest.mark.gpu


def _pts(sc, n, seed=0):
    rng = np.random.default_rng(seed)
    lo = np.array(sc.volume[0::2]); hi = np.array(sc.volume[1::2])
    return lo + (hi - lo) * rng.random((n, 3))


@pytest.mark.parametrize("kind", ["small", "u16"])
def test_project_and_los_bit_exact(kind):
    sc = _scenes.scene(kind)
    ref = _scenes.ref_oracle(kind)
    ctx = _scenes.gpu_context(sc)
    xyz = _pts(sc, 5000)
    for c in range(sc.n_cam):
        uv_g = ctx.project(c, xyz)
        uv_r = ref.project(c, xyz)
        assert np.array_equal(uv_g, uv_r), f"project cam {c}"
        los_g = ctx.los(c, uv_r)
        los_r = ref.los(c, uv_r)
        assert np.array_equal(los_g, los_r), f"los cam {c}"


def test_triangulation_bit_exact():
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    ctx = _scenes.gpu_context(sc)
    xyz = _pts(sc, 2000, seed=3)
    rng = np.random.default_rng(5)
    lines = []
    for c in range(sc.n_cam):
        uv = ref.project(c, xyz) + rng.normal(0, 0.3, size=(len(xyz), 2))
        lines.append(ref.los(c, uv))
    lines = np.stack(lines, axis=1)  # (n, 4, 6)
    for k in (2, 3, 4):
        out, ok = ctx.triangulate(lines[:, :k])
        for i in range(0, len(xyz), 7):
            r = ref.triangulate(lines[i, :k])
            assert ok[i] == (r is not None)
            if r is not None:
                assert np.array_equal(out[i], r), (k, i)


def test_otf_param_matches_reference():
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    ctx = _scenes.gpu_context(sc)
    xyz = _pts(sc, 1000, seed=9) * 1.2   # also outside the grid (clamped)
    for c in range(sc.n_cam):
        assert np.array_equal(ctx.otf_param(c, xyz), ref.otf_param(c, xyz))
