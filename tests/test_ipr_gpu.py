"""IPR driver parity (IPR::runIPR): object count and positions against the
reference on the same seeded images; recall and ghost rate against ground truth."""
import numpy as np
import pytest

from pyopenlpt_b200 import _ffi
from tests import _metrics, _scenes

pytestmark = pytest.mark.gpu


def _run(kind, precision, **over):
    sc = _scenes.scene(kind)
    s = _scenes.settings(kind)
    for k, v in over.items():
        setattr(s, k, v)
    ctx = _scenes.gpu_context(sc)
    ctx.upload_images(sc.images)
    n = ctx.ipr_run(_ffi.ipr_params(s, sc.volume, precision))
    xyz, uv = ctx.ipr_result(n)
    return sc, s, xyz, uv


def _ref(kind, s):
    from oracle.ref import RefOracle
    sc = _scenes.scene(kind)
    return RefOracle(sc, s, threads=0).ipr(sc.images)


@pytest.mark.parametrize("over", [{}, {"n_cam_reduced": 1, "n_loop_ipr": 2}])
def test_ipr_fp64_matches_reference(over):
    sc, s, xyz, uv = _run("small", 1, **over)
    want = _ref("small", s)
    n_ref = len(want["xyz"])
    print(f"IPR fp64: gpu {len(xyz)} ref {n_ref}")
    assert abs(len(xyz) - n_ref) <= max(3, 0.005 * n_ref)
    d = _metrics.match(want["xyz"], xyz)
    frac = np.mean(d <= 1e-4)
    print(f"  reference objects reproduced within 1e-4 mm: {frac:.4f}")
    assert frac >= 0.99


def test_ipr_fp32_recall_ghost():
    sc, s, xyz, uv = _run("small", 0)
    want = _ref("small", s)
    r_g, g_g = _metrics.recall_ghost(xyz, sc.xyz, 0.1)
    r_r, g_r = _metrics.recall_ghost(want["xyz"], sc.xyz, 0.1)
    print(f"IPR fp32: recall {r_g:.4f} ghost {g_g:.4f} | reference recall {r_r:.4f} ghost {g_r:.4f}")
    assert r_g >= r_r - 0.005
    assert g_g <= g_r + 0.005
