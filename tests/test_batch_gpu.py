"""olpt_ipr_run_batch: independent frames on several contexts at once give exactly
the objects each context gives on its own."""
import numpy as np
import pytest

from pyopenlpt_b200 import _ffi, learned as L, synth

pytestmark = pytest.mark.gpu


def test_batch_equals_one_at_a_time():
    scenes = [L.scene(700 + i, 0.02, size=512) for i in range(3)]
    s, _ = L.rig_settings(scenes[0])
    ctxs = [_ffi.Context(0) for _ in scenes]
    try:
        p = _ffi.ipr_params(s, scenes[0].volume)
        alone = []
        for c, sc in zip(ctxs, scenes):
            L.bind(c, sc)
            n = c.ipr_run(p)
            alone.append(c.ipr_result(n)[0])
        for c, sc in zip(ctxs, scenes):
            L.bind(c, sc)
        counts = _ffi.ipr_run_batch(ctxs, p)
        for c, n, want in zip(ctxs, counts, alone):
            got, _ = c.ipr_result(int(n))
            assert np.array_equal(got, want)
        with pytest.raises(_ffi.OlptError):
            _ffi.ipr_run_batch([ctxs[0], ctxs[0]], p)
    finally:
        for c in ctxs:
            c.close()
