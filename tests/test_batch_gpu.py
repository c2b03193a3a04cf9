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


def _tg_contexts(plan, n_frames):
    import bench  # the workloads' pixel settings
    seqs = [synth.make_tg_sequence(n_frames=n_frames, **p) for p in plan]
    w = bench.WORKLOADS["stb_batch64_tg_u8"]
    out = []
    for q in seqs:
        s, st = bench.px_settings(q, w)
        ctx = _ffi.Context(0)
        ctx.upload_cameras([_ffi.camera_desc(c) for c in q.cams])
        ctx.upload_otf(2, 2, 2, q.volume, q.otf_table)
        ctx.stb_configure(_ffi.stb_params(s, st, q.volume, 0, n_frames - 1, 0))
        out.append(ctx)
    return seqs, out


def test_stb_batch_equals_one_at_a_time():
    """olpt_stb_process_frame_batch over sequences of different camera counts and
    particle counts: every sequence's four track lists equal those of running it alone."""
    plan = [dict(n_particles=2500, n_cam=4, size=512, wavelength=30.0, seed=11),
            dict(n_particles=4000, n_cam=5, size=512, wavelength=45.0, seed=12),
            dict(n_particles=1500, n_cam=6, size=512, wavelength=25.0, seed=13)]
    nf = 7
    seqs, ctxs = _tg_contexts(plan, nf)
    solo_seqs, solo = _tg_contexts(plan, nf)
    try:
        for t in range(nf):
            for q, c in zip(seqs, ctxs):
                c.upload_images(list(q.frames[t]))
            _ffi.stb_process_frame_batch(ctxs, [t] * len(ctxs))
        for q, c in zip(solo_seqs, solo):
            for t in range(nf):
                c.upload_images(list(q.frames[t]))
                c.stb_process_frame(t)
        for i, (a, b) in enumerate(zip(ctxs, solo)):
            for k in range(4):
                ta, tb = a.stb_tracks(k), b.stb_tracks(k)
                print(f"sequence {i} list {k}: {len(np.unique(ta[0]))} tracks, "
                      f"{len(ta[0])} rows")
                assert all(np.array_equal(x, y) for x, y in zip(ta, tb))
        with pytest.raises(_ffi.OlptError):
            _ffi.stb_process_frame_batch([ctxs[0], ctxs[0]], [0, 0])
    finally:
        for c in ctxs + solo:
            c.close()


def test_autotune_keeps_results_and_images():
    """Every launch shape gives the same objects; the autotuner keeps the fastest and
    leaves the uploaded images as they were."""
    sc = L.scene(731, 0.02, size=512)
    s, _ = L.rig_settings(sc)
    ctx = _ffi.Context(0)
    try:
        L.bind(ctx, sc)
        p = _ffi.ipr_params(s, sc.volume)
        before = [ctx.image(c) for c in range(ctx.n_cam)]
        objs = {}
        for shape in [(4, 256, 64), (1, 128, 64), (2, 256, 128), (4, 128, 128)]:
            L.bind(ctx, sc)
            ctx.set_tuning(*shape)
            n = ctx.ipr_run(p)
            objs[shape] = ctx.ipr_result(n)[0]
        ref = objs[(4, 256, 64)]
        assert all(np.array_equal(v, ref) for v in objs.values())
        L.bind(ctx, sc)
        shape, ms = ctx.autotune_ipr(p, reps=1)
        print(f"autotuned launch shapes {shape}: {ms:.2f} ms per IPR")
        assert shape in {(w, r, g) for w in (1, 2, 4) for r in (128, 256) for g in (64, 128)}
        assert ms > 0
        assert ctx.tuning() == shape
        for c in range(ctx.n_cam):
            assert np.array_equal(ctx.image(c), before[c])
        with pytest.raises(_ffi.OlptError):
            ctx.set_tuning(3, 256)
    finally:
        ctx.close()
