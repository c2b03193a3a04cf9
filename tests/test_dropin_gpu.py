"""The drop-in classes (pyopenlpt_b200.openlpt) driven the way the reference's
users drive pyopenlpt, against the reference compiled here: ObjectFinder2D, IPR,
Shake and the whole STB pipeline from reference-format config files (OTF estimated
from the first frames as TracerConfig::readConfig does), and run(config)."""
import functools
import os
import tempfile

import numpy as np
import pytest

from pyopenlpt_b200 import openlpt as lpt
from pyopenlpt_b200 import synth
from tests import _metrics, _scenes

pytestmark = pytest.mark.gpu

N_FRAMES = 7


@functools.lru_cache(maxsize=None)
def _seq():
    return synth.make_sequence(n_particles=1500, n_frames=N_FRAMES, n_row=512, n_col=512,
                               focal=2500.0, volume=(-20, 20, -20, 20, -10, 10), a=200.0,
                               noise=2.0, bits=8, gamma=4e3, r_core=6.0, drift=(5.0, 0.0, 0.0),
                               seed=5)


def _settings(seq):
    ipr = synth.IPRSettings(n_loop_ipr=2, n_shake_loop=2)
    ipr.match_cam_count = min(ipr.match_cam_count, seq.n_cam)
    return ipr, synth.STBSettings(pf_nx=9, pf_ny=9, pf_nz=5)


def _tracer_config(sc, s):
    """A TracerConfig filled in Python (no config file), OTF from the scene's table."""
    cfg = lpt.TracerConfig()
    cfg._min_obj_int = int(s.min_obj_int)
    cfg._radius_obj = s.radius_obj
    cfg._shake_param._shake_width = s.shake_width
    cfg._shake_param._shakewidth_min = s.shakewidth_min
    cfg._shake_param._n_shake_loop = s.n_shake_loop
    cfg._shake_param._thred_ghost = s.thred_ghost
    cfg._sm_param.match_cam_count = s.match_cam_count
    cfg._sm_param.tol_2d_px = s.tol_2d_px
    cfg._sm_param.tol_3d_mm = s.tol_3d_mm
    cfg._sm_param.limit = lpt.AxisLimit(*sc.volume)
    cfg._ipr_param.n_cam_reduced = s.n_cam_reduced
    cfg._ipr_param.n_loop_ipr = s.n_loop_ipr
    cfg._ipr_param.n_loop_ipr_reduced = s.n_loop_ipr_reduced
    cfg.precision = 1
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "otf.txt"), "w") as f:
        f.write(synth.otf_text(sc.n_cam, sc.volume, *sc.otf_abc))
    cfg._otf = lpt.OTF(os.path.join(d, "otf.txt"))
    return cfg


def _cams(sc):
    d = tempfile.mkdtemp()
    return [lpt.Camera(p) for p in synth.write_scene_files(sc, d)]


def test_object_finder_bit_exact():
    sc = _scenes.scene("small")
    ref = _scenes.ref_oracle("small")
    cfg = _tracer_config(sc, _scenes.settings("small"))
    for c in range(sc.n_cam):
        objs = lpt.ObjectFinder2D().findObject2D(lpt.Image.from_numpy(sc.images[c]), cfg)
        xy = np.array([[o._pt_center[0], o._pt_center[1]] for o in objs])
        assert np.array_equal(xy, ref.find_peaks(sc.images[c]))
        assert all(o._r_px == cfg._radius_obj for o in objs[:5])


def test_ipr_and_shake_match_reference():
    sc = _scenes.scene("small")
    s = _scenes.settings("small")
    cfg = _tracer_config(sc, s)
    cams = _cams(sc)
    imgs = [lpt.Image.from_numpy(im) for im in sc.images]
    objs = lpt.IPR(cams).runIPR(cfg, imgs)
    want = _scenes.ref_oracle("small").ipr(sc.images)["xyz"]
    got = np.array([o._pt_center.to_list() for o in objs])
    print(f"drop-in IPR: {len(got)} objects, reference {len(want)}")
    assert abs(len(got) - len(want)) <= max(3, 0.005 * len(want))
    assert np.mean(_metrics.match(want, got) <= 1e-4) >= 0.99
    assert len(objs[0]) == sc.n_cam  # 2D projections on every camera
    # Shake of perturbed ground truth: same moves and flags as the reference's Shake
    truth = sc.xyz[:200]
    rng = np.random.default_rng(0)
    start = truth + rng.normal(0, 0.02, truth.shape)
    tr = [lpt.Tracer3D(lpt.Pt3D(*p)) for p in start]
    flags, out = lpt.Shake(cams, cfg).runShake(tr, imgs)
    assert out is not None and len(flags) == len(tr)
    moved = np.array([o._pt_center.to_list() for o in tr])
    want = _scenes.ref_oracle("small").shake(start, sc.images)
    assert np.max(np.abs(moved - want["xyz"])) <= 1e-4
    assert [int(f) for f in flags] == list(want["flags"])
    res = lpt.Shake(cams, cfg).calResidualImage(tr, imgs, flags)
    assert len(res) == sc.n_cam and res[0].getDimRow() == sc.images[0].shape[0]


def _write(seq, fmt):
    ipr, stb = _settings(seq)
    d = tempfile.mkdtemp()
    return synth.write_stb_config(seq, d, ipr, stb, image_format=fmt), d


def test_stb_from_config_matches_reference():
    """STB(setting, "Tracer", cfg) on TIFF frames against the reference STB built from
    the same configs: the estimated OTF and the four track lists after every frame."""
    from oracle.ref import RefSTB
    seq = _seq()
    ipr, stb = _settings(seq)
    ref = RefSTB(seq, ipr, stb, threads=0, otf_override=False)
    main, folder = _write(seq, "tif")
    bs = lpt.BasicSetting()
    assert bs.readConfig(main)
    st = lpt.STB(bs, "Tracer", bs._object_config_paths[0], precision=1)
    otf = st._obj_config._otf
    ours = np.stack([otf.a, otf.b, otf.c, otf.alpha])
    want = ref.otf()
    print("OTF (a, b, c) cam 0:", ours[:3, 0, 0], "reference", want[:3, 0, 0])
    assert np.allclose(ours, want, rtol=1e-12, atol=1e-12)
    io = [lpt.ImageIO("", p) for p in bs._image_file_paths]
    names = {"long_active": "_long_track_active", "short_active": "_short_track_active",
             "long_inactive": "_long_track_inactive", "exit": "_exit_track"}
    for t in range(N_FRAMES):
        imgs = [x.loadImg(t) for x in io]
        out = st.process_frame(t, imgs)
        ref.frame(t)
        assert len(out) == seq.n_cam
        if t < stb.n_initial_frames:  # initial phase: img_list unchanged
            assert np.array_equal(out[0].to_numpy(), seq.frames[t][0].astype(np.float64))
        rt = ref.tracks()
        for k, attr in names.items():
            mine = getattr(st, attr)
            n_ref = len(np.unique(rt[k][:, 0])) if len(rt[k]) else 0
            print(f"frame {t} {k}: drop-in {len(mine)} reference {n_ref}")
            assert abs(len(mine) - n_ref) <= max(2, 0.01 * n_ref)
    ref.close()


def test_run_writes_reference_track_files():
    """run(config) -- the reference's command-line loop -- writes the track files."""
    seq = _seq()
    main, folder = _write(seq, "tif")
    assert lpt.run(main) == 0
    conv = os.path.join(folder, "out", "ConvergeTrack")
    names = sorted(os.listdir(conv))
    assert f"LongTrackActive_{N_FRAMES - 1}.csv" in names
    with open(os.path.join(conv, f"LongTrackActive_{N_FRAMES - 1}.csv")) as f:
        head = f.readline().strip()
    assert head.startswith("TrackID,FrameID,WorldX,WorldY,WorldZ,cam0_x(col),cam0_y(row)")
    assert sorted(os.listdir(os.path.join(folder, "out", "InitialTrack")))
