"""The C++ drop-in classes and their Python module (pyopenlpt) without a
GPU: module surface, the reference's config and camera formats, TIFF reading (against
the reference's own image fixtures when the reference tree is mounted)."""
import os
import tempfile

import numpy as np
import pytest

from oracle.refdir import reference_dir
from pyopenlpt_b200 import openlpt  # noqa: F401  (puts the compiled module on sys.path)
from pyopenlpt_b200 import synth

import pyopenlpt as lpt  # noqa: E402  the reference's own import line

REFERENCE = reference_dir()


def test_module_surface():
    for name in ("Camera", "OTF", "Image", "ImageIO", "Pt2D", "Pt3D", "Tracer2D", "Tracer3D",
                 "ObjFlag", "BasicSetting", "TracerConfig", "STBParam", "ShakeParam", "PFParam",
                 "SMParam", "IPRParam", "ObjectConfig", "ObjectFinder2D", "StereoMatch", "Shake", "IPR", "STB",
                 "Track", "run"):
        assert hasattr(lpt, name), name


def _seq():
    return synth.make_sequence(n_particles=300, n_frames=6, n_row=128, n_col=160, focal=1250.0,
                               volume=(-10, 10, -8, 8, -5, 5), a=200.0, noise=2.0, bits=8, seed=1)


def test_config_camera_and_tiff_round_trip():
    seq = _seq()
    with tempfile.TemporaryDirectory() as d:
        main = synth.write_stb_config(seq, d, synth.IPRSettings(), synth.STBSettings(),
                                      image_format="tif")
        bs = lpt.BasicSetting()
        assert bs.readConfig(main)
        assert bs._n_cam == 4 and bs._frame_start == 0 and bs._frame_end == 5
        assert bs._output_path.endswith("/") and bs._object_types == ["Tracer"]
        assert (bs._axis_limit.x_min, bs._axis_limit.z_max) == (-10.0, 5.0)
        for cam, sc in zip(bs._cam_list, seq.cams):
            assert (cam.getNRow(), cam.getNCol()) == (sc.n_row, sc.n_col)
            assert cam._max_intensity == seq.max_val and cam._is_active
        for c in range(4):
            io = lpt.ImageIO("", bs._image_file_paths[c])
            for t in (0, 5):
                im = io.loadImg(t)
                assert np.array_equal(im.to_numpy(), seq.frames[t][c])
        # Image.save writes a TIFF the reader reads back
        im = lpt.Image.from_numpy(seq.frames[1][2])
        p = os.path.join(d, "x.tif")
        im.save(p)
        with open(os.path.join(d, "l.txt"), "w") as f:
            f.write(p + "\n")
        assert np.array_equal(lpt.ImageIO("", os.path.join(d, "l.txt")).loadImg(0).to_numpy(),
                              seq.frames[1][2])


def test_bad_inputs_raise():
    with pytest.raises(RuntimeError):
        lpt.Camera("/nonexistent/cam.txt")
    bs = lpt.BasicSetting()
    assert not bs.readConfig("/nonexistent/config.txt")
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "cam.txt")
        with open(p, "w") as f:
            f.write("PINPLATE\n")
        with pytest.raises(RuntimeError):
            lpt.Camera(p)


def _load(path):
    with tempfile.TemporaryDirectory() as d:
        lst = os.path.join(d, "l.txt")
        with open(lst, "w") as f:
            f.write(path + "\n")
        return lpt.ImageIO("", lst).loadImg(0).to_numpy()


@pytest.mark.skipif(REFERENCE is None, reason="reference tree not mounted")
def test_tiff_reader_on_reference_fixtures():
    """PackBits and LZW+predictor TIFFs of the reference's tests: detections on the
    decoded images match the reference's known answers."""
    from scipy.spatial import cKDTree

    from oracle.ref import RefOracle
    sc = synth.make_scene(n_particles=10, size=1024, seed=1)
    ref = RefOracle(sc, synth.IPRSettings(min_obj_int=30), threads=4)
    img = _load(f"{REFERENCE}/test/inputs/test_ObjectFinder/test_function_1.tif")
    assert img.dtype == np.uint8 and img.shape == (1024, 1024)
    # the reference finds 8,030 tracers on this image with threshold 30
    assert len(ref.find_peaks(img)) == 8030
    img = _load(f"{REFERENCE}/test/inputs/test_IPR/img_cam1.tif")
    xy = ref.find_peaks(img)
    gt = np.loadtxt(f"{REFERENCE}/test/solutions/test_ObjectFinder/pt2d_list_cam1.csv",
                    delimiter=",")
    d, _ = cKDTree(xy).query(gt)
    assert np.mean(d < 1.0) > 0.99
