"""Shared seeded scenes and CPU oracles for the test-suite."""
import functools

import numpy as np

from pyopenlpt_b200 import synth


@functools.lru_cache(maxsize=None)
def scene(kind: str = "small"):
    if kind == "small":     # fast: 2,000 particles, 4 x 512^2 u8
        return synth.make_scene(n_particles=2000, size=512, focal=2500.0, seed=7)
    if kind == "cfg1":      # the single-frame IPR scene: 10k particles, 4 x 1024^2 u8
        return synth.make_scene()
    if kind == "u16":       # 12-bit images, 3 cameras, non-square
        return synth.make_scene(n_particles=1500, n_cam=3, n_row=400, n_col=640, focal=2500.0,
                                a=3000.0, noise=20.0, bits=12, seed=11)
    if kind == "poly":      # 6 cubic polynomial cameras, 512^2 12-bit, 5x5x5 OTF, 0.01 ppp
        return synth.make_poly_scene(ppp=0.01, size=512, n_cam=6, seed=7)
    raise KeyError(kind)


def settings(kind: str = "small") -> synth.IPRSettings:
    """IPR knobs; match_cam_count capped at n_cam as readCommonConfig does
    (src/srcSTB/Config.cpp:222-224)."""
    s = synth.IPRSettings()
    s.match_cam_count = min(s.match_cam_count, scene(kind).n_cam)
    if kind == "poly":
        # every camera in the build: with check cameras the reference's checkMatch
        # leaves e_check NaN and match() throws (StereoMatch.cpp:120-127, 505-600)
        s.min_obj_int, s.shake_width, s.tol_3d_mm = 300, 0.025, 0.03
        s.match_cam_count = scene(kind).n_cam
    return s


@functools.lru_cache(maxsize=None)
def ref_oracle(kind: str = "small", threads: int = 0):
    from oracle.ref import RefOracle
    return RefOracle(scene(kind), settings(kind), threads=threads)


def gpu_context(sc):
    from pyopenlpt_b200 import _ffi
    ctx = _ffi.Context(0)
    ctx.upload_cameras([_ffi.camera_desc(c) for c in sc.cams])
    if sc.otf_table is not None:
        ctx.upload_otf(*sc.otf_n, sc.volume, sc.otf_table)
    else:
        from oracle.ref import otf_table
        ctx.upload_otf(2, 2, 2, sc.volume, otf_table(sc.n_cam, sc.otf_abc))
    return ctx
