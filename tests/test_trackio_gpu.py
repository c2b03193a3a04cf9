"""Track files formatted on the device: every number as the C library's "%.6f" prints
it (the reference writes them with std::fixed and precision 6), checked value by value
against snprintf on rounding ties, carries, signed zeros, tiny and large magnitudes,
NaN and infinities; the writer thread's files against the synchronous ones."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from pyopenlpt_b200 import _ffi
from tests._scenes import gpu_context, scene

pytestmark = pytest.mark.gpu

_libc = ctypes.CDLL(None)


def _c_fixed6(v: float) -> str:
    b = ctypes.create_string_buffer(400)
    _libc.snprintf(b, ctypes.c_size_t(400), b"%.6f", ctypes.c_double(v))
    return b.value.decode()


def _cases(rng):
    edge = [0.0, -0.0, 1.0, -1.0, 0.5, 1e-7, -1e-7, 4e-7, 5e-7, -5e-7, 6e-7, 0.0000005,
            0.9999995, 0.99999949999, 9.9999995, -9.9999995, 0.0078125, -0.0078125,
            2.0 ** -7 * 3, 1.0000005, 123.4567895, 1e15 + 0.5, 2.0 ** 52 + 1.0,
            2.0 ** 53, 9.2e18, -9.2e18, float(np.nextafter(2.0 ** 63, 0)), 1e-320, -1e-320,
            5e-324, 2.2250738585072014e-308, float("nan"), float("-nan"), float("inf"),
            float("-inf")]
    # exact ties k / 2 * 10^-6 that are dyadic: odd multiples of 2^-7 (5^6 divides them)
    ties = [(2 * k + 1) * 15625 / 2e6 for k in range(-300, 300)]
    # values next to the rounding boundaries of a random decimal grid
    grid = rng.integers(-10 ** 12, 10 ** 12, 4000) / 1e6 + 5e-7
    near = np.concatenate([grid, np.nextafter(grid, np.inf), np.nextafter(grid, -np.inf)])
    mags = rng.standard_normal(20000) * 10.0 ** rng.integers(-9, 16, 20000)
    bits = rng.integers(0, 2 ** 63 - 1, 5000, dtype=np.int64).view(np.float64)
    bits = bits[np.isfinite(bits) & (np.abs(bits) < 2.0 ** 63)]
    return np.concatenate([np.array(edge), np.array(ties), near, mags, bits, -bits])


def test_fixed6_matches_snprintf():
    ctx = _ffi.Context(0)
    try:
        vals = _cases(np.random.default_rng(5))
        got = ctx.format_fixed6(vals).split("\n")
        assert got[-1] == "" and len(got) == len(vals) + 1
        bad = [(v, g, _c_fixed6(v)) for v, g in zip(vals, got) if g != _c_fixed6(v)]
        for v, g, w in bad[:10]:
            print(f"{v!r}: device {g!r}, C library {w!r}")
        assert not bad, f"{len(bad)} of {len(vals)} values differ"
        with pytest.raises(_ffi.OlptError):
            ctx.format_fixed6([1.0, 2.0 ** 63])
        assert ctx.format_fixed6([]) == ""
    finally:
        ctx.close()


def test_async_files_equal_sync_files():
    ctx = gpu_context(scene("small"))
    try:
        rng = np.random.default_rng(9)
        n_tracks = 3000
        lens = rng.integers(1, 9, n_tracks)
        tid = np.repeat(np.arange(n_tracks, dtype=np.int32), lens)
        fr = np.concatenate([np.arange(l, dtype=np.int32) + 7 for l in lens])
        xyz = rng.uniform(-20, 20, (tid.size, 3))
        ctx.stb_set_tracks(_ffi.TRACK_LONG_ACTIVE, tid, fr, xyz)
        with tempfile.TemporaryDirectory() as d:
            a, b = os.path.join(d, "sync.csv"), os.path.join(d, "async.csv")
            ctx.stb_save_tracks(_ffi.TRACK_LONG_ACTIVE, a)
            ctx.track_files_async(True)
            ctx.stb_save_tracks(_ffi.TRACK_LONG_ACTIVE, b)
            ctx.flush_track_files()
            ctx.track_files_async(False)
            with open(a, "rb") as f1, open(b, "rb") as f2:
                ra, rb = f1.read(), f2.read()
            assert ra == rb
            lines = ra.decode().splitlines()
            assert len(lines) == tid.size + 1
            # each row against the C library's formatting of the same numbers
            uv = [ctx.project(c, xyz) for c in range(ctx.n_cam)]
            for r in rng.integers(0, tid.size, 300):
                fields = [str(tid[r]), str(fr[r])] + [_c_fixed6(x) for x in xyz[r]]
                for c in range(ctx.n_cam):
                    fields += [_c_fixed6(uv[c][r, 0]), _c_fixed6(uv[c][r, 1])]
                assert lines[1 + r] == ",".join(fields)
            # a write error surfaces at the flush
            ctx.track_files_async(True)
            ctx.stb_save_tracks(_ffi.TRACK_LONG_ACTIVE, os.path.join(d, "no", "such.csv"))
            with pytest.raises(_ffi.OlptError):
                ctx.flush_track_files()
            ctx.flush_track_files()  # reported once
    finally:
        ctx.close()
