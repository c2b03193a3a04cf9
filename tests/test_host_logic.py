"""Host-side logic that needs no GPU: the many-sequence generator's flow and plan, the
bench's per-workload settings, and the rounding rule of the track-file formatter
(trackio.cu) restated with exact rationals against Python's own "%.6f"."""
import math
from fractions import Fraction

import numpy as np

from pyopenlpt_b200 import synth


def test_taylor_green_is_divergence_free_with_unit_peak_speed():
    rng = np.random.default_rng(1)
    p = rng.uniform(-20, 20, (2000, 3))
    lam, h = 33.0, 1e-4
    div = np.zeros(len(p))
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        div += (synth.taylor_green_velocity(p + e, lam)[:, k]
                - synth.taylor_green_velocity(p - e, lam)[:, k]) / (2 * h)
    assert np.max(np.abs(div)) < 1e-6
    v = synth.taylor_green_velocity(rng.uniform(-60, 60, (200000, 3)), lam)
    assert np.max(np.linalg.norm(v, axis=1)) <= 1.0 + 1e-12


def test_batch_plan_is_seeded_and_in_range():
    a, b = synth.batch_plan(64, seed=7), synth.batch_plan(64, seed=7)
    assert a == b and a != synth.batch_plan(64, seed=8)
    assert all(2000 <= p["n_particles"] <= 80000 for p in a)
    assert {p["n_cam"] for p in a} <= {4, 5, 6} and {p["size"] for p in a} <= {512, 1024, 2048}
    assert all(20.0 <= p["wavelength"] <= 60.0 for p in a)


def _fixed6_rule(v: float) -> str:
    """The device formatter's rule: f = frac(|v|), p = fl(f * 10^6), e = f * 10^6 - p
    (exact), d = p - floor(p); round up when d > 1/2, or d == 1/2 and (e > 0, or e == 0
    and floor(p) odd)."""
    neg = math.copysign(1.0, v) < 0
    a = abs(v)
    ip = math.floor(a)
    f = a - ip
    p = f * 1e6
    e = Fraction(f) * 1000000 - Fraction(p)
    q = math.floor(p)
    d = p - q
    up = d > 0.5 or (d == 0.5 and (e > 0 or (e == 0 and q % 2 == 1)))
    fr = int(q) + (1 if up else 0)
    if fr >= 1000000:
        fr -= 1000000
        ip += 1
    return ("-" if neg else "") + f"{int(ip)}.{fr:06d}"


def test_fixed6_rule_matches_correct_rounding():
    rng = np.random.default_rng(11)
    vals = [0.0, -0.0, 0.5, 5e-7, -5e-7, 0.9999995, 9.9999995, 0.0078125, 1.0000005,
            123.4567895, 2.0 ** 52 + 1.0, 9.2e18, 1e-320]
    vals += [(2 * k + 1) * 15625 / 2e6 for k in range(-200, 200)]  # exact ties
    grid = rng.integers(-10 ** 12, 10 ** 12, 2000) / 1e6 + 5e-7
    vals += list(grid) + list(np.nextafter(grid, np.inf)) + list(np.nextafter(grid, -np.inf))
    vals += list(rng.standard_normal(5000) * 10.0 ** rng.integers(-9, 16, 5000))
    bad = [v for v in vals if _fixed6_rule(float(v)) != "%.6f" % float(v)]
    assert not bad, bad[:5]
