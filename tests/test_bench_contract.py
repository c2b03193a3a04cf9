"""The bench's JSON line carries the keys its readers need (metric, value, unit, timing,
config, e2e, roofline with traffic, cpu_baseline, clocks, launches), built here from
fake per-kernel timings without a GPU."""
import contextlib
import io
import json
import types

import bench


def _line(workload, cams, dominant):
    args = types.SimpleNamespace(workload=workload, steps=2, warmup=3)
    me = types.SimpleNamespace(args=args, world=1, prec=0)
    prof = {k: (1.0, 4, 1e6) for k in list(bench.PROF_NAMES) + list(bench.PHASE_NAMES)}
    prof[dominant] = (20.0, 4, 4.0 * 1912 * 10000)
    cfg = {"workload": workload, "cameras": cams}
    cpu = {"value": 250.0, "unit": "particles/s", "cores": 16, "kind": "reference",
           "sample": "fake"}
    clk = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": []}
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.Ours.line(me, prof, 400.0, 2e5, 0.5, 2e5, 50_331_648, 2_835_220, 1480, clk, cfg,
                        cpu, {})
    return json.loads(buf.getvalue())


def test_line_keys_and_roofline():
    d = _line("stb_2048_u16_6cam_poly_419k", 6, 3)
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "e2e",
              "gpu_launches", "roofline", "cpu_baseline", "clocks"):
        assert k in d, k
    assert d["value"] == 2e5 / 0.4 and d["ms_per_step"] == 200.0
    assert d["e2e"]["value"] == 2e5 / 0.5 and d["e2e"]["h2d_bytes_per_step"] == 50_331_648
    r = d["roofline"]
    assert r["kernel"] == bench.PROF_NAMES[3] and r["bound"] == "hbm"
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    # measured DRAM bytes per object for 6 cameras, scaled by the launch's objects
    assert abs(r["traffic"] - 10000 * bench.SHAKE_TRAFFIC[6][0]) < 1e-3


def test_traffic_only_where_measured():
    assert _line("stb_2048_u16_6cam_poly_419k", 5, 3)["roofline"]["traffic"] is None
    assert _line("stb_2048_u16_6cam_poly_419k", 6, 2)["roofline"]["traffic"] is None
    assert _line("stb_batch64_tg_u8", 6, 3)["roofline"]["traffic"] is None
