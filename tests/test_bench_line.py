"""The last line bench.py prints is what a reader of the run's log tail gets:
it must carry the contract's keys and stay short (a few KB), with every
secondary leg reduced to a one-number summary.  CPU only: the line is built
from a made-up measurement."""
import argparse
import json

import bench


def fake_result():
    return {"step_ms": [0.037] * 20, "total_s": 20 * 37.1e-6, "e2e_s": 20 * 50.3e-6,
            "e2e_copy_s": 20 * 64.2e-6, "ok": True,
            "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965, "reasons": [], "samples": 9,
                       "window": "timed region + the same load, untimed, to 0.4 s"},
            "peak": {"returning": 814.7956780730, "fire_and_forget": 789.07644264598,
                     "per_sector_returning": 149.450346622663,
                     "per_sector_fire_and_forget": 150.0607722463892},
            "hot_word_rate": 1554315762.0585377, "lone_warp_us": 32.76799991726875}


def fake_legs():
    legs = {
        "phase": {"value": 2538803689.062011, "ok": True, "tuned_4_heads": {"value": 3.9e9},
                  "payload": {"frac_of_hbm": 0.0737263}},
        "batched": {"persistent_graph": {"value": 41000739.86064273}, "speedup": 3.31049387,
                    "small_only": {"speedup": 1.6529528388}, "ok": True},
        "graph": {"value": 26107100465.318874, "ok": True},
        "serve": {"points": [{"lambda": 1e6, "jobs_per_s": 944059.3, "p50_ns": 21384.7,
                              "p99_ns": 137697.0},
                             {"lambda": 1e8, "jobs_per_s": 1471859.755, "p50_ns": 11732.77,
                              "p99_ns": 118892.125}], "ok": True},
        "samples": {"ok": True},
        "halloc_programs": {"cases": [{"vs_published": 9.1}, {"vs_published": 0.8}]},
    }
    return {k: bench.leg_summary(k, v) for k, v in legs.items()}


def make_line():
    args = argparse.Namespace(steps=20, warmup=5)
    cpu = {"value": 6830538.278576698, "unit": "pairs/s", "cores": 16,
           "sample": "227 x the full workload (327680 pairs) on 16 threads",
           "kind": "reference"}
    glibc = {"value": 712345678.9, "unit": "pairs/s", "cores": 16, "sample": "..."}
    cm = {"value": 4471234.5678, "heap_bytes": 536870912, "ok": True}
    return bench.headline(args, 1, fake_result(), cpu, glibc, cm, fake_legs())


def test_headline_carries_the_contract_keys():
    line = make_line()
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "e2e", "roofline", "cpu_baseline", "gpu_launches", "clocks"):
        assert key in line, key
    assert line["e2e"]["h2d_bytes_per_step"] == 32768 * 4
    assert line["e2e"]["d2h_bytes_per_step"] == 16
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in line["roofline"], key
    for key in ("value", "unit", "cores", "kind", "sample"):
        assert key in line["cpu_baseline"], key
    assert abs(line["value"] - 327680 / 37.1e-6) / line["value"] < 1e-4
    assert line["legs"]["serve"]["lambda"] == 1e8
    assert line["legs"]["halloc_programs"] == {"rows": 2, "rows_ahead_of_published": 1}


def test_headline_is_short():
    """A 3-KB log tail must hold the whole line."""
    assert len(json.dumps(make_line())) < 2500


def test_leg_summary_of_a_failed_leg():
    assert bench.leg_summary("phase", {"error": "timed out"}) == {"error": "timed out"}
