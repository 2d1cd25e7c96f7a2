"""bench.py's measurement logic on the CPU: the spread schedule of timed
steps, the algorithmic-byte model of the roofline, the DRAM traffic read from
the committed ncu summaries, and the bf16 verdict."""
import importlib.util
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("warmup,steps,run", [(5, 20, 500), (3, 10, 1000), (5, 20, 300), (3, 2, 6), (5, 20, 10)])
def test_timed_steps_spread_over_the_run(bench, warmup, steps, run):
    idx = bench.timed_schedule(warmup, steps, run)
    span = max(run - warmup, steps)
    assert len(idx) == steps
    assert all(b > a for a, b in zip(idx, idx[1:]))
    assert idx[0] >= warmup and idx[-1] < warmup + span
    gaps = [b - a for a, b in zip(idx, idx[1:])]
    if gaps:
        assert max(gaps) - min(gaps) <= 1  # evenly spread
    if run - warmup >= 2 * steps:
        assert idx[-1] >= warmup + span - span // steps - 1  # reaches the end of the run


def test_algorithmic_bytes_follow_the_per_pass_model(bench):
    nd, n, P = 102400, 131296, 3_200_000
    ab = bench.algorithmic_bytes
    # one CG iteration: 32 B per stored pair + 112 B per fluid particle
    assert ab("cg_a", nd, n, P) + ab("cg_b", nd, n, P) == 32 * P + 112 * nd
    # build: lists written and read once more for density and Aii
    assert ab("nbr_build", nd, n, P) == 32 * P + 92 * n
    it = {"outer": 2.0, "cg": 4.0, "visc": 0.0, "visc_on": False, "st": 0.0}
    expect = (3 * ab("pack", nd, n, P) + 2 * ab("rhs", nd, n, P) + 4 * (32 * P + 112 * nd)
              + ab("divergence", nd, n, P) + 48 * nd)
    assert ab("ip_solve", nd, n, P, it) == pytest.approx(expect)
    # per-pass list bytes dominate: every pass streams 16 B per pair
    assert ab("ip_solve", nd, n, P, it) > 16 * P * (3 + 2 + 8)


def test_traffic_lines_of_the_profiles_parse(bench):
    pat = re.compile(r"traffic kernel=(\S+) workload=(\S+) dram_bytes_per_launch=(\d+)")
    found = {}
    d = os.path.join(REPO, "profiles")
    for name in os.listdir(d):
        with open(os.path.join(d, name)) as f:
            for line in f:
                m = pat.search(line)
                if m:
                    found[(m.group(1), m.group(2))] = int(m.group(3))
    # the dominant kernel of every benchmarked workload has a capture
    for key in [("ip_solve", "tall_column"), ("ip_solve", "dam_break"), ("ip_solve", "batch64")]:
        assert key in found and found[key] > 0, key
    known = {"ip_solve", "visc", "surface_tension", "nbr_build", "prj"}
    assert {k for k, _ in found} <= known


def test_traffic_scaled_only_where_rows_stream_from_dram(bench):
    dram, alg = bench.load_traffic("ip_solve", "dam_break")
    assert dram and alg
    t = bench.traffic_for("ip_solve", "dam_break", 2 * alg)
    assert t["traffic"] == pytest.approx(2 * dram) and t["traffic_captured"] == dram
    col = bench.traffic_for("ip_solve", "tall_column", 1e9)
    assert col["traffic"] == bench.load_traffic("ip_solve", "tall_column")[0]
    assert "unscaled" in col["traffic_note"]
    assert bench.traffic_for("ip_solve", "no_such_workload", 1e9) == {"traffic": None}


def test_bf16_variant_is_rejected(bench):
    slow = bench.bf16_verdict({"ms_per_step": 0.8, "valid": True}, 0.6)
    fast = bench.bf16_verdict({"ms_per_step": 0.5, "valid": True}, 0.6)
    assert slow["verdict"] == "rejected" and len(slow["reasons"]) == 2
    # faster alone does not accept it: its error misses the FP32 bound
    assert fast["verdict"] == "rejected" and len(fast["reasons"]) == 1
