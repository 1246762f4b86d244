"""CPU checks of bench.py's reporting helpers (no GPU work)."""
import importlib.util
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", REPO / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_traffic_estimate_scales_the_committed_captures():
    """Traffic = the capture's bytes per relaxation x this launch's
    relaxations (c2 from the c2 capture, c3/c5 from the c3-shaped one), only
    for a launch at the capture's near/far step; the DRAM rate is reported
    against the random-sector ceiling."""
    bench = load_bench()
    rows = []
    for line in (REPO / "profiles" / "frontier_push_traffic.txt").read_text().splitlines():
        parts = line.split()
        if parts and not line.startswith("#") and len(parts) == 5:
            rows.append((parts[0], int(parts[1]), int(parts[2]), parts[3]))
    assert {r[0] for r in rows} == {"c2", "c3small"}
    for name, b, rl, step in rows:
        for workload in (("c2",) if name == "c2" else ("c3", "c5")):
            t, src, ceil = bench.traffic_estimate(workload, 2 * rl, 10.0, step)
            assert t == pytest.approx(2 * b, rel=1e-9)
            assert f"(step {step})" in src and src.endswith(f"{2 * rl:,} relaxations")
            assert ceil["dram_gbs"] == pytest.approx(2 * b / 0.010 / 1e9)
            assert 0 < ceil["frac"] and ceil["peak_gbs"] > 0
            # a step without a capture: not scaled, and the source says why
            t, src, ceil = bench.traffic_estimate(workload, 2 * rl, 10.0, "another")
            assert t is None and ceil is None and "not scaled" in src
    assert bench.traffic_estimate("c2", 0, 10.0) == (None, None, None)


def test_step_label():
    bench = load_bench()
    inf = float("inf")
    assert bench.step_label([2, 2], [2.0, 2.0], 2.0) == "1"
    assert bench.step_label([2, 2], [inf, inf], 2.0) == "plain"
    assert bench.step_label([2, 0], [1.0, inf], 2.0) == "0.5"
    assert bench.step_label([2, 2], [1.0, 4.0], 2.0) == "mixed"
    assert bench.step_label([0, 1], [inf, inf], 2.0) == "none"


def test_traffic_estimate_without_file(tmp_path):
    bench = load_bench()
    assert bench.traffic_estimate("c2", 10, 1.0, path=tmp_path / "absent.txt") == (None, None, None)
