"""The benchmark's reference arm on the CPU: `bench.py --impl reference` times
the reference's own CPU engine (oracle/_ref, built from the reference's
sources) on the c2 workload and prints the bench JSON line with
impl = "reference".  The arm must run the reference alone: the process never
loads libbfx (the graph, layout and queries come from the reference library
and pure-Python samplers), so its number says nothing about this project's
code.  Run here on 16 of the 256 queries, one step."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent

PROBE = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--queries", "16", "--steps", "1", "--warmup", "0"]
runpy.run_path("bench.py", run_name="__main__")
libs = sorted({line.split()[-1] for line in open("/proc/self/maps") if line.rstrip().endswith(".so")})
print("LOADED " + " ".join(libs))
"""


def test_reference_arm_runs_the_reference_alone():
    sys.path.insert(0, str(REPO))
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("oracle/_ref is not built (the reference checkout is absent)")
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    line = json.loads(next(l for l in lines if l.startswith("{")))
    loaded = next(l for l in lines if l.startswith("LOADED ")).split()[1:]
    assert line["impl"] == "reference"
    assert line["metric"].startswith("batched SSSP queries/s (256 uneven regional queries")
    assert line["unit"] == "queries/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["config"]["queries_per_step"] == 16
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "queries/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert not any(Path(p).name == "libbfx.so" for p in loaded), loaded
    assert any("oracle/_ref" in p for p in loaded), loaded
