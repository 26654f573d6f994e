"""The benchmark's reference arm on the host (no GPU): `bench.py --impl reference` times the
reference's kernels built for the host (or the oracle's restatement where that build is absent)
on a bounded gene sample and prints one JSON line whose time is the sample's gene-independent
part plus its per-gene part scaled to all genes."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "0", "--steps", "2",
                        "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "evals/s"
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert "gene-independent part" in cb["sample"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["config"]["workload"].startswith("config 0")
