"""CPU: bench.py's reference arm prints one JSON line with the keys the
benchmark contract names (it runs the reference's own CPU build from
oracle/_ref, so it needs no GPU)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

import oracle

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(oracle.ref() is None, reason="oracle/_ref not built")
def test_reference_arm_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--workload", "plain4m", "--scale", "0.01", "--steps", "2",
                          "--warmup", "1"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["unit"] == "Gsym/s" and d["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": "Gsym/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["value"] == d["value"] and cpu["cores"] >= 1
    assert d["config"]["symbols_per_step"] < 100_000  # the scaled 4 Mbp workload
