"""bench.py's reference arm on the CPU: the JSON line carries the contract's keys (the
metric and config of the GPU arm, impl, cpu_baseline, e2e with zero copies), says which
samples of the workload it ran, honours --warmup, and uses every host core it asks for."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--cpu-n", "48", "--n", "512"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    # the line names the GPU arm's workload and what the CPU ran of it (one sample per core)
    assert "rain-on-terrain dense 512x512" in d["config"]["workload"]
    assert f"x 48x48 samples" in d["config"]["workload"]
    assert d["warmup"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
