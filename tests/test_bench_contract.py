"""bench.py's reference arm runs without a GPU: its one JSON line carries the benchmark contract's keys (the metric,
the whole-job value, the timing fields, the CPU-baseline description and an end-to-end figure without transfers) on
the same workload description as the package's arm."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup",
                        "0", "--cpu-budget", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["unit"] == "path·k/s" and d["config"]["paths_per_gpu"] == 189419 and d["config"]["nk"] == 401
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the timing is checkable from the line: a step is the measured sample, the full batch is extrapolated beside it
    t = d["timing"]
    assert t["timed_paths_per_step"] > 0 and t["timed_s"] > 0 and t["ms_full_batch_extrapolated"] > d["ms_per_step"]
    assert abs(t["timed_s"] * 1e3 - d["ms_per_step"] * d["steps"]) <= 0.5 * t["timed_s"] * 1e3
    assert sorted(d["config"]["legs"]) == [str(n) for n in range(2, 9)] or sorted(d["config"]["legs"]) == list(range(2, 9))
