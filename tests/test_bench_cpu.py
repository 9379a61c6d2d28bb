"""bench.py's reference arm (the CPU restatement timed on the host cores) on the CPU: one JSON
line with the GPU arm's metric, unit and workload shapes, the host sample named, e2e with no copies."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_line_with_the_gpu_arms_config():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                          "--cpu-per-core", "4"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["higher_is_better"] is True
    assert d["metric"] == "certified subdomain bounds/sec" and d["unit"] == "subdomains/s"
    assert d["config"]["workload"] == "dense_q_n200" and d["config"]["batch"] == 65536
    assert d["config"]["n"] == 200 and d["config"]["spec_rows"] == 51
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"]
