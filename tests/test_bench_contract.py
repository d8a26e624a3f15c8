"""bench.py's JSON line, reference arm (CPU only): the keys and types the measurement contract asks
for, on the same metric as the GPU arm. The arm runs here on the small cantilever (the full
workload's setup solves 3.2 M DOFs to 1e-8 on the CPU, minutes on this host); the default
workload's description is checked without running it."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--workload", "small"], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["metric"].startswith("Newton iters/s") and d["unit"] == "Newton iter/s"
    assert d["higher_is_better"] is True and d["value"] > 0 and d["steps"] == 1
    assert d["config"]["n_dof"] == 8019
    m = d["measured"]
    assert m["krylov_its"] > 0 and m["krylov_status"] == 0 and m["threads"] >= 1 and m["cg_iter_s"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_default_workload_is_the_3m_dof_cantilever():
    sys.path.insert(0, ROOT)
    import bench
    cfg = bench._config(bench._workload("large"), 1e-8)
    assert cfg["workload"].startswith("hex8_cantilever_256x64x64")
    assert cfg["n_dof"] == 3257475 and cfg["n_elem"] == 1048576
