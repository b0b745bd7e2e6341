"""bench.py's reference arm on the CPU (it runs the reference's own CPU solver,
or the oracle restatement where that library is absent; no GPU): one JSON line
on stdout with the keys and types the benchmark line carries, at a small grid
so the test takes seconds."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--solve-n", "16",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600, env=env,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1 and lines[0].startswith("{"), out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert isinstance(d["metric"], str) and d["unit"] == "ms/solve"
    assert d["value"] > 0 and d["ms_per_step"] == d["value"]
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3  # at least 3 warm-up steps
    assert d["higher_is_better"] is False and d["scaling"] == "weak" and d["vs_baseline"] is None
    assert d["dtype"] == "f64" and "synthetic" in d["data"]
    assert isinstance(d["config"], dict) and "workload" in d["config"] and d["config"]["grid"] == [16, 16, 16]
    cb = d["cpu_baseline"]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref

    kind = "reference" if ref.available() else "port"
    assert cb["value"] == d["value"] and cb["kind"] == kind and cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
