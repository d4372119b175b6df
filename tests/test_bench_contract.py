"""CPU: bench.py's reference arm prints one JSON line with the contract's
keys (run on a small cylinder so it takes seconds), and the CG byte model
counts the column stream only when the columns are not resident."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                          "--ncross", "10", "--naxial", "8"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["unit"] == "s/timestep" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "k-tet cylinder" in d["config"]["workload"]


def test_cg_byte_model():
    sys.path.insert(0, ROOT)
    import bench

    nnz, n = 1000, 100
    for m in (4, 8):
        streamed = bench.cg_iter_bytes(nnz, n, m, 1)
        resident = bench.cg_iter_bytes(nnz, n, m, 1, resident=True)
        assert streamed - resident == 8 * nnz
        assert resident == nnz * 7 * m + n * (16 + 8 * m + 24 + 16 + 16 + 16 + 16)
