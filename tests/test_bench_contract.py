"""bench.py's reference arm (the CPU oracle on the host cores) prints one JSON
line with the keys the benchmark contract asks for; no GPU needed."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    # a small grid (the contract, not the number, is under test here)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--size", "24"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["higher_is_better"] is False and d["unit"] == "s"
    assert d["value"] > 0 and d["iterations"] > 0
    assert d["config"]["rows"] == 24 ** 3 and "24^3" in d["config"]["workload"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_algorithmic_bytes_of_the_reported_kernels():
    # The per-launch byte counts that roofline.achieved divides by, for the
    # 128^3 benchmark operator: FP64 operator on its sliced copy, FP32
    # finest level on row tiles (2-byte columns) and on its sliced copy.
    import sys
    sys.path.insert(0, ROOT)
    import bench
    n, nnz, entries = 2097152, 14581760, 14614528
    assert bench.layout_bytes("sliced", n, entries, 8) == 179961860
    assert bench.layout_bytes("csr", n, nnz, 4) == 112656388
    assert bench.layout_bytes("sliced", n, entries, 4) == 104726532
    # ncu traffic per launch sits just below the algorithmic bytes (x partly in L2)
    assert 0.9 < bench.SPMV_TRAFFIC["sliced"] / 179961860 < 1.0
    assert 0.9 < bench.SPMV32_TRAFFIC["csr"] / 112656388 < 1.0
    assert 0.9 < bench.SPMV32_TRAFFIC["sliced"] / 104726532 < 1.0
