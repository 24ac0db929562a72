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
    # The per-launch byte counts that roofline.achieved divides by: the 128^3
    # benchmark operator on its sliced copy (FP64) and its FP32 finest level
    # on row tiles and on its sliced copy; the banded copy and 4-byte-column
    # CSR on the 256^3 operator.
    import sys
    sys.path.insert(0, ROOT)
    import bench
    n, nnz, entries = 2097152, 14581760, 14614528
    assert bench.layout_bytes("sliced", n, entries, 8) == 179961860
    assert bench.layout_bytes("csr", n, nnz, 4) == 112656388
    assert bench.layout_bytes("sliced", n, entries, 4) == 104726532
    n2, nnz2 = 16777216, 117047296
    assert bench.layout_bytes("csr32", n2, nnz2, 8) == 1740111876  # the CSR-int32 bytes of the 256^3 operator
    banded = bench.layout_bytes("banded", n2, 7 * n2, 8)
    assert banded == 7 * n2 * 8 + 7 * n2 // 32 * 8 + (n2 // 32 + 1) * 4 + 2 * n2 * 8
    assert banded < 0.72 * 1740111876
    # ncu traffic per launch sits just below the algorithmic bytes (x partly in L2)
    for ratio in bench.TRAFFIC_RATIO.values():
        assert 0.9 < ratio < 1.0
