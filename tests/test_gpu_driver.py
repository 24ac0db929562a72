"""The solve-matrix driver (example/solve-matrix.cu:54-180): a manufactured
solution on synthetic Matrix Market files (the reference's real matrices are
not shipped), the key=value report in the reference's order, exit codes."""
import os
import subprocess

import numpy as np
import pytest
import torch

import thermofem_b200 as tf
from conftest import to_device
from thermofem_b200 import build as B
from thermofem_b200 import problems as P

pytestmark = pytest.mark.gpu

KEYS = ["matrix", "rows", "nnz", "preconditioner", "read_seconds", "device", "gpu", "cuda_runtime", "rtol", "atol",
        "max_iterations", "refresh_interval", "phase", "setup_seconds"]


def run(*args, env=None):
    e = dict(os.environ, **(env or {}))
    r = subprocess.run([B.DRIVER, *args], capture_output=True, text=True, env=e, timeout=300)
    kv = {}
    order = []
    for line in r.stdout.splitlines():
        k, _, v = line.partition("=")
        if k == "level":
            kv.setdefault("levels_lines", []).append(line)
        else:
            kv[k] = v
        order.append(k)
    return r.returncode, kv, order, r.stderr


@pytest.fixture(scope="module")
def poisson_mtx(tmp_path_factory):
    path = str(tmp_path_factory.mktemp("mtx") / "laplace64.mtx")
    off, idx, val = P.laplace2d(64)
    P.write_matrix_market(path, off, idx, val, symmetric=True)
    return path, (off, idx, val)


@pytest.mark.parametrize("args", [("amg",), ("amg", "w"), ("amg", "f"), ("identity",)])
def test_driver_passes_manufactured_solution(poisson_mtx, args):
    path, _ = poisson_mtx
    rc, kv, order, err = run(path, *args)
    assert rc == 0, err
    assert kv["validation"] == "PASS" and kv["status"] == "Converged"
    assert order[:len(KEYS)] == KEYS
    assert kv["rows"] == "4096" and kv["preconditioner"] == args[0]
    assert float(kv["host_relative_residual"]) <= 1.01e-8
    assert float(kv["relative_solution_error"]) <= 1e-4
    if args[0] == "amg":
        assert kv["cycle"] == (args[1] if len(args) > 1 else "v")
        assert int(kv["levels"]) == len(kv["levels_lines"]) >= 2
        assert float(kv["grid_complexity"]) > 1.0 and float(kv["operator_complexity"]) > 1.0


def test_driver_matches_library_solve(poisson_mtx, ctx):
    # The driver's iteration count is the library's on the same b = A x_exact.
    path, m = poisson_mtx
    rc, kv, _, err = run(path, "amg")
    assert rc == 0, err
    n = len(m[0]) - 1
    i = np.arange(n, dtype=np.float64)
    exact = 1.0 + 0.25 * np.sin(i * 0.013) + 0.125 * np.cos(i * 0.007)
    off, idx, val = m
    rows = np.repeat(np.arange(n), np.diff(off))
    b = np.zeros(n)
    np.add.at(b, rows, val * exact[idx])
    s = tf.BiCgStab(tf.solver_options(relative_tolerance=1e-8), "amg", ctx=ctx)
    s.setup(to_device(m))
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep = s.apply(torch.tensor(b, device="cuda"), x)
    assert rep["status"] == "Converged"
    assert abs(rep["iterations"] - int(kv["iterations"])) <= 1


def test_driver_fp32_hierarchy(poisson_mtx):
    path, _ = poisson_mtx
    rc, kv, _, err = run(path, "amg", env={"THERMOFEM_B200_HIERARCHY": "f32"})
    assert rc == 0, err
    assert kv["validation"] == "PASS"


EXTRA = ["precision", "device_solve_ms", "operator_spmv_layout", "operator_spmv_gbs",
         "operator_spmv_roofline_fraction", "peak_gbs", "peak_source"]


@pytest.mark.parametrize("hierarchy", ["f64", "f32"])
def test_driver_performance_keys_are_opt_in(poisson_mtx, hierarchy):
    # THERMOFEM_B200_DRIVER_EXTRA=1 appends the precision mode, the device
    # solve time and the operator SpMV's bandwidth after the reference's
    # keys; without it the report carries the reference's keys only
    path, _ = poisson_mtx
    env = {"THERMOFEM_B200_HIERARCHY": hierarchy}
    rc, kv, order, err = run(path, "amg", env=env)
    assert rc == 0, err
    assert not set(EXTRA) & set(order)
    rc, kv2, order2, err = run(path, "amg", env=dict(env, THERMOFEM_B200_DRIVER_EXTRA="1",
                                                     THERMOFEM_B200_HBM_GBS="6540.8"))
    assert rc == 0, err
    assert order2[:len(order)] == order and order2[len(order):] == EXTRA
    assert kv2["precision"] == ("f32_hierarchy_f64_outer" if hierarchy == "f32" else "f64")
    assert float(kv2["device_solve_ms"]) > 0 and float(kv2["operator_spmv_gbs"]) > 0
    assert float(kv2["operator_spmv_roofline_fraction"]) == pytest.approx(
        float(kv2["operator_spmv_gbs"]) / 6540.8, rel=1e-4)
    assert kv2["peak_source"] == "THERMOFEM_B200_HBM_GBS" and kv2["operator_spmv_layout"] in ("sliced", "csr")
