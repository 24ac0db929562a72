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
