"""This library's solves against the reference's own GPU solve path.

The reference library (its Cg / BiCgStab with its aggregation Amg on
cuSPARSE, cuBLAS and CUB) is compiled for sm_100a from its sources by
`make -C oracle refgpu` into oracle/_ref/libref_gpu.so; these tests skip
where that build is absent.  Same inputs, same options (FP64 hierarchy,
Jacobi w = 2/3, coarse LU <= 64 rows, tolerance 1e-8): AMG-preconditioned
CG takes the same iterations and its solution agrees to 1e-12 relative;
BiCGStab, which amplifies the two implementations' different reduction
orders, agrees within one iteration and 1e-6.  The last test also reports
both solve times on the 128^3 benchmark problem.
"""
import json
import os
import subprocess

import numpy as np
import pytest
import torch

import thermofem_b200 as tf
from oracle import oracle as O
from thermofem_b200 import build as B
from thermofem_b200 import problems as P

REF_DRIVER = os.path.join(os.path.dirname(O.REF_GPU_LIB), "solve-matrix")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_gpu_available(), reason="reference GPU build absent (make -C oracle refgpu)")]


def _ours(m, b, kind, cycle, hierarchy="f64", jacobi_weight=2 / 3, coarse_rows=64, precond="amg"):
    solver = tf.BiCgStab if kind == "bicgstab" else tf.Cg
    if precond == "identity":
        s = solver(tf.solver_options(), "identity")
    else:
        s = solver(tf.solver_options(), "amg",
                   tf.amg_options(hierarchy_type=hierarchy, jacobi_weight=jacobi_weight, coarse_rows=coarse_rows,
                                  cycle=cycle))
    s.setup(tf.DeviceCsr.from_host(*m))
    x = torch.zeros(len(b), dtype=torch.float64, device="cuda")
    bd = torch.tensor(b, device="cuda")
    rep = s.apply(bd, x)
    return s, x, bd, rep


@pytest.mark.parametrize("problem,kind,cycle", [("heat", "cg", "v"), ("heat", "cg", "w"), ("heat", "cg", "f"),
                                                ("heat", "bicgstab", "v"), ("convdiff", "bicgstab", "w")])
def test_solves_match_the_reference_gpu_build(problem, kind, cycle):
    m = P.heat3d(24, seed=41) if problem == "heat" else P.convdiff3d(20, seed=43)
    n = len(m[0]) - 1
    b = P.rhs_uniform(n, 42)
    xr, rr = O.ref_gpu_solve(O.Csr(n, *m), b, kind=kind, cycle=cycle)
    _, x, _, rep = _ours(m, b, kind, cycle)
    assert rr["status"] == 0 and rep["status"] == "Converged"
    xo = x.cpu().numpy()
    err = np.linalg.norm(xo - xr) / np.linalg.norm(xr)
    print(f"\nvs reference GPU build {problem} {kind}-{cycle}: {rep['iterations']} vs {rr['iterations']} "
          f"iterations, relative difference {err:.3e}")
    if kind == "cg":
        # PCG on the same hierarchy: rounding differences (cuBLAS/cuSPARSE
        # reduction orders against this library's) stay at rounding level
        assert rep["iterations"] == rr["iterations"]
        assert err <= 1e-12
    else:
        # BiCGStab amplifies them over the iterations (measured 1e-12 on
        # heat 24^3, 1e-9 on convection-diffusion 20^3)
        assert abs(rep["iterations"] - rr["iterations"]) <= 1, (rep["iterations"], rr["iterations"])
        assert err < 1e-6


@pytest.mark.parametrize("case", ["laplace2d-128", "w-0.75", "coarse-16", "identity-cg", "identity-bicgstab"])
def test_more_solves_match_the_reference_gpu_build(case):
    # the 2-D 128^2 Laplacian of the small benchmark configuration; the
    # reference's default Jacobi weight 0.75; a 16-row coarse level; and the
    # solvers without a preconditioner (the reference's default identity)
    if case == "laplace2d-128":
        m, kw = P.laplace2d(128), {}
    elif case.startswith("identity"):
        m, kw = P.laplace2d(48), {}  # converges without a preconditioner within the default 1000 iterations
    else:
        m, kw = P.heat3d(20, seed=47), {}
    if case == "w-0.75":
        kw = {"jacobi_weight": 0.75}
    elif case == "coarse-16":
        kw = {"coarse_rows": 16}
    kind = "bicgstab" if case.endswith("bicgstab") else "cg"
    precond = "identity" if case.startswith("identity") else "amg"
    n = len(m[0]) - 1
    b = P.rhs_uniform(n, 48)
    xr, rr = O.ref_gpu_solve(O.Csr(n, *m), b, kind=kind, precond=precond, **kw)
    _, x, _, rep = _ours(m, b, kind, "v", precond=precond, **kw)
    assert rr["status"] == 0 and rep["status"] == "Converged"
    # without a preconditioner hundreds of iterations accumulate the two
    # implementations' different reduction orders (BiCGStab's iteration count
    # is erratic under them: a textbook restatement takes 107 here, the CPU
    # oracle 124), and a 1e-8 residual bounds the solution only to about
    # cond(A) * 1e-8
    if precond == "identity":
        slack = max(1, rr["iterations"] // (50 if kind == "cg" else 4))
        tol = 1e-4
    else:  # AMG-preconditioned CG: rounding level, as above
        slack, tol = 0, 1e-12
    assert abs(rep["iterations"] - rr["iterations"]) <= slack, (rep["iterations"], rr["iterations"])
    err = np.linalg.norm(x.cpu().numpy() - xr) / np.linalg.norm(xr)
    print(f"\nvs reference GPU build {case}: {rep['iterations']} vs {rr['iterations']} iterations, "
          f"relative difference {err:.3e}")
    assert err <= tol


def test_reference_gpu_build_on_the_benchmark_problem(capsys):
    # 128^3 log-normal heat, PCG + AMG V(1,1): the reference's FP64 solve and
    # this library's FP64 and mixed solves, device-synchronised wall times.
    m = P.heat3d(128, 1001)
    n = len(m[0]) - 1
    b = P.rhs_uniform(n, 1002)
    xr, rr = O.ref_gpu_solve(O.Csr(n, *m), b, kind="cg", cycle="v", repeats=2)
    out = {"reference_fp64": rr}
    for hierarchy in ("f64", "f32"):
        s, x, bd, rep = _ours(m, b, "cg", "v", hierarchy)
        times = []
        for _ in range(3):
            x.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            rep = s.apply(bd, x)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        out[f"ours_{hierarchy}"] = {"iterations": rep["iterations"], "solve_s": min(times)}
        if hierarchy == "f64":
            assert abs(rep["iterations"] - rr["iterations"]) <= 1
            assert np.linalg.norm(x.cpu().numpy() - xr) / np.linalg.norm(xr) < 1e-6
            assert min(times) < rr["solve_s"]
    with capsys.disabled():
        print("\nreference GPU build vs this library, heat3d 128^3 PCG V(1,1): " + json.dumps(out))


def _report(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    rows = [line.partition("=") for line in r.stdout.splitlines()]
    return r.returncode, [(k, v) for k, _, v in rows], r.stderr


# report lines that measure this run (times, device identity) rather than the solve
_RUN_KEYS = {"read_seconds", "setup_seconds", "solve_seconds", "device", "gpu", "cuda_runtime"}
_CLOSE_KEYS = {"reported_relative_residual", "host_relative_residual", "relative_solution_error"}


@pytest.mark.skipif(not os.path.exists(REF_DRIVER), reason="reference solve-matrix not built")
@pytest.mark.parametrize("matrix,args", [("laplace2d", ("amg",)), ("laplace2d", ("amg", "w")),
                                         ("laplace2d", ("amg", "f")), ("laplace2d", ("identity",)),
                                         ("convdiff", ("amg", "w"))])
def test_solve_matrix_driver_reports_what_the_reference_driver_reports(tmp_path, matrix, args):
    # Both drivers on the same synthetic Matrix Market file: the same report
    # lines in the same order with the same values (matrix, sizes, options,
    # cycle, levels, stop reason, coarse solver, per-level rows, nonzeros and
    # aggregate histograms, complexities, status, iterations, validation),
    # times and device lines aside and residuals to a relative 1e-3.
    path = str(tmp_path / f"{matrix}.mtx")
    if matrix == "laplace2d":
        P.write_matrix_market(path, *P.laplace2d(64), symmetric=True)
    else:
        P.write_matrix_market(path, *P.convdiff3d(16, seed=49))
    rc_r, ref, err_r = _report([REF_DRIVER, path, *args])
    rc_o, ours, err_o = _report([B.DRIVER, path, *args])
    assert rc_r == 0 and rc_o == 0, (err_r, err_o)
    assert [k for k, _ in ours] == [k for k, _ in ref]
    # unpreconditioned BiCGStab (the driver's identity mode) is erratic under
    # different reduction orders: iterations within a quarter, residuals
    # checked against the tolerance rather than against each other
    identity = args[0] == "identity"
    for (k, vo), (_, vr) in zip(ours, ref):
        if k in _RUN_KEYS:
            continue
        if k in _CLOSE_KEYS:
            if identity:
                assert float(vo) <= (1e-4 if k == "relative_solution_error" else 1.01e-8), (k, vo)
            else:
                assert abs(float(vo) - float(vr)) <= 1e-3 * abs(float(vr)) + 1e-12, (k, vo, vr)
        elif k == "iterations":
            assert abs(int(vo) - int(vr)) <= (max(1, int(vr) // 4) if identity else 1), (vo, vr)
        elif k in ("grid_complexity", "operator_complexity"):
            assert float(vo) == pytest.approx(float(vr), rel=1e-9), (k, vo, vr)
        else:
            assert vo == vr, (k, vo, vr)


@pytest.mark.skipif(os.environ.get("THERMOFEM_B200_REFERENCE_256") != "1",
                    reason="opt-in: THERMOFEM_B200_REFERENCE_256=1 (the reference's 256^3 setup takes minutes)")
@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_reference_gpu_build_at_256(kind, capsys):
    # 256^3 log-normal heat (16.8M rows, 117M nonzeros), V(1,1): the
    # reference's FP64 solve against this library's FP64 and mixed solves.
    m = P.heat3d(256, 1001)
    n = len(m[0]) - 1
    b = P.rhs_uniform(n, 1002)
    xr, rr = O.ref_gpu_solve(O.Csr(n, *m), b, kind=kind, cycle="v", repeats=1)
    out = {"reference_fp64": rr}
    for hierarchy in ("f64", "f32"):
        s, x, bd, rep = _ours(m, b, kind, "v", hierarchy)
        times = []
        for _ in range(2):
            x.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            rep = s.apply(bd, x)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        out[f"ours_{hierarchy}"] = {"iterations": rep["iterations"], "solve_s": min(times)}
        if hierarchy == "f64":
            # BiCGStab's count drifts with the reduction order over ~70 steps
            # of a 16.8M-row solve (71 here, 73 in the reference): 4 %
            slack = 1 if kind == "cg" else max(1, rr["iterations"] // 25)
            assert abs(rep["iterations"] - rr["iterations"]) <= slack
            assert min(times) < rr["solve_s"]
        del s
    with capsys.disabled():
        print(f"\nreference GPU build vs this library, heat3d 256^3 {kind} V(1,1): " + json.dumps(out))


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_float_solves_match_the_reference_gpu_build(kind):
    # the float components on both sides (FP32 operator, vectors and
    # hierarchy, the float default tolerance 1e-5), heat 20^3, AMG V(1,1)
    m = P.heat3d(20, seed=53)
    n = len(m[0]) - 1
    b = P.rhs_uniform(n, 54)
    # both sides see the same FP32 values: round them once here
    m32 = (m[0], m[1], m[2].astype(np.float32).astype(np.float64))
    b32 = b.astype(np.float32).astype(np.float64)
    xr, rr = O.ref_gpu_solve(O.Csr(n, *m32), b32, kind=kind, single=True)
    solver = tf.BiCgStab if kind == "bicgstab" else tf.Cg
    s = solver(tf.solver_options(torch.float32), "amg",
               tf.amg_options(jacobi_weight=2 / 3, coarse_rows=64, cycle="v"), dtype=torch.float32)
    s.setup(tf.DeviceCsr.from_host(*m32, dtype=torch.float32))
    x = torch.zeros(n, dtype=torch.float32, device="cuda")
    rep = s.apply(torch.tensor(b32, dtype=torch.float32, device="cuda"), x)
    assert rr["status"] == 0 and rep["status"] == "Converged"
    assert abs(rep["iterations"] - rr["iterations"]) <= 1, (rep["iterations"], rr["iterations"])
    xo = x.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(xo - xr) / np.linalg.norm(xr) < 1e-3
