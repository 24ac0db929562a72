"""GPU AMG cycles and Krylov solvers against the CPU oracle and the
reference's known answers.  Tolerances follow the reference tests: cycle vs
host recursion 2e-10 (FP64) and 2e-3 (FP32) (amg_native_test.cpp:348);
solver solutions to the exact 1-D Poisson solution (solver_test.cpp:196-205)."""
import numpy as np
import pytest
import torch

import thermofem_b200 as tf
from conftest import to_device
from oracle import oracle as O
from thermofem_b200 import problems as P

pytestmark = pytest.mark.gpu


def poisson(n, dtype=torch.float64, index_dtype=torch.int32, nonsymmetric=False):
    off, idx, val = P.poisson1d(n)
    if nonsymmetric:
        val = np.where(idx == np.repeat(np.arange(n), np.diff(off)), 3.0, np.where(idx > np.repeat(np.arange(n), np.diff(off)), -0.5, -1.0))
    return (off, idx, val), to_device((off, idx, val), dtype=dtype, index_dtype=index_dtype)


@pytest.mark.parametrize("cycle", ["v", "w", "f"])
@pytest.mark.parametrize("dtype,index_dtype,tol", [(torch.float64, torch.int32, 2e-10),
                                                    (torch.float32, torch.int64, 2e-3)])
def test_cycles_match_host_recursion(ctx, cycle, dtype, index_dtype, tol):
    # amg_native_test.cpp:303-395
    host, a = poisson(127, dtype, index_dtype)
    n = 127
    i = np.arange(n)
    b = (np.sin(0.13 * i) + 0.4).astype(np.float32 if dtype == torch.float32 else np.float64).astype(np.float64)
    c = np.cos(0.07 * i)
    amg = tf.Amg(tf.amg_options(coarse_rows=4, cycle=cycle), dtype=dtype, index_dtype=index_dtype, ctx=ctx)
    amg.setup(a)
    assert amg.level_count() >= 3
    ora = O.Amg(O.Csr(n, *host), coarse_rows=4, cycle={"v": 0, "w": 1, "f": 2}[cycle])
    x = amg.apply(torch.tensor(b, dtype=dtype, device="cuda")).cpu().numpy()
    want, visits = ora.apply(b)
    assert np.max(np.abs(x - want)) < tol
    assert amg.last_cycle_visits() == list(visits)
    L = amg.level_count()
    if cycle == "v":
        assert list(visits) == [1] * L
    elif cycle == "w":
        assert list(visits) == [2 ** d for d in range(L)]
    else:
        assert list(visits) == [d + 2 if d + 1 < L else L for d in range(L)]
    # linearity and rhs/x aliasing
    xc = amg.apply(torch.tensor(c, dtype=dtype, device="cuda")).cpu().numpy()
    xs = amg.apply(torch.tensor(b + c, dtype=dtype, device="cuda")).cpu().numpy()
    assert np.max(np.abs(xs - (x + xc))) < tol
    r = torch.tensor(b, dtype=dtype, device="cuda")
    amg.apply(r, r)
    assert np.max(np.abs(r.cpu().numpy() - x)) < tol


@pytest.mark.parametrize("cycle", ["v", "w", "f"])
def test_mixed_precision_cycle_tracks_fp64(ctx, cycle):
    m = P.heat3d(16, seed=3)
    n = len(m[0]) - 1
    b = P.rhs_uniform(n, 9)
    opts = dict(coarse_rows=64, cycle=cycle)
    a64 = to_device(m)
    full = tf.Amg(tf.amg_options(**opts), ctx=ctx)
    mixed = tf.Amg(tf.amg_options(hierarchy_type=tf.F32, **opts), ctx=ctx)
    full.setup(a64)
    mixed.setup(a64)
    tb = torch.tensor(b, device="cuda")
    x64, x32 = full.apply(tb).cpu().numpy(), mixed.apply(tb).cpu().numpy()
    assert np.max(np.abs(x32 - x64)) / np.max(np.abs(x64)) < 1e-4
    ora = O.Amg(O.Csr(n, *m), **opts | {"cycle": {"v": 0, "w": 1, "f": 2}[cycle]})
    assert np.max(np.abs(x64 - ora.apply(b)[0])) / np.max(np.abs(x64)) < 1e-12


def test_fallback_jacobi_equals_standalone_jacobi_and_zero_sweeps(ctx):
    # amg_native_test.cpp:398-424
    host, a = poisson(100)
    b = torch.ones(100, dtype=torch.float64, device="cuda")
    amg = tf.Amg(tf.amg_options(max_levels=1, coarse_sweeps=8), ctx=ctx)
    amg.setup(a)
    assert amg.coarse_solver() == "Jacobi (coarsening stopped)"
    x = amg.apply(b)
    j = tf.Jacobi(8, 0.75, ctx=ctx)
    j.setup(a)
    y = j.apply(b, torch.zeros(100, dtype=torch.float64, device="cuda"))
    assert torch.equal(x, y)
    for cycle in "vwf":
        m = tf.Amg(tf.amg_options(coarse_rows=4, pre_sweeps=0, post_sweeps=0, cycle=cycle), ctx=ctx)
        m.setup(a)
        first = m.apply(b).clone()
        assert torch.equal(first, m.apply(b))


def test_amg_lifecycle_and_coarse_paths(ctx):
    # solver_test.cpp:134-162
    a = to_device((np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32), np.array([1.0, 2, 4, 3])))
    amg = tf.Amg(ctx=ctx)
    with pytest.raises(tf.LogicError):
        amg.apply(torch.ones(2, dtype=torch.float64, device="cuda"))
    amg.setup(a)
    x = amg.apply(torch.tensor([5.0, 10.0], dtype=torch.float64, device="cuda")).cpu().numpy()
    assert np.allclose(x, [1, 2], atol=1e-12)
    invalid = to_device((np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32), np.array([0.0, 1, 1, 1])))
    with pytest.raises(tf.InvalidArgument):
        amg.setup(invalid)
    x = amg.apply(torch.tensor([5.0, 10.0], dtype=torch.float64, device="cuda")).cpu().numpy()
    assert np.allclose(x, [1, 2], atol=1e-12)  # failed setup kept the previous state
    amg.setup(to_device((np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32), np.ones(4))))
    assert amg.coarse_solver() == "Jacobi (singular LU)"
    bounded = tf.Amg(tf.amg_options(max_levels=1, coarse_rows=2), ctx=ctx)
    bounded.setup(poisson(100)[1])
    assert bounded.level_count() == 1 and bounded.coarse_solver() == "Jacobi (coarsening stopped)"
    with pytest.raises(tf.InvalidArgument):
        tf.Amg(tf.amg_options(max_levels=0), ctx=ctx)


@pytest.mark.parametrize("solver", [tf.Cg, tf.BiCgStab])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_amg_solves_poisson_known_answer(ctx, solver, dtype):
    # solver_test.cpp:180-213, cg_test.cpp:51-75
    n = 63
    _, a = poisson(n, dtype)
    rtol = 1e-9 if dtype == torch.float64 else 2e-4
    s = solver(tf.solver_options(dtype, relative_tolerance=rtol), "amg", tf.amg_options(coarse_rows=8), dtype=dtype,
               ctx=ctx)
    s.setup(a)
    b = torch.ones(n, dtype=dtype, device="cuda")
    x = torch.zeros(n, dtype=dtype, device="cuda")
    rep = s.apply(b, x)
    assert rep["status"] == "Converged" and rep["iterations"] < 100
    exact = np.array([(i + 1) * (n - i) / 2 for i in range(n)])
    xv = x.cpu().numpy().astype(np.float64)
    assert np.allclose(xv, exact, rtol=1e-8 if dtype == torch.float64 else 1e-3)
    r = 1 - 2 * xv + np.r_[0, xv[:-1]] + np.r_[xv[1:], 0]
    assert abs(rep["residual_norm"] - np.linalg.norm(r)) <= (1e-10 if dtype == torch.float64 else 1e-3)
    assert rep["relative_residual"] <= rtol
    again = s.apply(b, x)
    assert again["status"] == "Converged" and again["iterations"] == 0
    alias = torch.ones(n, dtype=dtype, device="cuda")
    assert s.apply(alias, alias)["status"] == "Converged"


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 1e-5)])
def test_bicgstab_identity_nonsymmetric_refresh(ctx, dtype, tol):
    # solver_test.cpp:214-237
    n = 80
    host, a = poisson(n, dtype, nonsymmetric=True)
    exact = 1 + (np.arange(n) % 7) / 7
    b = 3 * exact - np.r_[0, exact[:-1]] - 0.5 * np.r_[exact[1:], 0]
    s = tf.BiCgStab(tf.solver_options(dtype, residual_refresh_interval=3, relative_tolerance=tol), "identity",
                    dtype=dtype, ctx=ctx)
    s.setup(a)
    x = torch.full((n,), 0.2, dtype=dtype, device="cuda")
    rep = s.apply(torch.tensor(b, dtype=dtype, device="cuda"), x)
    assert rep["status"] == "Converged"
    assert np.allclose(x.cpu().numpy(), exact, atol=1e-9 if dtype == torch.float64 else 1e-4)


@pytest.mark.parametrize("solver", [tf.Cg, tf.BiCgStab])
def test_status_semantics(ctx, solver):
    # solver_test.cpp:238-287, cg_test.cpp:100-170
    _, a = poisson(5)
    zeros = torch.zeros(5, dtype=torch.float64, device="cuda")
    s = solver(tf.solver_options(absolute_tolerance=1e-12), "identity", ctx=ctx)
    s.setup(a)
    rep = s.apply(zeros.clone(), zeros.clone())
    assert rep["status"] == "Converged" and rep["iterations"] == 0
    rep = s.apply(zeros.clone(), torch.ones(5, dtype=torch.float64, device="cuda"))
    assert rep["status"] == "Converged" and rep["residual_norm"] <= 1e-12
    assert rep["relative_residual"] == rep["residual_norm"]
    host, a3 = poisson(3, nonsymmetric=True)
    b = torch.tensor([1.0, 2, 3], dtype=torch.float64, device="cuda")
    lim = solver(tf.solver_options(max_iterations=0), "identity", ctx=ctx)
    lim.setup(a3)
    rep = lim.apply(b, torch.zeros(3, dtype=torch.float64, device="cuda"))
    assert rep["status"] == "MaxIterations" and rep["iterations"] == 0
    one = solver(tf.solver_options(max_iterations=1, relative_tolerance=0.0), "identity", ctx=ctx)
    one.setup(a3)
    rep = one.apply(b, torch.zeros(3, dtype=torch.float64, device="cuda"))
    assert rep["status"] == "MaxIterations" and rep["iterations"] == 1
    zero_matrix = to_device((np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0)))
    z = solver(tf.solver_options(), "identity", ctx=ctx)
    z.setup(zero_matrix)
    rep = z.apply(b, torch.zeros(3, dtype=torch.float64, device="cuda"))
    assert rep["status"] == "Breakdown" and abs(rep["residual_norm"] - np.sqrt(14)) < 1e-12
    bad = torch.tensor([1.0, float("nan"), 3], dtype=torch.float64, device="cuda")
    assert z.apply(bad, torch.zeros(3, dtype=torch.float64, device="cuda"))["status"] == "NonFinite"


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_jacobi_analytic_sweeps_and_aliased_rhs(ctx, dtype):
    # solver_test.cpp:56-74: Jacobi(2 sweeps, weight 1) on the 2x2 Poisson
    # matrix from x = 0 gives (0.5, 0.25); with rhs and x the same vector
    # (1, 0) the right-hand side is kept before the update: (0.75, 0.25)
    j = tf.Jacobi(2, 1.0, dtype=dtype, ctx=ctx)
    j.setup(poisson(2, dtype=dtype)[1])
    b = torch.tensor([1.0, 0.0], dtype=dtype, device="cuda")
    x = torch.zeros(2, dtype=dtype, device="cuda")
    assert j.apply(b, x).cpu().tolist() == [0.5, 0.25]
    rhs = torch.tensor([1.0, 0.0], dtype=dtype, device="cuda")
    assert j.apply(rhs, rhs).cpu().tolist() == [0.75, 0.25]


def test_solver_lifecycle_errors(ctx):
    s = tf.BiCgStab(ctx=ctx, index_dtype=torch.int64)
    with pytest.raises(tf.LogicError):
        s.apply(torch.ones(2, dtype=torch.float64, device="cuda"), torch.zeros(2, dtype=torch.float64, device="cuda"))
    s.setup(poisson(2, index_dtype=torch.int64)[1])
    assert s.apply(torch.tensor([1.0, 0.0], dtype=torch.float64, device="cuda"),
                   torch.zeros(2, dtype=torch.float64, device="cuda"))["status"] == "Converged"
    with pytest.raises(tf.InvalidArgument):
        tf.BiCgStab(tf.solver_options(relative_tolerance=-1.0), ctx=ctx)
    with pytest.raises(tf.InvalidArgument):
        tf.Jacobi(0, ctx=ctx)


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
@pytest.mark.parametrize("hierarchy", [None, "f32"])
def test_heat3d_solve_matches_oracle(ctx, kind, hierarchy):
    m = P.heat3d(24, seed=21)
    n = len(m[0]) - 1
    b = P.rhs_uniform(n, 22)
    opts = dict(coarse_rows=64, jacobi_weight=2 / 3)
    solver = tf.Cg if kind == "cg" else tf.BiCgStab
    s = solver(tf.solver_options(), "amg", tf.amg_options(hierarchy_type=hierarchy, **opts), ctx=ctx)
    a = to_device(m)
    s.setup(a)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep = s.apply(torch.tensor(b, device="cuda"), x)
    assert rep["status"] == "Converged"
    xv = x.cpu().numpy()
    A = O.Csr(n, *m)
    true_rel = np.linalg.norm(b - O.spmv(A, xv)) / np.linalg.norm(b)
    assert true_rel <= 1e-8 * 1.0001
    ora = O.Amg(A, **opts)
    xo, orep = (O.cg if kind == "cg" else O.bicgstab)(A, ora, b, np.zeros(n))
    assert orep["status"] == "Converged"
    err = np.linalg.norm(xv - xo) / np.linalg.norm(xo)
    print(f"\nheat3d 24^3 {kind} hierarchy={hierarchy}: {rep['iterations']} vs oracle {orep['iterations']} "
          f"iterations, relative difference {err:.3e}")
    if hierarchy is None:
        # same precision, same hierarchy bits, same recurrence: the same
        # iterations, and the solutions differ only by rounding
        assert rep["iterations"] == orep["iterations"]
        assert err <= 1e-12
    else:  # FP32 cycle: a different trajectory, but no more than 25% more iterations
        assert rep["iterations"] <= 1.25 * orep["iterations"] + 2
        assert err < 1e-6


def test_host_buffer_apply(ctx):
    m = P.heat3d(12, seed=2)
    n = len(m[0]) - 1
    b = torch.tensor(P.rhs_uniform(n, 3)).pin_memory()
    x = torch.zeros(n, dtype=torch.float64).pin_memory()
    s = tf.Cg(ctx=ctx)
    s.setup(to_device(m))
    rep = s.apply(b, x)
    assert rep["status"] == "Converged"
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep2 = s.apply(b.cuda(), xd)
    assert rep2["iterations"] == rep["iterations"]
    assert torch.equal(xd.cpu(), x)


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_graph_modes_give_identical_solves(ctx, kind):
    m = P.heat3d(20, seed=31)
    n = len(m[0]) - 1
    b = torch.tensor(P.rhs_uniform(n, 32), device="cuda")
    solver = tf.Cg if kind == "cg" else tf.BiCgStab
    s = solver(tf.solver_options(), "amg", tf.amg_options(hierarchy_type="f32", jacobi_weight=2 / 3), ctx=ctx)
    s.setup(to_device(m))
    assert s.last_execution == -1
    xs, reps, runs = [], [], []
    for mode in (1, 0, 1):
        s.set_graph_mode(mode)
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        reps.append(s.apply(b, x))
        xs.append(x)
        runs.append(s.last_execution)
    assert runs == [2, 1, 2]  # no silent fallback to uncaptured launches
    assert reps[0]["status"] == "Converged"
    assert reps[0] == reps[1] == reps[2]
    assert torch.equal(xs[0], xs[1]) and torch.equal(xs[0], xs[2])


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_dependent_launch_gives_identical_solves(ctx, kind, monkeypatch):
    # Kernels overlap their predecessor's tail under programmatic dependent
    # launch; THERMOFEM_B200_PDL=0 restores plain stream order.  Both must
    # give the same bits.
    m = P.heat3d(20, seed=51)
    n = len(m[0]) - 1
    b = torch.tensor(P.rhs_uniform(n, 52), device="cuda")
    solver = tf.Cg if kind == "cg" else tf.BiCgStab
    out = []
    for pdl in ("1", "0"):
        monkeypatch.setenv("THERMOFEM_B200_PDL", pdl)
        c = tf.Context(0)
        s = solver(tf.solver_options(), "amg", tf.amg_options(hierarchy_type="f32", jacobi_weight=2 / 3), ctx=c)
        s.setup(to_device(m))
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        rep = s.apply(b, x)
        assert s.last_execution == 2
        out.append((rep, x.cpu()))
        del s
        c.close()
    assert out[0][0]["status"] == "Converged"
    assert out[0][0] == out[1][0]
    assert torch.equal(out[0][1], out[1][1])


@pytest.mark.parametrize("cycle", ["v", "w", "f"])
@pytest.mark.parametrize("hierarchy", ["f64", "f32"])
def test_transfer_fusion_is_bit_identical(ctx, cycle, hierarchy, monkeypatch):
    # Restriction fused into the coarse level's first kernel and
    # prolongation fused into its last one (THERMOFEM_B200_FUSE=1, the
    # default, and 2, every level) must reproduce the unfused cycle exactly.
    m = P.heat3d(56, seed=61)  # 175616 rows: the finest level exceeds the scatter threshold
    n = len(m[0]) - 1
    a = to_device(m)
    b = torch.tensor(P.rhs_uniform(n, 62), device="cuda")
    outs = []
    for fuse in ("0", "1", "2"):
        monkeypatch.setenv("THERMOFEM_B200_FUSE", fuse)
        amg = tf.Amg(tf.amg_options(cycle=cycle, hierarchy_type=hierarchy, jacobi_weight=2 / 3, post_sweeps=2),
                     ctx=ctx)
        amg.setup(a)
        outs.append(amg.apply(b).clone())
        amg.apply(b, outs[-1])  # the captured graph replays the same kernels
        outs.append(outs[-1].clone())
    assert torch.isfinite(outs[0]).all()
    for o in outs[1:]:
        assert torch.equal(outs[0], o)


@pytest.mark.parametrize("kind,hierarchy", [("cg", "f32"), ("cg", "f64"), ("bicgstab", "f32"), ("bicgstab", "f64")])
def test_transfer_fusion_solve_and_small_level_program(ctx, kind, hierarchy, monkeypatch):
    # THERMOFEM_B200_FUSE=0 also keeps the preconditioner's final conversion
    # apart from the PCG dot / BiCGStab SpMVs that follow it.
    m = P.heat3d(24, seed=71)
    n = len(m[0]) - 1
    b = torch.tensor(P.rhs_uniform(n, 72), device="cuda")
    res = []
    solver = tf.BiCgStab if kind == "bicgstab" else tf.Cg
    for fuse, small in (("0", 0), ("1", 0), ("1", 2000)):
        monkeypatch.setenv("THERMOFEM_B200_FUSE", fuse)
        s = solver(tf.solver_options(), "amg",
                   tf.amg_options(hierarchy_type=hierarchy, jacobi_weight=2 / 3, small_level_rows=small), ctx=ctx)
        s.setup(to_device(m))
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        rep = s.apply(b, x)
        res.append((rep, x))
    assert res[0][0]["status"] == "Converged"
    assert res[0][0] == res[1][0] and torch.equal(res[0][1], res[1][1])
    # the small-level cluster program (transfers fused into its launch)
    assert res[2][0] == res[0][0] and torch.equal(res[2][1], res[0][1])


def _far_coupled_poisson(n):
    # 1-D Poisson plus a symmetric coupling between the first and the last
    # row: one entry lies n-1 rows from the diagonal, beyond the 2-byte
    # column offsets, so the operator must keep its 4-byte column stream.
    rows, cols, vals = [], [], []
    for i in range(n):
        d = 2.0 + (0.5 if i in (0, n - 1) else 0.0)
        ent = {i: d}
        if i > 0:
            ent[i - 1] = -1.0
        if i < n - 1:
            ent[i + 1] = -1.0
        if i == 0:
            ent[n - 1] = -0.5
        if i == n - 1:
            ent[0] = -0.5
        for j in sorted(ent):
            rows.append(i)
            cols.append(j)
            vals.append(ent[j])
    off = np.zeros(n + 1, np.int32)
    np.add.at(off, np.array(rows) + 1, 1)
    return np.cumsum(off).astype(np.int32), np.array(cols, np.int32), np.array(vals)


@pytest.mark.parametrize("case", ["heat3d-cg", "heat3d-bicgstab", "far-coupling-cg"])
def test_two_byte_column_stream_gives_identical_solves(ctx, case, monkeypatch):
    # Operators whose couplings lie within 32767 rows of the diagonal are
    # streamed with 2-byte column offsets; THERMOFEM_B200_DELTA16=0 keeps the
    # 4-byte indices.  Same columns in the same order: the same bits.
    if case.startswith("heat3d"):
        m = P.heat3d(24, seed=81)
    else:
        m = _far_coupled_poisson(40000)
    n = len(m[0]) - 1
    b = torch.tensor(P.rhs_uniform(n, 82), device="cuda")
    solver = tf.BiCgStab if case.endswith("bicgstab") else tf.Cg
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("THERMOFEM_B200_DELTA16", flag)
        s = solver(tf.solver_options(), "amg", tf.amg_options(hierarchy_type="f32", jacobi_weight=2 / 3), ctx=ctx)
        s.setup(to_device(m))
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        out.append((s.apply(b, x), x))
    assert out[0][0]["status"] == "Converged"
    assert out[0][0] == out[1][0]
    assert torch.equal(out[0][1], out[1][1])


@pytest.mark.parametrize("shape", ["0,2", "1,3", "1,8", "0,5", "2,2,3", "2,3,5", "2,4,1"])
@pytest.mark.parametrize("case", ["heat3d-cg-f32", "heat3d-cg-f64", "heat3d-bicgstab-f32"])
def test_sliced_layout_gives_identical_solves(ctx, case, shape, monkeypatch):
    # Operators with 2-byte column offsets also carry a sliced copy (32-row
    # slices, entries column-major) that the SpMV family streams when it is
    # faster.  THERMOFEM_B200_SLICED_SHAPE="prefetch,ctas" forces the direct
    # kernel with that launch shape, "2,stages,ctas" the staged one (tiles
    # bulk-copied into a shared-memory ring), THERMOFEM_B200_SLICED=0 turns
    # the copy off.  Same
    # per-row order and the same 256-row-block partial sums: the same bits,
    # on every level (coarse levels have rows longer than one 8-entry group)
    # and on a row count that is no multiple of 32.
    m = P.heat3d(25, seed=83)
    n = len(m[0]) - 1
    b = torch.tensor(P.rhs_uniform(n, 84), device="cuda")
    solver = tf.BiCgStab if "bicgstab" in case else tf.Cg
    out = []
    # padding bound 10 %: the aggregated levels (30-50 % in row order) keep
    # CSR unless sorted; 50 % (the default): they take row-order slices too
    monkeypatch.setenv("THERMOFEM_B200_BANDED", "0")  # the 2-byte-offset sliced copy, not the banded one
    for flag, pad in (("0", "10"), ("1", "10"), ("sorted", "10"), ("1", "50")):
        monkeypatch.setenv("THERMOFEM_B200_SLICED", flag)
        monkeypatch.setenv("THERMOFEM_B200_SLICED_PAD", pad)
        monkeypatch.setenv("THERMOFEM_B200_SLICED_SHAPE", shape)
        s = solver(tf.solver_options(), "amg",
                   tf.amg_options(hierarchy_type=case[-3:], jacobi_weight=2 / 3, cycle="w"), ctx=ctx)
        s.setup(to_device(m))
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        rep = s.apply(b, x)
        xs = torch.randn(n, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
        out.append((rep, x, s.spmv(xs)))
        layout, entries = s.spmv_layout()
        if flag == "0":
            assert (layout, entries) == ("csr", len(m[1]))
        else:
            assert layout == "sliced" and len(m[1]) <= entries <= len(m[1]) * 1.5
            assert s.level_spmv_layout(0)[0] == "sliced"
            # coarse aggregated levels: with "sorted", rows ordered longest first within their tiles
            kinds = [s.level_spmv_layout(d)[0] for d in range(1, s.level_count())]
            assert ("sorted" in kinds) == (flag == "sorted"), kinds
            assert (kinds[0] == "sliced") == (pad == "50"), kinds
    assert out[0][0]["status"] == "Converged"
    for other in out[1:]:
        assert out[0][0] == other[0]
        assert torch.equal(out[0][1], other[1])
        assert torch.equal(out[0][2], other[2])


@pytest.mark.parametrize("shape", ["0,2", "1,3", "1,8", "0,5", "2,2,3", "2,3,2", "2,3,3,2", "2,2,2,4", "3,2,3",
                                   "3,3,2", None])
@pytest.mark.parametrize("case", ["heat3d25-cg-f32", "heat3d25-bicgstab-f64", "heat3d184-cg-f32"])
def test_banded_layout_gives_identical_solves(ctx, case, shape, monkeypatch):
    # Stencil operators (the solver's operator, the finest level) carry a
    # banded copy: 32-row slices whose rows share one column offset per entry
    # slot, with a padding mask, so SpMV streams values and an 8-byte pair
    # per 32 entries.  Each row still sums its entries left to right from +0
    # (padding lanes gather nothing): the same bits as the CSR arrays
    # (THERMOFEM_B200_SLICED=0), whatever the launch shape: "p,c" the direct
    # kernel (prefetch p, c CTAs per SM), "2,s,c[,g]" the staged one (s stages
    # of g tiles' values and slots copied in bulk into shared memory), "3,s,c"
    # the staged one with four rows per lane (reducing epilogues: one row per
    # lane, the same stages).  184^3:
    # couplings 33,856 rows apart, beyond 2-byte offsets, so the CSR arrays
    # stream 4-byte columns there.
    side = int(case.split("-")[0][6:])
    if side > 100 and shape not in (None, "1,3", "2,2,3", "2,3,3,2", "3,2,3"):
        pytest.skip("the large case runs five launch shapes")
    m = P.heat3d(side, seed=85)
    n = len(m[0]) - 1
    b = torch.tensor(P.rhs_uniform(n, 86), device="cuda")
    solver = tf.BiCgStab if "bicgstab" in case else tf.Cg
    if shape:
        monkeypatch.setenv("THERMOFEM_B200_SLICED_SHAPE", shape)
    out = []
    for flag in ("0", "1"):
        monkeypatch.setenv("THERMOFEM_B200_SLICED", flag)
        s = solver(tf.solver_options(), "amg", tf.amg_options(hierarchy_type=case[-3:], jacobi_weight=2 / 3),
                   ctx=ctx)
        s.setup(to_device(m))
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        rep = s.apply(b, x)
        xs = torch.randn(n, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(6))
        out.append((rep, x, s.spmv(xs), s.level_spmv_layout(0)[0], s.spmv_layout()))
        del s
    (r0, x0, y0, l0, op0), (r1, x1, y1, l1, op1) = out
    assert op0[0] == ("csr" if side < 100 else "csr32")
    if shape:  # a forced shape streams the copy
        assert op1[0] == "banded" and l1 == "banded"
        assert len(m[1]) <= op1[1] <= len(m[1]) * 1.1
    assert r0["status"] == "Converged" and r0 == r1
    assert torch.equal(x0, x1) and torch.equal(y0, y1)


@pytest.mark.parametrize("shape", [None, "1,4", "0,3", "2,2,4", "2,3,2", "2,3,2,2", "2,2,2,4"])
def test_operator_spmv_entry_points(ctx, shape, monkeypatch):
    # The solver's and the hierarchy's own operators (2-byte column stream,
    # sliced copy when the tuner picks it or a shape forces it) give the same
    # product as the plain CSR SpMV.
    if shape:
        monkeypatch.setenv("THERMOFEM_B200_SLICED_SHAPE", shape)
    m = P.heat3d(24, seed=91)
    n = len(m[0]) - 1
    a = to_device(m)
    x = torch.tensor(np.random.default_rng(92).standard_normal(n), device="cuda")
    s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(hierarchy_type="f32"), ctx=ctx)
    with pytest.raises(tf.LogicError):
        s.spmv(x)
    s.setup(a)
    assert torch.equal(s.spmv(x), tf.spmv(a, x, ctx=ctx))
    h = s  # the solver is a view of its hierarchy
    for d in range(h.level_count()):
        lm = h.level_matrix(d)
        xd = torch.tensor(np.random.default_rng(d).standard_normal(lm.rows), dtype=torch.float32, device="cuda")
        assert torch.equal(h.level_spmv(d, xd), tf.spmv(lm, xd, ctx=ctx))


@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_banded_level_spmv_on_unaligned_vectors(ctx, dtype, monkeypatch):
    # The four-rows-per-lane banded kernel reads four x values with one
    # 16-byte load where they are aligned; an x that starts one element into
    # its buffer takes the one-load-per-entry path: the same bits as the CSR
    # arrays either way.
    m = P.heat3d(25, seed=85)
    n = len(m[0]) - 1
    t = torch.float32 if dtype == "f32" else torch.float64
    base = torch.randn(n + 1, dtype=t, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    out = []
    monkeypatch.setenv("THERMOFEM_B200_SLICED_SHAPE", "3,2,3")
    for flag in ("1", "0"):
        monkeypatch.setenv("THERMOFEM_B200_SLICED", flag)
        s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(hierarchy_type=dtype, jacobi_weight=2 / 3), ctx=ctx)
        s.setup(to_device(m))
        assert s.level_spmv_layout(0)[0] == ("banded" if flag == "1" else "csr")
        out.append((s.level_spmv(0, base[1:]).clone(), s.level_spmv(0, base[:n]).clone()))
        del s
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
