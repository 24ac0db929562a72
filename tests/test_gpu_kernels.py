"""GPU parity of the kernel layer against the CPU oracle (FP64) and a plain
numpy FP64 evaluation of the same formula (FP32 kernels).  Tolerances:
FP64 kernels 1e-13 relative to the row's magnitude (FMA contraction and
summation order are the only differences); FP32 kernels 2e-6 relative."""
import numpy as np
import pytest
import torch

import thermofem_b200 as tf
from conftest import to_device
from oracle import oracle as O
from thermofem_b200 import problems as P

pytestmark = pytest.mark.gpu


def irregular(n=3000, seed=7):
    """Rows of very different lengths, including rows longer than one staged
    chunk (4096 entries) and empty rows."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 12, n)
    lens[5] = 9000
    lens[17] = 0
    lens[n - 1] = 5000
    off = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    idx = np.concatenate([np.sort(rng.choice(n, size=l, replace=l > n)) for l in lens]).astype(np.int32)
    val = rng.standard_normal(off[-1])
    for i in range(n):  # make every row have a diagonal where nonempty
        if lens[i]:
            idx[off[i]] = i
    return off.astype(np.int32), idx, val


def mats():
    yield "heat3d16", P.heat3d(16)
    yield "laplace2d40", P.laplace2d(40)
    yield "irregular", irregular()
    s = O.sample_matrix(61)
    yield "sample61", (s.offsets, s.indices, s.values)


def host_spmv(m, x):
    off, idx, val = m
    n = len(off) - 1
    y = np.zeros(n)
    np.add.at(y, np.repeat(np.arange(n), np.diff(off)), val * x[idx])
    return y


def rel_err(a, b):
    return np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b)))


@pytest.mark.parametrize("name,m", list(mats()))
@pytest.mark.parametrize("index_dtype", [torch.int32, torch.int64])
def test_spmv_f64_matches_oracle(ctx, name, m, index_dtype):
    off, idx, val = m
    n = len(off) - 1
    x = np.random.default_rng(1).standard_normal(n)
    a = to_device(m, index_dtype=index_dtype)
    y = tf.spmv(a, torch.tensor(x, device="cuda"), ctx=ctx).cpu().numpy()
    ref = O.spmv(O.Csr(n, off, idx, val), x)
    scale = host_spmv((off, idx, np.abs(val)), np.abs(x)) + 1e-300
    assert np.max(np.abs(y - ref) / scale) < 1e-13


@pytest.mark.parametrize("name,m", list(mats()))
def test_spmv_f32_matches_fp64_reference(ctx, name, m):
    off, idx, val = m
    n = len(off) - 1
    x = np.random.default_rng(2).standard_normal(n).astype(np.float32)
    a = to_device(m, dtype=torch.float32)
    y = tf.spmv(a, torch.tensor(x, device="cuda"), ctx=ctx).cpu().numpy().astype(np.float64)
    ref = host_spmv((off, idx, val.astype(np.float32).astype(np.float64)), x.astype(np.float64))
    scale = host_spmv((off, idx, np.abs(val)), np.abs(x.astype(np.float64))) + 1e-30
    assert np.max(np.abs(y - ref) / scale) < 2e-6


def test_spmv_empty_pattern_and_typed_entry(ctx):
    a = to_device((np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0)))
    y = tf.spmv(a, torch.ones(3, dtype=torch.float64, device="cuda"), ctx=ctx)
    assert y.abs().max().item() == 0.0
    off, idx, val = P.laplace2d(20)
    d = to_device((off, idx, val))
    x = torch.randn(400, dtype=torch.float64, device="cuda")
    y1 = tf.spmv(d, x, ctx=ctx)
    y2 = torch.empty_like(x)
    with ctx:
        tf.check(tf.lib().tf_spmv_f64(ctx.h, 400, 400, len(idx), d.offsets.data_ptr(), d.indices.data_ptr(),
                                      d.values.data_ptr(), x.data_ptr(), y2.data_ptr()))
    assert torch.equal(y1, y2)
    with pytest.raises(tf.InvalidArgument):
        tf.spmv(d, x, y=x, ctx=ctx)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 3e-6)])
def test_residual_and_jacobi_family(ctx, dtype, tol):
    off, idx, val = P.heat3d(12, seed=5)
    n = len(off) - 1
    rng = np.random.default_rng(3)
    b, x = rng.standard_normal(n), rng.standard_normal(n)
    hb = b.astype(np.float32).astype(np.float64) if dtype == torch.float32 else b
    hx = x.astype(np.float32).astype(np.float64) if dtype == torch.float32 else x
    hv = val.astype(np.float32).astype(np.float64) if dtype == torch.float32 else val
    a = to_device((off, idx, val), dtype=dtype)
    tb, tx = torch.tensor(b, dtype=dtype, device="cuda"), torch.tensor(x, dtype=dtype, device="cuda")
    ax = host_spmv((off, idx, hv), hx)
    scale = host_spmv((off, idx, np.abs(hv)), np.abs(hx)) + np.abs(hb)
    r = tf.residual(a, tb, tx, ctx=ctx).cpu().numpy()
    assert np.max(np.abs(r - (hb - ax)) / scale) < tol
    dinv = tf.inverse_diagonal(a, ctx=ctx)
    hd = dinv.cpu().numpy().astype(np.float64)
    diag = np.array([hv[off[i]:off[i + 1]][idx[off[i]:off[i + 1]] == i].sum() for i in range(n)])
    assert np.max(np.abs(hd * diag - 1)) < tol * 10
    w = 2.0 / 3.0
    xo = tf.jacobi_sweep(a, dinv, tb, tx, w, ctx=ctx).cpu().numpy()
    want = hx + w * hd * (hb - ax)
    assert np.max(np.abs(xo - want) / (np.abs(hx) + w * np.abs(hd) * scale)) < tol * 4
    # per-row weights
    rw = torch.linspace(0.3, 0.9, n, device="cuda", dtype=torch.float32)
    xo = tf.jacobi_sweep(a, dinv, tb, tx, w, row_weight=rw, ctx=ctx).cpu().numpy()
    hw = rw.cpu().numpy().astype(np.float64)
    want = hx + hw * hd * (hb - ax)
    assert np.max(np.abs(xo - want) / (np.abs(hx) + np.abs(hd) * scale)) < tol * 4
    # prolongation fused: x~ = x + e[map]
    nc = 97
    mp = rng.integers(0, nc, n).astype(np.int32)
    e = rng.standard_normal(nc)
    he = e.astype(np.float32).astype(np.float64) if dtype == torch.float32 else e
    xt = hx + he[mp]
    if dtype == torch.float32:
        xt = xt.astype(np.float32).astype(np.float64)
    axt = host_spmv((off, idx, hv), xt)
    xo = tf.jacobi_sweep(a, dinv, tb, tx, w, map=torch.tensor(mp, device="cuda"),
                         coarse=torch.tensor(e, dtype=dtype, device="cuda"), ctx=ctx).cpu().numpy()
    want = xt + w * hd * (hb - axt)
    scale2 = host_spmv((off, idx, np.abs(hv)), np.abs(xt)) + np.abs(hb)
    assert np.max(np.abs(xo - want) / (np.abs(xt) + w * np.abs(hd) * scale2)) < tol * 4
    z = tf.jacobi_zero(dinv, tb, w, ctx=ctx).cpu().numpy()
    assert np.max(np.abs(z - w * hd * hb) / (np.abs(w * hd * hb) + 1e-300)) < tol


def test_jacobi_sweep_matches_oracle_jacobi(ctx):
    # two sweeps of the fused kernel == Jacobi<double>(2, 1) on poisson(2): 0.5/0.25 (solver_test.cpp:56-74)
    off, idx, val = P.poisson1d(2)
    a = to_device((off, idx, val))
    dinv = tf.inverse_diagonal(a, ctx=ctx)
    b = torch.tensor([1.0, 0.0], dtype=torch.float64, device="cuda")
    x = torch.zeros(2, dtype=torch.float64, device="cuda")
    x = tf.jacobi_sweep(a, dinv, b, x, 1.0, ctx=ctx)
    x = tf.jacobi_sweep(a, dinv, b, x, 1.0, ctx=ctx)
    assert x.cpu().tolist() == [0.5, 0.25]


def test_inverse_diagonal_rejects_bad_diagonals(ctx):
    # duplicate diagonal entries are summed (multigrid_operations_test.cpp:63-83)
    a = to_device((np.array([0, 2, 4], np.int32), np.array([0, 0, 0, 1], np.int32), np.array([1.0, 1, 4, 3])))
    d = tf.inverse_diagonal(a, ctx=ctx).cpu().numpy()
    assert abs(d[0] - 0.5) < 1e-15 and abs(d[1] - 1 / 3) < 1e-15
    bad = to_device((np.array([0, 2, 4], np.int32), np.array([0, 0, 0, 1], np.int32), np.array([0.0, 0, 4, 3])))
    with pytest.raises(tf.InvalidArgument):
        tf.inverse_diagonal(bad, ctx=ctx)


def test_restrict_prolong_and_blas1(ctx):
    n = 5000
    rng = np.random.default_rng(4)
    nc = 1500
    mp = np.sort(rng.integers(0, nc, n)).astype(np.int32)
    mp[:nc] = np.arange(nc)  # every aggregate nonempty
    mp = np.sort(mp)
    off = np.zeros(nc + 1, np.int32)
    np.cumsum(np.bincount(mp, minlength=nc), out=off[1:])
    mem = np.argsort(mp, kind="stable").astype(np.int32)
    t = tf.Transfer(torch.tensor(mp, device="cuda"), torch.tensor(off, device="cuda"), torch.tensor(mem, device="cuda"),
                    n, nc, np.zeros(4))
    f = rng.standard_normal(n)
    c = tf.restrict_aggregates(t, torch.tensor(f, device="cuda"), ctx=ctx).cpu().numpy()
    want = np.array([sum(f[mem[off[k]:off[k + 1]]]) for k in range(nc)])  # member order, left to right
    assert np.array_equal(c, want)
    fine = torch.tensor(f, device="cuda")
    tf.prolong_aggregates(t, torch.tensor(want, device="cuda"), fine, ctx=ctx)
    assert np.array_equal(fine.cpu().numpy(), f + want[mp])
    xs = [torch.tensor(rng.standard_normal(n), device="cuda") for _ in range(3)]
    ys = [torch.tensor(rng.standard_normal(n), device="cuda") for _ in range(3)]
    d = tf.dot_multi(xs, ys, ctx=ctx).cpu().numpy()
    want = [float(np.dot(a.cpu().numpy(), b.cpu().numpy())) for a, b in zip(xs, ys)]
    assert np.allclose(d, want, rtol=1e-13, atol=1e-12)
    d2 = tf.dot_multi(xs, ys, ctx=ctx).cpu().numpy()
    assert np.array_equal(d, d2)  # deterministic
    y = ys[0].clone()
    tf.axpby(2.0, xs[0], -0.5, y, ctx=ctx)
    assert torch.allclose(y, 2.0 * xs[0] - 0.5 * ys[0], rtol=1e-15, atol=1e-15)


@pytest.mark.parametrize("n", [1, 7, 2048, 2049, 100000, 5_000_000])
def test_scan_exclusive(ctx, n):
    rng = np.random.default_rng(n)
    x = rng.integers(0, 5, n).astype(np.int32)
    out = tf.scan_exclusive(torch.tensor(x, device="cuda"), ctx=ctx).cpu().numpy()
    want = np.concatenate([[0], np.cumsum(x)[:-1]]).astype(np.int32)
    assert np.array_equal(out, want)
    t = torch.tensor(x, device="cuda")
    tf.scan_exclusive(t, out=t, ctx=ctx)  # in place
    assert np.array_equal(t.cpu().numpy(), want)


@pytest.mark.parametrize("src,dst", [(torch.float32, torch.float64), (torch.float64, torch.float32),
                                     (torch.float32, torch.float32), (torch.float64, torch.float64),
                                     (torch.int32, torch.int64), (torch.int64, torch.int32),
                                     (torch.int32, torch.int32), (torch.int64, torch.int64)])
def test_convert_matches_torch_casts(ctx, src, dst):
    # tf_convert is an elementwise static_cast, as the reference's convert
    # kernel (GpuAggregation.cu:1101-1108): FP64 -> FP32 rounds to nearest
    # even, int64 -> int32 keeps the low 32 bits (two's complement), exactly
    # what torch's casts do; the index range itself is checked by the
    # component layer (AMG native index capacity), not per element.
    g = torch.Generator(device="cuda").manual_seed(5)
    n = 1_000_003
    if src.is_floating_point:
        x = (torch.randn(n, dtype=torch.float64, device="cuda", generator=g) * 1e3).to(src)
        x[:4] = torch.tensor([0.0, -0.0, 1e-40, 3.4e38], dtype=torch.float64).to(src)
    else:
        x = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int64, device="cuda", generator=g).to(src)
        if src == torch.int64:
            x[:3] = torch.tensor([2**31, -2**31 - 1, 2**40 + 7], dtype=torch.int64)
    got = tf.convert(x, dst, ctx=ctx)
    ctx.synchronize()
    assert torch.equal(got, x.to(dst))
    assert tf.convert(x[:0], dst, ctx=ctx).numel() == 0


def test_convert_rejects_mixed_kinds(ctx):
    x = torch.ones(8, dtype=torch.float64, device="cuda")
    with pytest.raises(tf.InvalidArgument):
        tf.convert(x, torch.int32, ctx=ctx)
    with pytest.raises(tf.InvalidArgument):
        tf.convert(x.to(torch.int64), torch.float32, ctx=ctx)


@pytest.mark.parametrize("n,bits", [(1, 8), (1000, 12), (70000, 40), (1_000_003, 64)])
def test_radix_sort_is_stable_and_reduce_by_key(ctx, n, bits):
    rng = np.random.default_rng(n)
    hi = 1 << min(bits, 62)
    keys = rng.integers(0, min(hi, max(2, n // 3)), n, dtype=np.int64).astype(np.uint64)
    if bits == 64:
        keys = keys | (np.uint64(1) << np.uint64(63))
    vals = np.arange(n, dtype=np.float64)  # original positions expose stability
    tk = torch.tensor(keys.view(np.int64), device="cuda")
    tv = torch.tensor(vals, device="cuda")
    sk, sv = tf.radix_sort_pairs(tk, tv, end_bit=bits, ctx=ctx)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(sk.cpu().numpy().view(np.uint64), keys[order])
    assert np.array_equal(sv.cpu().numpy(), vals[order])
    w = rng.standard_normal(n)
    uk, uv = tf.reduce_by_key(sk, torch.tensor(w, device="cuda"), "sum", ctx=ctx)
    ks = keys[order]
    heads = np.flatnonzero(np.r_[True, ks[1:] != ks[:-1]])
    want = [float(sum(w[h:e])) for h, e in zip(heads, list(heads[1:]) + [n])] if n < 100000 else None
    assert np.array_equal(uk.cpu().numpy().view(np.uint64), ks[heads])
    if want is not None:
        assert np.array_equal(uv.cpu().numpy(), np.array(want))  # left-to-right sums: bit exact
    uk, um = tf.reduce_by_key(sk, torch.tensor(w, device="cuda"), "max", ctx=ctx)
    assert np.array_equal(um.cpu().numpy(), np.maximum.reduceat(w, heads))


def test_csr_validation_and_canonical(ctx):
    good = to_device(P.laplace2d(8))
    tf.csr_validate(good, ctx=ctx)
    assert tf.check_canonical(good, ctx=ctx) == 0
    bad = to_device((np.array([0, 7, 6], np.int32), np.array([1, 0, 0, 1, 0, 1], np.int32), np.ones(6)))
    with pytest.raises(tf.InvalidArgument):
        tf.csr_validate(bad, ctx=ctx)
    dup = to_device((np.array([0, 3, 6], np.int32), np.array([1, 0, 0, 1, 0, 1], np.int32),
                     np.array([-1.0, 1, 1, 1, -1, 1])))
    assert tf.check_canonical(dup, ctx=ctx) == 1
    c = tf.canonicalize(dup, ctx=ctx)
    assert c.values.cpu().tolist() == [2, -1, -1, 2]  # amg_native_test.cpp:115-121
    nan = to_device((np.array([0, 1, 2], np.int32), np.array([0, 1], np.int32), np.array([1.0, np.nan])))
    assert tf.check_canonical(nan, ctx=ctx) & 2


@pytest.mark.parametrize("n", [2, 17, 64, 150, 256])
def test_coarse_lu_matches_oracle(ctx, n):
    rng = np.random.default_rng(n)
    dense = rng.standard_normal((n, n)) + n * np.eye(n) * 0.1
    dense[rng.random((n, n)) < 0.3] = 0.0
    np.fill_diagonal(dense, np.diag(dense) + 1.0)
    off = np.concatenate([[0], np.cumsum((dense != 0).sum(axis=1))]).astype(np.int32)
    idx = np.concatenate([np.flatnonzero(r) for r in dense]).astype(np.int32)
    val = dense[dense != 0]
    ok, lu, piv = tf.coarse_lu_factor(to_device((off, idx, val)), ctx=ctx)
    ook, olu, opiv = O.lu_factor(O.Csr(n, off, idx, val))
    assert ok and ook
    assert np.array_equal(piv.cpu().numpy(), opiv)
    assert np.allclose(lu.cpu().numpy(), olu, rtol=1e-10, atol=1e-12)
    b = rng.standard_normal(n)
    x = tf.coarse_lu_solve(lu, piv, torch.tensor(b, device="cuda"), ctx=ctx).cpu().numpy()
    assert np.allclose(dense @ x, b, rtol=1e-10, atol=1e-10)


def test_coarse_lu_scale_invariance_and_singular(ctx):
    # amg_native_test.cpp:133-153
    off, idx = np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32)
    for scale in (1e-100, 1.0, 1e100):
        ok, lu, piv = tf.coarse_lu_factor(to_device((off, idx, np.array([1, 2, 4, 3.0]) * scale)), ctx=ctx)
        assert ok
        b = torch.tensor([5 * scale, 10 * scale], dtype=torch.float64, device="cuda")
        x = tf.coarse_lu_solve(lu, piv, b, ctx=ctx).cpu().numpy()
        assert abs(x[0] - 1) < 1e-12 and abs(x[1] - 2) < 1e-12
        tf.coarse_lu_solve(lu, piv, b, x=b, ctx=ctx)  # rhs and x alias
        assert np.array_equal(b.cpu().numpy(), x)
    ok, _, _ = tf.coarse_lu_factor(to_device((off, idx, np.ones(4))), ctx=ctx)
    assert not ok


def test_autotune_changes_speed_not_results(ctx):
    off, idx, val = P.heat3d(40, seed=8)
    n = len(off) - 1
    a = to_device((off, idx, val))
    x = torch.tensor(np.random.default_rng(5).standard_normal(n), device="cuda")
    before = tf.spmv(a, x, ctx=ctx).clone()
    stages, ctas, cap, rpt, ms = tf.autotune_spmv(a, x, ctx=ctx)
    assert 2 <= stages <= 4 and 1 <= ctas <= 6 and cap in (100, 125) and rpt in (1, 2) and ms > 0
    after = tf.spmv(a, x, ctx=ctx)
    assert torch.equal(before, after)
    r1 = tf.residual(a, x, x.clone(), ctx=ctx)
    assert torch.isfinite(r1).all()


# Launch shapes: (stages, ctas_per_sm, cap_pct, rows_per_thread).  cap 50%
# splits most tiles into several chunks, so rows straddle chunk boundaries.
SHAPES = [(2, 4, 125, 1), (4, 2, 100, 1), (2, 3, 100, 2), (3, 1, 125, 2), (2, 2, 50, 2), (3, 5, 50, 1)]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_every_launch_shape_gives_identical_results(ctx, dtype):
    off, idx, val = P.heat3d(40, seed=9)
    n = len(off) - 1
    a = to_device((off, idx, val), dtype=dtype)
    rng = np.random.default_rng(6)
    x = torch.tensor(rng.standard_normal(n), dtype=dtype, device="cuda")
    b = torch.tensor(rng.standard_normal(n), dtype=dtype, device="cuda")
    dinv = tf.inverse_diagonal(a, ctx=ctx)
    outs = []
    for shape in SHAPES:
        tf.set_spmv_config(a, *shape, ctx=ctx)
        outs.append((tf.spmv(a, x, ctx=ctx).clone(), tf.residual(a, b, x, ctx=ctx).clone(),
                     tf.jacobi_sweep(a, dinv, b, x, 0.7, ctx=ctx).clone()))
    for o in outs[1:]:
        for u, v in zip(outs[0], o):
            assert torch.equal(u, v)
    ref = O.spmv(O.Csr(n, off, idx, val.astype(np.float64)), x.double().cpu().numpy())
    tol = 1e-12 if dtype == torch.float64 else 1e-4
    assert np.abs(outs[0][0].double().cpu().numpy() - ref).max() <= tol * np.abs(ref).max()


def test_launch_shape_does_not_change_reductions(ctx):
    # The Krylov solve reduces r.z and p.Ap inside the SpMV epilogue: its
    # iterates must be bit-identical under every launch shape.
    m = P.heat3d(24, seed=41)
    n = len(m[0]) - 1
    a = to_device(m)
    b = torch.tensor(P.rhs_uniform(n, 42), device="cuda")
    xs, reps = [], []
    for shape in SHAPES[:4]:
        s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(jacobi_weight=2 / 3), ctx=ctx)
        s.setup(a)
        tf.set_spmv_config(a, *shape, ctx=ctx)  # after setup's own tuning
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        reps.append(s.apply(b, x))
        xs.append(x)
    assert reps[0]["status"] == "Converged"
    assert all(r == reps[0] for r in reps)
    assert all(torch.equal(xs[0], v) for v in xs[1:])


def test_set_spmv_config_rejects_bad_shapes(ctx):
    a = to_device(P.heat3d(8, seed=1))
    for bad in [(1, 2, 100, 1), (5, 2, 100, 1), (2, 0, 100, 1), (2, 9, 100, 1), (2, 2, 40, 1), (2, 2, 100, 3)]:
        with pytest.raises(tf.InvalidArgument):
            tf.set_spmv_config(a, *bad, ctx=ctx)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n", [1, 2047, 300001])
def test_fused_krylov_steps_match_torch(dtype, n):
    # the solvers' fused vector steps as standalone entry points, against the
    # same arithmetic in torch; the squared norms are the same bits as
    # tf_dot_multi of the result (same fixed partition and order)
    from thermofem_b200.api import _VT, _p, check, lib, default_context
    ctx = default_context()
    g = torch.Generator("cuda").manual_seed(n)

    def vec():
        return torch.randn(n, dtype=dtype, device="cuda", generator=g)

    vt, L = _VT[dtype], lib()
    rr = torch.zeros(1, dtype=torch.float64, device="cuda")
    tol = 1e-13 if dtype == torch.float64 else 1e-5

    def close(a, b):
        assert torch.allclose(a, b, rtol=tol, atol=tol)

    def same_norm(v):
        assert torch.equal(rr, tf.dot_multi([v], [v], ctx=ctx))
        assert float(rr) == pytest.approx(float((v.double() ** 2).sum()), rel=1e-10)

    alpha, beta, omega = 0.37, -1.25, 0.61
    # CG: x += alpha p, r -= alpha ap, r.r; p = z + beta p (or z)
    p, ap, x, r = vec(), vec(), vec(), vec()
    x0, r0 = x.clone(), r.clone()
    with ctx:
        check(L.tf_krylov_cg_update(ctx.h, vt, n, alpha, _p(p), _p(ap), _p(x), _p(r), _p(rr)))
    torch.cuda.synchronize()
    a = torch.tensor(alpha, dtype=dtype)
    close(x, x0 + a.item() * p)
    close(r, r0 - a.item() * ap)
    same_norm(r)
    z, pd = vec(), vec()
    pd0 = pd.clone()
    for restart in (0, 1):
        q = pd0.clone()
        with ctx:
            check(L.tf_krylov_cg_direction(ctx.h, vt, n, beta, restart, _p(z), _p(q)))
        torch.cuda.synchronize()
        close(q, z if restart else z + beta * pd0)
    # BiCGStab: p = r + beta (p - omega v) (or r); s = r - alpha v, x += alpha phat, s.s;
    # x += omega shat, r = s - omega t, r.r
    r, v, pb = vec(), vec(), vec()
    for restart in (0, 1):
        q = pb.clone()
        with ctx:
            check(L.tf_krylov_bicgstab_direction(ctx.h, vt, n, beta, omega, restart, _p(r), _p(v), _p(q)))
        torch.cuda.synchronize()
        close(q, r if restart else r + beta * (pb - omega * v))
    ph, x, s = vec(), vec(), torch.empty(n, dtype=dtype, device="cuda")
    x0 = x.clone()
    with ctx:
        check(L.tf_krylov_bicgstab_s(ctx.h, vt, n, alpha, _p(r), _p(v), _p(ph), _p(x), _p(s), _p(rr)))
    torch.cuda.synchronize()
    close(s, r - alpha * v)
    close(x, x0 + alpha * ph)
    same_norm(s)
    sh, t, x, r2 = vec(), vec(), vec(), torch.empty(n, dtype=dtype, device="cuda")
    x0 = x.clone()
    with ctx:
        check(L.tf_krylov_bicgstab_update(ctx.h, vt, n, omega, _p(sh), _p(s), _p(t), _p(x), _p(r2), _p(rr)))
    torch.cuda.synchronize()
    close(x, x0 + omega * sh)
    close(r2, s - omega * t)
    same_norm(r2)


def test_fused_krylov_steps_reject_aliases():
    from thermofem_b200.api import _VT, _p, lib, default_context
    ctx = default_context()
    v = torch.zeros(8, dtype=torch.float64, device="cuda")
    rr = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert lib().tf_krylov_cg_update(ctx.h, _VT[torch.float64], 8, 1.0, _p(v), _p(v), _p(v), _p(v), _p(rr)) == -1
    assert lib().tf_krylov_cg_direction(ctx.h, _VT[torch.float64], 8, 1.0, 0, _p(v), _p(v)) == -1


def test_null_vectors_are_rejected_before_any_launch(ctx):
    """A NULL device vector (or descriptor) of a nonempty operation comes back
    as TF_ERR_INVALID from the host checks and launches nothing."""
    import ctypes as C
    lib = tf.lib()
    invalid = -1
    a = to_device(P.heat3d(8))
    d = a.desc()
    n = a.rows
    v = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(4)]
    p = [t.data_ptr() for t in v]
    i32 = torch.zeros(n + 1, dtype=torch.int32, device="cuda").data_ptr()
    f64 = 1  # TF_F64
    before = lib.tf_ctx_launch_count(ctx.h)
    calls = {
        "spmv x": lambda: lib.tf_spmv(ctx.h, C.byref(d), None, p[1]),
        "spmv y": lambda: lib.tf_spmv(ctx.h, C.byref(d), p[0], None),
        "spmv descriptor": lambda: lib.tf_spmv(ctx.h, None, p[0], p[1]),
        "residual b": lambda: lib.tf_residual(ctx.h, C.byref(d), None, p[1], p[2]),
        "residual descriptor": lambda: lib.tf_residual(ctx.h, None, p[0], p[1], p[2]),
        "jacobi dinv": lambda: lib.tf_jacobi_sweep(ctx.h, C.byref(d), None, p[1], p[2], p[3], 0.5, None, None, None),
        "jacobi descriptor": lambda: lib.tf_jacobi_sweep(ctx.h, None, p[0], p[1], p[2], p[3], 0.5, None, None, None),
        "zero sweep x": lambda: lib.tf_jacobi_zero(ctx.h, n, f64, p[0], p[1], None, 0.5, None),
        "zero sweep length": lambda: lib.tf_jacobi_zero(ctx.h, -1, f64, p[0], p[1], p[2], 0.5, None),
        "inverse diagonal": lambda: lib.tf_inverse_diagonal(ctx.h, C.byref(d), None),
        "restrict members": lambda: lib.tf_restrict(ctx.h, f64, 4, i32, None, p[0], p[1]),
        "prolong map": lambda: lib.tf_prolong(ctx.h, f64, n, None, p[0], p[1]),
        "axpby y": lambda: lib.tf_axpby(ctx.h, f64, n, 1.0, p[0], 1.0, None),
        "scan out": lambda: lib.tf_scan_exclusive_i32(ctx.h, n, i32, None),
        "coarse solve lu": lambda: lib.tf_coarse_lu_solve(ctx.h, 4, None, i32, f64, p[0], p[1]),
    }
    for what, call in calls.items():
        assert call() == invalid, what
    assert lib.tf_ctx_launch_count(ctx.h) == before
    # the context is untouched: a valid call still runs
    assert lib.tf_spmv(ctx.h, C.byref(d), p[0], p[1]) == 0
    assert lib.tf_ctx_synchronize(ctx.h) == 0


def test_checked_context_rejects_malformed_operands_before_launching(monkeypatch):
    # THERMOFEM_B200_CHECKED=1 (read when the context is created): the
    # kernel-layer entry points validate the caller's CSR on the device
    # first; a column one past the last comes back as InvalidArgument and
    # only the validation kernel runs.  A well-formed operand gives the
    # unchecked result.
    import ctypes as C
    monkeypatch.setenv("THERMOFEM_B200_CHECKED", "1")
    ctx = tf.Context(0)
    lib = tf.lib()
    off, idx, val = P.poisson1d(4)
    good = to_device((off, idx, val))
    x = torch.arange(1.0, 5.0, dtype=torch.float64, device="cuda")
    assert torch.equal(tf.spmv(good, x, ctx=ctx), tf.spmv(good, x))
    bad_idx = idx.copy()
    bad_idx[-1] = 4  # n: one past the last column
    bad = to_device((off, bad_idx, val))
    dinv = tf.inverse_diagonal(good, ctx=ctx)
    for call in (lambda: tf.spmv(bad, x, ctx=ctx),
                 lambda: tf.residual(bad, x, x.clone(), ctx=ctx),
                 lambda: tf.jacobi_sweep(bad, dinv, x, x.clone(), 0.5, ctx=ctx)):
        before = lib.tf_ctx_launch_count(ctx.h)
        with pytest.raises(tf.InvalidArgument):
            call()
        assert lib.tf_ctx_launch_count(ctx.h) == before + 1  # the validation kernel only
    # an empty matrix may come without any arrays: valid, nothing to launch
    empty = tf.Csr(0, 0, 0, 2, 1, None, None, None)  # TF_I32, TF_F64
    assert lib.tf_csr_validate(ctx.h, C.byref(empty)) == 0


@pytest.mark.parametrize("dtype,index_dtype", [(torch.float64, torch.int32), (torch.float32, torch.int64)])
def test_unaligned_arrays_take_the_staged_kernel_with_the_same_bits(ctx, dtype, index_dtype):
    # A caller's CSR whose arrays start off a 16-byte boundary cannot be
    # bulk-copied: the staged row-tile kernel reads it (16-byte vector loads
    # over the aligned interior, scalar head and tail) and gives the bits of
    # the pipelined kernel on aligned copies of the same arrays.
    off, idx, val = P.heat3d(16, seed=9)
    a = to_device((off, idx, val), dtype=dtype, index_dtype=index_dtype)
    x = torch.randn(a.rows, dtype=dtype, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    b = torch.randn(a.rows, dtype=dtype, device="cuda", generator=torch.Generator("cuda").manual_seed(4))

    def shifted(t):  # the same values one element past an aligned start
        buf = torch.empty(t.numel() + 1, dtype=t.dtype, device="cuda")
        buf[1:].copy_(t)
        return buf[1:]

    u = tf.DeviceCsr(shifted(a.offsets), shifted(a.indices), shifted(a.values), a.cols)
    assert u.offsets.data_ptr() % 16 and u.indices.data_ptr() % 16 and u.values.data_ptr() % 16
    assert torch.equal(tf.spmv(u, x, ctx=ctx), tf.spmv(a, x, ctx=ctx))
    assert torch.equal(tf.residual(u, b, x, ctx=ctx), tf.residual(a, b, x, ctx=ctx))
