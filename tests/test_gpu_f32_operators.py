"""The hierarchy type TF_F32_VALUES: every level operator stored in FP32,
the cycle's vectors, diagonals and arithmetic in FP64 (each value widened
before its product).  No reference counterpart: it exists because
BiCGStab on strongly convective problems loses many iterations when the
preconditioner's vectors are rounded to FP32 (a preconditioner that is
linear only to ~4e-8), while FP32 operator values cost it nothing.

Parity: the levels are the FP64 hierarchy's levels rounded to FP32 (bit for
bit), and one cycle equals a numpy restatement of the cycle over those
rounded values with FP64 vectors (Cycle.cuh:35-63, the library's fused
transfers unrolled) to 1e-12."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import thermofem_b200 as tf
from conftest import to_device
from thermofem_b200 import problems as P

pytestmark = pytest.mark.gpu

OPTS = dict(jacobi_weight=2 / 3, coarse_rows=64)


def _arrays(amg, d):
    c = amg.level_matrix(d)
    return c.offsets.cpu(), c.indices.cpu(), c.values.cpu()


def _levels(amg):
    return [_arrays(amg, d) for d in range(amg.level_count())]


@pytest.mark.parametrize("case", ["heat3d16", "convdiff14"])
def test_levels_are_the_fp64_levels_rounded(ctx, case):
    m = P.heat3d(16, seed=3) if case == "heat3d16" else P.convdiff3d(14, seed=49)
    a = to_device(m)
    f64 = tf.Amg(tf.amg_options(hierarchy_type="f64", **OPTS), ctx=ctx)
    f32v = tf.Amg(tf.amg_options(hierarchy_type="f32v", **OPTS), ctx=ctx)
    f64.setup(a)
    f32v.setup(a)
    assert f64.level_count() == f32v.level_count() >= 3
    assert f64.level_statistics() == f32v.level_statistics()
    for d, (l64, l32) in enumerate(zip(_levels(f64), _levels(f32v))):
        o64, i64, v64 = l64
        o32, i32, v32 = l32
        assert torch.equal(o64, o32) and torch.equal(i64, i32), d
        assert v32.dtype == torch.float32
        assert torch.equal(v64.to(torch.float32), v32), d


def _restated_cycle(amg64, b, kind, w):
    """One cycle from a zero guess over the FP64 hierarchy's levels rounded to
    FP32, vectors and arithmetic in FP64."""
    mats, maps = [], []
    for d in range(amg64.level_count()):
        off, idx, val = (t.numpy() for t in _arrays(amg64, d))
        n = len(off) - 1
        mats.append(sp.csr_matrix((val.astype(np.float32).astype(np.float64), idx, off), shape=(n, n)))
        if d + 1 < amg64.level_count():
            maps.append(amg64.level_transfer(d)[0].cpu().numpy())
    # the coarse solve inverts the FP64 coarsest operator (its LU is factored
    # before any rounding)
    off, idx, val = (t.numpy() for t in _arrays(amg64, len(mats) - 1))
    inv = np.linalg.inv(sp.csr_matrix((val, idx, off)).toarray())
    L = len(mats)

    def cyc(d, rhs, x):
        A = mats[d]
        dinv = 1.0 / A.diagonal()
        if d == L - 1:
            return inv @ rhs
        x = w * dinv * rhs if x is None else x + w * dinv * (rhs - A @ x)
        r = rhs - A @ x
        rc = np.bincount(maps[d], weights=r, minlength=mats[d + 1].shape[0])
        xc = cyc(d + 1, rc, None)
        if kind == "w":
            xc = cyc(d + 1, rc, xc)
        x = x + xc[maps[d]]
        return x + w * dinv * (rhs - A @ x)

    return cyc(0, b, None)


@pytest.mark.parametrize("kind", ["v", "w"])
@pytest.mark.parametrize("case", ["heat3d16", "convdiff14"])
def test_cycle_matches_restatement(ctx, case, kind):
    m = P.heat3d(16, seed=3) if case == "heat3d16" else P.convdiff3d(14, seed=49)
    n = len(m[0]) - 1
    a = to_device(m)
    f64 = tf.Amg(tf.amg_options(hierarchy_type="f64", cycle=kind, **OPTS), ctx=ctx)
    f64.setup(a)
    b = P.rhs_uniform(n, 7)
    want = _restated_cycle(f64, b, kind, 2 / 3)
    tb = torch.tensor(b, device="cuda")
    for small in (1200, 0):  # the shared-memory region and every level launched: the same bits
        f32v = tf.Amg(tf.amg_options(hierarchy_type="f32v", cycle=kind, small_level_rows=small, **OPTS), ctx=ctx)
        f32v.setup(a)
        got = f32v.apply(tb).cpu().numpy()
        assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want)), small
        if small:
            region = got
        else:
            assert np.array_equal(got, region)


def test_bicgstab_iterations_on_convection_diffusion(ctx):
    # 192^3 convection-diffusion, BiCGStab + W(1,1): the FP32 hierarchy needs
    # ~1.5x the FP64 iterations (72 vs 46 on this right-hand side); FP32
    # operators under an FP64 cycle stay within 10 % of FP64 (49).
    m = P.convdiff3d(192, 1003)
    n = len(m[0]) - 1
    a = tf.DeviceCsr.from_host(*m)
    b = torch.tensor(P.rhs_uniform(n, 1002), device="cuda")
    its = {}
    for hier in ("f64", "f32v", "f32"):
        s = tf.BiCgStab(tf.solver_options(), "amg", tf.amg_options(hierarchy_type=hier, cycle="w", **OPTS), ctx=ctx)
        s.setup(a)
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        rep = s.apply(b, x)
        assert rep["status"] == "Converged"
        r = tf.residual(a, b, x, ctx=ctx)
        assert float(torch.linalg.norm(r) / torch.linalg.norm(b)) <= 1.0001e-8
        its[hier] = rep["iterations"]
        del s
    assert its["f32v"] <= 1.1 * its["f64"], its
    assert its["f32"] > 1.3 * its["f64"], its
