"""The small-level sub-cycle (tf_amg_options.small_level_rows): every level
below the threshold runs as one thread-block-cluster launch per sub-cycle.
It must give the cycle of the separately launched kernels bit for bit (same
arithmetic, same order) and match the oracle's host recursion like the
default path (amg_native_test.cpp:348)."""
import numpy as np
import pytest
import torch

import thermofem_b200 as tf
from conftest import to_device
from oracle import oracle as O
from thermofem_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cycle", ["v", "w", "f"])
@pytest.mark.parametrize("post", [1, 0, 2])
@pytest.mark.parametrize("fuse", ["1", "0"])
@pytest.mark.parametrize("rows", [700, 5000])  # one CTA; a cluster (levels too big for one)
def test_cluster_levels_match_launched_levels(ctx, cycle, post, fuse, rows, monkeypatch):
    monkeypatch.setenv("THERMOFEM_B200_FUSE", fuse)
    m = P.heat3d(24, seed=41)
    n = len(m[0]) - 1
    b = P.rhs_uniform(n, 42)
    a = to_device(m)
    opts = dict(coarse_rows=32, cycle=cycle, post_sweeps=post, jacobi_weight=2 / 3)
    plain = tf.Amg(tf.amg_options(small_level_rows=0, **opts), ctx=ctx)
    coop = tf.Amg(tf.amg_options(small_level_rows=rows, **opts), ctx=ctx)
    plain.setup(a)
    coop.setup(a)
    assert plain.level_count() >= 4
    tb = torch.tensor(b, device="cuda")
    x0, x1 = plain.apply(tb).cpu().numpy(), coop.apply(tb).cpu().numpy()
    scale = np.max(np.abs(x0))
    assert np.array_equal(x0, x1)
    assert plain.last_cycle_visits() == coop.last_cycle_visits()
    ora = O.Amg(O.Csr(n, *m), coarse_rows=32, cycle={"v": 0, "w": 1, "f": 2}[cycle], post_sweeps=post,
                jacobi_weight=2 / 3)
    assert np.max(np.abs(x1 - ora.apply(b)[0])) / scale < 1e-12
    again = coop.apply(tb).cpu().numpy()
    assert np.array_equal(again, x1)


def test_cluster_levels_in_solvers(ctx):
    m = P.convdiff3d(20, seed=43)
    n = len(m[0]) - 1
    b = torch.tensor(P.rhs_uniform(n, 44), device="cuda")
    reps = []
    for rows in (0, 5000):
        s = tf.BiCgStab(tf.solver_options(), "amg",
                        tf.amg_options(cycle="w", hierarchy_type="f32", small_level_rows=rows), ctx=ctx)
        s.setup(to_device(m))
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        reps.append(s.apply(b, x))
        assert reps[-1]["status"] == "Converged"
        r = tf.residual(to_device(m), b, x, ctx=ctx)
        assert float(torch.linalg.norm(r) / torch.linalg.norm(b)) <= 1.0001e-8
    assert reps[0] == reps[1]
