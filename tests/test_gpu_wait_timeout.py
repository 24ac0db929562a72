"""Failure detection without a GPU fault: a bounded device wait that nothing
ends gives up, surfaces as TF_ERR_TIMEOUT on the host, and leaves the context
usable (tf_ctx_check_bounded_wait runs the pipelined kernels' own bounded
mbarrier wait on a barrier that nothing completes)."""
import numpy as np
import pytest
import torch

import thermofem_b200 as tf
from thermofem_b200 import problems as P

pytestmark = pytest.mark.gpu

TF_ERR_TIMEOUT = -5


def test_expired_wait_is_reported_and_the_context_stays_usable():
    ctx = tf.Context(0)
    lib = tf.lib()
    m = P.heat3d(16, seed=61)
    a = tf.DeviceCsr.from_host(*m)
    x = torch.tensor(np.random.default_rng(62).standard_normal(a.rows), device="cuda")
    before = tf.spmv(a, x, ctx=ctx).clone()
    for _ in range(2):  # twice: the fault word is cleared after each report
        assert lib.tf_ctx_check_bounded_wait(ctx.h, 1000) == TF_ERR_TIMEOUT
        assert b"wait" in lib.tf_last_error()
        # the context keeps working: a solve and an SpMV give the same results
        assert lib.tf_ctx_synchronize(ctx.h) == 0
        assert torch.equal(tf.spmv(a, x, ctx=ctx), before)
    s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(), ctx=ctx)
    s.setup(a)
    xs = torch.zeros(a.rows, dtype=torch.float64, device="cuda")
    assert s.apply(torch.tensor(P.rhs_uniform(a.rows, 63), device="cuda"), xs)["status"] == "Converged"


def test_bounded_wait_check_rejects_bad_limits():
    ctx = tf.Context(0)
    lib = tf.lib()
    assert lib.tf_ctx_check_bounded_wait(ctx.h, 0) == -1  # TF_ERR_INVALID
    assert lib.tf_ctx_check_bounded_wait(ctx.h, (1 << 20) + 1) == -1
