"""Batched solves (tf_batch_*): independent systems as branches of one CUDA
graph.  Every system's iterations, report and solution must be those of its
own tf_solver_apply, bit for bit."""
import pytest
import torch

import thermofem_b200 as tf
from conftest import to_device
from thermofem_b200 import problems as P

pytestmark = pytest.mark.gpu


def make(kind, m, ctx, hierarchy="f32"):
    cls = tf.Cg if kind == "cg" else tf.BiCgStab
    s = cls(tf.solver_options(), "amg", tf.amg_options(hierarchy_type=hierarchy, jacobi_weight=2 / 3), ctx=ctx)
    s.setup(to_device(m))
    return s


def test_batch_equals_solo_solves(ctx):
    probs = P.batched_transient(6, seed=77, side_min=10, side_max=28)
    kinds = ["cg", "cg", "bicgstab", "cg", "bicgstab", "cg"]
    hier = ["f32", "f64", "f32", "f32", "f64", "f32"]
    solvers = [make(k, p[2], ctx, h) for k, p, h in zip(kinds, probs, hier)]
    rhs = [torch.tensor(p[3] / p[1], device="cuda") for p in probs]
    solo_x, solo_rep = [], []
    for s, b in zip(solvers, rhs):
        x = torch.zeros_like(b)
        solo_rep.append(s.apply(b, x))
        solo_x.append(x)
    batch = tf.Batch(solvers, ctx=ctx)
    for _ in range(2):  # the graph is built once and replayed
        xs = [torch.zeros_like(b) for b in rhs]
        reps = batch.apply(rhs, xs)
        assert reps == solo_rep
        assert all(torch.equal(a, b) for a, b in zip(xs, solo_x))
    assert all(r["status"] == "Converged" for r in reps)


def test_batch_time_steps_and_resetup(ctx):
    # Backward-Euler steps (rhs = T_prev / r) through one batch; a solver set
    # up again makes the batch rebuild its graph.
    probs = P.batched_transient(3, seed=88, side_min=12, side_max=20)
    solvers = [make("cg", p[2], ctx) for p in probs]
    batch = tf.Batch(solvers, ctx=ctx)
    temps = [torch.tensor(p[3], device="cuda") for p in probs]
    for _ in range(3):
        rhs = [t / p[1] for t, p in zip(temps, probs)]
        xs = [t.clone() for t in temps]  # previous step as the initial guess
        reps = batch.apply(rhs, xs)
        assert all(r["status"] == "Converged" for r in reps)
        for s, b, x, r in zip(solvers, rhs, xs, reps):
            x2 = temps[solvers.index(s)].clone()
            assert s.apply(b, x2) == r and torch.equal(x2, x)
        temps = xs
    # new operator for system 1
    m2 = P.transient3d(14, 0.5)
    solvers[1].setup(to_device(m2))
    b = torch.tensor(P.uniform(5, 14 ** 3), device="cuda")
    rhs = [temps[0], b, temps[2]]
    xs = [torch.zeros_like(t) for t in rhs]
    reps = batch.apply(rhs, xs)
    x1 = torch.zeros_like(b)
    assert solvers[1].apply(b, x1) == reps[1] and torch.equal(x1, xs[1])


def test_batch_errors(ctx):
    m = P.transient3d(8, 1.0)
    s = tf.Cg(tf.solver_options(), "amg", ctx=ctx)
    with pytest.raises(tf.InvalidArgument):
        tf.Batch([s, s], ctx=ctx)
    other = tf.Context(0)
    s2 = tf.Cg(tf.solver_options(), "amg", ctx=other)
    with pytest.raises(tf.InvalidArgument):
        tf.Batch([s, s2], ctx=ctx)
    batch = tf.Batch([s], ctx=ctx)
    b = torch.ones(512, dtype=torch.float64, device="cuda")
    with pytest.raises(tf.LogicError):
        batch.apply([b], [torch.zeros_like(b)])
    s.setup(to_device(m))
    rep = batch.apply([b], [torch.zeros_like(b)])[0]
    assert rep["status"] == "Converged"
