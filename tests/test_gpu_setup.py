"""GPU aggregation setup vs the reference oracle, bit for bit: canonical
form, strength graph, aggregates, member table, histogram and Galerkin
operator (structure and values) on the reference's own sweep
(amg_native_test.cpp:66-114) and on generated heat-conduction matrices
checked against the CPU oracle.  The summation order of every merged entry
is the stable left-to-right order, so even the values are exact."""
import numpy as np
import pytest
import torch

import thermofem_b200 as tf
from conftest import golden_csr, to_device
from oracle import oracle as O
from thermofem_b200 import problems as P

pytestmark = pytest.mark.gpu

CASES = [f"sample{n}" for n in (1, 2, 4, 17, 61, 128)] + ["galerkin4", "poisson127"]


def host(d: tf.DeviceCsr):
    off, idx, val = d.host()
    return O.Csr(len(off) - 1, off, idx, val)


def same(a, b):
    return (a.rows == b.rows and np.array_equal(a.offsets, b.offsets) and np.array_equal(a.indices, b.indices)
            and np.array_equal(a.values, b.values))


@pytest.mark.parametrize("name", CASES)
def test_setup_stages_match_reference_golden(ctx, golden, name):
    a = to_device(golden_csr(golden, f"{name}/input"))
    ca = tf.canonicalize(a, ctx=ctx)
    assert same(host(ca), golden_csr(golden, f"{name}/canonical"))
    for th in (0.0, 0.25, 1.0):
        g = tf.strength(ca, th, ctx=ctx)
        assert same(host(g), golden_csr(golden, f"{name}/strength{th}"))
        for rounds in (1, 8):
            for absorb in (0, 1):
                key = f"{name}/agg_t{th}_r{rounds}_a{absorb}"
                t = tf.aggregate(g, rounds, bool(absorb), ctx=ctx)
                assert np.array_equal(t.map.cpu().numpy(), golden[key + "/map"])
                assert np.array_equal(t.offsets.cpu().numpy(), golden[key + "/offsets"])
                assert np.array_equal(t.members.cpu().numpy(), golden[key + "/members"])
                assert np.array_equal(t.histogram, golden[key + "/histogram"])
                c = tf.galerkin(ca, t, ctx=ctx)
                assert same(host(c), golden_csr(golden, key + "/galerkin"))
                assert c.nnz <= ca.nnz
                ones = torch.ones(ca.rows, dtype=torch.float64, device="cuda")
                sums = tf.restrict_aggregates(t, ones, ctx=ctx)
                assert np.array_equal(sums.cpu().numpy(), np.diff(golden[key + "/offsets"]).astype(np.float64))
                tf.prolong_aggregates(t, sums, ones, ctx=ctx)
                assert np.array_equal(ones.cpu().numpy(), 1 + sums.cpu().numpy()[golden[key + "/map"]])


def test_match_and_contract_stages(ctx, golden):
    a = golden_csr(golden, "sample128/input")
    g = O.strength(O.canonical(a), 0.25)
    dg = to_device(g)
    for rounds in (1, 3, 8):
        m, cnt = tf.match(dg, rounds, ctx=ctx)
        om, ocnt = O.match_pairs(g, rounds)
        assert cnt == ocnt and np.array_equal(m.cpu().numpy(), om)
        c = tf.contract(dg, m, cnt, ctx=ctx)
        assert same(host(c), O.contract(g, om, ocnt))


def test_setup_validation_errors(ctx):
    # amg_native_test.cpp:115-131
    dup = to_device((np.array([0, 3, 6], np.int32), np.array([1, 0, 0, 1, 0, 1], np.int32),
                     np.array([-1.0, 1, 1, 1, -1, 1])))
    with pytest.raises(tf.InvalidArgument):
        tf.strength(tf.canonicalize(dup, ctx=ctx), -0.1, ctx=ctx)
    g = tf.strength(tf.canonicalize(dup, ctx=ctx), 0.25, ctx=ctx)
    with pytest.raises(tf.InvalidArgument):
        tf.aggregate(g, 0, True, ctx=ctx)
    zero_diag = to_device((np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32), np.array([0.0, 1, 1, 1])))
    with pytest.raises(tf.InvalidArgument):
        tf.strength(zero_diag, 0.25, ctx=ctx)


@pytest.mark.parametrize("gen", ["heat3d", "convdiff3d", "laplace2d"])
def test_hierarchy_matches_oracle(ctx, gen):
    m = {"heat3d": lambda: P.heat3d(20, seed=11), "convdiff3d": lambda: P.convdiff3d(14, seed=12),
         "laplace2d": lambda: P.laplace2d(64)}[gen]()
    off, idx, val = m
    n = len(off) - 1
    amg = tf.Amg(dtype=torch.float64, ctx=ctx, coarse_rows=32)
    amg.setup(to_device(m))
    ora = O.Amg(O.Csr(n, off, idx, val), coarse_rows=32)
    assert amg.level_count() == ora.levels
    assert amg.stop_reason() == ora.stop_reason()
    assert amg.coarse_solver() == ora.coarse_solver()
    stats = amg.level_statistics()
    for d in range(ora.levels):
        r, z, hist = ora.level_info(d)
        assert stats[d]["rows"] == r and stats[d]["nonzeros"] == z
        assert stats[d]["aggregate_sizes"] == hist.tolist()
        assert same(host(amg.level_matrix(d)), ora.matrix(d))
        if d + 1 < ora.levels:
            mp, _, _, nc = amg.level_transfer(d)
            assert np.array_equal(mp.cpu().numpy(), ora.map(d))


@pytest.mark.parametrize("hierarchy", ["f64", "f32"])
def test_setup_and_solve_are_deterministic(hierarchy):
    # the same setup twice, in two contexts: every level operator, the same
    # bytes; the same solve: the same report and the same bits
    m = P.heat3d(24, seed=71)
    n = len(m[0]) - 1
    b = torch.tensor(P.rhs_uniform(n, 72), device="cuda")
    runs = []
    for _ in range(2):
        ctx = tf.Context(0)
        s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(hierarchy_type=hierarchy), ctx=ctx)
        s.setup(to_device(m))
        levels = [s.level_matrix(d) for d in range(s.level_count())]
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        rep = s.apply(b, x)
        runs.append((levels, rep, x))
    (l0, r0, x0), (l1, r1, x1) = runs
    assert len(l0) == len(l1) >= 3
    for a, c in zip(l0, l1):
        assert torch.equal(a.offsets, c.offsets) and torch.equal(a.indices, c.indices)
        assert torch.equal(a.values, c.values)
    assert r0 == r1 and torch.equal(x0, x1)


def test_setup_phase_times():
    # every setup phase is timed and the phases cover the hierarchy build
    m = P.heat3d(24, seed=73)
    s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(hierarchy_type="f32"))
    s.setup(to_device(m))
    ph = s.setup_phases()
    assert list(ph) == ["level copies and diagonals", "column and sliced copies", "SpMV shape tuning",
                        "strength graphs", "aggregation", "Galerkin products", "coarse LU", "small-level region",
                        "layout selection"]
    assert all(v >= 0 for v in ph.values())
    assert ph["aggregation"] > 0 and ph["Galerkin products"] > 0 and ph["strength graphs"] > 0


def test_solvers_on_separate_threads_give_the_results_of_one_thread():
    # Separate solver instances, each with its own context, may be driven
    # from separate host threads at the same time: setups (tuning, layout
    # selection, graph captures) and solves interleave, and every report and
    # solution equals the one the same solve gives alone.
    import threading
    m = P.heat3d(20, seed=75)
    n = len(m[0]) - 1
    b_host = P.rhs_uniform(n, 76)

    def solve(hierarchy):
        # Each thread keeps its torch work on its own context's stream and
        # waits on that stream only: a device-wide synchronisation (or the
        # legacy default stream) would cut into another thread's graph
        # capture, which CUDA then invalidates.
        ctx = tf.Context(0)
        with torch.cuda.stream(ctx.stream):
            s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(hierarchy_type=hierarchy), ctx=ctx)
            s.setup(to_device(m))
            x = torch.zeros(n, dtype=torch.float64, device="cuda")
            rep = s.apply(torch.tensor(b_host, device="cuda"), x)
            ctx.stream.synchronize()
            assert s.last_execution == 2  # captured as one whole-solve graph, also beside other threads
            return rep, x.cpu()

    alone = {h: solve(h) for h in ("f64", "f32")}
    results, errors = {}, []

    def worker(h, k):
        try:
            results[(h, k)] = solve(h)
        except Exception as e:  # reported below, on the main thread
            errors.append(repr(e))

    threads = [threading.Thread(target=worker, args=(h, k)) for k in range(2) for h in ("f64", "f32")]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
    assert len(results) == 4
    for (h, _), (rep, x) in results.items():
        assert rep == alone[h][0] and rep["status"] == "Converged"
        assert torch.equal(x, alone[h][1])
