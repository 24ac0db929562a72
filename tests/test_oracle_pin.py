"""Pins the CPU oracle (oracle/oracle.c) before the tests trust it:
against the golden fixtures generated from the reference's own host oracle,
and, where this machine has the reference sources, against that oracle
directly (oracle/_ref).  CPU only."""
import numpy as np
import pytest

from conftest import golden_csr
from oracle import oracle as O

SIZES = [1, 2, 4, 17, 61, 128]


def same(a, b):
    return (a.rows == b.rows and np.array_equal(a.offsets, b.offsets) and np.array_equal(a.indices, b.indices)
            and np.array_equal(a.values, b.values))


@pytest.mark.parametrize("name", [f"sample{n}" for n in SIZES] + ["galerkin4", "poisson127"])
def test_oracle_matches_reference_golden(golden, name):
    a = golden_csr(golden, f"{name}/input")
    if name.startswith("sample"):
        # the oracle's sample(n) generator restates the reference's (MT19937, seed 173+n)
        assert same(O.sample_matrix(int(name[6:])), a)
    ca = O.canonical(a)
    assert same(ca, golden_csr(golden, f"{name}/canonical"))
    exercised = False
    for th in (0.0, 0.25, 1.0):
        g = O.strength(ca, th)
        assert same(g, golden_csr(golden, f"{name}/strength{th}"))
        for rounds in (1, 8):
            for absorb in (0, 1):
                key = f"{name}/agg_t{th}_r{rounds}_a{absorb}"
                t = O.aggregate(g, rounds, bool(absorb))
                assert np.array_equal(t.map, golden[key + "/map"])
                assert np.array_equal(t.offsets, golden[key + "/offsets"])
                assert np.array_equal(t.members, golden[key + "/members"])
                assert np.array_equal(t.histogram, golden[key + "/histogram"])
                c = O.galerkin(ca, t.map, t.coarse)
                assert same(c, golden_csr(golden, key + "/galerkin"))
                assert c.nnz <= ca.nnz
                if absorb:
                    exercised |= O.aggregate(g, rounds, False).coarse != t.coarse
    if name == "sample128":
        assert exercised, "absorption must change the aggregates somewhere in the sweep"


def test_four_point_galerkin_known_answer(golden):
    # multigrid_operations_test.cpp:28-44: 4x4 tridiagonal -> one aggregate, Ac = [2]
    a = golden_csr(golden, "galerkin4/input")
    t = O.aggregate(O.strength(a, 0.25), 8, True)
    c = O.galerkin(a, t.map, t.coarse)
    assert c.rows == 1 and list(c.values) == [2.0]


def test_four_point_residual_and_jacobi_known_answers(golden):
    # multigrid_operations_test.cpp:45-59 on the same 4x4 tridiagonal: the
    # residual of b = 0 at x = ones is (-1, 0, 0, -1); one Jacobi update with
    # weight 1 from x = 0 and b = ones is 0.5 everywhere
    a = golden_csr(golden, "galerkin4/input")
    ones = np.ones(4)
    assert list(np.zeros(4) - O.spmv(a, ones)) == [-1.0, 0.0, 0.0, -1.0]
    assert list(O.jacobi(a, 1, 1.0, ones, np.zeros(4))) == [0.5] * 4


def test_duplicate_canonicalisation_known_answer():
    # amg_native_test.cpp:115-121: duplicates summed -> {2, -1, -1, 2}
    a = O.Csr(2, np.array([0, 3, 6], np.int32), np.array([1, 0, 0, 1, 0, 1], np.int32),
              np.array([-1, 1, 1, 1, -1, 1], np.float64))
    assert list(O.canonical(a).values) == [2, -1, -1, 2]


def test_mt19937_matches_std_generator():
    if not O.ref_available():
        pytest.skip("reference sources not available on this machine")
    for seed in (5, 173, 174, 301):
        assert np.array_equal(O.mt19937(seed, 1500), O.ref_std_mt19937(seed, 1500))


def test_oracle_matches_reference_build_on_larger_samples():
    if not O.ref_available():
        pytest.skip("reference sources not available on this machine")
    for n in (300, 517):
        h = O.sample_matrix(n)
        ca = O.canonical(h)
        assert same(ca, O.ref_canonical(h))
        g = O.strength(ca, 0.25)
        assert same(g, O.ref_strength(h, 0.25))
        t, rt = O.aggregate(g, 8, True), O.ref_aggregate(g, 8, True)
        assert np.array_equal(t.map, rt.map) and np.array_equal(t.members, rt.members)
        assert same(O.galerkin(ca, t.map, t.coarse), O.ref_galerkin(h, rt))


def test_coarse_lu_scale_invariance():
    # amg_native_test.cpp:133-153
    for scale in (1e-100, 1.0, 1e100):
        a = O.Csr(2, np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32),
                  np.array([1, 2, 4, 3], np.float64) * scale)
        ok, lu, piv = O.lu_factor(a)
        assert ok
        x = O.lu_solve(lu, piv, np.array([5, 10]) * scale)
        assert abs(x[0] - 1) < 1e-12 and abs(x[1] - 2) < 1e-12
    ok, _, _ = O.lu_factor(O.Csr(2, np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32), np.ones(4)))
    assert not ok


def test_oracle_solvers_known_answers():
    # solver_test.cpp:180-213 / cg_test.cpp:51-75: 1-D Poisson, b = 1, x_i = (i+1)(n-i)/2
    n = 63
    from thermofem_b200 import problems as P
    off, idx, val = P.poisson1d(n)
    a = O.Csr(n, off, idx, val)
    exact = np.array([(i + 1) * (n - i) / 2 for i in range(n)])
    amg = O.Amg(a, coarse_rows=8)
    for solve in (O.cg, O.bicgstab):
        x, rep = solve(a, amg, np.ones(n), np.zeros(n), rtol=1e-9)
        assert rep["status"] == "Converged"
        assert np.allclose(x, exact, rtol=1e-8)


def test_oracle_cycle_visits():
    # amg_native_test.cpp:352-369
    from thermofem_b200 import problems as P
    off, idx, val = P.poisson1d(127)
    a = O.Csr(127, off, idx, val)
    for cyc in (0, 1, 2):
        amg = O.Amg(a, coarse_rows=4, cycle=cyc)
        _, visits = amg.apply(np.ones(127))
        L = amg.levels
        assert L >= 3
        if cyc == 0:
            assert list(visits) == [1] * L
        elif cyc == 1:
            assert list(visits) == [2 ** d for d in range(L)]
        else:
            assert list(visits) == [d + 2 if d + 1 < L else L for d in range(L)]
