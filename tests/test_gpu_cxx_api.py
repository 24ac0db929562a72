"""The reference's own C++ callers, compiled UNCHANGED against this
repository's C++ headers (include/) and linked against libthermofem_b200.so
only (oracle/Makefile `refapi`, built from the reference sources where they
lie, into oracle/_ref):

  - its tests of the solve path -- solver_test.cpp, cg_test.cpp,
    matrix_market_test.cpp, amg_native_test.cpp (with its own host
    aggregation oracle and host V/W/F recursion), version_test.cpp -- through
    tests/cxx's GoogleTest-compatible harness: every test passes (the two
    that need a second GPU skip themselves);
  - its example-4 (BiCGStab + AMG on a 2-D Poisson problem);
  - its solve-matrix driver, whose report must equal the one the reference's
    own driver prints for the same Matrix Market file.

The tests that need no device also run on the CPU (test_reference_api_host_tests)."""
import os
import re
import subprocess

import pytest

from thermofem_b200 import problems as P

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "oracle", "_ref")
API_TESTS = os.path.join(REF, "api-tests")
API_EXAMPLE = os.path.join(REF, "api-example-4")
API_DRIVER = os.path.join(REF, "api-solve-matrix")
REF_DRIVER = os.path.join(REF, "solve-matrix")

built = pytest.mark.skipif(not os.path.exists(API_TESTS), reason="reference callers not built (make -C oracle refapi)")


def _summary(out):
    m = re.search(r"(\d+) tests ran, (\d+) passed, (\d+) skipped, (\d+) failed", out)
    assert m, out[-2000:]
    return tuple(int(v) for v in m.groups())


@built
def test_reference_api_host_tests():
    # the reference tests that need no GPU: Matrix Market parsing and
    # rejection, option validation, the version
    r = subprocess.run([API_TESTS, "--gtest_filter=MatrixMarketTest.*:CgOptionsTest.*:VersionTest.*"],
                       capture_output=True, text=True, timeout=300)
    ran, passed, skipped, failed = _summary(r.stdout)
    assert r.returncode == 0 and failed == 0, r.stdout[-4000:]
    assert ran == passed == 5


@pytest.mark.gpu
@built
def test_reference_test_suite_passes_against_these_headers(capsys):
    r = subprocess.run([API_TESTS], capture_output=True, text=True, timeout=900)
    ran, passed, skipped, failed = _summary(r.stdout)
    with capsys.disabled():
        print(f"\nreference C++ tests against this library: {ran} ran, {passed} passed, {skipped} skipped, "
              f"{failed} failed")
    assert r.returncode == 0 and failed == 0, r.stdout[-6000:]
    # only the tests that need a second GPU may skip
    skipped_names = re.findall(r"\[  SKIPPED \] (\S+)", r.stdout)
    assert all("emptyPattern" in s or "prolongationKeepsOwner" in s for s in skipped_names), skipped_names
    assert passed >= 45


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(API_EXAMPLE), reason="reference example not built")
def test_reference_example_4_runs_against_these_headers():
    r = subprocess.run([API_EXAMPLE], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    err = float(re.search(r"Maximum error: (\S+)", r.stdout).group(1))
    assert err < 1e-6 and "Iterations:" in r.stdout


def _report(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    rows = [line.partition("=") for line in r.stdout.splitlines()]
    return r.returncode, [(k, v) for k, _, v in rows], r.stderr


_RUN_KEYS = {"read_seconds", "setup_seconds", "solve_seconds", "device", "gpu", "cuda_runtime"}
_CLOSE_KEYS = {"reported_relative_residual", "host_relative_residual", "relative_solution_error"}


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(API_DRIVER) and os.path.exists(REF_DRIVER)),
                    reason="reference solve-matrix builds absent")
@pytest.mark.parametrize("matrix,args", [("laplace2d", ("amg",)), ("laplace2d", ("amg", "w")),
                                         ("laplace2d", ("amg", "f")), ("laplace2d", ("identity",)),
                                         ("convdiff", ("amg", "w")), ("heat3d", ("amg",))])
def test_reference_driver_on_these_headers_reports_what_the_reference_reports(tmp_path, matrix, args):
    # The same driver source twice: built on the reference library and on
    # this one.  Same report lines in the same order, same values (sizes,
    # cycle, levels, stop reason, coarse solver, per-level rows, nonzeros and
    # aggregate histograms, complexities, status, iterations, validation);
    # times and device lines aside; residuals to 1e-3 relative.
    path = str(tmp_path / f"{matrix}.mtx")
    if matrix == "laplace2d":
        P.write_matrix_market(path, *P.laplace2d(64), symmetric=True)
    elif matrix == "heat3d":
        P.write_matrix_market(path, *P.heat3d(32, seed=51), symmetric=True)
    else:
        P.write_matrix_market(path, *P.convdiff3d(16, seed=49))
    rc_r, ref, err_r = _report([REF_DRIVER, path, *args])
    rc_o, ours, err_o = _report([API_DRIVER, path, *args])
    assert rc_r == 0 and rc_o == 0, (err_r, err_o)
    assert [k for k, _ in ours] == [k for k, _ in ref]
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


COMPONENT_TESTS = os.path.join(HERE, "cxx", "bin", "component-tests")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(COMPONENT_TESTS), reason="component tests not built (make -C tests/cxx)")
def test_host_driven_component_paths(capsys):
    # this repository's own C++ tests of what the reference's tests do not
    # reach: caller-written preconditioners and factory smoothers, which run
    # the Krylov loop and the cycle from the host, against the fused paths
    r = subprocess.run([COMPONENT_TESTS], capture_output=True, text=True, timeout=600)
    ran, passed, skipped, failed = _summary(r.stdout)
    with capsys.disabled():
        print(f"\ncomponent tests: {ran} ran, {passed} passed, {skipped} skipped, {failed} failed")
    assert r.returncode == 0 and failed == 0 and skipped == 0, r.stdout[-6000:]
