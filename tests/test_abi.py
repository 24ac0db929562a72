"""C ABI checks that need no GPU: the library loads, exports every entry
point the header declares, the host-side Matrix Market reader matches the
reference reader on the reference's own test inputs, and compute entry
points fail loudly (no CPU fallback) when no device is present."""
import ctypes
import json
import os
import re

import numpy as np
import pytest
import torch

import thermofem_b200 as tf
from conftest import GOLDEN, ROOT

HEADER = os.path.join(ROOT, "include", "thermofem_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    names = declared()
    assert len(names) > 60
    lib = ctypes.CDLL(tf.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert sorted(tf.SIGNATURES) == declared()


def test_version_and_status_strings():
    assert "sm_100a" in tf.version()
    for code in (0, -1, -2, -3, -4, -5, -6, -7):
        assert tf.lib().tf_status_string(code)


def test_matrix_market_matches_reference_reader():
    g = json.load(open(os.path.join(GOLDEN, "matrix_market_golden.json")))
    for name, case in g["accepted"].items():
        m = tf.read_matrix_market(case["text"])
        assert m["rows"] == case["rows"], name
        assert m["offsets"].tolist() == case["offsets"], name
        assert m["indices"].tolist() == case["indices"], name
        assert m["values"].tolist() == case["values"], name
    for text in g["rejected"]:
        with pytest.raises(tf.ParseError):
            tf.read_matrix_market(text)


def test_matrix_market_file_and_known_answers(tmp_path):
    # matrix_market_test.cpp:8-25
    m = tf.read_matrix_market("%%MatrixMarket matrix coordinate real general\n% comment\n3 3 4\n3 1 2\n1 2 4\n1 2 -1\n3 3 5\n")
    assert m["offsets"].tolist() == [0, 2, 2, 4]
    assert m["indices"].tolist() == [1, 1, 0, 2]
    assert m["values"].tolist() == [4, -1, 2, 5]
    p = tmp_path / "poisson.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n4 4 7\n1 1 2\n2 1 -1\n2 2 2\n3 2 -1\n3 3 2\n4 3 -1\n4 4 2\n")
    m = tf.read_matrix_market_file(str(p))
    assert m["offsets"].tolist() == [0, 2, 5, 8, 10]
    with pytest.raises(tf.ParseError):
        tf.read_matrix_market_file(str(tmp_path / "missing.mtx"))


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device error path")
def test_no_cpu_fallback_without_a_device():
    h = ctypes.c_void_p()
    status = tf.lib().tf_ctx_create(0, None, ctypes.byref(h))
    assert status in (tf.ERR_CUDA, tf.ERR_INVALID)
    assert tf.device_count() == 0
    with pytest.raises(RuntimeError):
        tf.Context(0)


def test_null_arguments_are_rejected():
    assert tf.lib().tf_spmv(None, None, None, None) == tf.ERR_INVALID
    assert tf.lib().tf_solver_apply(None, None, None, 0, None) == tf.ERR_INVALID
    assert b"null" in tf.lib().tf_last_error()


def test_problem_generators_match_the_benchmark_sizes():
    # 2-D 128^2 Poisson: 16,384 rows, 81,408 nonzeros; 3-D 7-point stencil
    # on n^3 cells: 7 n^3 - 6 n^2 nonzeros
    from thermofem_b200 import problems as P
    off, idx, val = P.laplace2d(128)
    assert len(off) - 1 == 16384 and len(idx) == 81408
    off, idx, val = P.heat3d(32, seed=1)
    assert len(off) - 1 == 32 ** 3 and len(idx) == 7 * 32 ** 3 - 6 * 32 ** 2
    assert np.array_equal(P.uniform(5, 10), P.uniform(5, 10))  # pure function of (seed, index)
    assert not np.array_equal(P.uniform(5, 10), P.uniform(6, 10))


def test_solve_matrix_driver_input_errors(tmp_path):
    # Argument and input errors exit 1 with error=... before touching a GPU
    # (example/solve-matrix.cu:59-78).
    import subprocess
    from thermofem_b200 import build as B
    from thermofem_b200 import problems as P
    B.build_driver()

    def run(*args):
        r = subprocess.run([B.DRIVER, *args], capture_output=True, text=True, timeout=60)
        return r.returncode, r.stderr.strip()

    assert run() == (1, "error=Usage: solve-matrix path [amg|identity] [v|w|f]")
    assert run("a", "b", "c", "d") == (1, "error=Usage: solve-matrix path [amg|identity] [v|w|f]")
    assert run("x.mtx", "amg", "z") == (1, "error=Unknown cycle")
    assert run("x.mtx", "jacobi") == (1, "error=Unknown preconditioner")
    assert run(str(tmp_path / "missing.mtx")) == (1, "error=Cannot open matrix file")
    rect = tmp_path / "rect.mtx"
    rect.write_text("%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1.0\n")
    assert run(str(rect)) == (1, "error=Expected nonempty square matrix")
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1.0 0.0\n")
    rc, err = run(str(bad))
    assert rc == 1 and err.startswith("error=")
    # the synthetic writer round-trips through the library's reader
    off, idx, val = P.laplace2d(5)
    path = tmp_path / "lap.mtx"
    P.write_matrix_market(str(path), off, idx, val, symmetric=True)
    back = tf.read_matrix_market_file(str(path))

    def triplets(o, i, v):
        r = np.repeat(np.arange(len(o) - 1), np.diff(o))
        return sorted(zip(r.tolist(), np.asarray(i).tolist(), np.asarray(v).tolist()))

    assert triplets(back["offsets"], back["indices"], back["values"]) == triplets(off, idx, val)


def test_header_binds_from_strict_c99(tmp_path):
    # A plain C caller: the header compiles as C99 with -pedantic and every
    # warning on, links against the library and calls two entry points that
    # need no device (device count, status strings).
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "thermofem_b200", "lib")
    src = tmp_path / "caller.c"
    src.write_text('#include "thermofem_b200.h"\n'
                   "int main(void) {\n"
                   "    int n = -1;\n"
                   "    if (tf_device_count(&n) != TF_OK || n < 0) return 2;\n"
                   "    if (tf_status_string(TF_ERR_INVALID)[0] != 'i') return 3;\n"
                   "    return tf_device_count(0) == TF_ERR_INVALID ? 0 : 4;\n"
                   "}\n")
    exe = tmp_path / "caller"
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(root, "include"),
                        str(src), "-L", libdir, "-lthermofem_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert subprocess.run([str(exe)], timeout=120).returncode == 0
