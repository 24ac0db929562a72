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


def _mm_random_text(rng):
    """One Matrix Market text built from fields that probe the stream
    extractors' number grammar, white space, comments, line endings and the
    header / size / entry rules; most are valid, many are not."""
    pick = lambda xs: xs[int(rng.integers(len(xs)))]  # noqa: E731
    sep = lambda: pick([" ", " ", "\t", "  ", " \t "])  # noqa: E731
    eol = pick(["\n", "\n", "\r\n"])
    field = pick(["real", "real", "integer", "Real", "complex"])
    symmetry = pick(["general", "general", "symmetric", "hermitian"])
    banner = pick(["%%MatrixMarket", "%%MatrixMarket", "%%matrixmarket", " %%MatrixMarket"])
    words = [banner, "matrix", "coordinate", field, symmetry]
    if rng.random() < 0.05:
        words = words[:4]
    if rng.random() < 0.05:
        words.append("extra")
    lines = [sep().join(words)]
    junk = ["", "   ", "% comment", "  % indented", "\t%", "\r", "\v", "%"]
    for _ in range(int(rng.integers(3))):
        lines.append(pick(junk) if rng.random() < 0.8 else "")
    rows = int(rng.integers(0, 6))
    cols = rows if rng.random() < 0.8 else int(rng.integers(0, 6))
    count = int(rng.integers(0, 7))
    size = [str(rows), str(cols), str(count)]
    r = rng.random()
    if r < 0.04:
        size = size[:2]
    elif r < 0.08:
        size.append("1")
    elif r < 0.12:
        size[int(rng.integers(3))] = pick(["+3", "-1", "2147483648", "3x", "3.0", "x", "03"])
    lines.append(sep().join(size))
    value_pool = ["2", "-1.5", "+3", ".5", "5.", "1e3", "1E-3", "1e", "1e+", "1.5.3", "0x10", "inf", "nan", "-",
                  "+", "1e400", "1e-400", "1.e5", ".e5", "e5", "-.5", "+-5", "007", "2abc", "1,5", "4", "-0",
                  "1e5.3", "2.5e-3x", "9" * 30, "4.0"]
    index_pool = ["+1", "01", "1.0", "-1", "0", "99999999999999999999", "1x", "1"]
    n_entries = count + (int(rng.integers(-1, 2)) if rng.random() < 0.15 else 0)
    for _ in range(max(n_entries, 0)):
        i = str(int(rng.integers(1, max(rows, 1) + 1)))
        j = str(int(rng.integers(1, max(cols, 1) + 1)))
        if rng.random() < 0.06:
            i = pick(index_pool)
        if rng.random() < 0.06:
            j = pick(index_pool)
        v = pick(value_pool) if rng.random() < 0.3 else str(int(rng.integers(-9, 10)))
        fields = [i, j, v]
        if rng.random() < 0.03:
            fields.append(pick(["extra", "1", "%"]))
        lines.append(sep().join(fields) + (sep() if rng.random() < 0.1 else ""))
        if rng.random() < 0.1:
            lines.append(pick(junk))
    text = eol.join(lines)
    return text + (eol if rng.random() < 0.9 else "")


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_oracle.so")),
                    reason="the reference reader is built only where the reference sources are")
def test_matrix_market_reader_agrees_with_the_reference_reader_on_random_inputs():
    # 8000 seeded texts: every text the reference reader accepts gives the
    # same CSR here; every text it rejects is rejected with the same message.
    from oracle import oracle as O
    rng = np.random.default_rng(2024)
    accepted = rejected = 0
    messages = set()
    for k in range(8000):
        text = _mm_random_text(rng)
        try:
            want = O.ref_read_matrix_market(text)
        except O.OracleError as e:
            rejected += 1
            messages.add(str(e))
            with pytest.raises(tf.ParseError) as got:
                tf.read_matrix_market(text)
            assert str(e) in str(got.value), (k, text)
            continue
        accepted += 1
        m = tf.read_matrix_market(text)
        assert m["rows"] == want.rows, (k, text)
        assert np.array_equal(m["offsets"], want.offsets), (k, text)
        assert np.array_equal(m["indices"], want.indices), (k, text)
        assert np.array_equal(m["values"], want.values), (k, text)
    assert accepted > 600 and rejected > 2000
    # every rule that a text can break was met (the index-range and read-error
    # rules need inputs larger than these)
    assert messages == {"Unsupported Matrix Market header", "Unexpected Matrix Market field",
                        "Invalid Matrix Market dimensions", "Truncated Matrix Market entries",
                        "Invalid Matrix Market entry", "Mixed triangles in symmetric storage",
                        "Extra Matrix Market entries"}, messages


def test_matrix_market_stream_reader_crosses_block_boundaries(tmp_path):
    # a file much larger than one read block, with a line longer than a block:
    # the file reader cuts lines across block boundaries correctly
    n = 200_000
    rng = np.random.default_rng(3)
    cols = rng.integers(1, n + 1, n)
    vals = rng.standard_normal(n)
    body = "".join(f"{i + 1} {c} {float(v)!r}\n" for i, (c, v) in enumerate(zip(cols, vals)))
    long_comment = "%" + "x" * (40 << 20) + "\n"
    text = "%%MatrixMarket matrix coordinate real general\n" + long_comment + f"{n} {n} {n}\n" + body
    p = tmp_path / "big.mtx"
    p.write_text(text)
    for m in (tf.read_matrix_market_file(str(p)), tf.read_matrix_market_stream(open(p, "rb"))):
        assert m["offsets"].tolist() == list(range(n + 1))
        assert np.array_equal(m["indices"], cols - 1)
        assert np.array_equal(m["values"], vals)

    class Failing:
        def read(self, k):
            raise OSError("device gone")
    with pytest.raises(tf.ParseError, match="read failure"):
        tf.read_matrix_market_stream(Failing())


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
