"""ctypes binding of the CPU oracle (oracle/liboracle.so) and of the
oracle built from the reference sources (oracle/_ref/libref_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_oracle.so")


class _Csr(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("nnz", C.c_int64),
                ("offsets", C.POINTER(C.c_int)), ("indices", C.POINTER(C.c_int)),
                ("values", C.POINTER(C.c_double))]


class AmgOptions(C.Structure):
    _fields_ = [("max_levels", C.c_int), ("coarse_rows", C.c_int), ("matching_rounds", C.c_int),
                ("pre_sweeps", C.c_int), ("post_sweeps", C.c_int), ("coarse_sweeps", C.c_int),
                ("jacobi_weight", C.c_double), ("strength_threshold", C.c_double),
                ("absorb_singletons", C.c_int), ("cycle", C.c_int), ("coarse_lu_rows", C.c_int)]

    @staticmethod
    def make(max_levels=20, coarse_rows=64, matching_rounds=8, pre_sweeps=1, post_sweeps=1,
             coarse_sweeps=8, jacobi_weight=0.75, strength_threshold=0.25, absorb_singletons=True,
             cycle=0, coarse_lu_rows=64):
        return AmgOptions(max_levels, coarse_rows, matching_rounds, pre_sweeps, post_sweeps, coarse_sweeps,
                          jacobi_weight, strength_threshold, int(absorb_singletons), cycle, coarse_lu_rows)


class _SolveResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("residual_norm", C.c_double),
                ("relative_residual", C.c_double)]


class _SolverOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("relative_tolerance", C.c_double),
                ("absolute_tolerance", C.c_double), ("refresh_interval", C.c_int)]


@dataclass
class Csr:
    rows: int
    offsets: np.ndarray
    indices: np.ndarray
    values: np.ndarray

    @property
    def nnz(self):
        return int(self.indices.shape[0])


def build():
    """Builds liboracle.so (and oracle/_ref when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    P, I, D, L = C.c_void_p, C.c_int, C.c_double, C.c_int64
    pc = C.POINTER(_Csr)
    lib.or_canonical.argtypes = [I, P, P, P, L, pc]
    lib.or_strength.argtypes = [pc, D, pc]
    lib.or_match_pairs.argtypes = [pc, I, P, P]
    lib.or_contract.argtypes = [pc, P, I, pc]
    lib.or_aggregate.argtypes = [pc, I, I, P, P, P, P, P]
    lib.or_galerkin.argtypes = [pc, P, I, pc]
    lib.or_csr_free.argtypes = [pc]
    lib.or_validate.argtypes = [pc, P]
    lib.or_lu_factor.argtypes = [pc, P, P]
    lib.or_lu_solve.argtypes = [I, P, P, P, P]
    lib.or_spmv.argtypes = [pc, P, P]
    lib.or_jacobi.argtypes = [pc, I, D, P, P]
    lib.or_amg_setup.argtypes = [pc, C.POINTER(AmgOptions), C.POINTER(C.c_int)]
    lib.or_amg_setup.restype = C.c_void_p
    lib.or_amg_free.argtypes = [P]
    lib.or_amg_levels.argtypes = [P]
    lib.or_amg_level_info.argtypes = [P, I, P, P, P]
    lib.or_amg_stop_reason.argtypes = [P]
    lib.or_amg_stop_reason.restype = C.c_char_p
    lib.or_amg_coarse_solver.argtypes = [P]
    lib.or_amg_coarse_solver.restype = C.c_char_p
    lib.or_amg_map.argtypes = [P, I]
    lib.or_amg_map.restype = C.POINTER(C.c_int)
    lib.or_amg_matrix.argtypes = [P, I]
    lib.or_amg_matrix.restype = pc
    lib.or_amg_apply.argtypes = [P, P, P, P]
    lib.or_cg.argtypes = [pc, P, P, P, C.POINTER(_SolverOptions)]
    lib.or_cg.restype = _SolveResult
    lib.or_bicgstab.argtypes = [pc, P, P, P, C.POINTER(_SolverOptions)]
    lib.or_bicgstab.restype = _SolveResult
    lib.or_sample_matrix.argtypes = [I, pc]
    lib.or_mt19937.argtypes = [C.c_uint32, I, P]
    lib.or_num_threads.restype = I
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _view(a: Csr):
    off = np.ascontiguousarray(a.offsets, dtype=np.int32)
    idx = np.ascontiguousarray(a.indices, dtype=np.int32)
    val = np.ascontiguousarray(a.values, dtype=np.float64)
    s = _Csr(a.rows, a.rows, idx.shape[0], off.ctypes.data_as(C.POINTER(C.c_int)),
             idx.ctypes.data_as(C.POINTER(C.c_int)), val.ctypes.data_as(C.POINTER(C.c_double)))
    s._keep = (off, idx, val)
    return s


def _take(s: _Csr, free) -> Csr:
    n, m = s.rows, s.nnz
    out = Csr(n, np.ctypeslib.as_array(s.offsets, (n + 1,)).copy(),
              np.ctypeslib.as_array(s.indices, (max(m, 1),))[:m].copy(),
              np.ctypeslib.as_array(s.values, (max(m, 1),))[:m].copy())
    free(C.byref(s))
    return out


class OracleError(ValueError):
    pass


def _check(status):
    if status != 0:
        raise OracleError(f"oracle status {status}")


def canonical(a: Csr) -> Csr:
    v = _view(a)
    out = _Csr()
    _check(lib().or_canonical(a.rows, C.cast(v.offsets, C.c_void_p), C.cast(v.indices, C.c_void_p),
                              C.cast(v.values, C.c_void_p), v.nnz, C.byref(out)))
    return _take(out, lib().or_csr_free)


def row_max(a: Csr):
    out = np.zeros(a.rows)
    status = lib().or_validate(C.byref(_view(a)), _ptr(out))
    return status, out


def strength(a: Csr, theta: float) -> Csr:
    out = _Csr()
    _check(lib().or_strength(C.byref(_view(a)), theta, C.byref(out)))
    return _take(out, lib().or_csr_free)


def match_pairs(g: Csr, rounds: int):
    m = np.zeros(g.rows, np.int32)
    cnt = C.c_int()
    _check(lib().or_match_pairs(C.byref(_view(g)), rounds, _ptr(m), C.byref(cnt)))
    return m, cnt.value


def contract(g: Csr, mp, count) -> Csr:
    mp = np.ascontiguousarray(mp, np.int32)
    out = _Csr()
    _check(lib().or_contract(C.byref(_view(g)), _ptr(mp), count, C.byref(out)))
    return _take(out, lib().or_csr_free)


@dataclass
class Transfer:
    map: np.ndarray
    offsets: np.ndarray
    members: np.ndarray
    coarse: int
    histogram: np.ndarray


def aggregate(g: Csr, rounds: int, absorb: bool) -> Transfer:
    n = g.rows
    mp = np.zeros(n, np.int32)
    off = np.zeros(n + 1, np.int32)
    mem = np.zeros(n, np.int32)
    cnt = C.c_int()
    hist = np.zeros(4, np.int64)
    _check(lib().or_aggregate(C.byref(_view(g)), rounds, int(absorb), _ptr(mp), _ptr(off), _ptr(mem),
                              C.byref(cnt), _ptr(hist)))
    return Transfer(mp, off[:cnt.value + 1].copy(), mem, cnt.value, hist)


def galerkin(a: Csr, mp, coarse) -> Csr:
    mp = np.ascontiguousarray(mp, np.int32)
    out = _Csr()
    _check(lib().or_galerkin(C.byref(_view(a)), _ptr(mp), coarse, C.byref(out)))
    return _take(out, lib().or_csr_free)


def lu_factor(a: Csr):
    n = a.rows
    lu = np.zeros(n * n)
    piv = np.zeros(n, np.int32)
    ok = lib().or_lu_factor(C.byref(_view(a)), _ptr(lu), _ptr(piv))
    return bool(ok), lu, piv


def lu_solve(lu, piv, b):
    n = piv.shape[0]
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(n)
    lib().or_lu_solve(n, _ptr(lu), _ptr(piv), _ptr(b), _ptr(x))
    return x


def spmv(a: Csr, x):
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(a.rows)
    lib().or_spmv(C.byref(_view(a)), _ptr(x), _ptr(y))
    return y


def jacobi(a: Csr, sweeps, weight, b, x):
    b = np.ascontiguousarray(b, np.float64)
    x = np.array(x, np.float64, copy=True)
    _check(lib().or_jacobi(C.byref(_view(a)), sweeps, weight, _ptr(b), _ptr(x)))
    return x


class Amg:
    """Oracle AMG hierarchy (setup in the constructor)."""

    def __init__(self, a: Csr, **opts):
        self.opts = AmgOptions.make(**opts)
        self._v = _view(a)
        st = C.c_int()
        self._free = lib().or_amg_free  # kept: module globals are cleared at interpreter shutdown
        self.h = lib().or_amg_setup(C.byref(self._v), C.byref(self.opts), C.byref(st))
        if st.value != 0 or not self.h:
            raise OracleError(f"oracle AMG setup status {st.value}")
        self.n = a.rows

    def __del__(self):
        if getattr(self, "h", None):
            self._free(self.h)
            self.h = None

    @property
    def levels(self):
        return lib().or_amg_levels(self.h)

    def level_info(self, d):
        r, z, hist = np.zeros(1, np.int64), np.zeros(1, np.int64), np.zeros(4, np.int64)
        lib().or_amg_level_info(self.h, d, _ptr(r), _ptr(z), _ptr(hist))
        return int(r[0]), int(z[0]), hist

    def stop_reason(self):
        return lib().or_amg_stop_reason(self.h).decode()

    def coarse_solver(self):
        return lib().or_amg_coarse_solver(self.h).decode()

    def map(self, d):
        n = self.level_info(d)[0]
        p = lib().or_amg_map(self.h, d)
        return np.ctypeslib.as_array(p, (n,)).copy() if p else None

    def matrix(self, d) -> Csr:
        s = lib().or_amg_matrix(self.h, d).contents
        n, m = s.rows, s.nnz
        return Csr(n, np.ctypeslib.as_array(s.offsets, (n + 1,)).copy(),
                   np.ctypeslib.as_array(s.indices, (max(m, 1),))[:m].copy(),
                   np.ctypeslib.as_array(s.values, (max(m, 1),))[:m].copy())

    def apply(self, rhs):
        rhs = np.ascontiguousarray(rhs, np.float64)
        x = np.zeros(self.n)
        visits = np.zeros(self.levels, np.int64)
        lib().or_amg_apply(self.h, _ptr(rhs), _ptr(x), _ptr(visits))
        return x, visits


STATUS = ["Converged", "MaxIterations", "Breakdown", "NonFinite"]


def _solve(fn, a, precond, b, x0, max_iterations, rtol, atol, refresh):
    b = np.ascontiguousarray(b, np.float64)
    x = np.array(x0, np.float64, copy=True)
    o = _SolverOptions(max_iterations, rtol, atol, refresh)
    r = fn(C.byref(_view(a)), precond.h if precond is not None else None, _ptr(b), _ptr(x), C.byref(o))
    return x, {"status": STATUS[r.status], "iterations": r.iterations, "residual_norm": r.residual_norm,
               "relative_residual": r.relative_residual}


def cg(a, precond, b, x0, max_iterations=1000, rtol=1e-8, atol=0.0, refresh=50):
    return _solve(lib().or_cg, a, precond, b, x0, max_iterations, rtol, atol, refresh)


def bicgstab(a, precond, b, x0, max_iterations=1000, rtol=1e-8, atol=0.0, refresh=50):
    return _solve(lib().or_bicgstab, a, precond, b, x0, max_iterations, rtol, atol, refresh)


def sample_matrix(n) -> Csr:
    out = _Csr()
    _check(lib().or_sample_matrix(n, C.byref(out)))
    return _take(out, lib().or_csr_free)


def mt19937(seed, count):
    out = np.zeros(count, np.uint32)
    lib().or_mt19937(seed, count, _ptr(out))
    return out


def num_threads():
    return lib().or_num_threads()


# --------------------------------------------------------------------------
# Oracle built from the reference sources (oracle/_ref): available where the reference
# sources were present at build time.
# --------------------------------------------------------------------------
_ref = None


def ref_available():
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        r = C.CDLL(REF_LIB)
        P, I, D = C.c_void_p, C.c_int, C.c_double
        pc = C.POINTER(_Csr)
        r.ref_canonical.argtypes = [I, P, P, P, pc]
        r.ref_strength.argtypes = [I, P, P, P, D, pc]
        r.ref_aggregate.argtypes = [I, P, P, P, I, I, P, P, P, P, P]
        r.ref_galerkin.argtypes = [I, P, P, P, P, I, P, P, pc]
        r.ref_read_matrix_market.argtypes = [C.c_char_p, pc]
        r.ref_csr_free.argtypes = [pc]
        r.ref_last_error.restype = C.c_char_p
        r.ref_std_mt19937.argtypes = [C.c_uint32, I, P]
        _ref = r
    return _ref


def _arrs(a: Csr):
    return (np.ascontiguousarray(a.offsets, np.int32), np.ascontiguousarray(a.indices, np.int32),
            np.ascontiguousarray(a.values, np.float64))


def _refcheck(status):
    if status != 0:
        raise OracleError(ref().ref_last_error().decode())


def ref_canonical(a: Csr) -> Csr:
    o, i, v = _arrs(a)
    out = _Csr()
    _refcheck(ref().ref_canonical(a.rows, _ptr(o), _ptr(i), _ptr(v), C.byref(out)))
    return _take(out, ref().ref_csr_free)


def ref_strength(a: Csr, theta) -> Csr:
    o, i, v = _arrs(a)
    out = _Csr()
    _refcheck(ref().ref_strength(a.rows, _ptr(o), _ptr(i), _ptr(v), theta, C.byref(out)))
    return _take(out, ref().ref_csr_free)


def ref_aggregate(g: Csr, rounds, absorb) -> Transfer:
    o, i, v = _arrs(g)
    n = g.rows
    mp, off, mem = np.zeros(n, np.int32), np.zeros(n + 1, np.int32), np.zeros(n, np.int32)
    cnt = C.c_int()
    hist = np.zeros(4, np.int64)
    _refcheck(ref().ref_aggregate(n, _ptr(o), _ptr(i), _ptr(v), rounds, int(absorb), _ptr(mp), _ptr(off),
                                  _ptr(mem), C.byref(cnt), _ptr(hist)))
    return Transfer(mp, off[:cnt.value + 1].copy(), mem, cnt.value, hist)


def ref_galerkin(a: Csr, t: Transfer) -> Csr:
    o, i, v = _arrs(a)
    out = _Csr()
    _refcheck(ref().ref_galerkin(a.rows, _ptr(o), _ptr(i), _ptr(v), _ptr(np.ascontiguousarray(t.map, np.int32)),
                                 t.coarse, _ptr(np.ascontiguousarray(t.offsets, np.int32)),
                                 _ptr(np.ascontiguousarray(t.members, np.int32)), C.byref(out)))
    return _take(out, ref().ref_csr_free)


def ref_read_matrix_market(text: str) -> Csr:
    out = _Csr()
    _refcheck(ref().ref_read_matrix_market(text.encode(), C.byref(out)))
    return _take(out, ref().ref_csr_free)


def ref_std_mt19937(seed, count):
    out = np.zeros(count, np.uint32)
    ref().ref_std_mt19937(seed, count, _ptr(out))
    return out


# ---- learned damping: a NumPy restatement of the row features and the MLP
# (thermofem_b200/csrc/mlp.cu), FP64 arithmetic on the BF16-rounded weights.

MLP_F, MLP_H = 4, 32
MLP_P = MLP_H * MLP_F + 2 * MLP_H + 1


def bf16_round(p):
    """float32 values rounded to BF16 (nearest, ties to even), as float32."""
    u = np.ascontiguousarray(p, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (u & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def mlp_features(off, idx, val, level):
    off = np.asarray(off, np.int64)
    n = len(off) - 1
    rows = np.repeat(np.arange(n), np.diff(off))
    val = np.asarray(val, np.float64)
    on = np.asarray(idx) == rows
    d = np.zeros(n)
    np.add.at(d, rows[on], val[on])
    offs = np.zeros(n)
    np.add.at(offs, rows[~on], np.abs(val[~on]))
    ad = np.abs(d)
    mean = ad.sum() / n
    f = np.zeros((n, MLP_F))
    ok = (ad > 0) & (mean > 0)
    f[ok, 0] = np.log(ad[ok] / mean)
    f[ad > 0, 1] = offs[ad > 0] / ad[ad > 0]
    f[:, 2] = np.diff(off) * 0.125
    f[:, 3] = level * 0.1
    return f.astype(np.float32)


def _mlp_parts(params):
    w = bf16_round(params).astype(np.float64)
    k = MLP_H * MLP_F
    return w[:k].reshape(MLP_H, MLP_F), w[k:k + MLP_H], w[k + MLP_H:k + 2 * MLP_H], w[-1]


def mlp_forward(params, x, lo, hi):
    W1, b1, w2, b2 = _mlp_parts(params)
    a = np.asarray(x, np.float64) @ W1.T + b1
    z = np.maximum(a, 0.0) @ w2 + b2
    return lo + (hi - lo) / (1.0 + np.exp(-z))


def mlp_gradient(params, x, target, lo, hi):
    """Sum over rows of the gradient of (omega - target)^2, and the loss sum."""
    W1, b1, w2, b2 = _mlp_parts(params)
    x = np.asarray(x, np.float64)
    a = x @ W1.T + b1
    h = np.maximum(a, 0.0)
    s = 1.0 / (1.0 + np.exp(-(h @ w2 + b2)))
    e = lo + (hi - lo) * s - np.asarray(target, np.float64)
    dz = 2.0 * e * (hi - lo) * s * (1.0 - s)
    dh = np.where(a > 0, dz[:, None] * w2[None, :], 0.0)
    g = np.concatenate([(dh.T @ x).ravel(), dh.sum(0), (dz[:, None] * h).sum(0), [dz.sum()]])
    return g, float((e * e).sum())


# --------------------------------------------------------------------------
# The reference's own GPU solve path (oracle/_ref/libref_gpu.so, built by
# `make -C oracle refgpu` from the reference sources): Cg / BiCgStab with its
# aggregation Amg in FP64 (ref_gpu_shim.cu).  A second oracle for the GPU tests.
# --------------------------------------------------------------------------
REF_GPU_LIB = os.path.join(HERE, "_ref", "libref_gpu.so")
_ref_gpu = None


def ref_gpu_available():
    return os.path.exists(REF_GPU_LIB)


def ref_gpu_solve(a: Csr, b, x0=None, kind="cg", cycle="v", jacobi_weight=2.0 / 3.0, coarse_rows=64, repeats=1,
                  precond="amg", single=False):
    """The reference's solve of a x = b (from x0, default zero) with its
    aggregation AMG (precond "amg") or its identity preconditioner, in FP64
    or (single) with its float components and their default tolerance.  Returns (x, report) with iterations, status (0 Converged,
    1 MaxIterations, 2 Breakdown, 3 NonFinite), relative_residual, setup_s
    and solve_s (the fastest of `repeats` solves, host clock around
    device-synchronised calls)."""
    global _ref_gpu
    if _ref_gpu is None:
        r = C.CDLL(REF_GPU_LIB)
        P, I, D = C.c_void_p, C.c_int, C.c_double
        r.ref_gpu_solve.argtypes = [I, P, P, P, C.c_int64, P, P, I, I, D, I, I, I, P, P, P, P, P]
        r.ref_gpu_solve.restype = I
        _ref_gpu = r
    rp, ci, val = _arrs(a)
    n = a.rows
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    it, st = np.zeros(1, np.int32), np.zeros(1, np.int32)
    rel, ts, tv = np.zeros(1), np.zeros(1), np.zeros(1)
    rc = _ref_gpu.ref_gpu_solve({"cg": 0, "bicgstab": 1}[kind], _ptr(rp), _ptr(ci), _ptr(val), n, _ptr(b), _ptr(x),
                                {"identity": 0, "amg": 1}[precond], {"v": 0, "w": 1, "f": 2}[cycle], float(jacobi_weight), int(coarse_rows),
                                int(repeats), int(bool(single)), _ptr(it), _ptr(st), _ptr(rel), _ptr(ts), _ptr(tv))
    if rc != 0:
        raise OracleError("reference GPU solve failed")
    return x, {"iterations": int(it[0]), "status": int(st[0]), "relative_residual": float(rel[0]),
               "setup_s": float(ts[0]), "solve_s": float(tv[0])}


def ref_gpu_amg_levels(a: Csr, jacobi_weight=2.0 / 3.0, coarse_rows=64):
    """The reference's own Amg<double> built on a (its GPU build): a list of
    (rows, nonzeros, histogram) per level, the stop reason and the coarse
    solver, as Amg::levelStatistics / stopReason / coarseSolver give them."""
    r = C.CDLL(REF_GPU_LIB)
    P, I, D = C.c_void_p, C.c_int, C.c_double
    r.ref_gpu_amg_levels.argtypes = [P, P, P, C.c_int64, D, I, I, P, P, P, C.c_char_p, C.c_char_p]
    r.ref_gpu_amg_levels.restype = I
    rp, ci, val = _arrs(a)
    cap = 32
    rows, nnz, hist = np.zeros(cap, np.int64), np.zeros(cap, np.int64), np.zeros(4 * cap, np.int64)
    stop, coarse = C.create_string_buffer(64), C.create_string_buffer(64)
    levels = r.ref_gpu_amg_levels(_ptr(rp), _ptr(ci), _ptr(val), a.rows, float(jacobi_weight), int(coarse_rows), cap,
                                  _ptr(rows), _ptr(nnz), _ptr(hist), stop, coarse)
    if levels < 0:
        raise OracleError("reference AMG setup failed")
    stats = [(int(rows[d]), int(nnz[d]), hist[4 * d:4 * d + 4].tolist()) for d in range(levels)]
    return stats, stop.value.decode(), coarse.value.decode()


def ref_gpu_solve_pair(a: Csr, b, jacobi_weight=2.0 / 3.0, coarse_rows=64, repeats=1, keep_x=False):
    """The reference's own FP64 PCG and BiCGStab with one shared AMG V-cycle
    setup (its GPU build).  Returns {"setup_s", "pcg": {...}, "bicgstab":
    {...}} with iterations, status (0 Converged), relative_residual, solve_s
    (fastest of `repeats`) and, with keep_x, x."""
    r = C.CDLL(REF_GPU_LIB)
    P, I, D = C.c_void_p, C.c_int, C.c_double
    r.ref_gpu_solve_pair.argtypes = [P, P, P, C.c_int64, P, D, I, I, P, P, P, P, P, P, P]
    r.ref_gpu_solve_pair.restype = I
    rp, ci, val = _arrs(a)
    n = a.rows
    b = np.ascontiguousarray(b, np.float64)
    setup = np.zeros(1)
    it, st = np.zeros(2, np.int32), np.zeros(2, np.int32)
    rel, ts = np.zeros(2), np.zeros(2)
    xs = [np.zeros(n), np.zeros(n)] if keep_x else [None, None]
    rc = r.ref_gpu_solve_pair(_ptr(rp), _ptr(ci), _ptr(val), n, _ptr(b), float(jacobi_weight), int(coarse_rows),
                              int(repeats), _ptr(setup), _ptr(it), _ptr(st), _ptr(rel), _ptr(ts),
                              _ptr(xs[0]) if keep_x else None, _ptr(xs[1]) if keep_x else None)
    if rc != 0:
        raise OracleError("reference GPU solve failed")
    out = {"setup_s": float(setup[0])}
    for k, name in enumerate(("pcg", "bicgstab")):
        out[name] = {"iterations": int(it[k]), "status": int(st[k]), "relative_residual": float(rel[k]),
                     "solve_s": float(ts[k])}
        if keep_x:
            out[name]["x"] = xs[k]
    return out
