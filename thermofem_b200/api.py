"""Typed Python wrappers over the C ABI: context, CSR views of torch tensors,
the kernel entry points and the component objects (Amg, Jacobi, Cg,
BiCgStab), named after the reference's C++ components."""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import (AmgOptions, Csr, HostCsr, SolveResult, SolverOptions, F32, F64, F32_VALUES, I32, I64, CYCLE, SOLVER_CG,
               SOLVER_BICGSTAB, PRECOND_AMG, PRECOND_IDENTITY, check, lib)

__all__ = ["Context", "DeviceCsr", "Transfer", "Amg", "Jacobi", "Cg", "BiCgStab", "Batch", "Mlp", "row_features", "MLP_PARAMS",
           "MLP_FEATURES", "MLP_HIDDEN", "amg_options", "solver_options",
           "read_matrix_market", "read_matrix_market_file", "read_matrix_market_stream", "spmv", "autotune_spmv", "set_spmv_config", "residual", "jacobi_sweep", "jacobi_zero",
           "inverse_diagonal", "restrict_aggregates", "prolong_aggregates", "dot_multi", "axpby", "convert",
           "csr_validate", "check_canonical", "canonicalize", "row_stats", "strength", "match", "contract",
           "aggregate", "galerkin", "radix_sort_pairs", "reduce_by_key", "scan_exclusive", "coarse_lu_factor",
           "coarse_lu_solve", "default_context"]

_VT = {torch.float32: F32, torch.float64: F64}
_IT = {torch.int32: I32, torch.int64: I64}


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _release(fn: str, handle):
    """Destroys a handle; at interpreter shutdown the library may already be gone."""
    try:
        getattr(lib(), fn)(handle)
    except Exception:  # module globals cleared during shutdown
        pass


class Context:
    """tf_ctx bound to a dedicated torch stream of one device.

    Calls order themselves after the work torch has queued on its current
    stream and make torch's current stream wait for them, so tensors can be
    used on either side without explicit synchronisation."""

    def __init__(self, device: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("thermofem_b200 needs a CUDA device (there is no CPU path)")
        self.device = device
        self.stream = torch.cuda.Stream(device=device)
        h = C.c_void_p()
        check(lib().tf_ctx_create(device, C.c_void_p(self.stream.cuda_stream), C.byref(h)))
        self.h = h

    def close(self, _release=_release):  # bound now: module globals are cleared at interpreter shutdown
        if getattr(self, "h", None):
            _release("tf_ctx_destroy", self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        return self

    def __exit__(self, *exc):
        torch.cuda.current_stream(self.device).wait_stream(self.stream)

    def synchronize(self):
        check(lib().tf_ctx_synchronize(self.h))

    @property
    def launches(self) -> int:
        return int(lib().tf_ctx_launch_count(self.h))


_default = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


class DeviceCsr:
    """CSR on the device as torch tensors (offsets, indices, values)."""

    def __init__(self, offsets, indices, values, cols=None):
        self.offsets, self.indices, self.values = offsets, indices, values
        self.rows = offsets.numel() - 1
        self.cols = self.rows if cols is None else cols

    @staticmethod
    def from_host(offsets, indices, values, device="cuda", dtype=torch.float64, index_dtype=torch.int32, cols=None):
        return DeviceCsr(torch.as_tensor(np.asarray(offsets), device=device).to(index_dtype),
                         torch.as_tensor(np.asarray(indices), device=device).to(index_dtype),
                         torch.as_tensor(np.asarray(values), device=device).to(dtype), cols)

    @property
    def nnz(self):
        return self.indices.numel()

    @property
    def dtype(self):
        return self.values.dtype

    def desc(self) -> Csr:
        return Csr(self.rows, self.cols, self.nnz, _IT[self.offsets.dtype], _VT[self.values.dtype],
                   self.offsets.data_ptr(), self.indices.data_ptr() if self.nnz else None,
                   self.values.data_ptr() if self.nnz else None)

    def to(self, dtype=None, index_dtype=None):
        return DeviceCsr(self.offsets.to(index_dtype or self.offsets.dtype),
                         self.indices.to(index_dtype or self.indices.dtype),
                         self.values.to(dtype or self.values.dtype), self.cols)

    def host(self):
        return (self.offsets.cpu().numpy(), self.indices.cpu().numpy(), self.values.cpu().numpy())


def _take_dcsr(ctx: Context, handle) -> DeviceCsr:
    """Copies a library-owned tf_dcsr into torch tensors and frees it."""
    v = Csr()
    check(lib().tf_dcsr_view(handle, C.byref(v)))
    dev = torch.device("cuda", ctx.device)
    off = torch.empty(v.rows + 1, dtype=torch.int32, device=dev)
    idx = torch.empty(v.nnz, dtype=torch.int32, device=dev)
    val = torch.empty(v.nnz, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    _memcpy(off, v.offsets, 4 * (v.rows + 1))
    if v.nnz:
        _memcpy(idx, v.indices, 4 * v.nnz)
        _memcpy(val, v.values, 8 * v.nnz)
    torch.cuda.synchronize(dev)
    check(lib().tf_dcsr_free(handle))
    return DeviceCsr(off, idx, val)


def _memcpy(dst: torch.Tensor, src_ptr: int, nbytes: int):
    """Device-to-device copy from a raw pointer into a tensor."""
    src = _RawDevice(src_ptr, nbytes, dst.device)
    dst.view(torch.uint8).copy_(src.tensor())


class _RawDevice:
    """Wraps a raw device pointer as a uint8 tensor (via __cuda_array_interface__)."""

    def __init__(self, ptr, nbytes, device):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3, "strides": None}
        self.device = device

    def tensor(self):
        return torch.as_tensor(self, device=self.device)


def _view_i32(ptr, n, device):
    if n == 0:
        return torch.empty(0, dtype=torch.int32, device=device)
    return torch.as_tensor(_RawDevice(ptr, 4 * n, device), device=device).view(torch.int32)


# ---------------------------------------------------------------------------
# kernels
# ---------------------------------------------------------------------------
def _ctx(ctx):
    return ctx if ctx is not None else default_context()


def spmv(a: DeviceCsr, x, y=None, ctx=None):
    ctx = _ctx(ctx)
    y = torch.empty(a.rows, dtype=a.dtype, device=x.device) if y is None else y
    d = a.desc()
    with ctx:
        check(lib().tf_spmv(ctx.h, C.byref(d), _p(x), _p(y)))
    return y


def autotune_spmv(a: DeviceCsr, x, y=None, ctx=None):
    """Times the pipelined SpMV shapes on this operator and caches the best;
    returns (stages, ctas_per_sm, cap_pct, rows_per_thread, ms_per_launch)."""
    ctx = _ctx(ctx)
    y = torch.empty(a.rows, dtype=a.dtype, device=x.device) if y is None else y
    d = a.desc()
    st, ct, cp, rpt, ms = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_float()
    with ctx:
        check(lib().tf_autotune_spmv(ctx.h, C.byref(d), _p(x), _p(y), C.byref(st), C.byref(ct), C.byref(cp),
                                     C.byref(rpt), C.byref(ms)))
    return st.value, ct.value, cp.value, rpt.value, ms.value


def set_spmv_config(a: DeviceCsr, stages: int, ctas_per_sm: int, cap_pct: int, rows_per_thread: int, ctx=None):
    """Caches a launch shape for operators of a's shape (no timing)."""
    ctx = _ctx(ctx)
    d = a.desc()
    check(lib().tf_spmv_set_config(ctx.h, C.byref(d), int(stages), int(ctas_per_sm), int(cap_pct),
                                   int(rows_per_thread)))


def residual(a: DeviceCsr, b, x, r=None, ctx=None):
    ctx = _ctx(ctx)
    r = torch.empty_like(b) if r is None else r
    d = a.desc()
    with ctx:
        check(lib().tf_residual(ctx.h, C.byref(d), _p(b), _p(x), _p(r)))
    return r


def jacobi_sweep(a: DeviceCsr, dinv, b, x, weight, row_weight=None, map=None, coarse=None, out=None, ctx=None):
    ctx = _ctx(ctx)
    out = torch.empty_like(x) if out is None else out
    d = a.desc()
    with ctx:
        check(lib().tf_jacobi_sweep(ctx.h, C.byref(d), _p(dinv), _p(b), _p(x), _p(out), float(weight),
                                    _p(row_weight), _p(map), _p(coarse)))
    return out


def jacobi_zero(dinv, b, weight, row_weight=None, out=None, ctx=None):
    ctx = _ctx(ctx)
    out = torch.empty_like(b) if out is None else out
    with ctx:
        check(lib().tf_jacobi_zero(ctx.h, b.numel(), _VT[b.dtype], _p(dinv), _p(b), _p(out), float(weight),
                                   _p(row_weight)))
    return out


def inverse_diagonal(a: DeviceCsr, ctx=None):
    ctx = _ctx(ctx)
    out = torch.empty(a.rows, dtype=a.dtype, device=a.values.device)
    d = a.desc()
    with ctx:
        check(lib().tf_inverse_diagonal(ctx.h, C.byref(d), _p(out)))
    return out


def restrict_aggregates(t: "Transfer", fine, coarse=None, ctx=None):
    ctx = _ctx(ctx)
    coarse = torch.empty(t.coarse_rows, dtype=fine.dtype, device=fine.device) if coarse is None else coarse
    with ctx:
        check(lib().tf_restrict(ctx.h, _VT[fine.dtype], t.coarse_rows, _p(t.offsets), _p(t.members), _p(fine),
                                _p(coarse)))
    return coarse


def prolong_aggregates(t: "Transfer", coarse, fine, ctx=None):
    ctx = _ctx(ctx)
    with ctx:
        check(lib().tf_prolong(ctx.h, _VT[fine.dtype], t.fine_rows, _p(t.map), _p(coarse), _p(fine)))
    return fine


def dot_multi(xs, ys, ctx=None):
    ctx = _ctx(ctx)
    k = len(xs)
    out = torch.empty(k, dtype=torch.float64, device=xs[0].device)
    px = (C.c_void_p * k)(*[t.data_ptr() for t in xs])
    py = (C.c_void_p * k)(*[t.data_ptr() for t in ys])
    with ctx:
        check(lib().tf_dot_multi(ctx.h, _VT[xs[0].dtype], xs[0].numel(), k, px, py, _p(out)))
    return out


def axpby(a, x, b, y, ctx=None):
    ctx = _ctx(ctx)
    with ctx:
        check(lib().tf_axpby(ctx.h, _VT[x.dtype], x.numel(), float(a), _p(x), float(b), _p(y)))
    return y


def convert(src, dtype, ctx=None):
    ctx = _ctx(ctx)
    out = torch.empty(src.numel(), dtype=dtype, device=src.device)
    tmap = {torch.float32: F32, torch.float64: F64, torch.int32: I32, torch.int64: I64}
    with ctx:
        check(lib().tf_convert(ctx.h, src.numel(), tmap[src.dtype], _p(src), tmap[dtype], _p(out)))
    return out


def csr_validate(a: DeviceCsr, ctx=None):
    ctx = _ctx(ctx)
    d = a.desc()
    with ctx:
        check(lib().tf_csr_validate(ctx.h, C.byref(d)))


def check_canonical(a: DeviceCsr, ctx=None) -> int:
    ctx = _ctx(ctx)
    d = a.desc()
    f = C.c_int()
    with ctx:
        check(lib().tf_csr_check_canonical(ctx.h, C.byref(d), C.byref(f)))
    return f.value


def canonicalize(a: DeviceCsr, ctx=None) -> DeviceCsr:
    ctx = _ctx(ctx)
    d = a.desc()
    h = C.c_void_p()
    with ctx:
        check(lib().tf_canonicalize(ctx.h, C.byref(d), C.byref(h)))
    return _take_dcsr(ctx, h)


def row_stats(a: DeviceCsr, ctx=None):
    ctx = _ctx(ctx)
    d = a.desc()
    out = torch.empty(a.rows, dtype=torch.float64, device=a.values.device)
    bad = C.c_int()
    with ctx:
        check(lib().tf_row_stats(ctx.h, C.byref(d), _p(out), C.byref(bad)))
    return out, bool(bad.value)


def strength(a: DeviceCsr, threshold: float, ctx=None) -> DeviceCsr:
    """Validates the level (as GpuAggregation::strength does) and builds the graph."""
    ctx = _ctx(ctx)
    mx, bad = row_stats(a, ctx)
    if bad:
        from . import InvalidArgument, ERR_INVALID
        raise InvalidArgument(ERR_INVALID, "Native AMG: missing/zero diagonal, non-finite value or reciprocal in hierarchy")
    d = a.desc()
    h = C.c_void_p()
    with ctx:
        check(lib().tf_strength(ctx.h, C.byref(d), _p(mx), float(threshold), C.byref(h)))
    return _take_dcsr(ctx, h)


def match(g: DeviceCsr, rounds: int, ctx=None):
    ctx = _ctx(ctx)
    d = g.desc()
    m = torch.empty(g.rows, dtype=torch.int32, device=g.values.device)
    cnt = C.c_int()
    with ctx:
        check(lib().tf_match(ctx.h, C.byref(d), rounds, _p(m), C.byref(cnt)))
    return m, cnt.value


def contract(g: DeviceCsr, map, count, ctx=None) -> DeviceCsr:
    ctx = _ctx(ctx)
    d = g.desc()
    h = C.c_void_p()
    with ctx:
        check(lib().tf_contract(ctx.h, C.byref(d), _p(map), int(count), C.byref(h)))
    return _take_dcsr(ctx, h)


@dataclass
class Transfer:
    """AggregateTransfer: map[fine], offsets[coarse+1], members[fine], histogram."""
    map: torch.Tensor
    offsets: torch.Tensor
    members: torch.Tensor
    fine_rows: int
    coarse_rows: int
    histogram: np.ndarray
    _handle: object = None

    def __del__(self, _release=_release):  # bound now: globals are cleared at shutdown
        if self._handle is not None:
            _release("tf_transfer_free", self._handle)
            self._handle = None


def aggregate(g: DeviceCsr, rounds: int, absorb: bool, ctx=None) -> Transfer:
    ctx = _ctx(ctx)
    d = g.desc()
    h = C.c_void_p()
    with ctx:
        check(lib().tf_aggregate(ctx.h, C.byref(d), int(rounds), int(absorb), C.byref(h)))
    fine, coarse = C.c_int(), C.c_int()
    hist = np.zeros(4, np.int32)
    check(lib().tf_transfer_info(h, C.byref(fine), C.byref(coarse), hist.ctypes.data_as(C.c_void_p)))
    pm, po, pe = C.c_void_p(), C.c_void_p(), C.c_void_p()
    check(lib().tf_transfer_arrays(h, C.byref(pm), C.byref(po), C.byref(pe)))
    dev = g.values.device
    return Transfer(_view_i32(pm.value, fine.value, dev).clone(), _view_i32(po.value, coarse.value + 1, dev).clone(),
                    _view_i32(pe.value, fine.value, dev).clone(), fine.value, coarse.value, hist, h)


def galerkin(a: DeviceCsr, t: Transfer, ctx=None) -> DeviceCsr:
    ctx = _ctx(ctx)
    d = a.desc()
    h = C.c_void_p()
    with ctx:
        check(lib().tf_galerkin(ctx.h, C.byref(d), t._handle, C.byref(h)))
    return _take_dcsr(ctx, h)


def radix_sort_pairs(keys, values, end_bit=64, ctx=None):
    ctx = _ctx(ctx)
    ko, vo = torch.empty_like(keys), torch.empty_like(values)
    with ctx:
        check(lib().tf_radix_sort_pairs_u64f64(ctx.h, keys.numel(), _p(keys), _p(values), _p(ko), _p(vo), end_bit))
    return ko, vo


def reduce_by_key(keys, values, op="sum", ctx=None):
    ctx = _ctx(ctx)
    ko, vo = torch.empty_like(keys), torch.empty_like(values)
    cnt = C.c_int64()
    with ctx:
        check(lib().tf_reduce_by_key_u64f64(ctx.h, keys.numel(), _p(keys), _p(values), 0 if op == "sum" else 1,
                                            _p(ko), _p(vo), C.byref(cnt)))
    return ko[:cnt.value], vo[:cnt.value]


def scan_exclusive(x, out=None, ctx=None):
    ctx = _ctx(ctx)
    out = torch.empty_like(x) if out is None else out
    with ctx:
        check(lib().tf_scan_exclusive_i32(ctx.h, x.numel(), _p(x), _p(out)))
    return out


def coarse_lu_factor(a: DeviceCsr, ctx=None):
    ctx = _ctx(ctx)
    n = a.rows
    lu = torch.empty(n * n, dtype=torch.float64, device=a.values.device)
    piv = torch.empty(n, dtype=torch.int32, device=a.values.device)
    ok = C.c_int()
    d = a.desc()
    with ctx:
        check(lib().tf_coarse_lu_factor(ctx.h, C.byref(d), _p(lu), _p(piv), C.byref(ok)))
    return bool(ok.value), lu, piv


def coarse_lu_solve(lu, piv, b, x=None, ctx=None):
    ctx = _ctx(ctx)
    x = torch.empty_like(b) if x is None else x
    with ctx:
        check(lib().tf_coarse_lu_solve(ctx.h, piv.numel(), _p(lu), _p(piv), _VT[b.dtype], _p(b), _p(x)))
    return x


# ---------------------------------------------------------------------------
# components
# ---------------------------------------------------------------------------
def amg_options(**kw) -> AmgOptions:
    o = AmgOptions()
    lib().tf_amg_options_default(C.byref(o))
    for k, v in kw.items():
        if k == "cycle" and isinstance(v, str):
            v = CYCLE[v.lower()]
        if k == "damping_model":
            o._damping_model_ref = v  # the model must live until the options are used
            v = v.h.value if v is not None else None
        if k == "hierarchy_type" and not isinstance(v, int):
            v = {torch.float32: F32, torch.float64: F64, "f32": F32, "f64": F64, "f32v": F32_VALUES, None: -1}[v]
        if not hasattr(o, k):
            raise TypeError(f"unknown AMG option {k}")
        setattr(o, k, v)
    return o


def solver_options(dtype=torch.float64, **kw) -> SolverOptions:
    o = SolverOptions()
    lib().tf_solver_options_default(_VT[dtype], C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown solver option {k}")
        setattr(o, k, v)
    return o


# tf_*_spmv_layout codes
LAYOUTS = ("csr", "sliced", "sorted", "banded", "csr32")


class _AmgView:
    """Read access to a hierarchy (statistics, level operators, transfers)."""

    def _h(self):
        raise NotImplementedError

    def level_count(self) -> int:
        return lib().tf_amg_level_count(self._h())

    def level_statistics(self):
        out = []
        for d in range(self.level_count()):
            r, z = C.c_int64(), C.c_int64()
            hist = np.zeros(4, np.int32)
            check(lib().tf_amg_level_stats(self._h(), d, C.byref(r), C.byref(z), hist.ctypes.data_as(C.c_void_p)))
            out.append({"rows": r.value, "nonzeros": z.value, "aggregate_sizes": hist.tolist()})
        return out

    def setup_phases(self):
        """{phase name: ms} of the last setup (CUDA events on the context stream)."""
        k = lib().tf_amg_setup_phase_count()
        ms = np.zeros(k, np.float64)
        check(lib().tf_amg_setup_phases(self._h(), ms.ctypes.data_as(C.c_void_p), k))
        return {lib().tf_amg_setup_phase_name(i).decode(): float(ms[i]) for i in range(k)}

    def stop_reason(self) -> str:
        return lib().tf_amg_stop_reason(self._h()).decode()

    def coarse_solver(self) -> str:
        return lib().tf_amg_coarse_solver(self._h()).decode()

    def last_cycle_visits(self):
        n = self.level_count()
        v = np.zeros(n, np.int64)
        check(lib().tf_amg_last_visits(self._h(), v.ctypes.data_as(C.c_void_p), n))
        return v.tolist()

    def level_matrix(self, d, device="cuda"):
        c = Csr()
        check(lib().tf_amg_level_matrix(self._h(), d, C.byref(c)))
        dev = torch.device(device)
        off = _view_i32(c.offsets, c.rows + 1, dev).clone()
        idx = _view_i32(c.indices, c.nnz, dev).clone()
        es = 8 if c.value_type == F64 else 4
        raw = torch.as_tensor(_RawDevice(c.values, es * c.nnz, dev), device=dev) if c.nnz else None
        dt = torch.float64 if c.value_type == F64 else torch.float32
        val = raw.view(dt).clone() if raw is not None else torch.empty(0, dtype=dt, device=dev)
        return DeviceCsr(off, idx, val)

    def level_spmv(self, d, x, y=None):
        """y = A_d x with level d's operator as the cycle streams it (x, y of
        the hierarchy's storage type)."""
        y = torch.empty_like(x) if y is None else y
        ctx = getattr(self, "ctx", None) or default_context()
        with ctx:
            check(lib().tf_amg_level_spmv(self._h(), int(d), _p(x), _p(y)))
        return y

    def level_spmv_layout(self, d):
        """(layout, entries streamed) of level d's SpMV: "sliced", "sorted",
        "banded", "csr" (2-byte column offsets) or "csr32" (4-byte columns)."""
        sl, n = C.c_int(), C.c_int64()
        check(lib().tf_amg_level_spmv_layout(self._h(), int(d), C.byref(sl), C.byref(n)))
        return LAYOUTS[sl.value], n.value

    def level_transfer(self, d, device="cuda"):
        pm, po, pe = C.c_void_p(), C.c_void_p(), C.c_void_p()
        cr = C.c_int()
        check(lib().tf_amg_level_transfer(self._h(), d, C.byref(pm), C.byref(po), C.byref(pe), C.byref(cr)))
        st = self.level_statistics()[d]
        dev = torch.device(device)
        n = st["rows"]
        return (_view_i32(pm.value, n, dev).clone(), _view_i32(po.value, cr.value + 1, dev).clone(),
                _view_i32(pe.value, n, dev).clone(), cr.value)

    def coarse_factor(self, device="cuda"):
        """(lu as rows x rows FP64, pivots) of the coarse LU, None for a
        Jacobi coarse solve (CoarseFactor, GpuAggregation.cuh:19-25)."""
        rows, plu, ppiv = C.c_int(), C.c_void_p(), C.c_void_p()
        check(lib().tf_amg_coarse_factor(self._h(), C.byref(rows), C.byref(plu), C.byref(ppiv)))
        n = rows.value
        if n == 0:
            return None
        dev = torch.device(device)
        lu = _view_i32(plu.value, 2 * n * n, dev).view(torch.float64).clone().view(n, n)
        return lu, _view_i32(ppiv.value, n, dev).clone()


class Amg(_AmgView):
    """Aggregation AMG preconditioner (Amg<T,I>): setup(matrix), apply(rhs, x)."""

    def __init__(self, options: AmgOptions | None = None, dtype=torch.float64, index_dtype=torch.int32, ctx=None,
                 **kw):
        self.ctx = _ctx(ctx)
        self.options = options if options is not None else amg_options(**kw)
        self.dtype = dtype
        h = C.c_void_p()
        check(lib().tf_amg_create(self.ctx.h, _VT[dtype], _IT[index_dtype], C.byref(self.options), C.byref(h)))
        self.h = h

    def _h(self):
        return self.h

    def __del__(self, _release=_release):  # bound now: globals are cleared at shutdown
        if getattr(self, "h", None):
            _release("tf_amg_destroy", self.h)
            self.h = None

    def setup(self, a: DeviceCsr):
        d = a.desc()
        with self.ctx:
            check(lib().tf_amg_setup(self.h, C.byref(d)))

    def apply(self, rhs, x=None):
        x = torch.empty_like(rhs) if x is None else x
        with self.ctx:
            check(lib().tf_amg_apply(self.h, _p(rhs), _p(x)))
        return x

    def save(self, path):
        """Writes the built hierarchy to `path` (tf_amg_save)."""
        with self.ctx:
            check(lib().tf_amg_save(self.h, os.fsencode(path)))

    def load(self, path):
        """Restores a hierarchy written by save() into this component, which
        must have the same types and smoothing (tf_amg_load)."""
        with self.ctx:
            check(lib().tf_amg_load(self.h, os.fsencode(path)))


class Jacobi:
    """Weighted Jacobi smoother (Jacobi<T,I>(sweeps, weight))."""

    def __init__(self, sweeps=2, weight=2.0 / 3.0, dtype=torch.float64, index_dtype=torch.int32, ctx=None):
        self.ctx = _ctx(ctx)
        h = C.c_void_p()
        check(lib().tf_jacobi_create(self.ctx.h, _VT[dtype], _IT[index_dtype], int(sweeps), float(weight),
                                     C.byref(h)))
        self.h = h

    def __del__(self, _release=_release):  # bound now: globals are cleared at shutdown
        if getattr(self, "h", None):
            _release("tf_jacobi_destroy", self.h)
            self.h = None

    def setup(self, a: DeviceCsr):
        d = a.desc()
        with self.ctx:
            check(lib().tf_jacobi_setup(self.h, C.byref(d)))

    def apply(self, rhs, x):
        with self.ctx:
            check(lib().tf_jacobi_apply(self.h, _p(rhs), _p(x)))
        return x


class _Solver(_AmgView):
    KIND = SOLVER_CG

    def __init__(self, options: SolverOptions | None = None, preconditioner="amg", amg: AmgOptions | None = None,
                 dtype=torch.float64, index_dtype=torch.int32, ctx=None):
        self.ctx = _ctx(ctx)
        self.options = options if options is not None else solver_options(dtype)
        pre = PRECOND_AMG if preconditioner == "amg" else PRECOND_IDENTITY
        self.amg_options = amg if amg is not None else amg_options()
        h = C.c_void_p()
        check(lib().tf_solver_create(self.ctx.h, self.KIND, _VT[dtype], _IT[index_dtype], C.byref(self.options), pre,
                                     C.byref(self.amg_options), C.byref(h)))
        self.h = h

    def _h(self):
        p = lib().tf_solver_amg(self.h)
        if not p:
            raise ValueError("solver has no AMG preconditioner")
        return p

    def __del__(self, _release=_release):  # bound now: globals are cleared at shutdown
        if getattr(self, "h", None):
            _release("tf_solver_destroy", self.h)
            self.h = None

    def setup(self, a: DeviceCsr):
        d = a.desc()
        with self.ctx:
            check(lib().tf_solver_setup(self.h, C.byref(d)))

    def apply(self, rhs, x):
        """Solves A x = rhs from the initial guess in x (device or host tensors)."""
        res = SolveResult()
        host = not rhs.is_cuda
        if host:
            check(lib().tf_solver_apply(self.h, C.c_void_p(rhs.data_ptr()), C.c_void_p(x.data_ptr()), 1,
                                        C.byref(res)))
        else:
            with self.ctx:
                check(lib().tf_solver_apply(self.h, _p(rhs), _p(x), 0, C.byref(res)))
        return res.as_dict()

    @property
    def last_apply_ms(self) -> float:
        return lib().tf_solver_last_apply_ms(self.h)

    def set_graph_mode(self, mode: int):
        """1: one graph per solve with a device-side loop (default); 0: one
        graph per iteration and a host loop (for kernel profilers)."""
        check(lib().tf_solver_set_graph_mode(self.h, int(mode)))

    def spmv(self, x, y=None):
        """y = A x with the solver's own operator (as its iterations stream it)."""
        y = torch.empty_like(x) if y is None else y
        with self.ctx:
            check(lib().tf_solver_spmv(self.h, _p(x), _p(y)))
        return y

    def spmv_layout(self):
        """(layout, entries streamed) of the solver's operator SpMV, as
        level_spmv_layout names them."""
        sl, n = C.c_int(), C.c_int64()
        check(lib().tf_solver_spmv_layout(self.h, C.byref(sl), C.byref(n)))
        return LAYOUTS[sl.value], n.value

    @property
    def last_execution(self) -> int:
        """2: the last apply ran as one graph; 1: a graph per iteration;
        0: uncaptured launches; -1: no apply yet."""
        return lib().tf_solver_last_execution(self.h)


class Cg(_Solver):
    """Preconditioned CG (Cg<T,I>); preconditioner 'amg' or 'identity'."""
    KIND = SOLVER_CG


class BiCgStab(_Solver):
    """Right-preconditioned BiCGStab (BiCgStab<T,I>)."""
    KIND = SOLVER_BICGSTAB


def _take_host(h: HostCsr):
    n, m = h.rows, h.nnz
    off = np.ctypeslib.as_array(h.offsets, (n + 1,)).copy() if h.offsets else np.zeros(n + 1, np.int32)
    idx = np.ctypeslib.as_array(h.indices, (max(m, 1),))[:m].copy() if m else np.zeros(0, np.int32)
    val = np.ctypeslib.as_array(h.values, (max(m, 1),))[:m].copy() if m else np.zeros(0, np.float64)
    out = {"rows": n, "cols": h.cols, "offsets": off, "indices": idx, "values": val}
    lib().tf_host_csr_free(C.byref(h))
    return out


def read_matrix_market(text: str):
    """io::readMatrixMarket over a text buffer (host; no GPU needed)."""
    b = text.encode()
    h = HostCsr()
    check(lib().tf_read_matrix_market(b, len(b), C.byref(h)))
    return _take_host(h)


def read_matrix_market_file(path: str):
    h = HostCsr()
    check(lib().tf_read_matrix_market_file(path.encode(), C.byref(h)))
    return _take_host(h)


def read_matrix_market_stream(stream):
    """io::readMatrixMarket over a binary file-like object, read in blocks
    through tf_read_matrix_market_stream."""
    from . import MM_READ

    def read(_user, buf, capacity):
        try:
            data = stream.read(capacity)
        except OSError:
            return C.c_size_t(-1).value
        C.memmove(buf, data, len(data))
        return len(data)

    fn = MM_READ(read)
    h = HostCsr()
    check(lib().tf_read_matrix_market_stream(fn, None, C.byref(h)))
    return _take_host(h)


class Batch:
    """Independent set-up solvers (sharing one Context) solved together: one
    CUDA graph launch per apply, the systems' solves as concurrent branches
    (tf_batch_*).  apply(rhs_list, x_list) -> list of reports."""

    def __init__(self, solvers, ctx=None):
        self.ctx = _ctx(ctx)
        self.solvers = list(solvers)  # keep them alive as long as the batch
        arr = (C.c_void_p * len(self.solvers))(*[s.h.value for s in self.solvers])
        h = C.c_void_p()
        check(lib().tf_batch_create(self.ctx.h, len(self.solvers), arr, C.byref(h)))
        self.h = h

    def __del__(self, _release=_release):  # bound now: globals are cleared at shutdown
        if getattr(self, "h", None):
            _release("tf_batch_destroy", self.h)
            self.h = None

    def apply(self, rhs, xs):
        n = len(self.solvers)
        if len(rhs) != n or len(xs) != n:
            raise ValueError("one rhs and one x per solver")
        r = (C.c_void_p * n)(*[t.data_ptr() for t in rhs])
        x = (C.c_void_p * n)(*[t.data_ptr() for t in xs])
        res = (SolveResult * n)()
        with self.ctx:
            check(lib().tf_batch_apply(self.h, r, x, res))
        return [res[k].as_dict() for k in range(n)]


MLP_FEATURES, MLP_HIDDEN = 4, 32
MLP_PARAMS = MLP_HIDDEN * MLP_FEATURES + 2 * MLP_HIDDEN + 1


class Mlp:
    """Learned per-row Jacobi damping (tf_mlp_*): 4 row features -> 32 ReLU
    units -> omega in [omega_min, omega_max]; BF16 weights, FP32 master
    copy, trained with the library's forward/backward/SGD kernels."""

    def __init__(self, seed=0, omega_min=0.3, omega_max=1.2, ctx=None, params=None):
        self.ctx = _ctx(ctx)
        h = C.c_void_p()
        check(lib().tf_mlp_create(self.ctx.h, int(seed), float(omega_min), float(omega_max), C.byref(h)))
        self.h = h
        self.omega_min, self.omega_max = float(omega_min), float(omega_max)
        if params is not None:
            self.set_params(params)

    def __del__(self, _release=_release):  # bound now: globals are cleared at shutdown
        if getattr(self, "h", None):
            _release("tf_mlp_destroy", self.h)
            self.h = None

    def params(self) -> np.ndarray:
        p = np.zeros(MLP_PARAMS, np.float32)
        check(lib().tf_mlp_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != MLP_PARAMS:
            raise ValueError(f"expected {MLP_PARAMS} parameters")
        check(lib().tf_mlp_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def forward(self, features):
        out = torch.empty(features.shape[0], dtype=torch.float32, device=features.device)
        with self.ctx:
            check(lib().tf_mlp_forward(self.h, features.shape[0], _p(features), _p(out)))
        return out

    def backward(self, features, target) -> float:
        loss = C.c_double()
        with self.ctx:
            check(lib().tf_mlp_backward(self.h, features.shape[0], _p(features), _p(target), C.byref(loss)))
        return loss.value

    def gradient(self) -> np.ndarray:
        g = np.zeros(MLP_PARAMS, np.float64)
        check(lib().tf_mlp_get_gradient(self.h, g.ctypes.data_as(C.POINTER(C.c_double))))
        return g

    def sgd(self, lr, momentum=0.9):
        with self.ctx:
            check(lib().tf_mlp_sgd(self.h, float(lr), float(momentum)))


def row_features(a: DeviceCsr, level=0, ctx=None):
    """n x 4 row features of a level operator (tf_row_features)."""
    ctx = _ctx(ctx)
    out = torch.empty((a.rows, MLP_FEATURES), dtype=torch.float32, device=a.values.device)
    d = a.desc()
    with ctx:
        check(lib().tf_row_features(ctx.h, C.byref(d), int(level), _p(out)))
    return out
