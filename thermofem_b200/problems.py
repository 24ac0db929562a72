"""Seeded synthetic heat-conduction problems (host CSR, numpy).

The reference ships no matrices (its data/ folder is empty by design), so the
workloads are generated: every random number comes from a counter-based
splitmix64 stream, u = (splitmix64(seed, i) >> 11) * 2^-53, normals by
Box-Muller, so a problem is a pure function of (size, seed) on any machine.

  laplace2d(m)          2-D 5-point Laplacian on an m x m interior grid,
                        homogeneous Dirichlet boundary eliminated, h = 1/(m+1).
  heat3d(m, seed)       3-D 7-point cell-centred finite volumes on m^3 cells,
                        h = 1/m, log-normal conductivity k = exp(N(0,1)) per
                        cell, harmonic-mean face coefficients 2 k_i k_j/(k_i+k_j),
                        Dirichlet T=0 on the face x=0 (half-cell coefficient
                        2 k_i/h^2), Neumann elsewhere.
  convdiff3d(m, seed)   7-point diffusion (k=1) plus first-order upwind
                        convection with a seeded unit velocity direction and a
                        cell Peclet number uniform in [1,10]; Robin (h=10) on
                        the faces x=0 and x=1, Neumann elsewhere.  Nonsymmetric.
  poisson1d(n)          tridiagonal [-1, 2, -1].
  rhs_uniform(n, seed)  right-hand side uniform in [-1, 1].
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    z = x + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def uniform(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """n uniforms in [0, 1) of stream `stream` of `seed`."""
    with np.errstate(over="ignore"):
        base = _splitmix64(np.array([seed * 0x100000001B3 + stream], dtype=np.uint64))[0]
        i = np.arange(n, dtype=np.uint64) + base
        return (_splitmix64(i) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, n: int, stream: int = 0) -> np.ndarray:
    u1 = 1.0 - uniform(seed, n, 2 * stream + 1)  # (0, 1]
    u2 = uniform(seed, n, 2 * stream + 2)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def rhs_uniform(n: int, seed: int) -> np.ndarray:
    return 2.0 * uniform(seed, n, 1000) - 1.0


def _csr_from_stencil(cols: np.ndarray, vals: np.ndarray, mask: np.ndarray):
    """Rows of at most S candidate entries (already column-sorted) -> CSR."""
    counts = mask.sum(axis=1).astype(np.int64)
    offsets = np.zeros(cols.shape[0] + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    return (offsets.astype(np.int32), cols[mask].astype(np.int32), vals[mask].astype(np.float64))


def poisson1d(n: int):
    i = np.arange(n)
    cols = np.stack([i - 1, i, i + 1], axis=1)
    vals = np.stack([-np.ones(n), 2 * np.ones(n), -np.ones(n)], axis=1)
    mask = (cols >= 0) & (cols < n)
    return _csr_from_stencil(cols, vals, mask)


def laplace2d(m: int):
    n = m * m
    h2 = 1.0 / float(m + 1) ** 2
    i = np.arange(n)
    ix, iy = i % m, i // m
    cols = np.stack([i - m, i - 1, i, i + 1, i + m], axis=1)
    mask = np.stack([iy > 0, ix > 0, np.ones(n, bool), ix < m - 1, iy < m - 1], axis=1)
    off = -1.0 / h2
    vals = np.stack([np.full(n, off), np.full(n, off), np.full(n, 4.0 / h2), np.full(n, off), np.full(n, off)], axis=1)
    return _csr_from_stencil(cols, vals, mask)


def _grid3(m):
    n = m * m * m
    i = np.arange(n, dtype=np.int64)
    return n, i, i % m, (i // m) % m, i // (m * m)


def heat3d(m: int, seed: int = 1001):
    n, i, ix, iy, iz = _grid3(m)
    h2 = 1.0 / float(m) ** 2
    k = np.exp(normal(seed, n))
    mm = m * m
    steps = [-mm, -m, -1, 1, m, mm]
    valid = [iz > 0, iy > 0, ix > 0, ix < m - 1, iy < m - 1, iz < m - 1]
    cols = np.empty((n, 7), np.int64)
    vals = np.empty((n, 7), np.float64)
    mask = np.empty((n, 7), bool)
    diag = np.zeros(n)
    slot = [0, 1, 2, 4, 5, 6]
    for s, step, ok in zip(slot, steps, valid):
        j = np.where(ok, i + step, i)
        kf = 2.0 * k * k[j] / (k + k[j]) / h2
        kf = np.where(ok, kf, 0.0)
        cols[:, s] = j
        vals[:, s] = -kf
        mask[:, s] = ok
        diag += kf
    diag += np.where(ix == 0, 2.0 * k / h2, 0.0)  # Dirichlet T=0 on x=0
    cols[:, 3] = i
    vals[:, 3] = diag
    mask[:, 3] = True
    return _csr_from_stencil(cols, vals, mask)


def convdiff3d(m: int, seed: int = 1003, robin_h: float = 10.0):
    n, i, ix, iy, iz = _grid3(m)
    h = 1.0 / float(m)
    u = uniform(seed, 3, 7)
    z = 2.0 * u[0] - 1.0
    phi = 2.0 * np.pi * u[1]
    r = np.sqrt(max(0.0, 1.0 - z * z))
    vel_dir = np.array([r * np.cos(phi), r * np.sin(phi), z])
    peclet = 1.0 + 9.0 * u[2]
    speed = peclet * 2.0 / h  # cell Peclet = |v| h / (2 k) with k = 1
    v = speed * vel_dir      # (vx, vy, vz)
    mm = m * m
    d = 1.0 / (h * h)
    steps = [-mm, -m, -1, 1, m, mm]
    valid = [iz > 0, iy > 0, ix > 0, ix < m - 1, iy < m - 1, iz < m - 1]
    comp = [2, 1, 0, 0, 1, 2]
    sign = [-1, -1, -1, 1, 1, 1]
    cols = np.empty((n, 7), np.int64)
    vals = np.empty((n, 7), np.float64)
    mask = np.empty((n, 7), bool)
    diag = np.zeros(n)
    slot = [0, 1, 2, 4, 5, 6]
    for s, step, ok, c, sg in zip(slot, steps, valid, comp, sign):
        j = np.where(ok, i + step, i)
        vn = sg * v[c]  # outward normal velocity on this face
        # first-order upwind: outflow adds vn/h to the diagonal, inflow couples -|vn|/h to the neighbour
        out_coef = max(vn, 0.0) / h
        in_coef = max(-vn, 0.0) / h
        cols[:, s] = j
        vals[:, s] = np.where(ok, -d - in_coef, 0.0)
        mask[:, s] = ok
        diag += np.where(ok, d + out_coef, 0.0)
    # Robin (convective) boundary h (T - 0) on x=0 and x=1: half-cell coupling
    robin = 1.0 / (h / 2.0 + 1.0 / robin_h) / h
    diag += np.where(ix == 0, robin, 0.0) + np.where(ix == m - 1, robin, 0.0)
    cols[:, 3] = i
    vals[:, 3] = diag
    mask[:, 3] = True
    return _csr_from_stencil(cols, vals, mask)


def manufactured_solution(n: int) -> np.ndarray:
    """x_i = 1 + 0.25 sin(0.013 i) + 0.125 cos(0.007 i), the solve driver's
    manufactured solution."""
    i = np.arange(n, dtype=np.float64)
    return 1.0 + 0.25 * np.sin(i * 0.013) + 0.125 * np.cos(i * 0.007)


def write_matrix_market(path: str, offsets, indices, values, symmetric: bool = False) -> None:
    """Writes a CSR matrix as Matrix Market coordinate real text (1-based;
    with symmetric=True only the lower triangle, as `general` otherwise) --
    the synthetic stand-in for the reference's real `.mtx` inputs."""
    offsets = np.asarray(offsets)
    indices = np.asarray(indices)
    values = np.asarray(values, dtype=np.float64)
    n = len(offsets) - 1
    rows = np.repeat(np.arange(n), np.diff(offsets))
    keep = indices <= rows if symmetric else np.ones(len(indices), bool)
    r, c, v = rows[keep] + 1, indices[keep] + 1, values[keep]
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {'symmetric' if symmetric else 'general'}\n")
        f.write(f"{n} {n} {len(v)}\n")
        for a, b, x in zip(r.tolist(), c.tolist(), v.tolist()):
            f.write(f"{a} {b} {x!r}\n")


def transient3d(m: int, r: float):
    """Backward-Euler step operator of 3-D heat conduction on m^3 cells,
    scaled by 1/(k h): A = (1/r) I + K7, K7 the 7-point stencil (6 on the
    diagonal, -1 per interior neighbour; Dirichlet walls), r = dt k / h^2."""
    n, i, ix, iy, iz = _grid3(m)
    mm = m * m
    steps = [-mm, -m, -1, 1, m, mm]
    valid = [iz > 0, iy > 0, ix > 0, ix < m - 1, iy < m - 1, iz < m - 1]
    cols = np.empty((n, 7), np.int64)
    vals = np.empty((n, 7), np.float64)
    mask = np.empty((n, 7), bool)
    for s, step, ok in zip([0, 1, 2, 4, 5, 6], steps, valid):
        cols[:, s] = np.where(ok, i + step, i)
        vals[:, s] = -1.0
        mask[:, s] = ok
    cols[:, 3] = i
    vals[:, 3] = 6.0 + 1.0 / r
    mask[:, 3] = True
    return _csr_from_stencil(cols, vals, mask)


def batched_transient_params(count: int = 48, seed: int = 1004, side_min: int = 16, side_max: int = 96):
    """(side m, r = dt k / h^2) of each problem of the batched transient
    workload: m uniform in [side_min, side_max], r uniform in [0.1, 10]
    (problem k uses streams of seed + k)."""
    out = []
    for k in range(count):
        u = uniform(seed + k, 2, 7)
        m = side_min + min(int(u[0] * (side_max - side_min + 1)), side_max - side_min)
        out.append((m, 0.1 + 9.9 * float(u[1])))
    return out


def transient3d_nnz(m: int) -> int:
    """Nonzeros of transient3d(m, r): the diagonal plus two per interior
    face of the m^3 grid."""
    return m ** 3 + 6 * m * m * (m - 1)


def batched_transient(count: int = 48, seed: int = 1004, side_min: int = 16, side_max: int = 96, only=None):
    """The batched transient workload: the problems of
    batched_transient_params with initial temperatures uniform in [0, 1].
    Returns [(m, r, (offsets, indices, values), T0)]; with `only` (problem
    indices) just those problems, in that order."""
    params = batched_transient_params(count, seed, side_min, side_max)
    out = []
    for k in (range(count) if only is None else only):
        m, r = params[k]
        out.append((m, r, transient3d(m, r), uniform(seed + k, m * m * m, 8)))
    return out
