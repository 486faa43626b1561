"""Synthetic workloads of the spectrum-slicing path (host-side generators).

Dirichlet Laplacians on nx x ny x nz grids: 5-point (2-D, diagonal 4) or
7-point (3-D, diagonal 6) stencils with off-diagonals -1, x fastest, rows
sorted by column -- the matrices the reference's Laplacian drivers build
(TESTS/COMMON/lapl.c:13-65) -- and their analytic spectrum
4 (sin^2(i pi/(2(nx+1))) + sin^2(j pi/(2(ny+1))) + sin^2(k pi/(2(nz+1)))).
"""
from __future__ import annotations

import numpy as np


def laplacian_csr(nx: int, ny: int, nz: int):
    """(ia, ja, a) of the Dirichlet Laplacian, int32 indices, float64 values."""
    n = nx * ny * nz
    idx = np.arange(n, dtype=np.int64)
    k = idx // (nx * ny)
    i = (idx - k * nx * ny) // nx
    j = idx - k * nx * ny - i * nx
    # neighbour offsets in increasing column order: -nx*ny, -nx, -1, 0, +1, +nx, +nx*ny
    offs = [(-nx * ny, k > 0), (-nx, i > 0), (-1, j > 0), (0, None), (1, j < nx - 1), (nx, i < ny - 1),
            (nx * ny, k < nz - 1)]
    diag = 6.0 if nz > 1 else 4.0
    counts = np.ones(n, dtype=np.int64)
    for off, mask in offs:
        if mask is not None:
            counts += mask
    ia = np.zeros(n + 1, dtype=np.int64)
    ia[1:] = np.cumsum(counts)
    ja = np.empty(ia[-1], dtype=np.int32)
    a = np.empty(ia[-1], dtype=np.float64)
    pos = ia[:-1].copy()
    for off, mask in offs:
        rows = idx if mask is None else idx[mask]
        p = pos[rows]
        ja[p] = (rows + off).astype(np.int32)
        a[p] = diag if off == 0 else -1.0
        pos[rows] += 1
    return ia.astype(np.int32), ja, a


def laplacian_eigenvalues(nx: int, ny: int, nz: int) -> np.ndarray:
    """All eigenvalues of the Dirichlet Laplacian, ascending."""
    tx = np.sin(np.arange(1, nx + 1) * (0.5 * np.pi / (nx + 1.0))) ** 2
    ty = np.sin(np.arange(1, ny + 1) * (0.5 * np.pi / (ny + 1.0))) ** 2
    tz = np.sin(np.arange(1, nz + 1) * (0.5 * np.pi / (nz + 1.0))) ** 2 if nz > 1 else np.zeros(1)
    ev = 4.0 * (tx[:, None, None] + ty[None, :, None] + tz[None, None, :])
    return np.sort(ev.ravel())


def count_in(ev: np.ndarray, a: float, b: float) -> int:
    """Eigenvalues in [a, b] with the reference's 10*DBL_EPSILON slack."""
    s = 10 * np.finfo(np.float64).eps
    return int(np.count_nonzero((ev >= a - s) & (ev <= b + s)))


def gap_interval(ev: np.ndarray, lo: float, count: int):
    """An interval holding exactly `count` distinct-position eigenvalues
    starting at the first eigenvalue above `lo`, with both end points at the
    midpoints of the gaps around it (so counts are robust to rounding)."""
    i0 = int(np.searchsorted(ev, lo))
    i1 = i0 + count
    # move the ends off clusters of equal eigenvalues
    while i1 < len(ev) and ev[i1] - ev[i1 - 1] < 1e-10:
        i1 += 1
    a = 0.5 * (ev[i0 - 1] + ev[i0]) if i0 > 0 else ev[0] - 1e-3
    b = 0.5 * (ev[i1 - 1] + ev[i1]) if i1 < len(ev) else ev[-1] + 1e-3
    return float(a), float(b), i1 - i0


def random_spd_csr(n: int, offdiag: int = 16, seed: int = 0):
    """Random sparse symmetric positive definite matrix: each row draws
    `offdiag` column indices uniformly (seeded), values U(-1, 1); the matrix
    is symmetrised as (M + M^T)/2 and each diagonal entry set to the row's
    absolute off-diagonal sum plus U(0, 1) (strict diagonal dominance).
    Returns (ia, ja, a) with sorted rows and duplicates summed (in the order
    of the stable sort of (row, column) keys)."""
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n, dtype=np.int64), offdiag)
    cols = rng.integers(0, n, size=n * offdiag, dtype=np.int64)
    vals = rng.uniform(-1.0, 1.0, size=n * offdiag)
    keep = rows != cols
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    key = np.concatenate([rows * n + cols, cols * n + rows])
    v = np.concatenate([vals, vals]) * 0.5
    del rows, cols, vals
    order = np.argsort(key, kind="stable")
    key, v = key[order], v[order]
    del order
    if np.any(key[1:] == key[:-1]):
        start = np.flatnonzero(np.concatenate([[True], key[1:] != key[:-1]]))
        v = np.add.reduceat(v, start)
        key = key[start]
    r = key // n
    c = key - r * n
    diag = np.bincount(r, weights=np.abs(v), minlength=n) + rng.uniform(0.0, 1.0, size=n)
    # the diagonal entry goes between the row's columns below and above it
    pos = np.searchsorted(key, np.arange(n, dtype=np.int64) * (n + 1))
    c = np.insert(c, pos, np.arange(n, dtype=np.int64))
    v = np.insert(v, pos, diag)
    ia = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=n) + 1, out=ia[1:])
    return ia.astype(np.int32), c.astype(np.int32), v


def gershgorin_bounds(ia, ja, a):
    """[min(d_i - r_i), max(d_i + r_i)] over the rows (contains the spectrum)."""
    n = len(ia) - 1
    rows = np.repeat(np.arange(n), np.diff(ia))
    on = rows == ja
    diag = np.bincount(rows[on], weights=a[on], minlength=n)
    absum = np.bincount(rows[~on], weights=np.abs(a[~on]), minlength=n)
    return float(np.min(diag - absum)), float(np.max(diag + absum))
