"""Seeded synthetic inputs for the SpGEMM configurations.

The reference benchmarks on SuiteSparse/SNAP matrices (``bin/launch.sh``) that
are not available here; these generators stand in for them with the shapes,
sizes and value distributions of the five configurations:

* ``er``         Erdos-Renyi pattern (each entry present with probability d/n,
                 columns drawn without replacement per row), values U[-1, 1];
* ``rmat``       R-MAT graph adjacency (level-wise quadrant sampler with
                 probabilities a, b, c, d), duplicates removed, values U(0, 1];
* ``stencil27``  27-point stencil on an s^3 grid (entries to every neighbour
                 inside the grid) with random-sign, log-uniform magnitudes, or
                 the classic 26/-1 operator;
* ``prolongator``  piecewise-constant prolongator over 2x2x2 aggregates;
* ``batch``      independent (A_i, B_i) pairs with log-uniform sizes and
                 Poisson row lengths, half ER and half R-MAT.

All matrices are returned as CSR: (rowptr int32, col int32, val float32) with
columns sorted inside each row, in a small ``Csr`` container.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Csr:
    rows: int
    cols: int
    rowptr: np.ndarray  # int32 [rows + 1]
    col: np.ndarray     # int32 [nnz]
    val: np.ndarray     # float32 [nnz]

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def to_csc(self) -> "Csc":
        """Column-major copy (stable: rows ascending inside each column)."""
        r = np.repeat(np.arange(self.rows, dtype=np.int64), np.diff(self.rowptr))
        order = np.argsort(self.col, kind="stable")
        colptr = np.zeros(self.cols + 1, np.int64)
        np.add.at(colptr, self.col.astype(np.int64) + 1, 1)
        colptr = np.cumsum(colptr)
        return Csc(self.rows, self.cols, colptr.astype(np.int32), r[order].astype(np.int32),
                   self.val[order].astype(np.float32))

    def transpose(self) -> "Csr":
        c = self.to_csc()
        return Csr(self.cols, self.rows, c.colptr, c.rowidx, c.val)


@dataclass
class Csc:
    rows: int
    cols: int
    colptr: np.ndarray  # int32 [cols + 1]
    rowidx: np.ndarray  # int32 [nnz]
    val: np.ndarray     # float32 [nnz]

    @property
    def nnz(self) -> int:
        return int(self.colptr[-1])


def from_coo(rows: int, cols: int, r: np.ndarray, c: np.ndarray, v: np.ndarray) -> Csr:
    """CSR from coordinate arrays (duplicates must already be removed)."""
    r = np.asarray(r, np.int64)
    c = np.asarray(c, np.int64)
    v = np.asarray(v, np.float32)
    key = r * cols + c
    if len(key) > 1 and not bool(np.all(key[1:] >= key[:-1])):
        order = np.lexsort((c, r))
        r, c, v = r[order], c[order], v[order]
    rowptr = np.zeros(rows + 1, np.int64)
    rowptr[1:] = np.cumsum(np.bincount(r, minlength=rows)[:rows])
    return Csr(rows, cols, rowptr.astype(np.int32), c.astype(np.int32), v)


def _unique_keys(keys: np.ndarray) -> np.ndarray:
    """Sorted distinct values (np.unique's result, by sorting)."""
    keys = np.sort(keys)
    if len(keys) < 2:
        return keys
    return keys[np.concatenate(([True], keys[1:] != keys[:-1]))]


def _rows_without_replacement(rng, n_rows: int, n_cols: int, deg: np.ndarray) -> tuple:
    """Per row i, deg[i] distinct columns drawn uniformly from [0, n_cols)."""
    deg = np.minimum(deg.astype(np.int64), n_cols)
    keys = np.empty(0, np.int64)
    need = deg.copy()
    for _ in range(64):
        tot = int(need.sum())
        if tot == 0:
            break
        r = np.repeat(np.arange(n_rows, dtype=np.int64), need)
        c = rng.integers(0, n_cols, size=tot, dtype=np.int64)
        keys = _unique_keys(np.concatenate([keys, r * n_cols + c]))
        have = np.bincount(keys // n_cols, minlength=n_rows)
        need = np.maximum(deg - have, 0)
    return keys // n_cols, keys % n_cols


def er(n: int, avg_deg: float, seed: int, cols: int | None = None, low=-1.0, high=1.0) -> Csr:
    """Erdos-Renyi: row i holds Binomial(cols, avg_deg/cols) distinct columns."""
    rng = np.random.default_rng(seed)
    cols = n if cols is None else cols
    deg = rng.binomial(cols, min(avg_deg / cols, 1.0), size=n)
    r, c = _rows_without_replacement(rng, n, cols, deg)
    v = rng.uniform(low, high, size=len(r)).astype(np.float32)
    return from_coo(n, cols, r, c, v)


def er_poisson(n: int, lam: float, seed: int, low=-1.0, high=1.0) -> Csr:
    """Row lengths Poisson(lam), columns uniform without replacement."""
    rng = np.random.default_rng(seed)
    deg = rng.poisson(lam, size=n)
    r, c = _rows_without_replacement(rng, n, n, deg)
    v = rng.uniform(low, high, size=len(r)).astype(np.float32)
    return from_coo(n, n, r, c, v)


def _rmat_edges(rng, scale: int, m: int, a: float, b: float, c: float):
    r = np.zeros(m, np.int64)
    cc = np.zeros(m, np.int64)
    for lvl in range(scale):
        u = rng.random(m)
        rb = (u >= a + b).astype(np.int64)
        cb = (((u >= a) & (u < a + b)) | (u >= a + b + c)).astype(np.int64)
        bit = scale - 1 - lvl
        r |= rb << bit
        cc |= cb << bit
    return r, cc


def rmat(scale: int, edge_factor: float, seed: int, a=0.57, b=0.19, c=0.19,
         n: int | None = None, values: str = "unit_open") -> Csr:
    """R-MAT adjacency with 2^scale vertices (or the first n < 2^scale, by
    rejection) and edge_factor * n sampled edges, duplicates removed.
    values: "unit_open" -> U(0, 1]; "sym" -> U[-1, 1]."""
    rng = np.random.default_rng(seed)
    nv = 1 << scale
    n = nv if n is None else n
    target = int(round(edge_factor * n))
    rs, cs = [], []
    got = 0
    while got < target:
        want = target - got if n == nv else int((target - got) * (nv * nv) / (n * n) * 1.05) + 16
        r, cc = _rmat_edges(rng, scale, want, a, b, c)
        keep = (r < n) & (cc < n)
        r, cc = r[keep], cc[keep]
        if got + len(r) > target:
            r, cc = r[: target - got], cc[: target - got]
        rs.append(r)
        cs.append(cc)
        got += len(r)
    r = np.concatenate(rs)
    cc = np.concatenate(cs)
    keys = _unique_keys(r * n + cc)
    r, cc = keys // n, keys % n
    if values == "unit_open":
        v = (1.0 - rng.random(len(r))).astype(np.float32)
    else:
        v = rng.uniform(-1.0, 1.0, size=len(r)).astype(np.float32)
    return from_coo(n, n, r, cc, v)


def stencil27(s: int, seed: int = 0, values: str = "loguniform") -> Csr:
    """27-point stencil on an s x s x s grid (row-major index x + s*(y + s*z)).
    values: "loguniform" -> random sign, |v| log-uniform in [1e-4, 1e4];
            "laplace"    -> 26 on the diagonal, -1 off it."""
    rng = np.random.default_rng(seed)
    n = s ** 3
    idx = np.arange(n, dtype=np.int64)
    x, y, z = idx % s, (idx // s) % s, idx // (s * s)
    rs, cs = [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ok = ((x + dx >= 0) & (x + dx < s) & (y + dy >= 0) & (y + dy < s) &
                      (z + dz >= 0) & (z + dz < s))
                rs.append(idx[ok])
                cs.append(idx[ok] + dx + s * (dy + s * dz))
    r = np.concatenate(rs)
    c = np.concatenate(cs)
    if values == "laplace":
        v = np.where(r == c, 26.0, -1.0).astype(np.float32)
    else:
        mag = 10.0 ** rng.uniform(-4.0, 4.0, size=len(r))
        sign = np.where(rng.random(len(r)) < 0.5, -1.0, 1.0)
        v = (mag * sign).astype(np.float32)
    return from_coo(n, n, r, c, v)


def prolongator(s: int) -> Csr:
    """Piecewise-constant prolongator of an s^3 grid onto (s/2)^3 aggregates of
    2x2x2 points: one entry of value 1 per fine row."""
    assert s % 2 == 0
    n = s ** 3
    h = s // 2
    idx = np.arange(n, dtype=np.int64)
    x, y, z = idx % s, (idx // s) % s, idx // (s * s)
    agg = (x // 2) + h * ((y // 2) + h * (z // 2))
    return Csr(n, h ** 3, np.arange(n + 1, dtype=np.int32), agg.astype(np.int32),
               np.ones(n, np.float32))


@dataclass
class BatchItem:
    kind: str
    n: int
    lam: float
    seed: int
    A: Csr
    B: Csr


def batch_specs(count: int, seed: int, n_lo=1000, n_hi=200000, lam_lo=4.0, lam_hi=32.0):
    """(kind, n, lam, seed) of each instance: n log-uniform, lam uniform,
    even instances ER and odd instances R-MAT, per-instance seed = seed + i."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), size=count)).astype(np.int64)
    lams = rng.uniform(lam_lo, lam_hi, size=count)
    return [("er" if i % 2 == 0 else "rmat", int(ns[i]), float(lams[i]), seed + i)
            for i in range(count)]


def _rmat_columns(rng, size: int, n: int, col_bit_p: float) -> np.ndarray:
    """`size` columns in [0, n) from the R-MAT column marginal: each of the
    ceil(log2 n) bits is 1 with probability col_bit_p (b + d of the R-MAT
    quadrant probabilities), values >= n redrawn."""
    scale = max(int(np.ceil(np.log2(max(n, 2)))), 1)
    out = np.empty(size, np.int64)
    todo = np.arange(size)
    while len(todo):
        c = np.zeros(len(todo), np.int64)
        for bit in range(scale - 1, -1, -1):
            c |= (rng.random(len(todo)) < col_bit_p).astype(np.int64) << bit
        ok = c < n
        out[todo[ok]] = c[ok]
        todo = todo[~ok]
    return out


def rmat_poisson(n: int, lam: float, seed: int, b=0.19, d=0.05, low=-1.0, high=1.0) -> Csr:
    """Row lengths Poisson(lam) (at most n), columns distinct within a row and
    drawn from the R-MAT column marginal (bit probability b + d): the R-MAT
    pattern's skewed column popularity with bounded rows."""
    rng = np.random.default_rng(seed)
    deg = np.minimum(rng.poisson(lam, size=n).astype(np.int64), n)
    keys = np.empty(0, np.int64)
    need = deg.copy()
    for _ in range(64):
        tot = int(need.sum())
        if tot == 0:
            break
        r = np.repeat(np.arange(n, dtype=np.int64), need)
        c = _rmat_columns(rng, tot, n, b + d)
        keys = _unique_keys(np.concatenate([keys, r * n + c]))
        have = np.bincount(keys // n, minlength=n)
        need = np.maximum(deg - have, 0)
    r, c = keys // n, keys % n
    v = rng.uniform(low, high, size=len(r)).astype(np.float32)
    return from_coo(n, n, r, c, v)


def batch_item(kind: str, n: int, lam: float, seed: int) -> BatchItem:
    """One product of the batch: A and B n x n, Poisson(lam) entries per row,
    columns uniform ("er") or from the R-MAT column marginal ("rmat"),
    values U[-1, 1]; independent patterns for A and B."""
    if kind == "er":
        A = er_poisson(n, lam, seed * 2 + 0)
        B = er_poisson(n, lam, seed * 2 + 1)
    else:
        A = rmat_poisson(n, lam, seed * 2 + 0)
        B = rmat_poisson(n, lam, seed * 2 + 1)
    return BatchItem(kind, n, lam, seed, A, B)


def batch(count: int = 512, seed: int = 1000, **kw):
    return [batch_item(*spec) for spec in batch_specs(count, seed, **kw)]
