"""Row sharding of one product over ranks (one GPU per rank).

Rows of C are independent: rank r computes C[r0:r1, :] = A[r0:r1, :] * B with
B replicated, so the only exchange is an optional gather of the result. The
row ranges are balanced by intermediate products (P_i = sum over A(i,k) of
nnz(B(k,:))), not by row count, because power-law inputs concentrate the work
in few rows.

`shard_multiply` takes the per-rank compute as a callable, so the same
partition / gather logic runs with the GPU engine on GPU ranks and with any
other product routine elsewhere.
"""
from __future__ import annotations

from typing import Callable

import numpy as np

from .workloads import Csr


def row_products(A: Csr, B: Csr) -> np.ndarray:
    """P_i of every row of C = A*B (int64)."""
    deg_b = np.diff(B.rowptr).astype(np.int64)
    rows_of = np.repeat(np.arange(A.rows), np.diff(A.rowptr))
    p = np.zeros(A.rows, np.int64)
    np.add.at(p, rows_of, deg_b[A.col])
    return p


def partition_rows(work: np.ndarray, parts: int) -> list[tuple[int, int]]:
    """Split rows [0, len(work)) into `parts` contiguous ranges of nearly
    equal total work (each row also counts 1, so empty rows spread too)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    w = np.asarray(work, np.float64) + 1.0
    csum = np.concatenate([[0.0], np.cumsum(w)])
    total = csum[-1]
    cuts = [0]
    for r in range(1, parts):
        cuts.append(int(np.searchsorted(csum, total * r / parts, side="left")))
    cuts.append(len(work))
    cuts = np.maximum.accumulate(np.clip(cuts, 0, len(work)))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(parts)]


def row_slice(A: Csr, r0: int, r1: int) -> Csr:
    """Rows [r0, r1) of a CSR matrix (same column count)."""
    s, e = int(A.rowptr[r0]), int(A.rowptr[r1])
    return Csr(r1 - r0, A.cols, (A.rowptr[r0:r1 + 1] - s).astype(np.int32), A.col[s:e], A.val[s:e])


def concat_rows(parts: list[Csr]) -> Csr:
    """Stack row blocks (in order) into one CSR matrix."""
    cols = parts[0].cols
    rowptr = [np.zeros(1, np.int64)]
    off = 0
    for p in parts:
        rowptr.append(p.rowptr[1:].astype(np.int64) + off)
        off += p.nnz
    return Csr(sum(p.rows for p in parts), cols, np.concatenate(rowptr).astype(np.int32),
               np.concatenate([p.col for p in parts]), np.concatenate([p.val for p in parts]))


def shard_multiply(A: Csr, B: Csr, rank: int, world: int,
                   compute: Callable[[Csr, Csr], Csr], group=None, gather: bool = True):
    """This rank's block of C = A*B, and (gather=True) the whole C on every
    rank via torch.distributed all_gather_object on `group` (any backend)."""
    ranges = partition_rows(row_products(A, B), world)
    r0, r1 = ranges[rank]
    local = compute(row_slice(A, r0, r1), B)
    if not gather or world == 1:
        return local, (r0, r1)
    import torch.distributed as dist
    blocks = [None] * world
    dist.all_gather_object(blocks, (r0, r1, local.rowptr, local.col, local.val), group=group)
    parts = [Csr(b[1] - b[0], B.cols, b[2], b[3], b[4]) for b in blocks]
    return concat_rows(parts), (r0, r1)
