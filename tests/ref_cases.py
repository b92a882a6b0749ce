"""Inputs on which the reference's own engine (src/mm.cu) computes C = A*B
correctly, shared by the reference-pin tests (CPU: oracle against the
reference; GPU: the engine against the reference).

The reference is exact only inside these limits, all from reading src/mm.cu:
  * values are small positive integers: its dense accumulator is int* and
    atomicAdd(int*, float) truncates each partial (:33, :386), and a column is
    emitted when the old accumulator value is within 1e-4 of zero (:387), which
    for positive sums happens exactly once, at the first touch;
  * every row of B has fewer than 128 entries: columns k with 128 or more B
    entries that are not "heavy" fall into no bin and are dropped (:211-221);
  * P < 2^31 (int offsets, :176-184) and every sum < 2^24 (exact in float);
  * B is square (cudaCOO2CM copies num_cols + 1 row pointers of B, :130).
"""
import numpy as np

from spgemm_b200 import workloads as W


def _int_values(M, seed):
    rng = np.random.default_rng(seed)
    return W.Csr(M.rows, M.cols, M.rowptr, M.col, rng.integers(1, 4, M.nnz).astype(np.float32))


def _truncate_rows(M, max_len):
    """Keep the first max_len entries of every row."""
    keep = np.zeros(M.nnz, bool)
    rp = M.rowptr.astype(np.int64)
    for i in range(M.rows):
        keep[rp[i]:min(rp[i + 1], rp[i] + max_len)] = True
    r = np.repeat(np.arange(M.rows), np.diff(rp))[keep]
    return W.from_coo(M.rows, M.cols, r, M.col[keep], M.val[keep])


def _with_empty(M, rows, cols):
    """Zero out the given rows and columns (pattern entries removed)."""
    r = np.repeat(np.arange(M.rows), np.diff(M.rowptr.astype(np.int64)))
    keep = ~np.isin(r, rows) & ~np.isin(M.col, cols)
    return W.from_coo(M.rows, M.cols, r[keep], M.col[keep], M.val[keep])


def cases():
    """name -> (A, B), A m x k, B k x k, integer values in {1, 2, 3}."""
    er = _int_values(W.er(4096, 8.0, 0), 1)
    st = _int_values(W.stencil27(8), 2)
    rm = _int_values(_truncate_rows(W.rmat(10, 8, 0), 127), 3)
    ra = _int_values(W.er(300, 6.0, 5, cols=200), 4)
    rb = _int_values(W.er(200, 6.0, 6), 5)
    em = _int_values(_with_empty(W.er(500, 5.0, 7), rows=np.arange(0, 500, 7),
                                 cols=np.arange(3, 500, 11)), 6)
    return {"er4096": (er, er), "stencil8": (st, st), "rmat10_trunc127": (rm, rm),
            "rect300x200": (ra, rb), "empty_rows_cols": (em, em)}


def triplets(M):
    r = np.repeat(np.arange(M.rows, dtype=np.int32), np.diff(M.rowptr.astype(np.int64)))
    return r, M.col.astype(np.int32), M.val.astype(np.float32)


def run_reference(A, B, tmp_path):
    """The reference's output, rows sorted by column: (rowptr int64, col, val, printed)."""
    import oracle
    ar, ac, av = triplets(A)
    br, bc, bv = triplets(B)
    r = oracle.ref_multiply(A.rows, A.cols, B.cols, ar, ac, av, br, bc, bv, tmp_path)
    cnt = r["cnt"].astype(np.int64)
    rowptr = np.concatenate([[0], np.cumsum(cnt)])
    col = np.empty(int(rowptr[-1]), np.int32)
    val = np.empty(int(rowptr[-1]), np.float32)
    for i in np.nonzero(cnt)[0]:
        b = int(r["base"][i])
        ci = r["idx"][b:b + cnt[i]]
        o = np.argsort(ci, kind="stable")
        col[rowptr[i]:rowptr[i + 1]] = ci[o]
        val[rowptr[i]:rowptr[i + 1]] = r["val"][b:b + cnt[i]][o]
    return rowptr, col, val, r
