"""The FP64 oracle and the FP32 CPU baseline against hand-computed products,
scipy.sparse and the committed golden fixtures (CPU only)."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from spgemm_b200 import workloads as W


def run_oracle(A: W.Csr, B: W.Csr, **kw):
    a = A.to_csc()
    return oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val,
                         stats=True, **kw)


def dense_to_csr(D):
    D = np.asarray(D, np.float32)
    r, c = np.nonzero(D)
    return W.from_coo(D.shape[0], D.shape[1], r, c, D[r, c])


def csr_with_explicit(rows, cols, entries):
    r = [e[0] for e in entries]
    c = [e[1] for e in entries]
    v = [e[2] for e in entries]
    return W.from_coo(rows, cols, np.array(r, np.int64), np.array(c, np.int64), np.array(v, np.float32))


def test_kat_small_square():
    A = dense_to_csr([[1, 2, 0], [0, 0, 0], [3, 0, -1]])
    B = dense_to_csr([[1, 0, 2], [0, 5, 0], [4, 0, -6]])
    C = run_oracle(A, B)
    assert C["rowptr"].tolist() == [0, 3, 3, 5]
    assert C["col"].tolist() == [0, 1, 2, 0, 2]
    assert C["val"].tolist() == [1.0, 10.0, 2.0, -1.0, 12.0]
    assert C["nterms"].tolist() == [1, 1, 1, 2, 2]
    assert C["products"] == 7


def test_kat_cancellation_keeps_explicit_zero():
    # row 0: col 0 gets 1*2 + 1*(-2) = 0 and stays in the structure
    A = csr_with_explicit(1, 2, [(0, 0, 1.0), (0, 1, 1.0)])
    B = csr_with_explicit(2, 2, [(0, 0, 2.0), (0, 1, 3.0), (1, 0, -2.0)])
    C = run_oracle(A, B)
    assert C["rowptr"].tolist() == [0, 2]
    assert C["col"].tolist() == [0, 1]
    assert C["val"].tolist() == [0.0, 3.0]
    assert C["absum"].tolist() == [4.0, 3.0]


def test_kat_explicit_zero_input_entry():
    # a stored zero in A still produces (zero) products, so the entries exist
    A = csr_with_explicit(2, 2, [(0, 0, 0.0), (1, 1, 2.0)])
    B = csr_with_explicit(2, 3, [(0, 1, 5.0), (0, 2, 1.0), (1, 0, 1.5)])
    C = run_oracle(A, B)
    assert C["rowptr"].tolist() == [0, 2, 3]
    assert C["col"].tolist() == [1, 2, 0]
    assert C["val"].tolist() == [0.0, 0.0, 3.0]


def test_kat_rectangular():
    A = dense_to_csr([[1, 0, 2], [0, 3, 0]])            # 2 x 3
    B = dense_to_csr([[1, 1, 0, 0], [0, 0, 0, 2], [0, 4, 0, 1]])  # 3 x 4
    C = run_oracle(A, B)
    D = np.array([[1, 0, 2], [0, 3, 0]], np.float64) @ np.array([[1, 1, 0, 0], [0, 0, 0, 2], [0, 4, 0, 1]], np.float64)
    assert C["rowptr"].tolist() == [0, 3, 4]
    assert C["col"].tolist() == [0, 1, 3, 3]
    assert C["val"].tolist() == [D[0, 0], D[0, 1], D[0, 3], D[1, 3]]


def test_empty_operands():
    A = W.Csr(0, 3, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    B = dense_to_csr(np.eye(3))
    C = run_oracle(A, B)
    assert C["rowptr"].tolist() == [0] and len(C["col"]) == 0
    A = W.Csr(4, 3, np.zeros(5, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    C = run_oracle(A, B)
    assert C["rowptr"].tolist() == [0, 0, 0, 0, 0] and C["products"] == 0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_matches_scipy(seed):
    A = W.er(300, 6.0, seed)
    B = W.er(300, 6.0, seed + 100)
    C = run_oracle(A, B)
    sA = sp.csr_matrix((A.val, A.col, A.rowptr), shape=(A.rows, A.cols)).astype(np.float64)
    sB = sp.csr_matrix((B.val, B.col, B.rowptr), shape=(B.rows, B.cols)).astype(np.float64)
    # structure: the pattern product (all-positive values never cancel)
    pat = (abs(sA) @ abs(sB)).tocsr()
    pat.sort_indices()
    assert C["rowptr"].tolist() == pat.indptr.tolist()
    assert C["col"].tolist() == pat.indices.tolist()
    # values: scipy's product on the same pattern
    ref = (sA @ sB).toarray()
    r = np.repeat(np.arange(A.rows), np.diff(C["rowptr"]))
    np.testing.assert_allclose(C["val"], ref[r, C["col"]], rtol=1e-12, atol=1e-12)


def test_row_subset_matches_full():
    A = W.rmat(10, 8, 3)
    full = run_oracle(A, A)
    rows = np.array([5, 0, 700, 1023, 17], np.int32)
    sub = run_oracle(A, A, rows=rows)
    for t, i in enumerate(rows):
        a, b = full["rowptr"][i], full["rowptr"][i + 1]
        c, d = sub["rowptr"][t], sub["rowptr"][t + 1]
        assert full["col"][a:b].tolist() == sub["col"][c:d].tolist()
        assert full["val"][a:b].tolist() == sub["val"][c:d].tolist()


def test_threads_do_not_change_result():
    A = W.rmat(11, 8, 4)
    one = run_oracle(A, A, threads=1)
    many = run_oracle(A, A, threads=7)
    for k in ("rowptr", "col", "val", "absum", "nterms"):
        assert np.array_equal(one[k], many[k]), k


def test_fp32_baseline_close_to_fp64():
    A = W.er(500, 8.0, 5)
    ref = run_oracle(A, A)
    a = A.to_csc()
    b32 = oracle.spgemm(A.rows, A.cols, a.colptr, a.rowidx, a.val, A.rowptr, A.col, A.val, mode=1)
    assert np.array_equal(b32["rowptr"], ref["rowptr"]) and np.array_equal(b32["col"], ref["col"])
    from helpers import plain_tolerance
    assert (np.abs(b32["val"].astype(np.float64) - ref["val"]) <= plain_tolerance(ref)).all()


def test_count_products_matches_numpy():
    A = W.rmat(12, 16, 0)
    a = A.to_csc()
    P, per_row = oracle.count_products(A.rows, a.colptr, a.rowidx, A.rowptr, per_row=True)
    deg = np.diff(A.rowptr).astype(np.int64)
    want = np.zeros(A.rows, np.int64)
    np.add.at(want, np.repeat(np.arange(A.rows), np.diff(A.rowptr)), deg[A.col])
    assert P == int(want.sum())
    assert np.array_equal(per_row, want)
