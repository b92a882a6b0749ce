"""Full-size configurations on the GPU (through the C ABI, device-resident
inputs), every entry of C compared with the FP64 oracle:

* R-MAT 2^18 ef16 A*A, plain FP32: all 262,144 rows, the oracle streamed over
  row chunks so that host memory stays bounded;
* the 27-point 96^3 stencil A*A (random sign, log-uniform |v| in [1e-4, 1e4]),
  plain FP32 and compensated;
* the Galerkin triple product P^T A P at 64^3 (two chained products; A with
  26/-1 values and with the log-uniform values above), each product against
  the oracle of its own inputs, and the chain against the FP64 chain.

Each test records the maximum relative error against the oracle
(helpers.rel_error_report) as a test property and prints it."""
import numpy as np
import pytest

import oracle
import spgemm_b200 as sg
from spgemm_b200 import workloads as W
from helpers import (assert_structure_equal, assert_values_close, compensated_tolerance,
                     plain_tolerance, rel_error_report)

pytestmark = pytest.mark.gpu


def device_product(A, B, precision, a_csc=True):
    import torch
    d = lambda a, t: torch.from_numpy(np.ascontiguousarray(a)).cuda().to(t)
    if a_csc:
        Ac = A.to_csc()
        tA = [d(Ac.colptr, torch.int32), d(Ac.rowidx, torch.int32), d(Ac.val, torch.float32)]
        Acm = sg.device_cm(tA[0].data_ptr(), tA[1].data_ptr(), tA[2].data_ptr(), A.nnz, A.rows,
                           A.cols, sg.COL_MAJOR)
    else:
        tA = [d(A.rowptr, torch.int32), d(A.col, torch.int32), d(A.val, torch.float32)]
        Acm = sg.device_cm(tA[0].data_ptr(), tA[1].data_ptr(), tA[2].data_ptr(), A.nnz, A.rows,
                           A.cols, sg.ROW_MAJOR)
    tB = [d(B.rowptr, torch.int32), d(B.col, torch.int32), d(B.val, torch.float32)]
    Bcm = sg.device_cm(tB[0].data_ptr(), tB[1].data_ptr(), tB[2].data_ptr(), B.nnz, B.rows, B.cols, sg.ROW_MAJOR)
    h = sg.Handle(precision)
    h.set_stream(torch.cuda.current_stream().cuda_stream)
    nnz = h.symbolic(Acm, Bcm)
    rp = torch.empty(A.rows + 1, dtype=torch.int32, device="cuda")
    col = torch.empty(max(nnz, 1), dtype=torch.int32, device="cuda")
    val = torch.empty(max(nnz, 1), dtype=torch.float32, device="cuda")
    h.numeric(rp.data_ptr(), col.data_ptr(), val.data_ptr())
    torch.cuda.synchronize()
    stats = h.stats()
    h.close()
    return rp, col[:nnz], val[:nnz], stats


def merge_reports(reps):
    worst = max(reps, key=lambda r: r["max_rel"])
    return {"max_rel": worst["max_rel"], "worst_cond": worst["worst_cond"],
            "zero_entries": int(sum(r["zero_entries"] for r in reps))}


def test_rmat18_all_rows(record_property):
    A = W.rmat(18, 16, 0)
    rp, col, val, stats = device_product(A, A, sg.PLAIN)
    rp_h = rp.cpu().numpy().astype(np.int64)
    a = A.to_csc()
    P, p_i = oracle.count_products(A.rows, a.colptr, a.rowidx, A.rowptr, per_row=True)
    assert stats["intermediate_products"] == P
    assert stats["nnz_c"] == rp_h[-1]
    # row chunks of about 16M entries of C (host memory of one chunk ~0.5 GB)
    bounds = [0]
    while bounds[-1] < A.rows:
        lo = bounds[-1]
        hi = int(np.searchsorted(rp_h, rp_h[lo] + 16_000_000, side="right")) - 1
        bounds.append(min(max(hi, lo + 1), A.rows))
    reps = []
    for lo, hi in zip(bounds[:-1], bounds[1:]):
        rows = np.arange(lo, hi, dtype=np.int32)
        ref = oracle.spgemm(A.rows, A.cols, a.colptr, a.rowidx, a.val, A.rowptr, A.col, A.val,
                            rows=rows, stats=True)
        s, e = int(rp_h[lo]), int(rp_h[hi])
        got_rp = rp_h[lo:hi + 1] - s
        gc = col[s:e].cpu().numpy()
        gv = val[s:e].cpu().numpy()
        assert_structure_equal(got_rp, gc, ref["rowptr"], ref["col"])
        assert_values_close(gv, ref, plain_tolerance(ref))
        reps.append(rel_error_report(gv, ref))
    rep = merge_reports(reps)
    record_property("rmat18_plain", rep)
    print("rmat18 plain:", rep)


@pytest.mark.parametrize("precision", [sg.PLAIN, sg.COMPENSATED])
def test_stencil96_full(precision, record_property):
    A = W.stencil27(96, seed=0)
    rp, col, val, stats = device_product(A, A, precision)
    a = A.to_csc()
    ref = oracle.spgemm(A.rows, A.cols, a.colptr, a.rowidx, a.val, A.rowptr, A.col, A.val, stats=True)
    assert stats["intermediate_products"] == ref["products"]
    assert_structure_equal(rp.cpu().numpy(), col.cpu().numpy(), ref["rowptr"], ref["col"])
    v = val.cpu().numpy()
    tol = plain_tolerance(ref) if precision == sg.PLAIN else compensated_tolerance(ref)
    assert_values_close(v, ref, tol)
    rep = rel_error_report(v, ref)
    name = "plain" if precision == sg.PLAIN else "compensated"
    record_property(f"stencil96_{name}", rep)
    print(f"stencil96 {name}:", rep)
    if precision == sg.COMPENSATED:
        assert rep["max_rel"] <= 1e-6, rep


def _host(rp, col, val, rows, cols):
    return W.Csr(rows, cols, rp.cpu().numpy(), col.cpu().numpy(), val.cpu().numpy())


@pytest.mark.parametrize("precision,values", [(sg.COMPENSATED, "laplace"),
                                              (sg.COMPENSATED, "loguniform"),
                                              (sg.PLAIN, "loguniform")])
def test_galerkin64_chain(precision, values, record_property):
    A = W.stencil27(64, seed=0, values=values)
    P = W.prolongator(64)
    # A*P (A as CSC), then P^T * (AP) with P^T given as the CSC view of P
    rp, col, val, st1 = device_product(A, P, precision)
    AP = _host(rp, col, val, A.rows, P.cols)
    ref_ap = oracle.spgemm(A.rows, P.cols, *_csc3(A), P.rowptr, P.col, P.val, stats=True)
    assert st1["intermediate_products"] == ref_ap["products"]
    assert_structure_equal(AP.rowptr, AP.col, ref_ap["rowptr"], ref_ap["col"])
    tol = plain_tolerance if precision == sg.PLAIN else compensated_tolerance
    assert_values_close(AP.val, ref_ap, tol(ref_ap))
    Pt = P.transpose()
    rp2, col2, val2, st2 = device_product(Pt, AP, precision)
    ref = oracle.spgemm(Pt.rows, AP.cols, *_csc3(Pt), AP.rowptr, AP.col, AP.val, stats=True)
    assert st2["intermediate_products"] == ref["products"]
    assert_structure_equal(rp2.cpu().numpy(), col2.cpu().numpy(), ref["rowptr"], ref["col"])
    v = val2.cpu().numpy()
    assert_values_close(v, ref, tol(ref))
    # the chain against the FP64 chain (P^T (A P) with AP exact)
    ap64 = W.Csr(AP.rows, AP.cols, ref_ap["rowptr"], ref_ap["col"], ref_ap["val"])
    chain = _oracle_f64_product(Pt, ap64)
    assert len(chain["val"]) == len(v)
    rep = rel_error_report(v, {"val": chain["val"], "absum": chain["absum"]})
    name = ("plain" if precision == sg.PLAIN else "compensated") + "_" + values
    record_property(f"galerkin64_{name}", rep)
    print(f"galerkin64 {name} (chain vs FP64 chain):", rep)


def _csc3(M):
    c = M.to_csc()
    return c.colptr, c.rowidx, c.val


def _oracle_f64_product(A, B):
    """A*B in FP64 with FP64 B values (A has values 0/1, so its FP32 values are
    exact): sums of exact products, and sum |p| per entry."""
    import scipy.sparse as sp
    Am = sp.csr_matrix((A.val.astype(np.float64), A.col, A.rowptr), shape=(A.rows, A.cols))
    Bm = sp.csr_matrix((np.asarray(B.val, np.float64), B.col, B.rowptr), shape=(B.rows, B.cols))
    Ba = sp.csr_matrix((np.abs(np.asarray(B.val, np.float64)), B.col, B.rowptr), shape=(B.rows, B.cols))
    Aa = sp.csr_matrix((np.abs(A.val.astype(np.float64)), A.col, A.rowptr), shape=(A.rows, A.cols))
    C = (Am @ Bm).tocsr()
    S = (Aa @ Ba).tocsr()
    C.sort_indices()
    S.sort_indices()
    # align C's stored entries (scipy drops exact zeros) to the pattern of S
    val = np.zeros(S.nnz)
    for i in range(S.shape[0]):
        s, e = S.indptr[i], S.indptr[i + 1]
        cs, ce = C.indptr[i], C.indptr[i + 1]
        pos = np.searchsorted(S.indices[s:e], C.indices[cs:ce])
        val[s + pos] = C.data[cs:ce]
    return {"val": val, "absum": S.data}
