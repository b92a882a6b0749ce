"""Full-size configurations on the GPU (through the C ABI, device-resident
inputs): R-MAT 2^18 ef16 A*A checked on sampled rows (random + heaviest)
against the oracle plus size-independent properties over all of C; the 27-point
96^3 stencil A*A in compensated mode checked entry by entry, with the maximum
relative error reported."""
import numpy as np
import pytest

import oracle
import spgemm_b200 as sg
from spgemm_b200 import workloads as W
from helpers import (assert_structure_equal, assert_values_close, compensated_tolerance,
                     plain_tolerance, rel_error_report)

pytestmark = pytest.mark.gpu


def device_product(A, B, precision):
    import torch
    Ac = A.to_csc()
    d = lambda a, t: torch.from_numpy(np.ascontiguousarray(a)).cuda().to(t)
    tA = [d(Ac.colptr, torch.int32), d(Ac.rowidx, torch.int32), d(Ac.val, torch.float32)]
    tB = [d(B.rowptr, torch.int32), d(B.col, torch.int32), d(B.val, torch.float32)]
    Acm = sg.device_cm(tA[0].data_ptr(), tA[1].data_ptr(), tA[2].data_ptr(), A.nnz, A.rows, A.cols, sg.COL_MAJOR)
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


def check_sorted_rows_on_device(rp, col):
    """Columns strictly increasing inside every row (so no duplicates)."""
    import torch
    n = col.numel()
    if n < 2:
        return
    starts = torch.zeros(n, dtype=torch.bool, device=col.device)
    first = rp[:-1].long()
    first = first[first < n]
    starts[first] = True
    ok = (col[1:] > col[:-1]) | starts[1:]
    assert bool(ok.all())


def test_rmat18_sampled_rows():
    import torch
    A = W.rmat(18, 16, 0)
    rp, col, val, stats = device_product(A, A, sg.PLAIN)
    rp_h = rp.cpu().numpy().astype(np.int64)
    assert rp_h[0] == 0 and np.all(np.diff(rp_h) >= 0) and rp_h[-1] == col.numel()
    check_sorted_rows_on_device(rp, col)
    a = A.to_csc()
    P, p_i = oracle.count_products(A.rows, a.colptr, a.rowidx, A.rowptr, per_row=True)
    assert stats["intermediate_products"] == P
    rng = np.random.default_rng(0)
    heavy = np.argsort(p_i)[-40:]
    rows = np.unique(np.concatenate([rng.choice(A.rows, 600, replace=False), heavy])).astype(np.int32)
    ref = oracle.spgemm(A.rows, A.cols, a.colptr, a.rowidx, a.val, A.rowptr, A.col, A.val,
                        rows=rows, stats=True)
    col_h = col.cpu().numpy()
    val_h = val.cpu().numpy()
    got_rp = [0]
    gc, gv = [], []
    for i in rows:
        s, e = rp_h[i], rp_h[i + 1]
        gc.append(col_h[s:e]); gv.append(val_h[s:e]); got_rp.append(got_rp[-1] + e - s)
    assert_structure_equal(np.array(got_rp), np.concatenate(gc), ref["rowptr"], ref["col"])
    assert_values_close(np.concatenate(gv), ref, plain_tolerance(ref))


def test_stencil96_compensated_full(record_property):
    A = W.stencil27(96, seed=0)
    rp, col, val, stats = device_product(A, A, sg.COMPENSATED)
    a = A.to_csc()
    ref = oracle.spgemm(A.rows, A.cols, a.colptr, a.rowidx, a.val, A.rowptr, A.col, A.val, stats=True)
    assert_structure_equal(rp.cpu().numpy(), col.cpu().numpy(), ref["rowptr"], ref["col"])
    v = val.cpu().numpy()
    assert_values_close(v, ref, compensated_tolerance(ref))
    rep = rel_error_report(v, ref)
    record_property("stencil96_compensated", rep)
    print("stencil96 compensated:", rep)
