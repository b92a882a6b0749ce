"""spgemm_coo_to_cm_noalloc: the allocation-free conversion for callers that
cannot allocate device memory (device memory owned by another allocator, hot
loops where a cudaMalloc would synchronise). Called through the C ABI on
caller-owned device arrays, its output must equal cudaCOO2CM's (the same
conversion, which allocates its own workspace) and the CSR/CSC the triplets
were made from, on two calls in a row that share the static scratch array.
This file sorts last so that a run stopping at the first failure has run
every other test."""
import ctypes as C

import numpy as np
import pytest

import spgemm_b200 as sg
from spgemm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def lib():
    L = sg.lib()
    L.spgemm_coo_to_cm_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.POINTER(C.c_longlong)]
    return L


def sorted_triplets(M: W.Csr, kind):
    """Triplet array (ridx, cidx, val bits) sorted the way sortCOO sorts."""
    r = np.repeat(np.arange(M.rows, dtype=np.int32), np.diff(M.rowptr))
    c = M.col.astype(np.int32)
    v = M.val.astype(np.float32)
    order = np.lexsort((r, c)) if kind == sg.COL_MAJOR else np.lexsort((c, r))
    t = np.empty((M.nnz, 3), np.int32)
    t[:, 0], t[:, 1], t[:, 2] = r[order], c[order], v[order].view(np.int32)
    return t


def reference_conversion(t, rows, cols, kind):
    """The existing entry point: cudaCOO2CM on host triplets."""
    L = sg.lib()
    L.spgemm_set_exit_on_error(0)
    arr = (sg.Triplet * len(t)).from_buffer_copy(np.ascontiguousarray(t).tobytes())
    coo = sg.COO(C.cast(arr, C.POINTER(sg.Triplet)), len(t), cols, rows, kind)
    out = L.cudaCOO2CM(coo)
    assert L.spgemm_legacy_status() == 0
    nmaj = (rows if kind == sg.ROW_MAJOR else cols) + 1
    res = (np.ctypeslib.as_array(out.ptr, (nmaj,)).copy(),
           np.ctypeslib.as_array(out.idx, (max(len(t), 1),))[:len(t)].copy(),
           np.ctypeslib.as_array(out.val, (max(len(t), 1),))[:len(t)].copy())
    L.cmFree(C.byref(out))
    return res


def noalloc_conversion(t, rows, cols, kind):
    import torch
    nmaj = (rows if kind == sg.ROW_MAJOR else cols) + 1
    d_t = torch.from_numpy(np.ascontiguousarray(t)).cuda()
    d_ptr = torch.full((nmaj,), -7, dtype=torch.int32, device="cuda")  # garbage on purpose
    d_idx = torch.full((max(len(t), 1),), -7, dtype=torch.int32, device="cuda")
    d_val = torch.full((max(len(t), 1),), -7.0, dtype=torch.float32, device="cuda")
    total = C.c_longlong(-1)
    st = lib().spgemm_coo_to_cm_noalloc(d_t.data_ptr(), len(t), rows, cols, kind, d_ptr.data_ptr(),
                                        d_idx.data_ptr(), d_val.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream, C.byref(total))
    assert st == 0
    assert total.value == len(t)
    torch.cuda.synchronize()
    return d_ptr.cpu().numpy(), d_idx.cpu().numpy()[:len(t)], d_val.cpu().numpy()[:len(t)]


def test_noalloc_matches_cudaCOO2CM_twice():
    cases = [(W.rmat(12, 8, 3, values="sym"), sg.ROW_MAJOR),
             (W.er(3000, 6.0, 4, cols=5000), sg.COL_MAJOR)]
    for M, kind in cases:  # two calls in a row share the static scratch
        t = sorted_triplets(M, kind)
        ref = reference_conversion(t, M.rows, M.cols, kind)
        got = noalloc_conversion(t, M.rows, M.cols, kind)
        for a, b in zip(ref, got):
            assert np.array_equal(a, b)
        # and the compressed matrix the triplets were made from
        src = M if kind == sg.ROW_MAJOR else M.to_csc()
        ptr, idx, val = ((src.rowptr, src.col, src.val) if kind == sg.ROW_MAJOR
                         else (src.colptr, src.rowidx, src.val))
        assert np.array_equal(got[0], ptr)
        assert np.array_equal(got[1], idx)
        assert np.array_equal(got[2], val)


def test_noalloc_empty_input():
    import torch
    d_ptr = torch.full((6,), -7, dtype=torch.int32, device="cuda")
    total = C.c_longlong(-1)
    st = lib().spgemm_coo_to_cm_noalloc(None, 0, 5, 9, sg.ROW_MAJOR, d_ptr.data_ptr(), None,
                                        None, None, C.byref(total))
    assert st == 0 and total.value == 0
    assert np.array_equal(d_ptr.cpu().numpy(), np.zeros(6, np.int32))


def test_noalloc_reports_out_of_range_index():
    import torch
    # row index 3 == num_rows: out of range
    t = np.array([[0, 1, 0], [1, 0, 0], [3, 2, 0]], np.int32)
    d_t = torch.from_numpy(t).cuda()
    bufs = [torch.zeros(4, dtype=torch.int32, device="cuda"),
            torch.zeros(3, dtype=torch.int32, device="cuda"),
            torch.zeros(3, dtype=torch.float32, device="cuda")]
    total = C.c_longlong()
    st = lib().spgemm_coo_to_cm_noalloc(d_t.data_ptr(), 3, 3, 3, sg.ROW_MAJOR, bufs[0].data_ptr(),
                                        bufs[1].data_ptr(), bufs[2].data_ptr(), None, C.byref(total))
    assert st == 1
    assert total.value == 2  # the two entries inside the dimensions were counted


def test_noalloc_rejects_oversize_and_reports_unsorted():
    import torch
    L = lib()
    assert L.spgemm_coo_to_cm_noalloc(None, 0, (1 << 26) + 1, 4, sg.ROW_MAJOR, 1, None, None,
                                      None, None) == 7
    t = np.array([[2, 0, 0], [0, 1, 0], [1, 0, 0]], np.int32)  # not sorted by row
    d_t = torch.from_numpy(t).cuda()
    bufs = [torch.zeros(4, dtype=torch.int32, device="cuda") for _ in range(2)] + \
           [torch.zeros(3, dtype=torch.float32, device="cuda")]
    total = C.c_longlong()
    st = L.spgemm_coo_to_cm_noalloc(d_t.data_ptr(), 3, 3, 3, sg.ROW_MAJOR, bufs[0].data_ptr(),
                                    bufs[1].data_ptr(), bufs[2].data_ptr(), None, C.byref(total))
    assert st == 1
