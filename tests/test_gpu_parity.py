"""GPU parity: the sm_100a engine (through the C ABI) against the FP64 oracle.

Structure (row pointers, sorted column indices, explicit zeros) must be
bit-exact; values must lie within the summation-error bounds stated in
helpers.py (plain FP32 and compensated modes)."""
import numpy as np
import pytest

import oracle
import spgemm_b200 as sg
from spgemm_b200 import workloads as W
from helpers import (assert_structure_equal, assert_values_close, compensated_tolerance,
                     plain_tolerance, rel_error_report)

pytestmark = pytest.mark.gpu


def ref_product(A, B, rows=None):
    a = A.to_csc()
    return oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val,
                         rows=rows, stats=True)


def check(A, B, precision=sg.PLAIN, a_format="csc", ref=None, tuning=None):
    Aop = A.to_csc() if a_format == "csc" else A
    with sg.Handle(precision) as h:
        if tuning:
            h.set_tuning(**tuning)
        C = h.multiply_host(Aop, B)
        stats = h.stats()
    ref = ref_product(A, B) if ref is None else ref
    assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
    tol = plain_tolerance(ref) if precision == sg.PLAIN else compensated_tolerance(ref)
    assert_values_close(C.val, ref, tol)
    assert stats["intermediate_products"] == ref["products"]
    assert stats["nnz_c"] == len(ref["col"])
    return C, ref, stats


def dense_csr(D):
    D = np.asarray(D, np.float32)
    r, c = np.nonzero(D)
    return W.from_coo(D.shape[0], D.shape[1], r, c, D[r, c])


def test_er4096_plain():
    A = W.er(4096, 8.0, 0)
    _, ref, stats = check(A, A)
    assert stats["kernel_launches"] > 0


def test_er4096_compensated():
    A = W.er(4096, 8.0, 0)
    check(A, A, sg.COMPENSATED)


def test_a_as_csr_equals_csc():
    A = W.er(2000, 10.0, 3)
    check(A, A, a_format="csr")


def test_kat_cancellation_and_empty_rows():
    A = W.from_coo(3, 2, np.array([0, 0, 2]), np.array([0, 1, 1]), np.array([1, 1, 4], np.float32))
    B = W.from_coo(2, 2, np.array([0, 0, 1]), np.array([0, 1, 0]), np.array([2, 3, -2], np.float32))
    C, _, _ = check(A, B)
    assert C.rowptr.tolist() == [0, 2, 2, 3]
    assert C.col.tolist() == [0, 1, 0]
    assert C.val.tolist() == [0.0, 3.0, -8.0]


def test_rectangular_and_empty_columns():
    rng = np.random.default_rng(7)
    D1 = (rng.random((37, 53)) < 0.1) * rng.uniform(-1, 1, (37, 53))
    D2 = (rng.random((53, 91)) < 0.1) * rng.uniform(-1, 1, (53, 91))
    D1[:, 5] = 0
    D2[10, :] = 0
    check(dense_csr(D1), dense_csr(D2))


def test_empty_product():
    A = W.Csr(5, 4, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    B = dense_csr(np.eye(4))
    C, _, _ = check(A, B)
    assert C.nnz == 0 and C.rowptr.tolist() == [0] * 6


def test_rmat_all_bins():
    A = W.rmat(14, 16, 1)
    _, ref, stats = check(A, A)
    assert stats["rows_per_symbolic_bin"][9] > 0, stats   # long rows
    assert stats["rows_per_symbolic_bin"][12] > 0, stats  # sorted rows (2K-4K products)
    assert stats["long_row_slices"] == 0, stats           # every long row taken whole
    # with sorting off, the mid rows take the fused span bitmap
    _, _, st1 = check(A, A, ref=ref, tuning=dict(esc_p_min=4096))
    assert st1["rows_per_symbolic_bin"][8] > 0, st1
    assert sum(st1["rows_per_symbolic_bin"][10:13]) == 0, st1
    # with the whole-row kernel off, long rows take column slices
    with sg.Handle() as h:
        h.set_tuning(long_rows=0)
        C = h.multiply_host(A.to_csc(), A)
        st0 = h.stats()
    ref = ref_product(A, A)
    assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
    assert_values_close(C.val, ref, plain_tolerance(ref))
    assert st0["rows_per_numeric_bin"][8] > 0, st0        # column slices


def test_rmat_all_bins_compensated():
    A = W.rmat(14, 16, 2)
    check(A, A, sg.COMPENSATED)


def test_long_rows_multi_slice_multi_window():
    # one C row with ~1e5 outputs over 1.2M columns: several numeric slices
    # and two symbolic bitmap windows
    rng = np.random.default_rng(11)
    n = 1_200_000
    kk = 220
    rows, cols = [], []
    for k in range(kk):
        c = np.unique(rng.integers(0, n, 600))
        rows.append(np.full(len(c), k))
        cols.append(c)
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    B = W.from_coo(kk, n, r, c, rng.uniform(-1, 1, len(r)).astype(np.float32))
    A = W.from_coo(3, kk, np.array([0] * kk + [2] * 50), np.concatenate([np.arange(kk), np.arange(50)]),
                   rng.uniform(-1, 1, kk + 50).astype(np.float32))
    _, _, stats = check(A, B)
    assert stats["long_row_slices"] >= 3, stats
    check(A, B, sg.COMPENSATED)


def test_galerkin_chain_small():
    A = W.stencil27(8, values="laplace")
    P = W.prolongator(8)
    with sg.Handle(sg.COMPENSATED) as h:
        AP = h.multiply_host(A.to_csc(), P)
        PtAP = h.multiply_host(P.transpose().to_csc(), AP)
    ref_ap = ref_product(A, P)
    assert_structure_equal(AP.rowptr, AP.col, ref_ap["rowptr"], ref_ap["col"])
    assert_values_close(AP.val, ref_ap, compensated_tolerance(ref_ap))
    ref = ref_product(P.transpose(), AP)
    assert_structure_equal(PtAP.rowptr, PtAP.col, ref["rowptr"], ref["col"])
    assert_values_close(PtAP.val, ref, compensated_tolerance(ref))


@pytest.mark.parametrize("precision", [sg.PLAIN, sg.COMPENSATED])
def test_stencil_small(precision):
    A = W.stencil27(14, seed=3)
    C, ref, _ = check(A, A, precision)
    if precision == sg.COMPENSATED:
        rep = rel_error_report(C.val, ref)
        assert rep["max_rel"] < 1e-6 or rep["worst_cond"] > 1e7, rep


def test_repeat_calls_reuse_workspace():
    A = W.er(3000, 8.0, 9)
    B = W.rmat(11, 8, 9)
    with sg.Handle() as h:
        for M in (A, W.er(1000, 4.0, 1), A):
            C = h.multiply_host(M.to_csc(), M)
            ref = ref_product(M, M)
            assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
        C = h.multiply_host(B.to_csc(), B)
        ref = ref_product(B, B)
        assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])


TUNINGS = [
    dict(keep_bitmaps=0),                                   # numeric rebuilds long-row bitmaps
    dict(slice_cap=2048, slice_cols=8192, long_rows=0),     # many column slices per long row
    dict(warp_p_max=0),                                     # no fused warp rows: block / bitmap
    dict(warp_table_max=64),                                # most warp rows overflow and are redone
    dict(warp_table_max=1024, warp_cap_max=4096),           # large warp tables
    dict(long_p=256, long_o_num=256),                       # mid rows take the two-pass path
    dict(long_p=64, long_o_num=64, mid_o_min=0),            # long path + span bitmap numeric
    dict(sym_window=4096, slice_cols=4096, slice_cap=2048,  # multi-window symbolic pass,
         keep_bitmaps=0),                                   # restricted numeric slices
    dict(mid_cols=0),                                       # no bitmaps: hash tables only
    dict(long_rows=1),                                      # whole long rows, reductions into C
    dict(long_rows=2),                                      # whole long rows, shared memory
    dict(long_rows=1, long_p=256, long_o_num=256),          # ... with many short long rows
    dict(long_rows=2, keep_bitmaps=0),                      # no kept bitmaps: column slices
    dict(long_rows=3),                                      # shared memory, L2 reductions above
    dict(long_rows=3, long_p=256, long_o_num=256),          # ... with many short long rows
    dict(warp_cap_max=0),                                   # every fused row sorted
    dict(esc_p_min=4096),                                   # no sorted rows: bitmap / block hash
    dict(warp_cap_max=64, esc_p_min=32, esc_span_min=20000),  # sorted only when the span is wide
    dict(warp_cap_max=0, long_p=1024),                      # sorted rows up to 1024 products
]


@pytest.mark.parametrize("tuning", TUNINGS, ids=lambda t: ",".join(f"{k}={v}" for k, v in t.items()))
@pytest.mark.parametrize("precision", [sg.PLAIN, sg.COMPENSATED])
def test_tuning_overrides(tuning, precision):
    A = W.rmat(14, 16, 5)
    ref = ref_product(A, A)
    with sg.Handle(precision) as h:
        h.set_tuning(**tuning)
        C = h.multiply_host(A.to_csc(), A)
        stats = h.stats()
    assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
    tol = plain_tolerance(ref) if precision == sg.PLAIN else compensated_tolerance(ref)
    assert_values_close(C.val, ref, tol)
    if "slice_cap" in tuning:
        assert stats["long_row_slices"] > stats["rows_per_numeric_bin"][8], stats


@pytest.mark.parametrize("long_rows", [1, 2, 3])
def test_whole_row_path_with_wide_and_narrow_rows(long_rows):
    """Long rows of both kinds in one product: row 0 has ~90K outputs (beyond
    the shared-memory capacity of long_rows=2, so it takes column slices
    there), rows 1..3 a few thousand; n = 200K keeps every span inside the
    whole-row directory."""
    rng = np.random.default_rng(21)
    n, kk = 200_000, 300
    rows, cols = [], []
    for k in range(kk):
        c = np.unique(rng.integers(0, n, 400))
        rows.append(np.full(len(c), k))
        cols.append(c)
    rows.append(np.full(2, kk)); cols.append(np.array([7, 8]))
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    B = W.from_coo(kk + 1, n, r, c, rng.uniform(-1, 1, len(r)).astype(np.float32))
    ar = np.array([0] * kk + [1] * 20 + [2] * 25 + [3] * 30)
    ac = np.array(list(range(kk)) + list(range(20)) + list(range(100, 125)) + list(range(200, 230)))
    A = W.from_coo(4, kk + 1, ar, ac, rng.uniform(-1, 1, len(ar)).astype(np.float32))
    with sg.Handle() as h:
        h.set_tuning(long_rows=long_rows)
        C = h.multiply_host(A.to_csc(), B)
        stats = h.stats()
    ref = ref_product(A, B)
    assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
    assert_values_close(C.val, ref, plain_tolerance(ref))
    assert np.diff(ref["rowptr"])[0] > 40_000
    if long_rows == 2:
        assert stats["long_row_slices"] >= 2, stats  # row 0 was sliced
    else:
        assert stats["long_row_slices"] == 0, stats


def test_bad_tuning_rejected():
    with sg.Handle() as h:
        with pytest.raises(sg.SpgemmError):
            h.set_tuning(long_o_num=5000)
        with pytest.raises(sg.SpgemmError):
            h.set_tuning(slice_cols=1000)
        with pytest.raises(sg.SpgemmError):
            h.set_tuning(long_p=5000)
        with pytest.raises(sg.SpgemmError):
            h.set_tuning(warp_table_max=100)
        with pytest.raises(sg.SpgemmError):
            h.set_tuning(long_rows=4)


def _dev(a, dtype, offset=0):
    """Device copy of a, starting `offset` elements into a larger buffer (to
    misalign it on purpose)."""
    import torch
    t = torch.zeros(len(a) + offset + 1, dtype=dtype, device="cuda")
    t[offset:offset + len(a)] = torch.from_numpy(np.ascontiguousarray(a)).to(dtype)
    return t, t[offset:]


@pytest.mark.parametrize("offset", [0, 1])
def test_device_api_two_phase(offset):
    """spgemm_symbolic + spgemm_numeric on device pointers into caller buffers;
    offset 1 misaligns B's arrays so the 128-bit load path is disabled."""
    import torch
    A = W.rmat(13, 12, 7, values="sym")
    Ac = A.to_csc()
    keep = []
    a_ptr = _dev(Ac.colptr, torch.int32)[1]; a_idx = _dev(Ac.rowidx, torch.int32)[1]
    a_val = _dev(Ac.val, torch.float32)[1]
    b_ptr = _dev(A.rowptr, torch.int32)[1]
    b_idx_base, b_idx = _dev(A.col, torch.int32, offset)
    b_val_base, b_val = _dev(A.val, torch.float32, offset)
    keep += [b_idx_base, b_val_base]
    Acm = sg.device_cm(a_ptr.data_ptr(), a_idx.data_ptr(), a_val.data_ptr(), A.nnz, A.rows, A.cols, sg.COL_MAJOR)
    Bcm = sg.device_cm(b_ptr.data_ptr(), b_idx.data_ptr(), b_val.data_ptr(), A.nnz, A.rows, A.cols, sg.ROW_MAJOR)
    with sg.Handle() as h:
        h.set_stream(torch.cuda.current_stream().cuda_stream)
        nnz = h.symbolic(Acm, Bcm)
        rp = torch.empty(A.rows + 1, dtype=torch.int32, device="cuda")
        col = torch.empty(nnz, dtype=torch.int32, device="cuda")
        val = torch.empty(nnz, dtype=torch.float32, device="cuda")
        h.numeric(rp.data_ptr(), col.data_ptr(), val.data_ptr())
        torch.cuda.synchronize()
    ref = ref_product(A, A)
    assert_structure_equal(rp.cpu().numpy(), col.cpu().numpy(), ref["rowptr"], ref["col"])
    assert_values_close(val.cpu().numpy(), ref, plain_tolerance(ref))


def test_numeric_before_symbolic_is_an_error():
    with sg.Handle() as h:
        with pytest.raises(sg.SpgemmError) as e:
            h.numeric(0, 0, 0)
        assert e.value.status == 5


def test_invalid_inputs_rejected():
    A = W.er(100, 4.0, 1)
    bad = W.Csr(A.rows, A.cols, A.rowptr.copy(), A.col.copy(), A.val.copy())
    bad.col[3] = A.cols + 5            # column out of range
    with sg.Handle() as h:
        with pytest.raises(sg.SpgemmError) as e:
            h.multiply_host(A.to_csc(), bad)
        assert e.value.status == 1
        uns = W.Csr(A.rows, A.cols, A.rowptr.copy(), A.col.copy(), A.val.copy())
        r = int(np.argmax(np.diff(A.rowptr) >= 2))
        s = A.rowptr[r]
        uns.col[s], uns.col[s + 1] = A.col[s + 1], A.col[s]   # unsorted B row
        with pytest.raises(sg.SpgemmError):
            h.multiply_host(A.to_csc(), uns)
        # the handle stays usable after rejected inputs
        C = h.multiply_host(A.to_csc(), A)
        ref = ref_product(A, A)
        assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])


def _run_twice(A, B, precision, tuning):
    out = []
    for _ in range(2):
        with sg.Handle(precision) as h:
            h.set_tuning(**tuning)
            C = h.multiply_host(A, B)  # A as CSR: its entry order is the caller's
        out.append(C)
    return out


@pytest.mark.parametrize("precision", [sg.PLAIN, sg.COMPENSATED])
def test_sorted_rows_are_deterministic(precision):
    # rows merged by sorting sum every column's products in product order
    # (A's entries in row order, each B row in order), so two runs give the
    # same bits when A is given as CSR (a CSC A is transposed with atomics,
    # which leaves the entry order inside a row to arrival order); stencil
    # rows repeat columns ~6 times each
    A = W.stencil27(14, seed=3)
    C1, C2 = _run_twice(A, A, precision, dict(warp_cap_max=0))
    assert np.array_equal(C1.rowptr, C2.rowptr) and np.array_equal(C1.col, C2.col)
    assert np.array_equal(C1.val.view(np.uint32), C2.val.view(np.uint32))
    ref = ref_product(A, A)
    assert_structure_equal(C1.rowptr, C1.col, ref["rowptr"], ref["col"])
    tol = plain_tolerance(ref) if precision == sg.PLAIN else compensated_tolerance(ref)
    assert_values_close(C1.val, ref, tol)


def test_sorted_rows_edge_cases():
    # rows with a single column (one-bit keys), stored zeros and exact
    # cancellation to an explicit zero, a wide span (25-bit column offsets:
    # four radix passes), and rows at each sorted-bin capacity (1024 / 2048 /
    # 4096 products)
    rng = np.random.default_rng(11)
    n = 1 << 25
    # row 0: 64 products all in column 5 (A row of 64 entries, each B row {5})
    # row 1: products cancelling to zero in column 7; row 2: span ~2^25
    ra, ca, va, rb, cb, vb = [], [], [], [], [], []
    for k in range(64):
        ra.append(0); ca.append(k); va.append(1.0)
        rb.append(k); cb.append(5); vb.append(float(k % 3) - 1.0)
    ra += [1, 1]; ca += [64, 65]; va += [2.0, 2.0]
    rb += [64, 65]; cb += [7, 7]; vb += [1.5, -1.5]
    for k in range(66, 66 + 300):
        ra.append(2); ca.append(k); va.append(rng.uniform(-1, 1))
        rb += [k, k]; cb += [int(rng.integers(0, n // 2)) * 2, n - 1 - 2 * (k - 66)]
        vb += [rng.uniform(-1, 1), rng.uniform(-1, 1)]
    A = W.from_coo(3, 400, np.array(ra), np.array(ca), np.array(va, np.float32))
    B = W.from_coo(400, n, np.array(rb), np.array(cb), np.array(vb, np.float32))
    C, _, st = check(A, B, tuning=dict(warp_cap_max=0))
    assert C.col[C.rowptr[1]:C.rowptr[2]].tolist() == [7]
    assert C.val[C.rowptr[1]:C.rowptr[2]].tolist() == [0.0]  # explicit zero kept
    assert C.col[0:C.rowptr[1]].tolist() == [5]
    # full bins: R-MAT rows of up to 4096 products, all sorted
    A = W.rmat(13, 24, 9)
    _, _, st = check(A, A, tuning=dict(warp_cap_max=0))
    assert min(st["rows_per_symbolic_bin"][10:13]) > 0, st
    check(A, A, sg.COMPENSATED, tuning=dict(warp_cap_max=0))


PIECE_TUNINGS = [
    dict(),                                         # whole long rows (shared memory), sorted mid rows
    dict(long_rows=0, slice_cap=2048, slice_cols=8192),  # column slices of long rows
    dict(long_rows=3),                              # whole rows, L2 reductions for the longest
    dict(long_p=256, long_o_num=256, mid_o_min=0),  # long rows in the span-bitmap and hash bins
    dict(long_p=256, long_o_num=4096, mid_o_min=100000),  # long rows in the block-hash bins
]


@pytest.mark.parametrize("tuning", PIECE_TUNINGS, ids=lambda t: ",".join(f"{k}={v}" for k, v in t.items()) or "default")
@pytest.mark.parametrize("precision", [sg.PLAIN, sg.COMPENSATED])
def test_host_copy_in_pieces(tuning, precision):
    # the host-buffer calls compute C in row ranges and copy each range back
    # while the next computes; a 4 KiB piece size gives the maximum of 16
    # ranges, so every numeric kernel runs on partial row ranges
    A = W.rmat(13, 16, 2)
    ref = ref_product(A, A)
    tol = plain_tolerance(ref) if precision == sg.PLAIN else compensated_tolerance(ref)
    with sg.Handle(precision) as h:
        h.set_tuning(**tuning)
        h.set_copy_chunk(4096)
        C = h.multiply_host(A.to_csc(), A)
        assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
        assert_values_close(C.val, ref, tol)
        nnz = len(ref["col"])
        rp = np.full(A.rows + 1, -1, np.int32)
        col = np.full(nnz, -1, np.int32)
        val = np.full(nnz, np.nan, np.float32)
        assert h.multiply_host_to(A.to_csc(), A, rp, col, val) == nnz
        assert_structure_equal(rp, col, ref["rowptr"], ref["col"])
        assert_values_close(val, ref, tol)
        h.set_copy_chunk(0)  # one piece
        C1 = h.multiply_host(A.to_csc(), A)
        assert_structure_equal(C1.rowptr, C1.col, ref["rowptr"], ref["col"])
