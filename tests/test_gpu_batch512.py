"""The full 512-product batch configuration on the GPU (n_i log-uniform in
[1k, 200k], Poisson(lam_i) entries per row with lam_i ~ U[4, 32], half
Erdos-Renyi, half R-MAT, values U[-1, 1], seed 1000 + i), planned and then
replayed as one CUDA graph through the C ABI (spgemm_batch_plan /
spgemm_batch_execute), and checked product by product against the oracle:

* every product: P_i (the oracle's product count) and the complete structure
  (row pointers and sorted column indices, the oracle's FP32 mode);
* 32 products, the largest among them: every value against the FP64 oracle
  within the FP32 summation bound, with the maximum relative error recorded.
"""
import multiprocessing as mp
import os

import numpy as np
import pytest

import oracle
import spgemm_b200 as sg
from spgemm_b200 import workloads as W
from helpers import assert_structure_equal, assert_values_close, plain_tolerance, rel_error_report

pytestmark = pytest.mark.gpu


def _item(spec):
    it = W.batch_item(*spec)
    return it.A, it.B


def _batch512():
    specs = W.batch_specs(512, 1000)
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 1, 32)) as pool:
        return pool.map(_item, specs, chunksize=1)


def test_batch512_every_product(record_property):
    import torch
    pairs = _batch512()
    keep = []

    def up(a, dt):
        t = torch.from_numpy(np.ascontiguousarray(a)).to(dt).cuda()
        keep.append(t)
        return t.data_ptr()
    A_list = [sg.device_cm(up(A.rowptr, torch.int32), up(A.col, torch.int32), up(A.val, torch.float32),
                           A.nnz, A.rows, A.cols, sg.ROW_MAJOR) for A, _ in pairs]
    B_list = [sg.device_cm(up(B.rowptr, torch.int32), up(B.col, torch.int32), up(B.val, torch.float32),
                           B.nnz, B.rows, B.cols, sg.ROW_MAJOR) for _, B in pairs]
    sizes = np.array([int(np.diff(B.rowptr.astype(np.int64))[A.col].sum()) for A, B in pairs])
    sampled = set(np.random.default_rng(5).choice(512, 31, replace=False).tolist())
    sampled.add(int(np.argmax(sizes)))
    reps = []
    with sg.Handle(sg.PLAIN) as h:
        h.set_stream(torch.cuda.current_stream().cuda_stream)
        total = h.batch_plan(A_list, B_list)
        assert h.stats()["intermediate_products"] == int(sizes.sum())
        h.batch_execute(graph=True)  # the replayed graph's output is what is checked
        torch.cuda.synchronize()
        nnz_sum = 0
        for i, (A, B) in enumerate(pairs):
            a = A.to_csc()
            assert oracle.count_products(A.rows, a.colptr, a.rowidx, B.rowptr) == sizes[i]
            C = h.batch_copy_result(i)
            assert (C.rows, C.cols) == (A.rows, B.cols)
            nnz_sum += len(C.col)
            if i in sampled:
                ref = oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col,
                                    B.val, stats=True)
                assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
                assert_values_close(C.val, ref, plain_tolerance(ref))
                reps.append(rel_error_report(C.val, ref))
            else:
                ref = oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col,
                                    B.val, mode=1)
                assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
        assert nnz_sum == total
    worst = max(reps, key=lambda r: r["max_rel"])
    record_property("batch512_plain", worst)
    print("batch512 plain (32 sampled products):", worst)
