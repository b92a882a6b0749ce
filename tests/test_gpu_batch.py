"""GPU parity of the batched entry points (spgemm_batch_*) through the C ABI:
every product of a packed batch must match the FP64 oracle exactly in
structure and within the FP32 bounds in value, after the planning run, after
graph replays with new values, and without the graph."""
import numpy as np
import pytest

import oracle
import spgemm_b200 as sg
from spgemm_b200 import workloads as W
from helpers import (assert_structure_equal, assert_values_close, compensated_tolerance,
                     plain_tolerance)

pytestmark = pytest.mark.gpu


def ref_product(A, B):
    a = A.to_csc()
    return oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val,
                         stats=True)


class DeviceBatch:
    """Device copies (torch) of a list of (A, B) host pairs, as CM structs."""

    def __init__(self, pairs, a_format="csr"):
        import torch
        self.torch = torch
        self.pairs = pairs
        self.keep = []
        self.A, self.B, self.a_val = [], [], []
        for A, B in pairs:
            if a_format == "csc":
                a = A.to_csc()
                ta = self._up(a.colptr, a.rowidx, a.val)
                self.A.append(sg.device_cm(*(t.data_ptr() for t in ta), A.nnz, A.rows, A.cols,
                                           sg.COL_MAJOR))
            else:
                ta = self._up(A.rowptr, A.col, A.val)
                self.A.append(sg.device_cm(*(t.data_ptr() for t in ta), A.nnz, A.rows, A.cols,
                                           sg.ROW_MAJOR))
            self.a_val.append(ta[2])
            tb = self._up(B.rowptr, B.col, B.val)
            self.B.append(sg.device_cm(*(t.data_ptr() for t in tb), B.nnz, B.rows, B.cols,
                                       sg.ROW_MAJOR))

    def _up(self, ptr, idx, val):
        t = self.torch
        out = [t.from_numpy(np.ascontiguousarray(ptr, np.int32)).cuda(),
               t.from_numpy(np.ascontiguousarray(idx, np.int32).copy() if len(idx) else np.zeros(1, np.int32)).cuda(),
               t.from_numpy(np.ascontiguousarray(val, np.float32).copy() if len(val) else np.zeros(1, np.float32)).cuda()]
        self.keep.append(out)
        return out


def small_batch(count, seed, n_lo=200, n_hi=4000):
    return [(it.A, it.B) for it in W.batch(count, seed, n_lo=n_lo, n_hi=n_hi)]


def check_all(h, pairs, precision=sg.PLAIN, refs=None):
    refs = refs or [ref_product(A, B) for A, B in pairs]
    for i, (A, B) in enumerate(pairs):
        C = h.batch_copy_result(i)
        ref = refs[i]
        assert (C.rows, C.cols) == (A.rows, B.cols)
        assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
        tol = plain_tolerance(ref) if precision == sg.PLAIN else compensated_tolerance(ref)
        assert_values_close(C.val, ref, tol)
    return refs


@pytest.mark.parametrize("a_format", ["csr", "csc"])
def test_batch_plan_matches_oracle(a_format):
    pairs = small_batch(24, 77)
    db = DeviceBatch(pairs, a_format)
    with sg.Handle() as h:
        tot = h.batch_plan(db.A, db.B)
        refs = check_all(h, pairs)
        assert tot == sum(len(r["col"]) for r in refs)
        ro, no = h.batch_offsets()
        assert ro[-1] == sum(A.rows for A, _ in pairs)
        assert no[-1] == tot


def test_batch_graph_replay_new_values():
    pairs = small_batch(16, 91)
    db = DeviceBatch(pairs)
    with sg.Handle() as h:
        h.batch_plan(db.A, db.B)
        # new values in the same arrays: scale every A_i, negate a few entries
        rng = np.random.default_rng(5)
        new_pairs = []
        for (A, B), tv in zip(pairs, db.a_val):
            v = (A.val * 2.0).astype(np.float32)
            if len(v):
                flip = rng.random(len(v)) < 0.3
                v[flip] = -v[flip]
                tv.copy_(db.torch.from_numpy(v))
            new_pairs.append((W.Csr(A.rows, A.cols, A.rowptr, A.col, v), B))
        refs = [ref_product(A, B) for A, B in new_pairs]
        for graph in (True, True, False):  # record, replay, direct launches
            h.batch_execute(graph=graph)
            check_all(h, new_pairs, refs=refs)
        st = h.stats()
        assert st["kernel_launches"] > 0


def test_batch_compensated():
    pairs = small_batch(12, 5)
    db = DeviceBatch(pairs)
    with sg.Handle(sg.COMPENSATED) as h:
        h.batch_plan(db.A, db.B)
        refs = check_all(h, pairs, sg.COMPENSATED)
        h.batch_execute(graph=True)
        check_all(h, pairs, sg.COMPENSATED, refs)


def test_batch_with_long_rows_and_empty_products():
    # a power-law product with rows above 4096 partials next to empty and tiny ones
    big = W.rmat(12, 16, 4, values="sym")
    empty = W.Csr(7, 5, np.zeros(8, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    eye5 = W.from_coo(5, 5, np.arange(5), np.arange(5), np.ones(5, np.float32))
    tiny = W.er(30, 3.0, 2)
    pairs = [(tiny, tiny), (empty, eye5), (big, big), (eye5, eye5), (tiny, tiny)]
    db = DeviceBatch(pairs)
    with sg.Handle() as h:
        h.batch_plan(db.A, db.B)
        st = h.stats()
        assert st["rows_per_symbolic_bin"][9] > 0  # long rows present in the packed product
        refs = check_all(h, pairs)
        h.batch_execute(graph=True)
        check_all(h, pairs, refs=refs)


def test_batch_plan_invalidated_by_other_product():
    pairs = small_batch(4, 3)
    db = DeviceBatch(pairs)
    with sg.Handle() as h:
        h.batch_plan(db.A, db.B)
        A, B = pairs[0]
        h.multiply_host(A.to_csc(), B)
        with pytest.raises(sg.SpgemmError) as e:
            h.batch_execute(graph=True)
        assert e.value.status == 5


def test_batch_rejects_mixed_formats_and_bad_shapes():
    pairs = small_batch(3, 8)
    db_csr = DeviceBatch(pairs, "csr")
    db_csc = DeviceBatch(pairs, "csc")
    with sg.Handle() as h:
        with pytest.raises(sg.SpgemmError) as e:
            h.batch_plan([db_csr.A[0], db_csc.A[1], db_csr.A[2]], db_csr.B)
        assert e.value.status == 1
        bad_b = list(db_csr.B)
        bad_b[1], bad_b[2] = bad_b[2], bad_b[1]
        if pairs[1][0].cols != pairs[2][1].rows:
            with pytest.raises(sg.SpgemmError) as e:
                h.batch_plan(db_csr.A, bad_b)
            assert e.value.status == 1
        with pytest.raises(sg.SpgemmError) as e:
            h.batch_execute()
        assert e.value.status == 5  # no successful plan


@pytest.mark.parametrize("precision", [sg.PLAIN, sg.COMPENSATED])
def test_batch_large_warp_tables(precision):
    # 1024-slot warp tables: uniform (ER) rows take the bucket sort, rows with
    # R-MAT-skewed columns crowd the low buckets and take the radix passes
    pairs = small_batch(12, 31, n_lo=3000, n_hi=30000)
    db = DeviceBatch(pairs)
    with sg.Handle(precision) as h:
        h.set_tuning(warp_table_max=1024, warp_p_max=1024, warp_cap_max=2048, esc_p_min=4096)
        h.batch_plan(db.A, db.B)
        st = h.stats()
        assert st["rows_per_symbolic_bin"][4] > 0  # rows in 1024-slot tables
        refs = check_all(h, pairs, precision)
        h.batch_execute(graph=True)
        check_all(h, pairs, precision, refs)
