"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py):
the oracle must reproduce them exactly (CPU), and the GPU engine must match
their structure bit for bit and their values within the FP32 bound."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from spgemm_b200 import workloads as W

GOLD = sorted((Path(__file__).parent / "golden").glob("*.npz"))


def load(p):
    d = np.load(p)
    A = W.Csr(int(d["a_rows"]), int(d["a_cols"]), d["a_rowptr"], d["a_col"], d["a_val"])
    B = W.Csr(int(d["b_rows"]), int(d["b_cols"]), d["b_rowptr"], d["b_col"], d["b_val"])
    ref = {"rowptr": d["c_rowptr"], "col": d["c_col"], "val": d["c_val"], "absum": d["c_absum"],
           "nterms": d["c_nterms"], "products": int(d["products"])}
    return A, B, ref


def test_fixtures_present():
    assert len(GOLD) >= 5


@pytest.mark.parametrize("path", GOLD, ids=lambda p: p.stem)
def test_oracle_reproduces_golden(path):
    A, B, ref = load(path)
    a = A.to_csc()
    C = oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val,
                      stats=True, threads=3)
    for k in ("rowptr", "col", "val", "absum", "nterms"):
        assert np.array_equal(C[k], ref[k]), k
    assert C["products"] == ref["products"]


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLD, ids=lambda p: p.stem)
def test_gpu_matches_golden(path):
    import spgemm_b200 as sg
    from helpers import assert_structure_equal, assert_values_close, plain_tolerance
    A, B, ref = load(path)
    with sg.Handle() as h:
        C = h.multiply_host(A.to_csc(), B)
    assert_structure_equal(C.rowptr, C.col, ref["rowptr"], ref["col"])
    assert_values_close(C.val, ref, plain_tolerance(ref))
