"""The oracle pinned to the reference's own multiply.

`oracle/_ref/ref_mm` is the reference's live engine, src/mm.cu, compiled
unmodified for the CPU (the launch syntax rewritten mechanically, the CUDA
runtime emulated by oracle/ref_shim/cuda_host_shim.h) and driven through its
own call protocol (sortCOO, cudaCOO2CM x2, cudaInitGEMM, cudaCategorizeGEMM,
cudaBinGEMM, cudaMergeGEMM). On inputs inside the reference's limits
(tests/ref_cases.py) it must agree with the FP64 oracle exactly:
  * the printed intermediate-product count P (src/mm.cu:181) and merged
    nnz(C) (src/mm.cu:449);
  * per row, the set of merged columns and their values (the reference
    emits columns in atomic-arrival order, so rows are compared sorted).
"""
import numpy as np
import pytest

import oracle
from ref_cases import cases, run_reference

CASES = cases()

pytestmark = pytest.mark.skipif(not oracle.ref_available(),
                                reason="oracle/_ref/ref_mm not built (needs the reference tree)")


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_multiply(name, tmp_path):
    A, B = CASES[name]
    rowptr, col, val, printed = run_reference(A, B, tmp_path)
    a = A.to_csc()
    ref = oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val)
    assert printed["p"] == printed["p_again"] == ref["products"]
    assert printed["nnzc"] == len(ref["col"])
    assert printed["nnzcf"] == int((ref["val"] > 1e-4).sum())
    assert np.array_equal(rowptr, ref["rowptr"])
    assert np.array_equal(col, ref["col"])
    assert np.array_equal(val.astype(np.float64), ref["val"])


def test_reference_sums_are_exact_in_these_cases():
    """The cases stay where the reference is exact: integer values, sums
    below 2^24, B rows under 128 entries, P below 2^31."""
    for name, (A, B) in CASES.items():
        assert np.diff(B.rowptr).max() < 128, name
        a = A.to_csc()
        ref = oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val)
        assert ref["products"] < 2 ** 31
        assert np.all(ref["val"] == np.round(ref["val"])) and ref["val"].max() < 2 ** 24
