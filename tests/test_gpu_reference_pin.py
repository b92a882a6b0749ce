"""The sm_100a engine against the reference's own multiply.

The same inputs as tests/test_reference_pin.py (inside the reference's
limits, integer values), multiplied by the engine through the C ABI and by
the reference's src/mm.cu run on the CPU (oracle/_ref/ref_mm). Integer sums
below 2^24 are exact in FP32, so structure AND values must be identical, and
the engine's P and nnz(C) must equal what the reference prints
(src/mm.cu:181, :449). Both precision modes and both A layouts are run.
"""
import numpy as np
import pytest

import oracle
import spgemm_b200 as sg
from ref_cases import cases, run_reference

CASES = cases()

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(),
                                 reason="oracle/_ref/ref_mm not built (needs the reference tree)")]


@pytest.mark.parametrize("precision", [sg.PLAIN, sg.COMPENSATED])
@pytest.mark.parametrize("name", sorted(CASES))
def test_engine_matches_reference_multiply(name, precision, tmp_path):
    A, B = CASES[name]
    rowptr, col, val, printed = run_reference(A, B, tmp_path)
    with sg.Handle(precision) as h:
        C = h.multiply_host(A.to_csc(), B)
        stats = h.stats()
    assert stats["intermediate_products"] == printed["p"]
    assert stats["nnz_c"] == printed["nnzc"]
    assert np.array_equal(C.rowptr.astype(np.int64), rowptr)
    assert np.array_equal(C.col, col)
    assert np.array_equal(C.val, val)


def test_engine_matches_reference_with_a_as_csr(tmp_path):
    A, B = CASES["rect300x200"]
    rowptr, col, val, _ = run_reference(A, B, tmp_path)
    with sg.Handle() as h:
        C = h.multiply_host(A, B)
    assert np.array_equal(C.rowptr.astype(np.int64), rowptr)
    assert np.array_equal(C.col, col)
    assert np.array_equal(C.val, val)
