"""Generate the golden fixtures in this directory: small seeded inputs and
their FP64 products from the oracle (oracle/spgemm_oracle.c), cross-checked
here against scipy.sparse before being written. Run from the repository root:

    python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np
import scipy.sparse as sp

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle  # noqa: E402
from spgemm_b200 import workloads as W  # noqa: E402

CASES = {
    "er64": lambda: (W.er(64, 5.0, 11), W.er(64, 5.0, 12)),
    "rmat8": lambda: (W.rmat(8, 8, 3, values="sym"),) * 2,
    "stencil6": lambda: (W.stencil27(6, seed=1),) * 2,
    "rect_40x70x50": lambda: (W.er(40, 6.0, 5, cols=70), W.er(70, 4.0, 6, cols=50)),
    "galerkin4_AP": lambda: (W.stencil27(4, values="laplace"), W.prolongator(4)),
}


def product(A, B):
    a = A.to_csc()
    return oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val,
                         stats=True, threads=1)


def main():
    out = Path(__file__).resolve().parent
    for name, make in CASES.items():
        A, B = make()
        C = product(A, B)
        sA = sp.csr_matrix((A.val, A.col, A.rowptr), shape=(A.rows, A.cols)).astype(np.float64)
        sB = sp.csr_matrix((B.val, B.col, B.rowptr), shape=(B.rows, B.cols)).astype(np.float64)
        ref = (sA @ sB).toarray()
        r = np.repeat(np.arange(A.rows), np.diff(C["rowptr"]))
        assert np.allclose(C["val"], ref[r, C["col"]], rtol=1e-12, atol=1e-12), name
        np.savez_compressed(
            out / f"{name}.npz",
            a_rows=A.rows, a_cols=A.cols, a_rowptr=A.rowptr, a_col=A.col, a_val=A.val,
            b_rows=B.rows, b_cols=B.cols, b_rowptr=B.rowptr, b_col=B.col, b_val=B.val,
            c_rowptr=C["rowptr"], c_col=C["col"], c_val=C["val"], c_absum=C["absum"],
            c_nterms=C["nterms"], products=C["products"])
        print(name, A.rows, B.cols, len(C["col"]))


if __name__ == "__main__":
    main()
