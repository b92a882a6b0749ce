"""The reference's mm.h call protocol end to end: a C driver equivalent to the
reference's src/main.cu, compiled against include/ and the library, run on a
Matrix-Market file. Its printed P and nnzC, and the C it writes, are checked
against the oracle (values are sums of 1.1 * 1.1: the reader forces 1.1)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import spgemm_b200 as sg
from spgemm_b200 import workloads as W

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def outer_bin(tmp_path_factory):
    d = tmp_path_factory.mktemp("outer")
    exe = d / "outer"
    libdir = sg.LIB_PATH.parent
    subprocess.run(["gcc", "-O2", f"-I{ROOT / 'include'}", str(ROOT / "spgemm_b200/examples/outer.c"),
                    f"-L{libdir}", "-lspgemm_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    return exe


def write_mtx(path, M: W.Csr):
    r = np.repeat(np.arange(M.rows), np.diff(M.rowptr))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{M.cols} {M.rows} {M.nnz}\n")     # first token -> num_cols (reference reader)
        for i, j in zip(r, M.col):
            f.write(f"{i + 1} {j + 1} 0.5\n")


@pytest.mark.parametrize("scale", [9, 12])
def test_outer_driver_matches_oracle(outer_bin, tmp_path, scale):
    A = W.rmat(scale, 8, 21)
    mtx = tmp_path / "a.mtx"
    write_mtx(mtx, A)
    out = tmp_path / "c.txt"
    res = subprocess.run([str(outer_bin), str(mtx), str(mtx), str(out)], capture_output=True,
                         text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    lines = res.stdout.strip().splitlines()
    # readMTX prints twice, then "P P", then "nnzC nnzCf"
    ones = W.Csr(A.rows, A.cols, A.rowptr, A.col, np.full(A.nnz, 1.1, np.float32))
    a = ones.to_csc()
    ref = oracle.spgemm(A.rows, A.cols, a.colptr, a.rowidx, a.val, ones.rowptr, ones.col, ones.val,
                        stats=True)
    p1, p2 = map(int, lines[2].split())
    assert p1 == p2 == ref["products"]
    nnzc, nnzcf = map(int, lines[3].split())
    assert nnzc == len(ref["col"]) and nnzcf == nnzc
    data = np.loadtxt(out, skiprows=1, ndmin=2)
    assert np.array_equal(data[:, 1].astype(np.int64), ref["col"])
    rows = np.repeat(np.arange(A.rows), np.diff(ref["rowptr"]))
    assert np.array_equal(data[:, 0].astype(np.int64), rows)
    tol = 2.0 * (ref["nterms"] * 2.0 ** -24 * ref["absum"] + 2.0 ** -24 * np.abs(ref["val"])) + 1e-6
    assert (np.abs(data[:, 2] - ref["val"]) <= tol).all()


def test_unsorted_coo_is_sorted_on_the_device():
    """cudaCOO2CM on triplets that skip sortCOO: the reference protocol
    requires sorted input; the library sorts on the device and returns the
    same compressed matrix as for the sorted triplets."""
    import ctypes as C
    L = sg.lib()
    L.spgemm_set_verbose(0)
    try:
        rng = np.random.default_rng(4)
        n = 300
        r = rng.integers(0, n, 4000)
        c = rng.integers(0, n, 4000)
        v = rng.uniform(-1, 1, 4000).astype(np.float32)
        key = np.unique(r * n + c)  # distinct positions
        r, c, v = key // n, key % n, v[:len(key)]
        perm = rng.permutation(len(key))
        for major in ("row", "col"):
            kind = sg.ROW_MAJOR if major == "row" else sg.COL_MAJOR
            order = np.lexsort((c, r)) if major == "row" else np.lexsort((r, c))
            outs = []
            for idx in (order, perm):
                trip = (sg.Triplet * len(idx))(*[(int(r[k]), int(c[k]), float(v[k])) for k in idx])
                coo = sg.COO(C.cast(trip, C.POINTER(sg.Triplet)), len(idx), n, n, kind)
                M = L.cudaCOO2CM(coo)
                assert L.spgemm_legacy_status() == 0
                outs.append([np.ctypeslib.as_array(M.ptr, (n + 1,)).copy(),
                             np.ctypeslib.as_array(M.idx, (M.nnz,)).copy(),
                             np.ctypeslib.as_array(M.val, (M.nnz,)).copy()])
                L.cmFree(C.byref(M))
            for a, b in zip(*outs):
                assert np.array_equal(a, b)
    finally:
        L.spgemm_set_verbose(1)


def _coo_of(M, col_major):
    """Triplets of host CSR M sorted as the protocol wants: by (column, row)
    for the COL_MAJOR operand A, by (row, column) for the ROW_MAJOR B."""
    r = np.repeat(np.arange(M.rows), np.diff(M.rowptr)).astype(np.int64)
    c = M.col.astype(np.int64)
    order = np.lexsort((r, c)) if col_major else np.lexsort((c, r))
    trip = (sg.Triplet * max(M.nnz, 1))()
    for t, k in enumerate(order):
        trip[t] = (int(r[k]), int(c[k]), float(M.val[k]))
    return trip


def test_dense_chunk_product_matches_oracle():
    """cudaDCGEMM (dense-chunk strategy: rows in dense column windows) right
    after cudaInitGEMM gives the oracle's C, and leaves the handle's tuning
    in place for a following cudaBinGEMM + cudaMergeGEMM product."""
    import ctypes as C
    L = sg.lib()
    L.spgemm_set_verbose(0)
    try:
        A = W.rmat(12, 12, 8, values="sym")
        B = W.rmat(12, 10, 9, values="sym")
        ta, tb = _coo_of(A, True), _coo_of(B, False)
        ca = sg.COO(C.cast(ta, C.POINTER(sg.Triplet)), A.nnz, A.cols, A.rows, sg.COL_MAJOR)
        cb = sg.COO(C.cast(tb, C.POINTER(sg.Triplet)), B.nnz, B.cols, B.rows, sg.ROW_MAJOR)
        Ah = L.cudaCOO2CM(ca)
        Bh = L.cudaCOO2CM(cb)
        a = A.to_csc()
        ref = oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val,
                            stats=True)
        L.spgemm_get_result.restype = C.c_int
        for dense in (True, False):
            Cm = L.cudaInitGEMM(Ah, Bh)
            if dense:
                L.cudaDCGEMM(Ah, Bh, Cm)
            else:
                L.cudaBinGEMM(Ah, Bh, Cm)
                L.cudaMergeGEMM(Cm)
            R = sg.CM()
            assert L.spgemm_get_result(C.byref(R)) == 0
            ptr = np.ctypeslib.as_array(R.ptr, (R.num_rows + 1,)).copy()
            col = np.ctypeslib.as_array(R.idx, (max(R.nnz, 1),))[:R.nnz].copy()
            val = np.ctypeslib.as_array(R.val, (max(R.nnz, 1),))[:R.nnz].copy()
            L.cmFree(C.byref(R))
            from helpers import assert_structure_equal, assert_values_close, plain_tolerance
            assert_structure_equal(ptr, col, ref["rowptr"], ref["col"])
            assert_values_close(val, ref, plain_tolerance(ref))
        for M in (Ah, Bh):
            L.cmFree(C.byref(M))
    finally:
        L.spgemm_set_verbose(1)
