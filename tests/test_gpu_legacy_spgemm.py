"""The legacy spGEMM() family (include/spGEMM.h) end to end: a C driver
compiled against include/ and the library runs both the one-call spGEMM()
and the individual passes on Matrix-Market files; C, nnzC and the heavy-row
count are checked against the oracle (values are sums of 1.1 * 1.1: the
reference reader forces 1.1). Also drives the passes through ctypes to check
the module globals and the out-of-order error path."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import spgemm_b200 as sg
from spgemm_b200 import workloads as W
from helpers import assert_structure_equal, assert_values_close, plain_tolerance

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("legacy")
    exe = d / "legacy_spgemm"
    libdir = sg.LIB_PATH.parent
    subprocess.run(["gcc", "-O2", f"-I{ROOT / 'include'}",
                    str(ROOT / "spgemm_b200/examples/legacy_spgemm.c"),
                    f"-L{libdir}", "-lspgemm_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                   check=True)
    return exe


def write_mtx(path, M: W.Csr):
    r = np.repeat(np.arange(M.rows), np.diff(M.rowptr))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{M.cols} {M.rows} {M.nnz}\n")
        for i, j in zip(r, M.col):
            f.write(f"{i + 1} {j + 1} 0.5\n")


def ref_of(A, B):
    a1 = W.Csr(A.rows, A.cols, A.rowptr, A.col, np.full(A.nnz, 1.1, np.float32))
    b1 = W.Csr(B.rows, B.cols, B.rowptr, B.col, np.full(B.nnz, 1.1, np.float32))
    a = a1.to_csc()
    return oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, b1.rowptr, b1.col, b1.val,
                         stats=True)


@pytest.mark.parametrize("mode", ["spGEMM", "passes"])
@pytest.mark.parametrize("scale", [9, 13])
def test_legacy_driver_matches_oracle(driver, tmp_path, mode, scale):
    A = W.rmat(scale, 8, 40 + scale)
    B = W.rmat(scale, 8, 50 + scale)
    write_mtx(tmp_path / "a.mtx", A)
    write_mtx(tmp_path / "b.mtx", B)
    out = tmp_path / "c.txt"
    args = [str(driver), str(tmp_path / "a.mtx"), str(tmp_path / "b.mtx"), str(out)]
    if mode == "passes":
        args.append("passes")
    res = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    lines = res.stdout.strip().splitlines()
    ref = ref_of(A, B)
    p_i = oracle.count_products(A.rows, A.to_csc().colptr, A.to_csc().rowidx, B.rowptr,
                                per_row=True)[1]
    assert int(lines[-2]) == int((p_i > 4096).sum())  # heavy rows printed by cudaPassC
    assert lines[-1] == f"nnzC {len(ref['col'])}"
    data = np.loadtxt(out, skiprows=1, ndmin=2)
    rows = np.repeat(np.arange(A.rows), np.diff(ref["rowptr"]))
    assert np.array_equal(data[:, 0].astype(np.int64), rows)
    assert np.array_equal(data[:, 1].astype(np.int64), ref["col"])
    assert_values_close(data[:, 2].astype(np.float32), ref, plain_tolerance(ref))


class CSC(C.Structure):
    _fields_ = [("header", C.POINTER(C.c_int)), ("ridx", C.POINTER(C.c_int)),
                ("val", C.POINTER(C.c_float)), ("n", C.c_int), ("e", C.c_int)]


class CSR(C.Structure):
    _fields_ = [("header", C.POINTER(C.c_int)), ("cidx", C.POINTER(C.c_int)),
                ("val", C.POINTER(C.c_float)), ("n", C.c_int), ("e", C.c_int)]


def test_legacy_globals_and_state_errors():
    L = sg.lib()
    L.spgemm_set_exit_on_error(0)
    L.spgemm_set_verbose(0)
    try:
        A = W.rmat(11, 12, 3, values="sym")
        B = W.er(A.cols, 9.0, 4)
        a = A.to_csc()
        keep = [np.ascontiguousarray(x) for x in (a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val)]
        ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
        fp = lambda x: x.ctypes.data_as(C.POINTER(C.c_float))
        C.c_int.in_dll(L, "nnzC").value = 0
        # a pass before cudaPass_ is an out-of-order call: reported, not run
        L.cudaPassC.argtypes = [C.c_int]
        L.cudaPassC(A.rows)
        assert L.spgemm_legacy_status() == 5
        CSC.in_dll(L, "CSC_HOST").__init__(ip(keep[0]), ip(keep[1]), fp(keep[2]), A.cols, A.nnz)
        CSR.in_dll(L, "CSR_HOST").__init__(ip(keep[3]), ip(keep[4]), fp(keep[5]), B.rows, B.nnz)
        L.cudaPass0.argtypes = [C.c_int, C.c_int]
        L.cudaPass0(A.rows, A.nnz)
        L.cudaPass2.restype = C.c_int
        nnz = L.cudaPass2()
        ref = oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val,
                            stats=True)
        assert nnz == len(ref["col"]) == C.c_int.in_dll(L, "nnzC").value
        n = A.rows
        ptr = np.ctypeslib.as_array(C.POINTER(C.c_int).in_dll(L, "c_ptr_h"), (n + 1,)).copy()
        col = np.ctypeslib.as_array(C.POINTER(C.c_int).in_dll(L, "c_idx_h"), (nnz,)).copy()
        val = np.ctypeslib.as_array(C.POINTER(C.c_float).in_dll(L, "c_val_h"), (nnz,)).copy()
        assert_structure_equal(ptr, col, ref["rowptr"], ref["col"])
        assert_values_close(val, ref, plain_tolerance(ref))
        rupp = np.ctypeslib.as_array(C.POINTER(C.c_int).in_dll(L, "RUPP_HOST"), (n + 1,)).copy()
        p_i = oracle.count_products(A.rows, a.colptr, a.rowidx, B.rowptr, per_row=True)[1]
        assert rupp[0] == 0 and np.array_equal(rupp[1:], p_i)
        wls = np.ctypeslib.as_array(C.POINTER(C.c_int).in_dll(L, "WLS_HOST"), (n,)).copy()
        assert np.array_equal(wls, np.diff(a.colptr) * np.diff(B.rowptr))
        dom_n = np.ctypeslib.as_array(C.POINTER(C.c_int).in_dll(L, "domN"), (1,))[0]
        assert dom_n == int((p_i > 4096).sum())
    finally:
        L.spgemm_set_exit_on_error(1)
        L.spgemm_set_verbose(1)


class WltData(C.Structure):
    _fields_ = [("idx", C.c_int), ("base_idx", C.c_int), ("num_of_row_elements", C.c_int),
                ("num_of_col_elements", C.c_int)]


class Wlt(C.Structure):
    _fields_ = [("data", C.POINTER(WltData)), ("threadblocks", C.c_int), ("workloads", C.c_int)]


class WltDataCheat(C.Structure):
    _fields_ = [("ridx", C.c_int), ("cidx", C.c_int), ("base_idx", C.c_int),
                ("num_of_row_elements", C.c_int), ("num_of_col_elements", C.c_int)]


class WltCheat(C.Structure):
    _fields_ = [("data", C.POINTER(WltDataCheat)), ("threadblocks", C.c_int), ("workloads", C.c_int)]


def test_spgemm_with_workload_tables():
    """spGEMM() with a per-k table and a non-trivial 2-D tile table (heavy
    outer products split into 7 x 5 tiles) gives the oracle's C; tables that
    do not describe the operands are rejected with SPGEMM_ERR_INVALID."""
    L = sg.lib()
    L.spgemm_set_exit_on_error(0)
    L.spgemm_set_verbose(0)
    try:
        A = W.rmat(11, 12, 8, values="sym")
        B = W.rmat(11, 10, 9, values="sym")
        a = A.to_csc()
        keep = [np.ascontiguousarray(x) for x in (a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val)]
        ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
        fp = lambda x: x.ctypes.data_as(C.POINTER(C.c_float))
        csc = CSC(ip(keep[0]), ip(keep[1]), fp(keep[2]), A.cols, A.nnz)
        csr = CSR(ip(keep[3]), ip(keep[4]), fp(keep[5]), B.rows, B.nnz)
        L.makeWLT.restype = Wlt
        L.makeWLT.argtypes = [CSC, CSR]
        L.makeWLT_cheat.restype = WltCheat
        L.makeWLT_cheat.argtypes = [CSC, CSR, C.c_int, C.c_int, C.c_int]
        L.spGEMM.restype = C.c_int
        L.spGEMM.argtypes = [CSC, CSR, Wlt, WltCheat, C.c_int]
        wl = L.makeWLT(csc, csr)
        wc = L.makeWLT_cheat(csc, csr, 7, 5, 200)
        assert wl.threadblocks > 0 and wc.threadblocks > 0
        # at least one outer product is split into several tiles
        tiles = [wc.data[t] for t in range(wc.threadblocks)]
        assert any(t.num_of_col_elements == 7 or t.num_of_row_elements == 5 for t in tiles)
        ref = oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val,
                            stats=True)
        nnz = L.spGEMM(csc, csr, wl, wc, 1)
        assert nnz == len(ref["col"])
        n = A.rows
        ptr = np.ctypeslib.as_array(C.POINTER(C.c_int).in_dll(L, "c_ptr_h"), (n + 1,)).copy()
        col = np.ctypeslib.as_array(C.POINTER(C.c_int).in_dll(L, "c_idx_h"), (nnz,)).copy()
        val = np.ctypeslib.as_array(C.POINTER(C.c_float).in_dll(L, "c_val_h"), (nnz,)).copy()
        assert_structure_equal(ptr, col, ref["rowptr"], ref["col"])
        assert_values_close(val, ref, plain_tolerance(ref))
        # a tile that leaves its B row
        t0 = wc.data[0]
        saved = t0.num_of_row_elements
        wc.data[0].num_of_row_elements = saved + 10 ** 6
        assert L.spGEMM(csc, csr, wl, wc, 1) == -1
        assert L.spgemm_legacy_status() == 1
        # with cheat == 0 the tile table is not consulted
        assert L.spGEMM(csc, csr, wl, wc, 0) == len(ref["col"])
        wc.data[0].num_of_row_elements = saved
        # a dropped tile leaves its outer product uncovered
        short = WltCheat(wc.data, wc.threadblocks - 1, wc.workloads)
        if wc.threadblocks > 1:
            assert L.spGEMM(csc, csr, wl, short, 1) == -1
        # a per-k record with the wrong element count
        wl.data[0].num_of_col_elements += 1
        assert L.spGEMM(csc, csr, wl, wc, 1) == -1
        wl.data[0].num_of_col_elements -= 1
        assert L.spGEMM(csc, csr, wl, wc, 1) == len(ref["col"])
        L.freeWLT.argtypes = [C.POINTER(Wlt)]
        L.freeWLTC.argtypes = [C.POINTER(WltCheat)]
        L.freeWLT(C.byref(wl))
        L.freeWLTC(C.byref(wc))
    finally:
        L.spgemm_set_exit_on_error(1)
        L.spgemm_set_verbose(1)
