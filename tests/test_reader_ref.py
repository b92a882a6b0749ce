"""Host reader / sort / copy: ours against the reference's own code
(src/coo.cpp, src/cm.cpp compiled in place into oracle/_ref by
`make -C oracle ref`). CPU only; skipped when the reference build is absent."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
import spgemm_b200 as sg

REF = oracle.REF_LIB_PATH
pytestmark = pytest.mark.skipif(not REF.exists(), reason="oracle/_ref not built (no reference tree)")


def ref_lib():
    L = C.CDLL(str(REF))
    L.readMTX.argtypes = [C.POINTER(sg.COO), C.c_char_p]
    L.readCOO.argtypes = [C.POINTER(sg.COO), C.c_char_p]
    L.sortCOO.argtypes = [sg.COO]
    L.copyCOO.argtypes = [sg.COO]
    L.copyCOO.restype = sg.COO
    L.initCOO.argtypes = [C.POINTER(sg.COO)]
    L.setCOOtype.argtypes = [C.POINTER(sg.COO), C.c_bool]
    return L


def ours():
    L = sg.lib()
    L.copyCOO.argtypes = [sg.COO]
    L.copyCOO.restype = sg.COO
    L.setCOOtype.argtypes = [C.POINTER(sg.COO), C.c_bool]
    return L


def triplets(c: sg.COO):
    n = c.nnz
    if n == 0:
        return np.zeros((0, 3))
    arr = np.ctypeslib.as_array(C.cast(c.data, C.POINTER(C.c_int)), (n * 3,)).copy()
    r, cc = arr[0::3], arr[1::3]
    v = arr[2::3].view(np.float32)
    return np.stack([r.astype(np.float64), cc.astype(np.float64), v.astype(np.float64)], 1)


def read_both(path, fn="readMTX", typ=sg.ROW_MAJOR):
    res = []
    for L in (ref_lib(), ours()):
        c = sg.COO()
        L.initCOO(C.byref(c))
        L.setCOOtype(C.byref(c), typ)
        getattr(L, fn)(C.byref(c), str(path).encode())
        res.append(c)
    return res


def assert_same(a: sg.COO, b: sg.COO):
    assert (a.nnz, a.num_cols, a.num_rows) == (b.nnz, b.num_cols, b.num_rows)
    assert np.array_equal(triplets(a), triplets(b))


GENERAL = """%%MatrixMarket matrix coordinate real general
% a comment line
%another
5 4 7
1 1 1.5
2 3 -2
5 4 3.25
3 3 1
1 4 0
4 2 7
2 1 2
"""
SYMMETRIC = """%%MatrixMarket matrix coordinate real symmetric
4 4 5
1 1 2
2 1 3
3 2 1
4 4 1
4 1 7
"""
PATTERN = """%%MatrixMarket matrix coordinate pattern general
3 3 4
1 1
2 2
3 1
1 3
"""


@pytest.mark.parametrize("text", [GENERAL, SYMMETRIC, PATTERN], ids=["general", "symmetric", "pattern"])
def test_readmtx_matches_reference(tmp_path, text, capfd):
    p = tmp_path / "m.mtx"
    p.write_text(text)
    a, b = read_both(p)
    assert_same(a, b)
    out = capfd.readouterr().out.splitlines()
    assert len(out) == 2 and out[0] == out[1]      # both print "0 num_cols num_rows"


def test_readmtx_random_and_sort(tmp_path):
    rng = np.random.default_rng(0)
    n, nnz = 300, 2000
    keys = np.unique(rng.integers(0, n * n, nnz))
    lines = ["%%MatrixMarket matrix coordinate real general", f"{n} {n} {len(keys)}"]
    for k in rng.permutation(keys):
        lines.append(f"{k // n + 1} {k % n + 1} {rng.uniform(-1, 1):.6f}")
    p = tmp_path / "r.mtx"
    p.write_text("\n".join(lines) + "\n")
    for typ in (sg.ROW_MAJOR, sg.COL_MAJOR):
        a, b = read_both(p, typ=typ)
        assert_same(a, b)
        ref_lib().sortCOO(a)
        ours().sortCOO(b)
        assert_same(a, b)
        ca, cb = ref_lib().copyCOO(a), ours().copyCOO(b)
        assert_same(ca, cb)


def test_readcoo_matches_reference(tmp_path):
    p = tmp_path / "a.coo"
    p.write_text("2 5 3\n0 1\n2 3\n4 4\n")
    a, b = read_both(p, fn="readCOO")
    assert_same(a, b)
    p.write_text("3 4 2\n0 1 1.5\n3 2 -0.25\n")
    a, b = read_both(p, fn="readCOO")
    assert_same(a, b)


def test_printcm_matches_reference(tmp_path, capfd):
    # printCM is not in the reference header (C++ linkage there)
    L = C.CDLL(str(REF))
    f = getattr(L, "_Z7printCM16CompressedMatrix")
    f.argtypes = [sg.CM]
    ours_f = sg.lib().printCM
    ours_f.argtypes = [sg.CM]
    ptr = np.array([0, 2, 2, 3], np.int32)
    idx = np.array([0, 2, 1], np.int32)
    val = np.array([1.5, -2.0, 0.25], np.float32)
    for typ in (sg.ROW_MAJOR, sg.COL_MAJOR):
        m, keep = sg.host_cm(ptr, idx, val, 3, 3, typ)
        f(m)
        ref_out = capfd.readouterr().out
        ours_f(m)
        assert capfd.readouterr().out == ref_out
