"""CPU oracle for the SpGEMM path -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only to check results against / as
the timed CPU baseline. The product path (``spgemm_b200``) never imports it.

``liboracle.so`` is the C restatement in ``spgemm_oracle.c`` (see its header
for the reference lines it follows); ``_ref/libref_host.so`` is the
reference's own host reader/sort, compiled from the reference sources by
``make ref`` when the reference tree is present.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_LIB_PATH = HERE / "_ref" / "libref_host.so"


class OracleCSR(C.Structure):
    _fields_ = [
        ("nrows", C.c_int),
        ("nnz", C.c_longlong),
        ("products", C.c_longlong),
        ("rowptr", C.POINTER(C.c_longlong)),
        ("col", C.POINTER(C.c_int)),
        ("val", C.POINTER(C.c_double)),
        ("val32", C.POINTER(C.c_float)),
        ("absum", C.POINTER(C.c_double)),
        ("nterms", C.POINTER(C.c_int)),
    ]


_lib = None


def build() -> None:
    """Compile liboracle.so (and _ref/ when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        ip = C.POINTER(C.c_int)
        fp = C.POINTER(C.c_float)
        L.oracle_spgemm.restype = C.POINTER(OracleCSR)
        L.oracle_spgemm.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, fp, ip, ip, fp, ip,
                                    C.c_int, C.c_int, C.c_int, C.c_int]
        L.oracle_free.argtypes = [C.POINTER(OracleCSR)]
        L.oracle_count_products.restype = C.c_longlong
        L.oracle_count_products.argtypes = [C.c_int, C.c_int, ip, ip, ip,
                                            C.POINTER(C.c_longlong)]
        _lib = L
    return _lib


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def count_products(m, a_colptr, a_rowidx, b_rowptr, per_row=False):
    """P (and optionally the per-row counts) of A*B; A in CSC, B in CSR."""
    a_colptr, a_rowidx, b_rowptr = _i32(a_colptr), _i32(a_rowidx), _i32(b_rowptr)
    kdim = len(a_colptr) - 1
    rp = np.zeros(max(m, 1), np.int64) if per_row else None
    total = lib().oracle_count_products(
        m, kdim, _p(a_colptr, C.c_int), _p(a_rowidx, C.c_int), _p(b_rowptr, C.c_int),
        _p(rp, C.c_longlong) if per_row else None)
    return (int(total), rp[:m]) if per_row else int(total)


def spgemm(m, n, a_colptr, a_rowidx, a_val, b_rowptr, b_colidx, b_val, rows=None,
           mode=0, stats=False, threads=None):
    """C = A*B for the given rows (default: all) on the CPU.

    A: CSC (colptr, rowidx, val); B: CSR (rowptr, colidx, val).
    mode 0: FP64 products and sums (the oracle); mode 1: FP32 (the baseline).
    Returns a dict with rowptr (int64, len(rows)+1), col (int32), val
    (float64 or float32) and, for mode 0 with stats, absum / nterms.
    """
    a_colptr, a_rowidx, a_val = _i32(a_colptr), _i32(a_rowidx), _f32(a_val)
    b_rowptr, b_colidx, b_val = _i32(b_rowptr), _i32(b_colidx), _f32(b_val)
    kdim = len(a_colptr) - 1
    if rows is not None:
        rows = _i32(rows)
    if threads is None:
        threads = os.cpu_count() or 1
    r = lib().oracle_spgemm(
        m, kdim, n, _p(a_colptr, C.c_int), _p(a_rowidx, C.c_int), _p(a_val, C.c_float),
        _p(b_rowptr, C.c_int), _p(b_colidx, C.c_int), _p(b_val, C.c_float),
        _p(rows, C.c_int) if rows is not None else None,
        len(rows) if rows is not None else m, mode, 1 if stats else 0, threads)
    if not r:
        raise MemoryError("oracle_spgemm failed")
    try:
        res = r.contents
        nr, nnz = res.nrows, res.nnz
        out = {
            "rowptr": np.ctypeslib.as_array(res.rowptr, (nr + 1,)).copy(),
            "col": np.ctypeslib.as_array(res.col, (max(nnz, 1),))[:nnz].copy(),
            "products": int(res.products),
        }
        if mode == 0:
            out["val"] = np.ctypeslib.as_array(res.val, (max(nnz, 1),))[:nnz].copy()
            if stats:
                out["absum"] = np.ctypeslib.as_array(res.absum, (max(nnz, 1),))[:nnz].copy()
                out["nterms"] = np.ctypeslib.as_array(res.nterms, (max(nnz, 1),))[:nnz].copy()
        else:
            out["val"] = np.ctypeslib.as_array(res.val32, (max(nnz, 1),))[:nnz].copy()
        return out
    finally:
        lib().oracle_free(r)


REF_MM_PATH = HERE / "_ref" / "ref_mm"


def ref_available() -> bool:
    """True when _ref/ref_mm (the reference's own src/mm.cu built for the CPU) exists."""
    return REF_MM_PATH.exists()


def ref_multiply(m, k, n, a_row, a_col, a_val, b_row, b_col, b_val, workdir):
    """C = A*B by the reference's own engine (src/mm.cu) run on the CPU.

    A (m x k) and B (k x n, square: n == k) are given as COO triplets in any
    order; the driver sorts them with the reference's sortCOO. Returns a dict:
    ``p`` and ``nnzc`` / ``nnzcf`` as the reference prints them
    (src/mm.cu:181, :449), and per row the merged bucket as the reference
    leaves it in its module globals: ``base`` (c_ptr_base), ``cnt``
    (c_ptr_nnz), ``idx`` / ``val`` (c_idx / c_val, columns in merge order).
    """
    if not ref_available():
        raise FileNotFoundError(f"{REF_MM_PATH} is not built (make -C oracle REF=...)")
    workdir = Path(workdir)
    inp, out = workdir / "ref_in.bin", workdir / "ref_out.bin"
    trip = np.dtype([("r", np.int32), ("c", np.int32), ("v", np.float32)])

    def pack(r, c, v):
        t = np.empty(len(r), trip)
        t["r"], t["c"], t["v"] = r, c, v
        return t.tobytes()

    with open(inp, "wb") as f:
        f.write(np.array([m, k, n, len(a_row), len(b_row)], np.int32).tobytes())
        f.write(pack(a_row, a_col, a_val))
        f.write(pack(b_row, b_col, b_val))
    r = subprocess.run([str(REF_MM_PATH), str(inp), str(out)], capture_output=True, text=True,
                       timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"ref_mm failed ({r.returncode}): {r.stderr[-2000:]}")
    lines = [ln.split() for ln in r.stdout.splitlines() if ln.strip()]
    raw = np.fromfile(out, dtype=np.int32)
    mm, p = int(raw[0]), int(raw[1])
    o = 2
    base = raw[o:o + mm + 1]; o += mm + 1
    cnt = raw[o:o + mm]; o += mm
    idx = raw[o:o + p]; o += p
    val = raw[o:o + p].view(np.float32)
    return {"p": int(lines[0][0]), "p_again": int(lines[0][1]), "nnzc": int(lines[1][0]),
            "nnzcf": int(lines[1][1]), "base": base, "cnt": cnt, "idx": idx, "val": val}
