"""spgemm_b200: sm_100a SpGEMM engine (C = A * B, sparse FP32).

Python view of the C ABI in ``include/spgemm_b200.h`` / ``include/mm.h``,
loaded from the in-tree ``libspgemm_b200.so`` with ctypes. There is no
fallback: if the library is missing, importing ``lib()`` raises.

* ``Handle``       -- the handle API (symbolic / numeric / multiply, device
                      pointers or host arrays, precision modes, statistics);
* ``legacy``       -- the reference's mm.h call protocol (cudaCOO2CM ->
                      cudaInitGEMM -> cudaCategorizeGEMM -> cudaBinGEMM ->
                      cudaMergeGEMM) plus readMTX / sortCOO;
* ``workloads``    -- seeded synthetic inputs of the benchmark configurations.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .workloads import Csc, Csr

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libspgemm_b200.so"

ROW_MAJOR = 0
COL_MAJOR = 1
PLAIN = 0
COMPENSATED = 1

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "allocation failed",
          4: "nnz(C) exceeds int32", 5: "call out of order", 6: "device-side check failed",
          7: "size exceeds a documented maximum"}


class SpgemmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"spgemm status {status} ({STATUS.get(status, '?')}): {msg}")
        self.status = status


class CM(C.Structure):
    """The reference's CompressedMatrix (include/cm.h)."""
    _fields_ = [("ptr", C.POINTER(C.c_int)), ("idx", C.POINTER(C.c_int)),
                ("val", C.POINTER(C.c_float)), ("nnz", C.c_int), ("num_rows", C.c_int),
                ("num_cols", C.c_int), ("type", C.c_bool)]


class Triplet(C.Structure):
    _fields_ = [("ridx", C.c_int), ("cidx", C.c_int), ("val", C.c_float)]


class COO(C.Structure):
    """The reference's coo (include/coo.h)."""
    _fields_ = [("data", C.POINTER(Triplet)), ("nnz", C.c_int), ("num_cols", C.c_int),
                ("num_rows", C.c_int), ("type", C.c_bool)]


class Tuning(C.Structure):
    """spgemm_tuning (include/spgemm_b200.h)."""
    _fields_ = [("warp_p_max", C.c_int), ("warp_table_max", C.c_int),
                ("warp_cap_max", C.c_int), ("long_p", C.c_int), ("long_o_num", C.c_int),
                ("slice_cap", C.c_int), ("slice_cols", C.c_int), ("sym_window", C.c_int),
                ("keep_bitmaps", C.c_int), ("mid_o_min", C.c_int), ("mid_cols", C.c_int),
                ("long_rows", C.c_int), ("esc_p_min", C.c_int), ("esc_span_min", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Stats(C.Structure):
    _fields_ = [("intermediate_products", C.c_longlong), ("nnz_c", C.c_longlong),
                ("rows_per_symbolic_bin", C.c_int * 16), ("rows_per_numeric_bin", C.c_int * 16),
                ("long_row_slices", C.c_int), ("kernel_launches", C.c_longlong),
                ("warp_overflow_rows", C.c_int)]


_lib = None


def lib():
    """The loaded libspgemm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m spgemm_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        vp, ip, fp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_float)
        L.spgemm_version.restype = C.c_char_p
        L.spgemm_status_string.restype = C.c_char_p
        L.spgemm_last_error.restype = C.c_char_p
        L.spgemm_last_error.argtypes = [vp]
        L.spgemm_create.argtypes = [C.POINTER(vp)]
        L.spgemm_destroy.argtypes = [vp]
        L.spgemm_set_stream.argtypes = [vp, vp]
        L.spgemm_set_precision.argtypes = [vp, C.c_int]
        L.spgemm_symbolic.argtypes = [vp, CM, CM, C.POINTER(C.c_longlong)]
        L.spgemm_numeric.argtypes = [vp, ip, ip, fp]
        L.spgemm_multiply.argtypes = [vp, CM, CM, C.POINTER(CM)]
        L.spgemm_get_stats.argtypes = [vp, C.POINTER(Stats)]
        L.spgemm_multiply_host.argtypes = [vp, CM, CM, C.POINTER(CM)]
        L.spgemm_multiply_host_to.argtypes = [vp, CM, CM, ip, ip, fp, C.c_longlong,
                                              C.POINTER(C.c_longlong)]
        L.spgemm_set_copy_chunk.argtypes = [vp, C.c_longlong]
        L.spgemm_get_result.argtypes = [C.POINTER(CM)]
        L.spgemm_set_verbose.argtypes = [C.c_int]
        L.spgemm_set_exit_on_error.argtypes = [C.c_int]
        L.spgemm_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.spgemm_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.spgemm_set_profiling.argtypes = [vp, C.c_int]
        L.spgemm_reset_kernel_times.argtypes = [vp]
        L.spgemm_get_kernel_times.argtypes = [vp, C.c_char_p, C.c_int, C.POINTER(C.c_double),
                                              C.POINTER(C.c_longlong), C.c_int]
        L.spgemm_batch_plan.argtypes = [vp, C.c_int, C.POINTER(CM), C.POINTER(CM),
                                        C.POINTER(C.c_longlong)]
        L.spgemm_batch_execute.argtypes = [vp, C.c_int]
        L.spgemm_batch_offsets.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.spgemm_batch_result.argtypes = [vp, C.c_int, C.POINTER(CM)]
        L.spgemm_batch_copy_result.argtypes = [vp, C.c_int, ip, ip, fp]
        L.spgemm_batch_copy_all.argtypes = [vp, vp, vp, vp]
        L.spgemm_read_mtx.argtypes = [C.POINTER(COO), C.c_char_p]
        L.spgemm_coo_to_cm.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp]
        L.cmFree.argtypes = [C.POINTER(CM)]
        L.cudaCOO2CM.restype = CM
        L.cudaCOO2CM.argtypes = [COO]
        L.cudaInitGEMM.restype = CM
        L.cudaInitGEMM.argtypes = [CM, CM]
        L.cudaCategorizeGEMM.argtypes = [CM, CM]
        L.cudaBinGEMM.argtypes = [CM, CM, CM]
        L.cudaSimpleGEMM.argtypes = [CM, CM, CM]
        L.cudaDCGEMM.argtypes = [CM, CM, CM]
        L.cudaMergeGEMM.argtypes = [CM]
        L.readMTX.argtypes = [C.POINTER(COO), C.c_char_p]
        L.readCOO.argtypes = [C.POINTER(COO), C.c_char_p]
        L.sortCOO.argtypes = [COO]
        L.freeCOO.argtypes = [C.POINTER(COO)]
        L.initCOO.argtypes = [C.POINTER(COO)]
        _lib = L
    return _lib


def read_mtx(path):
    """Matrix-Market file through the library's value-preserving reader
    (spgemm_read_mtx): (rows, cols, row indices, column indices, values) as
    numpy arrays, entries in file order with mirrored ones after their source.
    Raises SpgemmError on a malformed file."""
    L = lib()
    m = COO()
    st = L.spgemm_read_mtx(C.byref(m), str(path).encode())
    if st != 0:
        raise SpgemmError(st, f"spgemm_read_mtx({path})")
    try:
        n = m.nnz
        raw = np.ctypeslib.as_array(C.cast(m.data, C.POINTER(C.c_int)), (3 * n,)) if n else np.zeros(0, np.int32)
        t = raw.reshape(n, 3).copy() if n else np.zeros((0, 3), np.int32)
        vals = t[:, 2].view(np.float32).copy()
        return m.num_rows, m.num_cols, t[:, 0].astype(np.int64), t[:, 1].astype(np.int64), vals
    finally:
        L.freeCOO(C.byref(m))


def version() -> str:
    return lib().spgemm_version().decode()


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def host_cm(ptr, idx, val, rows, cols, kind):
    """A CM over host numpy arrays (the arrays must outlive the call)."""
    ptr, idx, val = _i32(ptr), _i32(idx), _f32(val)
    m = CM(ptr.ctypes.data_as(C.POINTER(C.c_int)), idx.ctypes.data_as(C.POINTER(C.c_int)),
           val.ctypes.data_as(C.POINTER(C.c_float)), len(idx), rows, cols, kind)
    return m, (ptr, idx, val)


def device_cm(ptr: int, idx: int, val: int, nnz: int, rows: int, cols: int, kind: int) -> CM:
    """A CM over device addresses (e.g. torch tensors' data_ptr())."""
    return CM(C.cast(C.c_void_p(ptr), C.POINTER(C.c_int)), C.cast(C.c_void_p(idx), C.POINTER(C.c_int)),
              C.cast(C.c_void_p(val), C.POINTER(C.c_float)), nnz, rows, cols, kind)


def as_host_cm(M):
    if isinstance(M, Csc):
        return host_cm(M.colptr, M.rowidx, M.val, M.rows, M.cols, COL_MAJOR)
    return host_cm(M.rowptr, M.col, M.val, M.rows, M.cols, ROW_MAJOR)


class Handle:
    """One engine instance (workspace, stream, precision)."""

    def __init__(self, precision: int = PLAIN):
        self._h = C.c_void_p()
        self._check(lib().spgemm_create(C.byref(self._h)))
        self.set_precision(precision)

    def close(self):
        if self._h:
            lib().spgemm_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st != 0:
            msg = lib().spgemm_last_error(self._h).decode() if self._h else ""
            raise SpgemmError(st, msg)

    def set_precision(self, p: int):
        self._check(lib().spgemm_set_precision(self._h, p))
        self.precision = p

    def set_stream(self, stream_ptr: int):
        self._check(lib().spgemm_set_stream(self._h, C.c_void_p(stream_ptr)))

    def stats(self) -> dict:
        s = Stats()
        self._check(lib().spgemm_get_stats(self._h, C.byref(s)))
        return {"intermediate_products": s.intermediate_products, "nnz_c": s.nnz_c,
                "rows_per_symbolic_bin": list(s.rows_per_symbolic_bin)[:13],
                "warp_overflow_rows": s.warp_overflow_rows,
                "rows_per_numeric_bin": list(s.rows_per_numeric_bin)[:10],
                "long_row_slices": s.long_row_slices, "kernel_launches": s.kernel_launches}

    def tuning(self) -> dict:
        t = Tuning()
        self._check(lib().spgemm_get_tuning(self._h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        """Change tuning fields by name (others keep their current value)."""
        t = Tuning()
        self._check(lib().spgemm_get_tuning(self._h, C.byref(t)))
        for k, v in kw.items():
            if not hasattr(t, k):
                raise KeyError(k)
            setattr(t, k, int(v))
        self._check(lib().spgemm_set_tuning(self._h, C.byref(t)))

    def set_copy_chunk(self, nbytes: int):
        """Bytes of C per device-to-host piece of the host-buffer calls
        (0: one piece after the whole product)."""
        self._check(lib().spgemm_set_copy_chunk(self._h, int(nbytes)))

    def set_profiling(self, on: bool = True):
        self._check(lib().spgemm_set_profiling(self._h, 1 if on else 0))

    def reset_kernel_times(self):
        self._check(lib().spgemm_reset_kernel_times(self._h))

    def kernel_times(self) -> dict:
        """{kernel name: (total ms, launches)} accumulated while profiling."""
        buf = C.create_string_buffer(8192)
        ms = (C.c_double * 128)()
        cnt = (C.c_longlong * 128)()
        k = lib().spgemm_get_kernel_times(self._h, buf, 8192, ms, cnt, 128)
        if k < 0:
            self._check(-k)
        names = buf.value.decode().split("\n")[:k]
        return {nm: (ms[i], cnt[i]) for i, nm in enumerate(names)}

    # ---- host arrays ----
    def multiply_host(self, A, B: Csr) -> Csr:
        """C = A*B from host arrays (A: Csc or Csr, B: Csr); returns host Csr."""
        a, keep_a = as_host_cm(A)
        b, keep_b = as_host_cm(B)
        out = CM()
        self._check(lib().spgemm_multiply_host(self._h, a, b, C.byref(out)))
        try:
            nnz, m = out.nnz, out.num_rows
            rowptr = np.ctypeslib.as_array(out.ptr, (m + 1,)).copy()
            col = np.ctypeslib.as_array(out.idx, (max(nnz, 1),))[:nnz].copy()
            val = np.ctypeslib.as_array(out.val, (max(nnz, 1),))[:nnz].copy()
        finally:
            lib().cmFree(C.byref(out))
        del keep_a, keep_b
        return Csr(m, B.cols, rowptr, col, val)

    def multiply_host_to(self, A, B: Csr, rowptr: np.ndarray, col: np.ndarray, val: np.ndarray) -> int:
        """C = A*B from host arrays into caller-provided host arrays (may be
        pinned); returns nnz(C)."""
        a, keep_a = as_host_cm(A)
        b, keep_b = as_host_cm(B)
        nnz = C.c_longlong()
        self._check(lib().spgemm_multiply_host_to(
            self._h, a, b, rowptr.ctypes.data_as(C.POINTER(C.c_int)),
            col.ctypes.data_as(C.POINTER(C.c_int)), val.ctypes.data_as(C.POINTER(C.c_float)),
            min(len(col), len(val)), C.byref(nnz)))
        del keep_a, keep_b
        return nnz.value

    # ---- device pointers ----
    def symbolic(self, A: CM, B: CM) -> int:
        nnz = C.c_longlong()
        self._check(lib().spgemm_symbolic(self._h, A, B, C.byref(nnz)))
        return nnz.value

    def numeric(self, rowptr: int, col: int, val: int):
        self._check(lib().spgemm_numeric(self._h, C.cast(C.c_void_p(rowptr), C.POINTER(C.c_int)),
                                         C.cast(C.c_void_p(col), C.POINTER(C.c_int)),
                                         C.cast(C.c_void_p(val), C.POINTER(C.c_float))))

    def multiply(self, A: CM, B: CM) -> CM:
        out = CM()
        self._check(lib().spgemm_multiply(self._h, A, B, C.byref(out)))
        return out

    def coo_to_cm(self, d_triplets: int, nnz: int, rows: int, cols: int, kind: int,
                  d_ptr: int, d_idx: int, d_val: int) -> None:
        """Device triplets in any order to CSR (ROW_MAJOR) or CSC (COL_MAJOR)
        in caller device arrays (spgemm_coo_to_cm)."""
        self._check(lib().spgemm_coo_to_cm(self._h, C.c_void_p(d_triplets), nnz, rows, cols, kind,
                                           C.c_void_p(d_ptr), C.c_void_p(d_idx),
                                           C.c_void_p(d_val)))

    # -- batched products (device operands) --------------------------------
    def batch_plan(self, A_list, B_list) -> int:
        """Plan and run the batch C_i = A_i * B_i once; returns total nnz."""
        n = len(A_list)
        if len(B_list) != n:
            raise ValueError("A_list and B_list differ in length")
        self._batch_A = (CM * n)(*A_list)
        self._batch_B = (CM * n)(*B_list)
        self._batch_count = n
        tot = C.c_longlong(0)
        self._check(lib().spgemm_batch_plan(self._h, n, self._batch_A, self._batch_B,
                                            C.byref(tot)))
        return tot.value

    def batch_execute(self, graph: bool = True) -> None:
        self._check(lib().spgemm_batch_execute(self._h, 1 if graph else 0))

    def batch_offsets(self):
        n = self._batch_count
        ro = np.zeros(n + 1, np.int64)
        no = np.zeros(n + 1, np.int64)
        self._check(lib().spgemm_batch_offsets(
            self._h, ro.ctypes.data_as(C.POINTER(C.c_longlong)),
            no.ctypes.data_as(C.POINTER(C.c_longlong))))
        return ro, no

    def batch_result(self, i: int) -> CM:
        out = CM()
        self._check(lib().spgemm_batch_result(self._h, i, C.byref(out)))
        return out

    def batch_copy_all(self, rowptr_ptr: int, col_ptr: int, val_ptr: int) -> None:
        """Copy the packed batch output to host memory at the given addresses."""
        self._check(lib().spgemm_batch_copy_all(self._h, C.c_void_p(rowptr_ptr),
                                                C.c_void_p(col_ptr), C.c_void_p(val_ptr)))

    def batch_copy_result(self, i: int) -> Csr:
        d = self.batch_result(i)
        rowptr = np.zeros(d.num_rows + 1, np.int32)
        col = np.zeros(max(d.nnz, 1), np.int32)
        val = np.zeros(max(d.nnz, 1), np.float32)
        self._check(lib().spgemm_batch_copy_result(
            self._h, i, rowptr.ctypes.data_as(C.POINTER(C.c_int)),
            col.ctypes.data_as(C.POINTER(C.c_int)), val.ctypes.data_as(C.POINTER(C.c_float))))
        return Csr(d.num_rows, d.num_cols, rowptr, col[:d.nnz], val[:d.nnz])


def multiply(A, B: Csr, precision: int = PLAIN) -> Csr:
    """One-shot host-array product."""
    with Handle(precision) as h:
        return h.multiply_host(A, B)
