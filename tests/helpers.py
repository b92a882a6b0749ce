"""Shared checks: structure and value comparison of a CSR product against the
FP64 oracle, with the floating-point tolerances stated here."""
import numpy as np

EPS32 = 2.0 ** -24   # unit roundoff of float32 (round to nearest)


def plain_tolerance(ref):
    """Bound on |c_fp32 - c_exact| for FP32 products summed in FP32 in any
    order: each of the n products carries one rounding and the n-1 additions
    at most (n-1) roundings of partial sums bounded by sum|p|, so
    |err| <= gamma_n * sum|p| with gamma_n = n*u/(1-n*u); the extra final
    store adds u*|c|. A factor 2 covers second-order terms."""
    n = ref["nterms"].astype(np.float64)
    g = n * EPS32 / (1.0 - n * EPS32)
    return 2.0 * (g * ref["absum"] + EPS32 * np.abs(ref["val"])) + 1e-37


def compensated_tolerance(ref):
    """Bound for the compensated mode (TwoProduct + TwoSum, i.e. Dot2 of
    Ogita-Rump-Oishi): |err| <= u*|c| + gamma_n^2 * sum|p| before the final
    rounding to float32, which adds u*|c|. FP64-accumulated rows are far
    inside this bound. A factor 2 on each term covers the accumulation of
    the compensation words themselves."""
    n = ref["nterms"].astype(np.float64)
    g = 2.0 * n * EPS32 / (1.0 - 2.0 * n * EPS32)
    return 2.0 * (2.0 * EPS32 * np.abs(ref["val"]) + g * g * ref["absum"]) + 1e-37


def assert_structure_equal(gpu_rowptr, gpu_col, ref_rowptr, ref_col):
    """Bit-exact structure: row pointers, sorted column indices, nnz per row."""
    gpu_rowptr = np.asarray(gpu_rowptr, np.int64)
    ref_rowptr = np.asarray(ref_rowptr, np.int64)
    assert gpu_rowptr.shape == ref_rowptr.shape, (gpu_rowptr.shape, ref_rowptr.shape)
    if not np.array_equal(gpu_rowptr, ref_rowptr):
        bad = np.nonzero(gpu_rowptr != ref_rowptr)[0][:5]
        raise AssertionError(f"row pointers differ at {bad}: gpu {gpu_rowptr[bad]} ref {ref_rowptr[bad]}")
    gpu_col = np.asarray(gpu_col)
    ref_col = np.asarray(ref_col)
    if not np.array_equal(gpu_col, ref_col):
        bad = np.nonzero(gpu_col != ref_col)[0][:5]
        raise AssertionError(f"column indices differ at {bad}: gpu {gpu_col[bad]} ref {ref_col[bad]}")


def assert_values_close(gpu_val, ref, tol):
    err = np.abs(np.asarray(gpu_val, np.float64) - ref["val"])
    bad = err > tol
    if bad.any():
        i = np.nonzero(bad)[0][:5]
        raise AssertionError(
            f"{int(bad.sum())} values out of tolerance, e.g. idx {i}: gpu {np.asarray(gpu_val)[i]} "
            f"ref {ref['val'][i]} tol {tol[i]} nterms {ref['nterms'][i]}")


def rel_error_report(gpu_val, ref):
    """max |c_hat - c| / |c| over entries with c != 0, the count of c == 0
    entries and the condition sum|p| / |c| of the worst entry."""
    c = ref["val"]
    nz = c != 0
    err = np.abs(np.asarray(gpu_val, np.float64) - c)
    rel = np.zeros_like(c)
    rel[nz] = err[nz] / np.abs(c[nz])
    worst = int(np.argmax(rel)) if rel.size else 0
    return {"max_rel": float(rel.max()) if rel.size else 0.0,
            "zero_entries": int((~nz).sum()),
            "worst_cond": float(ref["absum"][worst] / abs(c[worst])) if rel.size and nz[worst] else 0.0}
