"""Seeded generators of the benchmark configurations (no GPU): determinism,
CSR validity (sorted, distinct columns per row), and the distributions each
configuration states."""
import numpy as np
import pytest

from spgemm_b200 import workloads as W


def check_csr(M):
    rp = np.asarray(M.rowptr, np.int64)
    assert rp[0] == 0 and rp[-1] == M.nnz and np.all(np.diff(rp) >= 0)
    assert M.col.min(initial=0) >= 0 and (M.nnz == 0 or M.col.max() < M.cols)
    for i in range(min(M.rows, 2000)):
        c = M.col[rp[i]:rp[i + 1]]
        assert np.all(np.diff(c) > 0), i  # sorted, distinct


@pytest.mark.parametrize("gen", [
    lambda: W.er(3000, 8.0, 5),
    lambda: W.er_poisson(3000, 12.0, 6),
    lambda: W.rmat(12, 16, 7),
    lambda: W.rmat(12, 9.5, 8, n=3000, values="sym"),
    lambda: W.rmat_poisson(3000, 20.0, 9),
    lambda: W.stencil27(8, seed=1),
])
def test_generators_are_seeded_and_valid(gen):
    A, B = gen(), gen()
    check_csr(A)
    assert np.array_equal(A.rowptr, B.rowptr) and np.array_equal(A.col, B.col)
    assert np.array_equal(A.val, B.val)


def test_rmat_poisson_rows_and_skew():
    n, lam = 50000, 16.0
    A = W.rmat_poisson(n, lam, 3)
    deg = np.diff(A.rowptr)
    assert abs(deg.mean() - lam) < 0.2 and abs(deg.var() - lam) < 1.0   # Poisson(lam) rows
    cnt = np.bincount(A.col, minlength=n)
    # R-MAT column marginal: the lowest columns are far more popular than the top ones
    assert cnt[: n // 64].sum() > 10 * cnt[-(n // 64):].sum()
    assert np.all((A.val >= -1) & (A.val <= 1))


def test_batch_specs_follow_the_configuration():
    specs = W.batch_specs(512, 1000)
    assert len(specs) == 512
    kinds = [s[0] for s in specs]
    assert kinds.count("er") == kinds.count("rmat") == 256
    ns = np.array([s[1] for s in specs])
    lams = np.array([s[2] for s in specs])
    assert ns.min() >= 1000 and ns.max() <= 200000
    assert 4.0 <= lams.min() and lams.max() <= 32.0
    # log-uniform n: the median sits near the geometric mean of the range
    assert 0.5 < np.median(ns) / np.sqrt(1000 * 200000) < 2.0
    assert [s[3] for s in specs] == [1000 + i for i in range(512)]
    assert W.batch_specs(512, 1000) == specs


def test_stencil_counts_are_exact():
    A = W.stencil27(6, seed=0)
    assert A.rows == 216 and A.nnz == (3 * 6 - 2) ** 3  # 16^3 = 4096 couplings
