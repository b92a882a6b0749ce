"""The value-preserving Matrix-Market reader (spgemm_read_mtx, no GPU): every
field and symmetry the format defines for real matrices, against
scipy.io.mmread, and rejection of malformed files."""
import io

import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

import spgemm_b200 as sg


def canon(rows, cols, r, c, v):
    M = sp.coo_matrix((v.astype(np.float64), (r, c)), shape=(rows, cols)).tocsr()
    M.sum_duplicates()
    M.sort_indices()
    return M


def scipy_ref(path):
    M = scipy.io.mmread(str(path))
    return sp.csr_matrix(M)


@pytest.mark.parametrize("kind", ["general", "symmetric", "skew-symmetric", "integer", "pattern"])
def test_reader_matches_scipy(tmp_path, kind):
    rng = np.random.default_rng(11)
    n = 60
    D = sp.random(n, n, density=0.08, random_state=3, format="coo")
    D.data = rng.uniform(-5, 5, D.nnz)
    if kind == "symmetric":
        D = sp.tril(D) + sp.tril(D, -1).T
    elif kind == "skew-symmetric":
        D = sp.tril(D, -1) - sp.tril(D, -1).T
    elif kind == "integer":
        D.data = np.round(D.data * 10)
    elif kind == "pattern":
        D.data = np.ones(D.nnz)
    path = tmp_path / f"{kind}.mtx"
    field = {"integer": "integer", "pattern": "pattern"}.get(kind, "real")
    symmetry = kind if kind in ("symmetric", "skew-symmetric") else "general"
    scipy.io.mmwrite(str(path), sp.coo_matrix(D), field=field, symmetry=symmetry)
    rows, cols, r, c, v = sg.read_mtx(path)
    ref = scipy_ref(path)
    assert (rows, cols) == ref.shape
    got = canon(rows, cols, r, c, v)
    assert np.array_equal(got.indptr, ref.indptr) and np.array_equal(got.indices, ref.indices)
    np.testing.assert_allclose(got.data, ref.data.astype(np.float32), rtol=1e-6)


def test_rectangular_and_comments(tmp_path):
    path = tmp_path / "r.mtx"
    path.write_text("%%MatrixMarket matrix coordinate real general\n% comment\n\n"
                    "3 5 4\n1 1 1.5\n% mid comment\n3 5 -2e3\n2 4 0.25\n3 1 7\n")
    rows, cols, r, c, v = sg.read_mtx(path)
    assert (rows, cols) == (3, 5)
    assert r.tolist() == [0, 2, 1, 2] and c.tolist() == [0, 4, 3, 0]
    assert v.tolist() == [1.5, -2000.0, 0.25, 7.0]


@pytest.mark.parametrize("text", [
    "",                                                                    # empty
    "3 3 1\n1 1 1\n",                                                      # no banner
    "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",         # dense form
    "%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1 0\n",  # complex
    "%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n2 2 2\n",  # truncated
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n",        # row out of range
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1\n",        # bad token
    "%%MatrixMarket matrix coordinate real symmetric\n2 3 1\n1 1 1\n",      # non-square symmetric
])
def test_malformed_files_are_rejected(tmp_path, text):
    path = tmp_path / "bad.mtx"
    path.write_text(text)
    with pytest.raises(sg.SpgemmError) as e:
        sg.read_mtx(path)
    assert e.value.status == 1


def test_missing_file():
    with pytest.raises(sg.SpgemmError):
        sg.read_mtx("/nonexistent/file.mtx")
