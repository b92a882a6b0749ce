"""Device COO -> CSR/CSC of triplets in any order (spgemm_coo_to_cm) against
a stable numpy sort: short rows (warp sort), rows of 1024..8192 entries
(block sort), rows above 8192 entries (block-merged runs), duplicates kept in
input order, empty rows, and out-of-range indices reported."""
import numpy as np
import pytest

import spgemm_b200 as sg

pytestmark = pytest.mark.gpu

TRIP = np.dtype([("r", "<i4"), ("c", "<i4"), ("v", "<f4")])


def run(h, r, c, v, rows, cols, kind):
    import torch
    t = np.zeros(len(r), TRIP)
    t["r"], t["c"], t["v"] = r, c, v
    dt = torch.from_numpy(t.view(np.uint8).copy() if len(t) else np.zeros(12, np.uint8)).cuda()
    n_major = rows if kind == sg.ROW_MAJOR else cols
    ptr = torch.zeros(n_major + 1, dtype=torch.int32, device="cuda")
    idx = torch.zeros(max(len(r), 1), dtype=torch.int32, device="cuda")
    val = torch.zeros(max(len(r), 1), dtype=torch.float32, device="cuda")
    h.coo_to_cm(dt.data_ptr(), len(r), rows, cols, kind, ptr.data_ptr(), idx.data_ptr(),
                val.data_ptr())
    torch.cuda.synchronize()
    return ptr.cpu().numpy(), idx.cpu().numpy()[:len(r)], val.cpu().numpy()[:len(r)]


def expected(r, c, v, rows, cols, kind):
    major, minor = (r, c) if kind == sg.ROW_MAJOR else (c, r)
    n_major = rows if kind == sg.ROW_MAJOR else cols
    order = np.lexsort((np.arange(len(r)), minor, major))  # stable: ties in input order
    ptr = np.zeros(n_major + 1, np.int64)
    ptr[1:] = np.cumsum(np.bincount(major, minlength=n_major))
    return ptr, minor[order], v[order]


@pytest.mark.parametrize("kind", [sg.ROW_MAJOR, sg.COL_MAJOR])
def test_any_order_matches_stable_sort(kind):
    rng = np.random.default_rng(8)
    rows, cols = 5000, 40000
    lens = rng.integers(0, 40, rows)
    lens[7] = 3000     # block sort
    lens[11] = 8192    # block sort, full
    lens[13] = 30001   # runs + merges
    lens[17] = 0
    r = np.repeat(np.arange(rows), lens)
    c = rng.integers(0, cols, len(r))
    c[r == 13] = rng.integers(0, 500, int((r == 13).sum()))  # many duplicates in a long row
    v = rng.uniform(-1, 1, len(r)).astype(np.float32)
    if kind == sg.COL_MAJOR:
        r, c = c % rows, r  # long columns instead of long rows
        rows, cols = rows, 5000
    perm = rng.permutation(len(r))
    r, c, v = r[perm], c[perm], v[perm]
    with sg.Handle() as h:
        got = run(h, r, c, v, rows, cols, kind)
    exp = expected(r, c, v, rows, cols, kind)
    assert np.array_equal(got[0], exp[0])
    assert np.array_equal(got[1], exp[1])
    assert np.array_equal(got[2], exp[2])


def test_empty_and_out_of_range():
    with sg.Handle() as h:
        got = run(h, np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.float32), 4, 4,
                  sg.ROW_MAJOR)
        assert got[0].tolist() == [0, 0, 0, 0, 0]
        with pytest.raises(sg.SpgemmError) as e:
            run(h, np.array([0, 5]), np.array([1, 1]), np.ones(2, np.float32), 4, 4, sg.ROW_MAJOR)
        assert e.value.status == 1
