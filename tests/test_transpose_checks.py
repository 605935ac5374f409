"""Host-side pieces of the transpose: the oracle's counting-sort transpose
(src/lp.cpp:55-72) pinned against an independent NumPy restatement (stable
argsort of the column keys) and the package's Csr.transpose, and the C ABI
rejecting malformed input on the host, before any device work."""
import numpy as np
import pytest

from ganit_v2_b200.lp import Csr


def numpy_transpose(a):
    rows = np.repeat(np.arange(a.rows, dtype=np.int32), np.diff(a.ptr))
    order = np.argsort(a.idx, kind="stable")
    ptr = np.concatenate([[0], np.cumsum(np.bincount(a.idx, minlength=a.cols))]).astype(np.int32)
    return Csr(a.cols, a.rows, ptr, rows[order], a.val[order])


@pytest.mark.parametrize("seed", range(6))
def test_oracle_transpose_is_stable_counting_sort(oracle_built, seed):
    rng = np.random.default_rng(seed)
    rows, cols = int(rng.integers(1, 400)), int(rng.integers(1, 300))
    lens = rng.integers(0, 15, rows)
    ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    a = Csr(rows, cols, ptr, rng.integers(0, cols, int(ptr[-1])), rng.standard_normal(int(ptr[-1])))
    r = oracle_built.transpose(a)
    for other in (numpy_transpose(a), a.transpose()):
        np.testing.assert_array_equal(r.ptr, other.ptr)
        np.testing.assert_array_equal(r.idx, other.idx)
        np.testing.assert_array_equal(r.val, other.val)


@pytest.mark.parametrize("bad", ["col>=cols", "col<0", "ptr decreasing"])
def test_abi_rejects_malformed_csr(bad):
    import ganit_v2_b200 as gb

    ptr = np.array([0, 2, 3], np.int32)
    idx = np.array([0, 1, 2], np.int32)
    if bad == "col>=cols":
        idx[2] = 3
    elif bad == "col<0":
        idx[0] = -1
    else:
        ptr = np.array([0, 2, 1], np.int32)
        idx = idx[:1]
    a = Csr.__new__(Csr)  # bypass the dataclass checks to reach the C ABI's own
    a.rows, a.cols, a.ptr, a.idx, a.val = 2, 3, ptr, idx, np.ones(len(idx))
    with pytest.raises(gb.GanitError):
        gb.transpose(a)
