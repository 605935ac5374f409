"""The device transpose (gb_csr_transpose: the hand-written stable radix sort
and scan the solver builds A^T with) against the oracle's counting-sort
transpose, a restatement of src/lp.cpp:55-72: bit-identical ptr, idx and
val on every case -- empty matrices, a single column (no sort pass), key
widths of one to four 8-bit passes, a dense column, empty and 100,000-entry
rows, unsorted and repeated column indices inside a row, and the golden
fixtures' matrices."""
import os

import numpy as np
import pytest

from ganit_v2_b200.lp import Csr
from tests.golden.make_golden import load_lp

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rand_csr(rng, rows, cols, lens, sort=False):
    lens = np.asarray(lens, dtype=np.int64)
    ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    idx = rng.integers(0, cols, size=int(ptr[-1])).astype(np.int32)
    if sort:
        for i in range(rows):
            idx[ptr[i]:ptr[i + 1]].sort()
    return Csr(rows, cols, ptr, idx, rng.standard_normal(int(ptr[-1])))


def cases():
    rng = np.random.default_rng(11)
    yield "empty", Csr(3, 4, np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0))
    yield "no rows", Csr(0, 5, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    yield "one column", rand_csr(rng, 5000, 1, rng.integers(0, 2, 5000))
    for cols in (2, 200, 256, 257, 70_000):  # 1, 1, 1, 2 and 3 digit passes
        yield f"cols={cols}", rand_csr(rng, 3000, cols, rng.integers(0, 12, 3000))
    yield "cols=2^24+5", rand_csr(rng, 20_000, (1 << 24) + 5, rng.integers(0, 30, 20_000))  # 4 passes
    lens = rng.integers(0, 9, 50_000)
    lens[17] = 100_000  # one long row
    lens[100:2000] = 0  # a run of empty rows
    a = rand_csr(rng, 50_000, 40_000, lens)
    dense = a.idx.copy()
    dense[a.ptr[:-1][lens > 0]] = 123  # column 123 in every nonempty row
    yield "dense column + long row", Csr(a.rows, a.cols, a.ptr, dense, a.val)
    b = rand_csr(rng, 2000, 50, rng.integers(0, 40, 2000))  # repeated columns inside rows
    yield "repeats", b
    yield "sorted rows", rand_csr(rng, 10_000, 9_999, rng.integers(0, 20, 10_000), sort=True)
    for name in ("rand_free", "blend_small", "port_lifted_small"):
        p = os.path.join(GOLD, name + ".npz")
        if os.path.exists(p):
            lp, _ = load_lp(p)
            yield name, lp.A


@pytest.mark.parametrize("name,a", list(cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_transpose_matches_oracle(oracle_built, name, a):
    import ganit_v2_b200 as gb

    t = gb.transpose(a)
    r = oracle_built.transpose(a)
    assert (t.rows, t.cols) == (a.cols, a.rows)
    np.testing.assert_array_equal(t.ptr, r.ptr)
    np.testing.assert_array_equal(t.idx, r.idx)
    assert np.array_equal(t.val.view(np.int64), r.val.view(np.int64))
