"""MPS / QPS reader of the library (gb_read_mps, CPU only) against the
reference's own reader (src/mps.cpp, built into oracle/_ref) on the
reference's instance files, and on a hand-written file that exercises every
section, row type, range rule and bound type."""
import glob
import os

import numpy as np
import pytest

from oracle.oracle import REF_INSTANCES as REF_ROOT, REF_MISSING  # noqa: E402


def _files():
    out = []
    for ext in ("mps", "qps", "MPS", "QPS"):
        out += glob.glob(os.path.join(REF_ROOT, "**", "*." + ext), recursive=True)
    return sorted(set(out))


@pytest.fixture(scope="module")
def gb():
    from ganit_v2_b200 import build

    build.build()
    import ganit_v2_b200 as gb

    return gb


@pytest.mark.parametrize("path", _files() or ["<no reference instances>"], ids=lambda p: os.path.basename(p))
def test_matches_the_reference_reader(gb, oracle_built, path):
    if not os.path.exists(path) or not oracle_built.ref_available():
        pytest.skip(REF_MISSING)
    a = gb.read_mps(path)
    b = oracle_built.ref_read_mps(path)
    assert (a.m, a.n, a.maximize) == (b.m, b.n, b.maximize)
    assert a.obj_const == b.obj_const
    np.testing.assert_array_equal(a.A.ptr, b.A.ptr)
    np.testing.assert_array_equal(a.A.idx, b.A.idx)
    np.testing.assert_allclose(a.A.val, b.A.val, rtol=1e-15, atol=0)  # duplicates may sum in another order
    for k in ("c", "l", "u", "lo", "hi"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    assert (a.is_int is None) == (b.is_int is None)
    if a.is_int is not None:
        np.testing.assert_array_equal(a.is_int, b.is_int)
    assert (a.Q is None) == (b.Q is None)
    if a.Q is not None:
        np.testing.assert_array_equal(a.Q.ptr, b.Q.ptr)
        np.testing.assert_array_equal(a.Q.idx, b.Q.idx)
        np.testing.assert_allclose(a.Q.val, b.Q.val, rtol=1e-15, atol=0)


SAMPLE = """\
* every section, row type, range rule and bound type
NAME          SAMPLE
OBJSENSE
    MAX
ROWS
 N  COST
 E  R1
 L  R2
 G  R3
 N  SPARE
 E  R4
COLUMNS
    X1        COST         1.0   R1           2.0
    X1        R2           1.0   SPARE        9.0
    MARKER                 'MARKER'                 'INTORG'
    X2        COST        -3.0   R1           1.0
    X2        R3           4.0   R2           0.5
    MARKER                 'MARKER'                 'INTEND'
    X3        R1           1.0   R1           1.0
    X3        R4           7.0
    X4        R3           1.0   COST         2.5
    X5        R2           1.0
    X6        R4           1.0
    X7        R4           1.0
    X8        R3           1.0
    X9        R2           2.0
RHS
    RHS       R1           3.0   R2           4.0
    R3           5.0
    RHS       COST        -6.0   R4           1.5
RANGES
    RNG       R1           2.0   R2          -3.0
    RNG       R3           1.0   R4          -0.5
BOUNDS
 UP BND       X1           4.0
 UP BND       X2          -2.0
 LO BND       X3          -1.0
 UP BND       X3          -0.5
 FX BND       X4           2.0
 FR BND       X5
 MI BND       X6
 PL BND       X7
 BV BND       X8
 LI BND       X9           1.0
 UI BND       X9           3.0
QUADOBJ
    X1        X1           2.0
    X2        X1           0.5
ENDATA
"""


def test_every_section_and_rule(gb, tmp_path):
    p = tmp_path / "sample.mps"
    p.write_text(SAMPLE)
    lp = gb.read_mps(str(p))
    inf = np.inf
    assert (lp.m, lp.n, lp.maximize, lp.obj_const) == (4, 9, True, 6.0)
    assert lp.name == "SAMPLE"
    np.testing.assert_array_equal(lp.c, [1.0, -3.0, 0, 2.5, 0, 0, 0, 0, 0])
    A = np.zeros((4, 9))
    A[0, 0], A[1, 0] = 2.0, 1.0
    A[0, 1], A[2, 1], A[1, 1] = 1.0, 4.0, 0.5
    A[0, 2], A[3, 2] = 2.0, 7.0                    # duplicate R1 entries of X3 summed
    A[2, 3], A[1, 4], A[3, 5], A[3, 6], A[2, 7], A[1, 8] = 1, 1, 1, 1, 1, 2
    np.testing.assert_array_equal(lp.A.to_scipy().toarray(), A)
    # E + positive range widens up; L: lo = b - |r|; G: hi = b + |r|; E + negative range widens down
    np.testing.assert_array_equal(lp.lo, [3.0, 1.0, 5.0, 1.0])
    np.testing.assert_array_equal(lp.hi, [5.0, 4.0, 6.0, 1.5])
    # UP>0; negative UP with no lower given -> lower -inf; LO then negative UP keeps LO; FX; FR; MI; PL; BV; LI/UI
    np.testing.assert_array_equal(lp.l, [0.0, -inf, -1.0, 2.0, -inf, -inf, 0.0, 0.0, 1.0])
    np.testing.assert_array_equal(lp.u, [4.0, -2.0, -0.5, 2.0, inf, inf, inf, 1.0, 3.0])
    Q = lp.Q.to_scipy().toarray()
    expect = np.zeros((9, 9))
    expect[0, 0], expect[0, 1], expect[1, 0] = 2.0, 0.5, 0.5  # QUADOBJ lower triangle mirrored
    np.testing.assert_array_equal(Q, expect)
    # integer: X2 between the markers, X8 (BV), X9 (LI / UI)
    np.testing.assert_array_equal(lp.is_int, [0, 1, 0, 0, 0, 0, 0, 1, 1])


@pytest.mark.parametrize("text,msg", [
    ("NAME X\nROWS\n N C\nBOGUS\nENDATA\n", "unknown section"),
    ("NAME X\nROWS\n N C\n E R\nCOLUMNS\n    X1 Q 1.0\nENDATA\n", "unknown row"),
    ("NAME X\nROWS\n N C\n E R\nCOLUMNS\n    X1 R abc\nENDATA\n", "bad number"),
    ("NAME X\nROWS\n N C\n E R\nCOLUMNS\n    X1 R 1\nBOUNDS\n UP B X9 1\nENDATA\n", "unknown column"),
])
def test_errors_name_the_line(gb, tmp_path, text, msg):
    p = tmp_path / "bad.mps"
    p.write_text(text)
    with pytest.raises(gb.GanitError, match=msg):
        gb.read_mps(str(p))
