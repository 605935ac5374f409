"""Parity of the fused B200 solver (gb_solve through the C ABI) with the
reference CPU PDHG, on the golden fixtures the reference produced.

Bar (the engine's tolerance statement): same verdict; every OPTIMAL result
FP64-certified within tol (rel_p, rel_d, rel_gap <= tol); objective within
10 * tol relative of the reference's; at FP64 the trajectory matches the
reference's iteration count to within two KKT checks."""
import json
import os

import numpy as np
import pytest

from tests.golden.make_golden import load_lp

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLD, "golden.json")) as f:
    GOLDEN = json.load(f)

PREC = {"double": 0, "mixed": 1, "dynamic": 2}


@pytest.fixture(scope="module")
def gb():
    import ganit_v2_b200 as gb

    gb.load_library()
    return gb


def check_against(r, g, tol, prec, check_every=64):
    assert r.status_name == g["status"]
    if g["status"] == "OPTIMAL":
        assert r.rel_primal <= tol * 1.0000001 and r.rel_dual <= tol * 1.0000001 and r.rel_gap <= tol * 1.0000001
        assert abs(r.pobj - g["pobj"]) <= 10 * tol * (1 + abs(g["pobj"])), (r.pobj, g["pobj"])
        assert abs(r.dobj - g["dobj"]) <= 10 * tol * (1 + abs(g["dobj"])), (r.dobj, g["dobj"])
    if prec == "double":
        assert abs(r.iterations - g["iterations"]) <= 2 * check_every, (r.iterations, g["iterations"])


@pytest.mark.parametrize("name", sorted(GOLDEN["synthetic"]))
@pytest.mark.parametrize("prec", ["double", "mixed", "dynamic"])
def test_solve_matches_reference(gb, name, prec):
    lp, arr = load_lp(os.path.join(GOLD, name + ".npz"))
    entry = GOLDEN["synthetic"][name]
    tol = entry["options"].get("tol", 1e-4)
    r = gb.solve_pdhg_gpu(lp, gb.Options(tol=tol, precision=gb.Precision(PREC[prec])))
    check_against(r, entry["results"][prec], tol, prec)
    assert r.x.shape == (lp.n,) and r.y.shape == (lp.m,)
    assert np.all(np.isfinite(r.x)) and np.all(np.isfinite(r.y))
    if prec == "double" and entry["results"][prec]["status"] == "OPTIMAL":
        xr = arr["x_double"]
        assert np.linalg.norm(r.x - xr) <= 1e-3 * (1 + np.linalg.norm(xr))


def test_resident_problem_repeats_bit_identically(gb):
    lp, _ = load_lp(os.path.join(GOLD, "rand_cfg0.npz"))
    with gb.Problem(lp) as p:
        r1 = p.solve(gb.Options(precision=gb.Precision.Mixed))
        r2 = p.solve(gb.Options(precision=gb.Precision.Mixed))
    assert r1.iterations == r2.iterations and r1.pobj == r2.pobj
    np.testing.assert_array_equal(r1.x, r2.x)
    np.testing.assert_array_equal(r1.y, r2.y)


def test_iteration_limit_and_check_every(gb):
    lp, _ = load_lp(os.path.join(GOLD, "rand_small.npz"))
    r = gb.solve_pdhg_gpu(lp, gb.Options(max_iter=100, check_every=50))
    assert r.status == gb.Status.IterationLimit and r.iterations == 100
    r = gb.solve_pdhg_gpu(lp, gb.Options(check_every=33))
    assert r.status == gb.Status.Optimal and r.iterations % 33 == 0


def test_odd_check_every_matches_oracle(gb, oracle_built):
    lp, _ = load_lp(os.path.join(GOLD, "rand_small.npz"))
    o = oracle_built.solve(lp, check_every=37)
    r = gb.solve_pdhg_gpu(lp, gb.Options(check_every=37))
    assert r.status_name == o.status
    assert abs(r.iterations - o.iterations) <= 74
    assert abs(r.pobj - o.pobj) <= 1e-3 * (1 + abs(o.pobj))


def test_time_limit_reported(gb):
    lp, _ = load_lp(os.path.join(GOLD, "rand_tight.npz"))
    r = gb.solve_pdhg_gpu(lp, gb.Options(tol=1e-12, time_limit=0.0))
    assert r.status == gb.Status.TimeLimit


def test_invalid_problem_is_an_error_not_a_crash(gb):
    lp, _ = load_lp(os.path.join(GOLD, "rand_small.npz"))
    bad = gb.LP(gb.Csr(lp.m, lp.n, lp.A.ptr, np.where(lp.A.idx > 5, lp.n + 7, lp.A.idx), lp.A.val), lp.c, lp.l,
                lp.u, lp.lo, lp.hi)
    with pytest.raises(gb.GanitError) as e:
        gb.solve_pdhg_gpu(bad)
    assert e.value.code == -1 and "out of range" in str(e.value)
    nan = gb.LP(lp.A, np.full(lp.n, np.nan), lp.l, lp.u, lp.lo, lp.hi)
    r = gb.solve_pdhg_gpu(nan, gb.Options(max_iter=640))
    assert r.status in (gb.Status.NumericalError, gb.Status.IterationLimit)


def test_device_memory_cache_reuses_blocks_and_keeps_results():
    """Freed device blocks are kept and reused by the next problem of the same
    shape; the solve is unchanged and the cache can be emptied."""
    import ganit_v2_b200 as gb
    from ganit_v2_b200 import api, workloads as W

    lp = W.random_feasible_lp(300, 700, 5, seed=21)
    opt = gb.Options(precision=gb.Precision.Mixed)
    api.release_cached_memory()
    assert api.cached_memory_bytes() == 0
    r1 = gb.solve_pdhg_gpu(lp, opt)
    kept = api.cached_memory_bytes()
    assert kept > 0
    r2 = gb.solve_pdhg_gpu(lp, opt)
    assert api.cached_memory_bytes() == kept  # same shape: every block came from the cache and went back
    assert r1.status == r2.status and r1.iterations == r2.iterations
    np.testing.assert_array_equal(r1.x, r2.x)
    np.testing.assert_array_equal(r1.y, r2.y)
    api.release_cached_memory()
    assert api.cached_memory_bytes() == 0


@pytest.mark.parametrize("name", sorted(GOLDEN["synthetic"]))
def test_bf16_matrix_phase_reaches_the_reference_answer(gb, name):
    """GB_PREC_MIXED_BF16 (an extension: BF16 matrix values first, then FP32,
    then FP64) meets the same bar against the reference's mixed-precision
    results: same verdict, FP64-certified KKT within tol, objective within
    10 * tol.  QPs skip the BF16 phase."""
    lp, _ = load_lp(os.path.join(GOLD, name + ".npz"))
    entry = GOLDEN["synthetic"][name]
    tol = entry["options"].get("tol", 1e-4)
    r = gb.solve_pdhg_gpu(lp, gb.Options(tol=tol, precision=gb.Precision.MixedBf16))
    check_against(r, entry["results"]["mixed"], tol, "mixed")
    if lp.Q is None:
        assert r.bf16_iterations > 0
    else:
        assert r.bf16_iterations == 0


def test_problem_autotune_keeps_the_certified_answer(gb):
    lp, _ = load_lp(os.path.join(GOLD, "rand_cfg0.npz"))
    opt = gb.Options(precision=gb.Precision.Mixed)
    p = gb.Problem(lp, opt)
    try:
        a = p.solve(opt)
        t = p.autotune(10)
        assert 256 <= t["block_nnz"] <= 2048 and 32 <= t["max_rows"] <= 256
        assert t["ms_per_iter_tuned"] <= 1.05 * t["ms_per_iter_default"]
        assert t["ms_per_iter_tuned_f64"] <= 1.05 * t["ms_per_iter_default_f64"]
        assert 256 <= t["block_nnz_f64"] <= 2048
        b = p.solve(opt)
        assert a.status == b.status
        assert max(b.rel_primal, b.rel_dual, b.rel_gap) <= 1e-4 * 1.0000001
        assert abs(a.pobj - b.pobj) <= 1e-3 * (1 + abs(a.pobj))
    finally:
        p.close()


def _write_mps(lp, path):
    """Free-format MPS of an LP (row bounds as E / L / G rows with ranges)."""
    A = lp.A.to_scipy().tocsc()
    lines = ["NAME TEST", "ROWS", " N OBJ"]
    kind, rhs, rng = [], [], []
    for i in range(lp.m):
        lo, hi = lp.lo[i], lp.hi[i]
        if lo == hi:
            kind.append("E"); rhs.append(lo); rng.append(None)
        elif np.isinf(lo):
            kind.append("L"); rhs.append(hi); rng.append(None)
        elif np.isinf(hi):
            kind.append("G"); rhs.append(lo); rng.append(None)
        else:
            kind.append("G"); rhs.append(lo); rng.append(hi - lo)
        lines.append(f" {kind[-1]} R{i}")
    lines.append("COLUMNS")
    for j in range(lp.n):
        lines.append(f"    C{j} OBJ {float(lp.c[j])!r}")
        for p in range(A.indptr[j], A.indptr[j + 1]):
            lines.append(f"    C{j} R{A.indices[p]} {float(A.data[p])!r}")
    lines.append("RHS")
    lines += [f"    RHS R{i} {float(rhs[i])!r}" for i in range(lp.m) if rhs[i] != 0]
    lines.append("RANGES")
    lines += [f"    RNG R{i} {float(rng[i])!r}" for i in range(lp.m) if rng[i] is not None]
    lines.append("BOUNDS")
    for j in range(lp.n):
        l, u = lp.l[j], lp.u[j]
        if np.isinf(l) and np.isinf(u):
            lines.append(f" FR BND C{j}")
            continue
        if np.isinf(l):
            lines.append(f" MI BND C{j}")
        elif l != 0:
            lines.append(f" LO BND C{j} {float(l)!r}")
        if not np.isinf(u):
            lines.append(f" UP BND C{j} {float(u)!r}")
    lines.append("ENDATA")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def test_problem_read_from_an_mps_file_solves_like_the_in_memory_one(gb, tmp_path):
    lp, _ = load_lp(os.path.join(GOLD, "rand_small.npz"))
    path = str(tmp_path / "rand_small.mps")
    _write_mps(lp, path)
    fl = gb.read_mps(path)
    opt = gb.Options(precision=gb.Precision.Double)
    a = gb.solve_pdhg_gpu(lp, opt)
    b = gb.solve_pdhg_gpu(fl, opt)
    assert a.status == b.status and a.iterations == b.iterations
    np.testing.assert_array_equal(a.x, b.x)
    np.testing.assert_array_equal(a.y, b.y)


def test_graph_timed_kernels(gb):
    lp, _ = load_lp(os.path.join(GOLD, "rand_cfg0.npz"))
    opt = gb.Options(precision=gb.Precision.Mixed)
    p = gb.Problem(lp, opt)
    try:
        p.solve(opt, fetch=False)
        for level in (0, 2, 3):
            t = p.time_kernels_graph(level, 20)
            assert t["ms_primal"] > 0 and t["ms_dual"] > 0 and t["ms_iteration"] > 0
            assert t["ms_iteration"] <= 2.0 * (t["ms_primal"] + t["ms_dual"])
        r = p.solve(opt)  # the timing leaves the problem solvable
        assert r.status_name == "OPTIMAL"
    finally:
        p.close()
