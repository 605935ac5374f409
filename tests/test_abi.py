"""The C-ABI library loads and exports every symbol include/ganit_b200.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ganit_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gb_[A-Za-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from ganit_v2_b200 import build

    build.build()
    return ctypes.CDLL(build.LIB)


def test_header_declares_the_python_export_list():
    from ganit_v2_b200.api import EXPORTS

    assert declared_functions() == sorted(EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_version_and_defaults_without_gpu(lib):
    from ganit_v2_b200 import api

    L = api.load_library()
    assert L.gb_version() == 10000
    o = api._GbOptions()
    L.gb_default_options(ctypes.addressof(o))
    d = api.Options()
    assert (o.tol, o.max_iter, o.check_every, o.ruiz_iters, o.stall_checks, o.stall_checks_l2) == (
        d.tol, d.max_iter, d.check_every, d.ruiz_iters, d.stall_checks, d.stall_checks_l2)
    assert o.infeas_tol == d.infeas_tol and o.pock_chambolle == 1 and o.precision == 0


def test_library_is_sm100a_only():
    """The fatbin carries sm_100a code only (checked through the build recipe,
    not by reading the binary)."""
    from ganit_v2_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "-fmad=false" in build.FLAGS


def test_no_device_error_is_reported_not_thrown(lib):
    """Without a GPU every entry point returns an error code and a message."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ganit_v2_b200 import GanitError, solve_pdhg_gpu, workloads

    with pytest.raises(GanitError) as e:
        solve_pdhg_gpu(workloads.random_feasible_lp(20, 40, 3, seed=1))
    assert e.value.code in (-2, -4)


def test_diff_argument_checks_without_gpu(lib):
    """gb_diff_create validates K, R and the no-Hessian rule before touching a device."""
    import numpy as np

    from ganit_v2_b200 import GanitError, workloads as W
    from ganit_v2_b200.api import DiffSolver

    lp = W.random_feasible_lp(20, 40, 3, seed=1)
    with pytest.raises(GanitError, match="multiple of ckpt_every"):
        DiffSolver([lp], tail_iters=30, ckpt_every=20)
    with pytest.raises(GanitError, match="multiple of ckpt_every"):
        DiffSolver([lp], tail_iters=0, ckpt_every=1)
    qp = W.portfolio_qp(200, 3, seed=1)
    with pytest.raises(GanitError, match="LPs only"):
        DiffSolver([qp], tail_iters=20, ckpt_every=10)
