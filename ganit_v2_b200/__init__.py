"""B200-native restarted-PDHG engine for GANIT's LP / convex-QP path.

Public API (mirrors include/ganit/pdhg.hpp of the reference):
``Options``, ``Precision``, ``Status``, ``Result``, ``solve_pdhg_gpu`` (alias
``solve_pdhg_b200``), plus ``Problem`` (resident problem), ``Backend``
(Backend-concept operations), ``BatchSolver`` and ``DiffSolver`` (with the
``torch.autograd.Function`` wrapper in :mod:`ganit_v2_b200.diff`), and
``strong_branch`` (batched strong branching of a MILP node).
The compute path is libganit_b200.so (sm_100a); there is no CPU fallback.
"""
from .lp import LP, Csr
from .api import (Backend, BatchSolver, DiffSolver, FactorForm, GanitError, Options, Precision, Problem, Result, Status, load_library, set_device,
                  transpose, solve_pdhg_b200, solve_pdhg_gpu, read_mps, LIB_PATH, StrongBranch, strong_branch, fractional,
                  most_fractional, BRANCH_VAR, BRANCH_TIGHTEN, BRANCH_NODE_INFEASIBLE)

__all__ = ["LP", "Csr", "Backend", "BatchSolver", "DiffSolver", "FactorForm", "GanitError", "Options", "Precision", "Problem", "Result", "Status",
           "load_library", "set_device", "transpose", "solve_pdhg_b200", "solve_pdhg_gpu", "read_mps", "LIB_PATH",
           "StrongBranch", "strong_branch", "fractional", "most_fractional", "BRANCH_VAR", "BRANCH_TIGHTEN",
           "BRANCH_NODE_INFEASIBLE"]
