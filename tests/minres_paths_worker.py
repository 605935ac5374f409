"""Child process of tests/test_gpu_minres_paths.py: forward + backward of a
small differentiable batch, gradients saved to the .npz named in argv[1].
GANIT_B200_MR_ONE_LAUNCH is read once per process, hence the child."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import ganit_v2_b200 as gb  # noqa: E402
from ganit_v2_b200 import workloads as W  # noqa: E402


def main(path: str) -> None:
    lps = W.diff_batch(12, m=120, n=300, nnz_per_col=10, seed=3100)
    opt = gb.Options(tol=1e-6, precision=gb.Precision.Mixed)
    ds = gb.DiffSolver(lps, opt, tail_iters=40, ckpt_every=10)
    res, x, y = ds.forward(opt)
    rng = np.random.default_rng(5)
    g = ds.backward(rng.standard_normal(int(ds.n_off[-1])), rng.standard_normal(int(ds.m_off[-1])))
    infos = [ds.info(i) for i in range(len(lps))]
    np.savez(path, x=x, y=y, polished=np.array([i["polished"] for i in infos]),
             converged=np.array([i["implicit_converged"] for i in infos]), **{f"g_{k}": v for k, v in g.items()})
    ds.close()


if __name__ == "__main__":
    main(sys.argv[1])
