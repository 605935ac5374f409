"""The differentiable layer's two MINRES drivers give the same solutions: the
one-launch solve (one CTA per instance, used when every instance's reduced
system is small) and the graph of two launches per step (used for larger
systems, forced here with GANIT_B200_MR_ONE_LAUNCH=0).  Both stop at a
relative residual of 1e-10, so the polished points and the gradients agree
to far better than the layer's 1e-4; only their summation orders differ."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
WORKER = os.path.join(os.path.dirname(__file__), "minres_paths_worker.py")


def run(path: str, one_launch: bool):
    env = dict(os.environ, GANIT_B200_MR_ONE_LAUNCH="1" if one_launch else "0")
    p = subprocess.run([sys.executable, WORKER, path], env=env, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    return np.load(path)


def test_one_launch_and_graph_minres_agree(tmp_path):
    a = run(str(tmp_path / "one.npz"), True)
    b = run(str(tmp_path / "graph.npz"), False)
    assert a["polished"].all() and b["polished"].all()
    assert a["converged"].all() and b["converged"].all()
    rel = lambda u, v: float(np.linalg.norm(u - v) / max(np.linalg.norm(v), 1e-300))  # noqa: E731
    assert rel(a["x"], b["x"]) <= 1e-8 and rel(a["y"], b["y"]) <= 1e-8
    for k in ("g_c", "g_lo", "g_hi", "g_a_val"):
        assert rel(a[k], b[k]) <= 1e-6, (k, rel(a[k], b[k]))
