"""Phases that only some instances of a batch take part in launch the
iteration kernels on those instances' row blocks alone (the phase block
lists).  The blocks and their arithmetic are the same, so every result bit
must be: each workload is solved in two child processes, with the lists on
and off (GANIT_B200_PHASE_LISTS=0), and their digests of status, iteration
counts, objectives, points and (for the differentiable layer) gradients are
compared.  The trace of the lists-on run shows that lists were used."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
WORKER = os.path.join(os.path.dirname(__file__), "phase_lists_worker.py")


def run(which: str, lists: bool):
    env = dict(os.environ, GANIT_B200_TRACE="1", GANIT_B200_PHASE_LISTS="1" if lists else "0")
    # at 3e-6 a few of the 48 LPs go on to the FP64 phase
    args = [sys.executable, WORKER, which] + (["3e-6"] if which == "batch" else [])
    p = subprocess.run(args, env=env, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    return p.stdout.strip().splitlines()[-1], p.stderr


@pytest.mark.parametrize("which", ["batch", "diff"])
def test_phase_lists_change_no_result_bit(which):
    on, err_on = run(which, True)
    off, err_off = run(which, False)
    assert "phase lists" in err_on
    assert "phase lists" not in err_off
    assert on == off
