"""Row-block scheduler (ganit_v2_b200/csrc/gb_spmv.cuh), host logic, no GPU:
tests/schedule_check.cu builds schedules for short rows, a blending-LP-like
period (one 960-nonzero row among ~140 short ones), and a heavy tail with rows
past every threshold, at the default and at a tuned cut, and checks that
every nonzero is covered once and in order, that STREAM blocks respect their
nonzero, row and lane-sum caps (no lane of a row's group adds more than
kMaxLaneSum products), that long rows become LONG or CHUNK blocks with
consecutive slot ids, and that the lane-group table matches its definition."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_schedule_invariants(tmp_path):
    from ganit_v2_b200 import build

    exe = tmp_path / "schedule_check"
    cmd = [build.nvcc(), "-std=c++17", "-O2", *build.ARCH, "-o", str(exe), os.path.join(HERE, "schedule_check.cu")]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        pytest.fail("schedule_check.cu did not compile:\n" + out.stdout + out.stderr)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    lines = run.stdout.strip().splitlines()
    assert len(lines) == 6 and all(line.startswith("ok ") for line in lines), run.stdout
