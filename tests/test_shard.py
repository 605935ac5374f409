"""Instance sharding of batches over ranks (ganit_v2_b200.shard): the greedy
partition, and a two-rank gloo run on CPU in which each rank solves its
share (oracle standing in for the GPU) and the gathered results equal a
single-process solve of the whole batch, in input order."""
import json
import os
import socket
import subprocess
import sys

import numpy as np

from ganit_v2_b200 import shard, workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))


def test_partition_covers_every_instance_once_and_balances():
    rng = np.random.default_rng(0)
    w = rng.integers(1, 1000, size=101).tolist()
    for parts in (1, 2, 3, 8):
        p = shard.partition(w, parts)
        assert len(p) == parts
        flat = sorted(i for part in p for i in part)
        assert flat == list(range(len(w)))
        loads = [sum(w[i] for i in part) for part in p]
        assert max(loads) <= sum(w) / parts + max(w)
        assert p == shard.partition(w, parts)  # deterministic


def test_partition_more_parts_than_instances():
    p = shard.partition([5, 3], 4)
    assert sorted(i for part in p for i in part) == [0, 1]
    assert sum(1 for part in p if not part) == 2


def test_single_process_shard_solve_is_the_plain_solve():
    lps = W.lp_batch(3, seed=9, m_min=20, m_max=60)
    out = shard.shard_solve(lps, None, solve=lambda l, o: [lp.name for lp in l])
    assert out == [lp.name for lp in lps]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_rank_gloo_shard_solve_matches_single_process(tmp_path, oracle_built):
    out = tmp_path / "res.json"
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "shard_worker.py"), str(out)], env=env))
    codes = [p.wait(timeout=300) for p in procs]
    assert codes == [0, 0]
    got = json.loads(out.read_text())
    lps = W.lp_batch(7, seed=300, m_min=20, m_max=200)
    assert [g["name"] for g in got] == [lp.name for lp in lps]
    assert {g["rank"] for g in got} == {0, 1}
    parts = shard.partition([shard.instance_weight(lp) for lp in lps], 2)
    for r, part in enumerate(parts):
        assert all(got[i]["rank"] == r for i in part)
    for g, lp in zip(got, lps):
        ref = oracle_built.solve(lp, precision="double")
        assert g["status"] == ref.status and g["iterations"] == ref.iterations
        assert g["pobj"] == ref.pobj
