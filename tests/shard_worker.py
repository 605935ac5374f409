"""One rank of the two-rank gloo test of ganit_v2_b200.shard (run by
tests/test_shard.py as a child process; RANK / WORLD_SIZE / MASTER_* in the
environment).  Each rank solves its share of a small batch with the oracle
standing in for the GPU batch solver; rank 0 writes the gathered results."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def oracle_solve(lps, opt):
    from oracle import oracle as O

    out = []
    for lp in lps:
        r = O.solve(lp, precision="double")
        out.append({"name": lp.name, "status": r.status, "pobj": r.pobj, "iterations": r.iterations,
                    "rank": int(os.environ["RANK"])})
    return out


def main(path):
    from datetime import timedelta

    import torch.distributed as dist

    from ganit_v2_b200 import shard, workloads as W

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    lps = W.lp_batch(7, seed=300, m_min=20, m_max=200)
    res = shard.shard_solve(lps, None, solve=oracle_solve)
    if dist.get_rank() == 0:
        with open(path, "w") as f:
            json.dump(res, f)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1])
