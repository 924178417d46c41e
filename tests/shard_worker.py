"""One rank of the CPU (gloo) test of the instance-sharding host logic.

Run by tests/test_shard.py as WORLD_SIZE processes; each rank takes its LPT share
of a batch of instance sizes, computes a per-instance value for its share only and
combines the values with the same calls a multi-GPU batch run uses.  Rank r prints
one JSON line with what it saw.
"""
import json
import os
import sys
from datetime import timedelta

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402
import torch.distributed as dist  # noqa: E402

from flam_b200 import problems, shard  # noqa: E402


def main():
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    rank, world = shard.dist_info()
    Ns, _, _ = problems.instance_batch(257, seed=4, nmin=1024, nmax=16384)
    costs = [shard.instance_cost(n) for n in Ns]
    mine = shard.my_share(costs)
    # each rank reports the instances it owns: the assembled vector must count each once
    owners = shard.gather_by_instance(np.full(len(mine), rank + 1.0), mine, len(Ns))
    ones = shard.gather_by_instance(np.ones(len(mine)), mine, len(Ns))
    vals = shard.gather_by_instance(np.sqrt(Ns[mine].astype(float)), mine, len(Ns))
    load = float(np.sum(np.asarray(costs)[mine]))
    mx = shard.max_over_ranks(load)
    print(json.dumps({"rank": rank, "world": world, "n_mine": len(mine), "mine_head": mine[:5],
                      "ones_ok": bool(np.all(ones == 1.0)),
                      "vals_ok": bool(np.allclose(vals, np.sqrt(Ns.astype(float)))),
                      "owners": owners.tolist(), "load": load, "max_load": mx, "total": float(np.sum(costs)),
                      "max_cost": float(np.max(costs))}), flush=True)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
