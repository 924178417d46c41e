"""Instance sharding over several GPUs: the host logic (LPT shares, combining
per-instance results, max over ranks), tested on CPU with gloo ranks; and, on one
GPU, that a rank's batched share factors exactly as the same instances do in the
full batch."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from flam_b200 import problems, shard

HERE = os.path.dirname(os.path.abspath(__file__))


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.lognormal(0, 1, size=101)
    for k in (1, 2, 3, 8):
        parts = shard.lpt_partition(costs, k)
        assert sorted(i for p in parts for i in p) == list(range(101))
        loads = [costs[p].sum() for p in parts]
        # LPT bound: no part exceeds the mean load by more than the largest item
        assert max(loads) <= costs.sum() / k + costs.max() + 1e-9
        assert parts == shard.lpt_partition(costs, k)          # deterministic
    assert shard.lpt_partition([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard.lpt_partition([1.0], 0)


def test_instance_cost_grows_with_n():
    assert shard.instance_cost(16384) > shard.instance_cost(1024) * 16


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_share_and_combine():
    world = 2
    env0 = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), WORLD_SIZE=str(world))
    procs = []
    for r in range(world):
        env = dict(env0, RANK=str(r), LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "shard_worker.py")], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=240)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    Ns, _, _ = problems.instance_batch(257, seed=4, nmin=1024, nmax=16384)
    parts = shard.lpt_partition([shard.instance_cost(n) for n in Ns], world)
    for r, o in enumerate(sorted(outs, key=lambda o: o["rank"])):
        assert o["world"] == world and o["n_mine"] == len(parts[r]) and o["mine_head"] == parts[r][:5]
        assert o["ones_ok"] and o["vals_ok"]
        assert o["max_load"] == max(x["load"] for x in outs)
        assert o["max_load"] <= o["total"] / world + o["max_cost"] + 1e-6
    owners = np.asarray(outs[0]["owners"])
    assert owners.tolist() == outs[1]["owners"]
    for r in range(world):
        assert np.all(owners[parts[r]] == r + 1)


@pytest.mark.gpu
def test_rank_share_factors_like_the_full_batch():
    import flam_b200 as fb
    Ns, aa, kk = problems.instance_batch(5, seed=2, nmin=600, nmax=2000)
    items = [problems.instance(int(n), a, k) for n, a, k in zip(Ns, aa, kk)]
    As, xs = [it[1] for it in items], [it[0] for it in items]
    F, mine = shard.rskelf_sharded(As, xs, 64, 1e-10, items[0][2])       # one rank: everything
    assert mine == list(range(5))
    Fb = fb.rskelf_batched(As, xs, 64, 1e-10, items[0][2])
    for j in range(5):
        a, b = F.factors(j)["factors"], Fb.factors(j)["factors"]
        assert [len(f["sk"]) for f in a] == [len(f["sk"]) for f in b]
