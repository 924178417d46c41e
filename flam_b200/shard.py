"""Many independent rskelf problems over several GPUs (one process per GPU).

Independent instances (a batch of curves, each its own matrix) need no exchange
while they are factored or solved: each rank takes a share of the instances,
factors its share in one batched pipeline (`rskelf_batched`) and solves its
right-hand sides; only per-instance results (times, errors, log-determinants)
are combined at the end with one all-reduce of a small vector.  Shares are
chosen by LPT (longest processing time first) on an estimated cost, so ranks
finish at about the same time when instance sizes vary by an order of
magnitude.

    torchrun --nproc-per-node 8 --master-addr 127.0.0.1 -m flam_b200.shard --count 4096

Works with any `torch.distributed` process group (NCCL on GPUs, gloo on CPU for
the host logic).
"""
import argparse
import heapq
import math
import time

import numpy as np


def instance_cost(N, d=2):
    """Estimated factor+solve cost of one instance: N k^2 with skeleton size k ~ log N
    for boundary problems in 2D (k ~ N^(1/2) on 3D surfaces)."""
    N = max(int(N), 2)
    k = math.log2(N) if d == 2 else math.sqrt(N)
    return N * k * k


def lpt_partition(costs, nparts):
    """Split indices 0..len(costs)-1 into nparts lists by LPT: in decreasing cost order
    each index goes to the currently lightest part (ties: lowest part index).  Each
    list is returned in increasing index order.  Deterministic: every rank computes
    the same partition from the same costs."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, p) for p in range(nparts)]
    parts = [[] for _ in range(nparts)]
    for i in order:
        load, p = heapq.heappop(heap)
        parts[p].append(i)
        heapq.heappush(heap, (load + float(costs[i]), p))
    return [sorted(p) for p in parts]


def dist_info(group=None):
    """(rank, world size) of the default or given process group, (0, 1) without one."""
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(group), dist.get_world_size(group)
    except ImportError:
        pass
    return 0, 1


def gather_by_instance(values, mine, total, group=None, device=None):
    """Combine per-instance float values computed on each rank: `values[j]` belongs to
    instance `mine[j]`.  Every rank returns the full vector (length `total`).  Each
    instance is owned by exactly one rank, so a sum all-reduce assembles it."""
    out = np.zeros(total, dtype=np.float64)
    if len(mine):
        out[np.asarray(mine, dtype=np.int64)] = np.asarray(values, dtype=np.float64)
    rank, world = dist_info(group)
    if world == 1:
        return out
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(out)
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def max_over_ranks(v, group=None, device=None):
    """Largest value of v over the ranks (device timings are reported as the max)."""
    rank, world = dist_info(group)
    if world == 1:
        return float(v)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def my_share(costs, group=None):
    """Instances this rank factors (LPT over the group's ranks)."""
    rank, world = dist_info(group)
    return lpt_partition(costs, world)[rank]


def rskelf_sharded(As, xs, occ, rank_or_tol, pxyfun=None, opts=None, group=None, costs=None):
    """This rank's share of a batch of independent problems, factored in one batched
    pipeline.  Returns (Factor, indices): `Factor` is a batched handle whose instance j
    is problem `indices[j]` of the full batch (None when this rank has no share)."""
    from .api import rskelf_batched
    if costs is None:
        costs = [instance_cost(np.shape(x)[1], np.shape(x)[0]) for x in xs]
    mine = my_share(costs, group)
    if not mine:
        return None, mine
    F = rskelf_batched([As[i] for i in mine], [xs[i] for i in mine], occ, rank_or_tol, pxyfun, opts)
    return F, mine


def _main():
    ap = argparse.ArgumentParser(description="Batch of independent star-curve problems over the ranks")
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--nmin", type=int, default=1024)
    ap.add_argument("--nmax", type=int, default=16384)
    ap.add_argument("--nrhs", type=int, default=4)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    import os

    import torch
    import torch.distributed as dist

    from . import problems
    from .api import rskelf_sv
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    Ns, aa, kk = problems.instance_batch(args.count, seed=args.seed, nmin=args.nmin, nmax=args.nmax)
    costs = [instance_cost(n) for n in Ns]
    mine = my_share(costs)
    items = [problems.instance(int(Ns[i]), aa[i], kk[i]) for i in mine]
    pxy = problems.instance(1024, 0.2, 5)[2]
    B = [np.asfortranarray(np.random.default_rng(args.seed + i).standard_normal((int(Ns[i]), args.nrhs)))
         for i in mine]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    F = None
    if mine:
        from .api import rskelf_batched
        F = rskelf_batched([it[1] for it in items], [it[0] for it in items], 64, args.tol, pxy)
        X = rskelf_sv(F, np.asfortranarray(np.concatenate(B, axis=0)))
    torch.cuda.synchronize()
    t = max_over_ranks(time.perf_counter() - t0, device=dev)
    dofs = float(np.sum(Ns))
    if dist_info()[0] == 0:
        print(f"instances {args.count} on {world} GPU(s): {dofs / t:.4g} DOF/s ({t * 1e3:.1f} ms, LPT shares "
              f"{[len(p) for p in lpt_partition(costs, world)]})", flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    _main()
