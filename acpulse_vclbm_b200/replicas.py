"""Multi-GPU form: independent replicas, one process per GPU.

The reference has no parallelism beyond OpenMP threads and no exchange step
between solves (one case per process, main.cpp:37-271), so the engine shards
whole solves across GPUs and never moves lattice data between them.  The
only collective is the bookkeeping of a measurement: the slowest rank's time
(max over ranks) and the total node updates (sum over ranks), through
torch.distributed (NCCL between GPUs, gloo on the host).
"""
import datetime
import os


def init(backend="nccl", timeout_s=120):
    """Join the process group described by the torchrun environment
    (RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT); returns (dist, rank, world)
    or (None, 0, 1) outside torchrun."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None, 0, 1
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist, dist.get_rank(), dist.get_world_size()


def reduce(values, dist, op="max", device="cpu"):
    """Elementwise max or sum of a list of floats over all ranks."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return t.tolist()


def aggregate(ms, updates, dist, device="cpu"):
    """Whole-job throughput of replicas: total node updates over all ranks
    divided by the slowest rank's time; returns (mlups, ms_max, updates_sum)."""
    ms_max = reduce([ms], dist, "max", device)[0]
    total = reduce([float(updates)], dist, "sum", device)[0]
    return total / (ms_max * 1e-3) / 1e6, ms_max, total


def finish(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
