"""Multi-GPU search: DM trials sharded across ranks, one process per GPU.

The reference searches DM trials in parallel with a process pool, one trial per task
(pipeline/worker_pool.py:35-68). Trials are independent, so on several GPUs each rank
searches a contiguous shard of the trials (balanced by sample count, which the search cost
follows) and there is no exchange on the data path. The periodograms come back to the host
of their rank; gathering them on one rank is a host-side step (torch.distributed object
gather), and timings are reduced with a MAX over ranks.

Ranks are set up from the usual torchrun environment (RANK, WORLD_SIZE, LOCAL_RANK,
MASTER_ADDR, MASTER_PORT). The process group uses NCCL when CUDA is present and gloo
otherwise (the host-side logic is tested on CPU with gloo).
"""
import datetime
import os

import numpy as np


def init_from_env(backend=None, timeout_s=600):
    """Join the process group described by the environment. Returns (world, rank, local).
    With WORLD_SIZE unset or 1 no group is created."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def _group_device():
    import torch
    import torch.distributed as dist

    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def shard_bounds(lengths, world):
    """Contiguous shards of the trials, one per rank, with near-equal total samples: shard r
    is trials [bounds[r], bounds[r + 1]). Every shard is non-empty when there are at least
    `world` trials."""
    lengths = np.asarray(lengths, dtype=np.int64).ravel()
    n = lengths.size
    if world < 1:
        raise ValueError("world must be at least 1")
    if n == 0:
        return np.zeros(world + 1, dtype=np.int64)
    csum = np.concatenate([[0], np.cumsum(lengths)])
    total = csum[-1]
    bounds = [0]
    for r in range(1, world):
        # first trial boundary whose prefix reaches r / world of the samples
        k = int(np.searchsorted(csum, total * r / world, side="left"))
        if n >= world:  # every shard keeps at least one trial
            k = min(max(k, bounds[-1] + 1), n - (world - r))
        else:
            k = min(max(k, bounds[-1]), n)
        bounds.append(k)
    bounds.append(n)
    return np.asarray(bounds, dtype=np.int64)


def shard_range(lengths, rank, world):
    """(start, stop) of the trials that rank `rank` searches."""
    b = shard_bounds(lengths, world)
    return int(b[rank]), int(b[rank + 1])


def max_over_ranks(value, world=None):
    """Maximum of a per-rank float over all ranks (the job's time is the slowest rank's)."""
    if world is None:
        world = int(os.environ.get("WORLD_SIZE", "1"))
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=_group_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world=None):
    if world is None:
        world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def gather_to_root(local_items, rank, world, root=0):
    """Concatenate the per-rank lists (in rank order, i.e. trial order for contiguous shards)
    on `root`; other ranks get None. Host objects, no device traffic."""
    if world == 1:
        return list(local_items)
    import torch.distributed as dist

    out = [None] * world if rank == root else None
    dist.gather_object(list(local_items), out, dst=root)
    if rank != root:
        return None
    return [x for part in out for x in part]


def search_sharded(series, tsamp, rank, world, search=None, root=0, **search_kw):
    """Search the trials `series` (list of 1D float arrays, identical on every rank) with
    each rank taking its shard; returns the list of Periodogram on `root` (trial order) and
    None elsewhere. `search(shard_series, tsamp, **search_kw)` defaults to this package's
    GPU pipeline (SearchPipeline); any callable returning one result per trial works."""
    lengths = [int(np.asarray(s).size) for s in series]
    start, stop = shard_range(lengths, rank, world)
    local = list(series[start:stop])
    if search is None:
        search = _pipeline_search
    results = search(local, tsamp, **search_kw) if local else []
    return gather_to_root(results, rank, world, root=root)


def _pipeline_search(series, tsamp, chunk_trials=16, **search_kw):
    from .batched import SearchPipeline

    pipe = SearchPipeline([s.size for s in series], tsamp, chunk_trials=chunk_trials,
                          **search_kw)
    try:
        return pipe.search(series)
    finally:
        pipe.close()
