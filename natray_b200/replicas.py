"""Scenes on several GPUs: one process per GPU (torch.distributed, launched by torchrun), each
with its own batch, and no collective on the data path. A scene is one coupled system (two
global reductions per solver iteration; the membrane, air and block set are global every step)
that fits one B200, so the GPUs share out whole scenes: replicas, not a split scene.

    partition_requests   the request stream shared out across the ranks, least loaded first
                         (the rank with the most free device memory left takes the next request)
    merge_results        the ranks' serving results as one (throughput, p50/p99 latency)
    serve_replicas       the serving loop on every rank over its share, the results gathered
    max_over_ranks       a device time as the maximum over the ranks (the bench's clock)

Only host objects cross between the ranks (free memory, the plan is computed alike on every
rank, and the results at the end), with gloo or NCCL alike.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import check, lib
from .world import World, blob_arg


def device_bytes(world: World | bytes) -> int:
    """The device memory a simulation of the world takes (ntr_world_device_bytes)."""
    blob, size = blob_arg(world)
    n = C.c_uint64()
    check(lib().ntr_world_device_bytes(blob, size, C.byref(n)))
    return n.value


def partition_requests(need: list[int], free: list[int]) -> list[list[int]]:
    """Requests (in arrival order, each needing `need[i]` bytes) to ranks (with `free[r]` bytes
    free): each goes to the rank with the most free memory left (the lowest rank among equals),
    which is then charged for it. A request larger than every rank's remainder still goes to the
    rank with the most left, where it waits for memory in that rank's batch."""
    left = [int(f) for f in free]
    plan: list[list[int]] = [[] for _ in free]
    for i, b in enumerate(need):
        r = max(range(len(left)), key=lambda k: (left[k], -k))
        plan[r].append(i)
        left[r] -= int(b)
    return plan


def merge_results(results: list[dict]) -> dict:
    """One serving result from the ranks': requests summed, the makespan the longest, the
    latency percentiles over every request."""
    lat = np.concatenate([np.asarray(r.get("latencies", []), dtype=np.float64) for r in results]) if results else np.zeros(0)
    n = int(sum(r["requests"] for r in results))
    seconds = max((r["seconds"] for r in results), default=0.0)
    out = {"requests": n, "seconds": seconds, "scenes_per_s": n / seconds if seconds > 0 else 0.0, "ranks": len(results),
           "per_rank": [r["requests"] for r in results]}
    if lat.size:
        out.update({"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean())})
    return out


def serve_replicas(worlds: list[World], arrivals: list[float], steps: int, chunk: int = 4, max_scenes: int = 64,
                   serve_fn=None, free: int | None = None) -> dict | None:
    """The serving loop on every rank of the initialised process group, over the rank's share of
    the requests (partition_requests on every rank's free device memory). Returns the merged
    result on rank 0, None on the others. `serve_fn(worlds, arrivals, steps, chunk, max_scenes)`
    defaults to natray_b200.serve.serve; `free` to this rank's free device memory."""
    import torch.distributed as dist

    if serve_fn is None:
        from .serve import serve as serve_fn
    if free is None:
        import torch
        free = int(torch.cuda.mem_get_info()[0])
    rank, size = dist.get_rank(), dist.get_world_size()
    frees: list = [None] * size
    dist.all_gather_object(frees, int(free))
    plan = partition_requests([device_bytes(w) for w in worlds], frees)
    mine = plan[rank]
    dist.barrier()  # a common start for the arrival clock
    res = serve_fn([worlds[i] for i in mine], [arrivals[i] for i in mine], steps, chunk, max_scenes) if mine else \
        {"requests": 0, "seconds": 0.0, "latencies": []}
    res["requests_served"] = list(mine)
    gathered: list = [None] * size
    dist.all_gather_object(gathered, res)
    if rank != 0:
        return None
    out = merge_results(gathered)
    out["plan"] = plan
    return out


def max_over_ranks(x: float) -> float:
    """The maximum of x over the ranks (the bench's device time): a CPU tensor under gloo, a
    tensor on this rank's GPU under NCCL."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
