"""Scenes on several GPUs: one process per GPU (torch.distributed, launched by torchrun), each
with its own batch, and no collective on the data path. A scene is one coupled system (two
global reductions per solver iteration; the membrane, air and block set are global every step)
that fits one B200, so the GPUs share out whole scenes: replicas, not a split scene.

    serve_replicas       the serving loop on every rank, the requests dispatched as the ranks'
                         slots free up (each claims the next request in arrival order from a
                         counter in a shared store when it has room), the results gathered
    merge_results        the ranks' serving results as one (throughput, p50/p99 latency)
    max_over_ranks       a device time as the maximum over the ranks (the bench's clock)

Only host objects cross between the ranks: the claim counter (an atomic add on a TCP store),
and the results at the end, with gloo or NCCL alike.
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


def request_store(rank: int, world_size: int, port: int | None = None, host: str | None = None):
    """The store the ranks share the request counter through: a TCP store on MASTER_ADDR, one
    port above MASTER_PORT (rank 0 hosts it)."""
    import os
    from datetime import timedelta

    import torch.distributed as dist

    host = host or os.environ.get("MASTER_ADDR", "127.0.0.1")
    port = port or int(os.environ.get("MASTER_PORT", "29500")) + 1
    return dist.TCPStore(host, port, world_size, rank == 0, timeout=timedelta(seconds=120))


def serve_replicas(worlds, arrivals: list[float], steps: int, chunk: int = 4, max_scenes: int = 64, serve_fn=None,
                   store=None, build=None, batch_factory=None) -> dict | None:
    """The serving loop on every rank of the initialised process group, the requests dispatched
    as slots free up (natray_b200.serve.SharedRequests on `store`, request_store by default).
    `worlds` are the requests' worlds, or their parameters with `build` (each rank builds what it
    takes, on its arrival). Returns the merged result on rank 0, None on the others."""
    import torch.distributed as dist

    from .serve import SharedRequests, serve

    serve_fn = serve_fn or serve
    rank, size = dist.get_rank(), dist.get_world_size()
    if store is None:
        store = request_store(rank, size)
    dist.barrier()  # a common start for the arrival clock
    res = serve_fn(worlds, arrivals, steps, chunk, max_scenes, requests=SharedRequests(store, arrivals), build=build,
                   batch_factory=batch_factory)
    gathered: list = [None] * size
    dist.all_gather_object(gathered, res)
    if rank != 0:
        return None
    out = merge_results(gathered)
    out["served_by_rank"] = [r.get("requests_served", []) for r in gathered]
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
