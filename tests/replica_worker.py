"""A rank of the two-rank gloo tests of natray_b200.replicas (tests/test_replicas.py), started by
torch.multiprocessing.spawn. CPU only: the serving function is a stand-in that records what the
rank was given."""
import json
import os


def fake_serve(worlds, arrivals, steps, chunk, max_scenes):
    # every request finishes 10 ms after its arrival, the rank's run lasting until the last one
    lat = [0.01] * len(worlds)
    return {"requests": len(worlds), "seconds": (max(arrivals) + 0.01) if arrivals else 0.0, "latencies": lat,
            "arrivals": list(arrivals)}


def run(rank, port, blobs, arrivals, frees, out_dir):
    import torch.distributed as dist

    from natray_b200.replicas import max_over_ranks, serve_replicas
    from natray_b200.world import World

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2)
    try:
        worlds = [World(b) for b in blobs]
        res = serve_replicas(worlds, arrivals, 8, 4, 16, serve_fn=fake_serve, free=frees[rank])
        m = max_over_ranks(1.5 + rank)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"merged": res, "max": m}, f)
    finally:
        dist.destroy_process_group()
