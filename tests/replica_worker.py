"""A rank of the two-rank gloo tests of natray_b200.replicas (tests/test_replicas.py), started by
torch.multiprocessing.spawn. CPU only: the serving loop is the real one (natray_b200.serve.serve)
with a stand-in batch that finishes a scene after its steps, each of its steps taking
`step_ms[rank]` milliseconds, so that a slower rank has its slots free less often."""
import json
import os
import threading
import time


class FakeBatch:
    """Admission comes from the serving loop's admission thread, the rest from its own: a lock
    keeps the slots consistent, as the library's batch lock does."""

    def __init__(self, max_scenes: int, step_s: float):
        self.max_scenes, self.step_s = max_scenes, step_s
        self.slots: dict[int, list[int]] = {}
        self.mu = threading.Lock()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass

    def admit(self, world, steps):
        with self.mu:
            if len(self.slots) >= self.max_scenes:
                return None
            k = min(set(range(self.max_scenes)) - set(self.slots))
            self.slots[k] = [0, steps]
            return k

    def step(self, n):
        time.sleep(self.step_s)
        with self.mu:
            for v in self.slots.values():
                v[0] = min(v[0] + n, v[1])
            return sum(1 for v in self.slots.values() if v[0] < v[1])

    def poll(self, k):
        with self.mu:
            v = self.slots[k]
            return {"finished": v[0] >= v[1], "steps_done": v[0]}

    def retire(self, k):
        with self.mu:
            del self.slots[k]


def run(rank, port, n_requests, arrivals, step_ms, max_scenes, out_dir):
    import torch.distributed as dist

    from natray_b200.replicas import max_over_ranks, request_store, serve_replicas

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2)
    try:
        store = request_store(rank, 2, port=port + 1, host="127.0.0.1")
        worlds = [f"request {i}" for i in range(n_requests)]
        res = serve_replicas(worlds, arrivals, 8, 4, max_scenes, store=store,
                             batch_factory=lambda: FakeBatch(max_scenes, step_ms[rank] * 1e-3))
        m = max_over_ranks(1.5 + rank)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"merged": res, "max": m}, f)
    finally:
        dist.destroy_process_group()
