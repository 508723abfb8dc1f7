"""Batched runs and the serving loop over the batch engine (ntr_batch_*).

    python -m natray_b200.serve --scenes 64 --steps 500          # many mixed scenes in one batch
    python -m natray_b200.serve --serve 200 --steps 200 --rate 40 # Poisson arrivals, continuous batching

`mixed_scenes` draws seeded scenes of uneven size: particle counts log-uniform (or log-normal),
balloon diameter, projectile speed, and a membrane that is finer for bigger balloons. The batched
run builds its worlds before timing; the serving loop builds each request's world on a host
thread when the request arrives, so that its latency includes the build.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from .batch import Batch
from .sim import Sim
from .world import Params, World, build_world, sized_for


def scene_params(n_particles: int, diameter_cm: float, speed: float, seed: int) -> Params:
    """A balloon of `diameter_cm` filled with about `n_particles`, a steel sphere of 8 mm at
    `speed`; the membrane's level grows with the diameter (triangles ~ d^2), and the block and
    spray capacities are sized to the scene."""
    level = 4 if diameter_cm < 8.0 else (5 if diameter_cm < 12.0 else 6)
    return Params(diameter=diameter_cm, resolution=sized_for(n_particles, diameter_cm), mesh_level=level, bullet=6, caliber=8,
                  bullet_speed=speed, dt_max=2e-6, seed=seed, block_cap=min(65535, n_particles // 100 + 512),
                  spray_cap=max(16384, n_particles))


def mixed_scenes(n: int, seed: int, lo: int = 16_000, hi: int = 512_000, lognormal_median: int | None = None) -> list[Params]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if lognormal_median:
            npart = int(np.clip(rng.lognormal(math.log(lognormal_median), 1.0), lo, hi))
        else:
            npart = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        # Radius 3-8 cm; a balloon at the rubber's rest size (6 cm) does not inflate, so from 6.5 cm.
        d = float(rng.uniform(6.5, 16.0))
        v = float(rng.uniform(150.0, 400.0))
        out.append(scene_params(npart, d, v, seed * 1000 + i + 1))
    return out


def build_worlds(params: list[Params], threads: int = 16) -> list[World]:
    """The scenes' worlds, built on host threads (the builder releases the interpreter)."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        return list(ex.map(build_world, params))


def run_batched(worlds: list[World], steps: int, chunk: int = 4, max_scenes: int = 64, tune_steps: int = 0) -> dict:
    """All scenes admitted into one batch and stepped together to `steps` steps each. With
    `tune_steps`, the launch shapes are first chosen by the batch autotuner on a throwaway batch
    of the same scenes (its tuning steps are not part of the timed run)."""
    tuning = None
    if tune_steps:
        with Batch(max_scenes=max_scenes) as tb:
            for w in worlds:
                tb.admit(w, 1 << 30)
            tuning, _ = tb.autotune(tune_steps)
    with Batch(max_scenes=max_scenes) as b:
        if tuning:
            b.tuning = tuning
        slots = [b.admit(w, steps) for w in worlds]
        if None in slots:
            raise RuntimeError("the batch could not hold every scene")
        t0 = time.perf_counter()
        calls = 0
        while b.step(chunk):
            calls += 1
        wall = time.perf_counter() - t0
        done = [b.poll(s)["steps_done"] for s in slots]
        info = b.info()
    n_ps = sum(w.h.n_particles * d for w, d in zip(worlds, done))
    return {"seconds": wall, "scenes_per_s": len(worlds) / wall, "particle_steps_per_s": n_ps / wall, "calls": calls,
            "graph_captures": info["captures"], "graph_instantiations": info["instantiations"], "tuning": tuning}


def run_sequential(worlds, steps: int, chunk: int = 4, build=None) -> dict:
    """The same scenes one after the other, each a Sim of its own. With `build`, `worlds` are the
    scenes' parameters and each is built just before it runs (its time counts with its setup)."""
    times, with_setup = [], []
    t_all = time.perf_counter()
    n_ps = 0
    for w in worlds:
        t_setup = time.perf_counter()
        if build:
            w = build(w)
        s = Sim(world=w)
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            got = s.step(min(chunk, steps - done))
            if got == 0:
                break
            done += got
        times.append(time.perf_counter() - t0)
        n_ps += w.h.n_particles * done
        s.close()
        with_setup.append(time.perf_counter() - t_setup)
    wall = time.perf_counter() - t_all
    busy = sum(times)
    return {"seconds": busy, "seconds_with_setup": wall, "scenes_per_s": len(worlds) / busy, "particle_steps_per_s": n_ps / busy,
            "per_scene_seconds": times, "per_scene_seconds_with_setup": with_setup}


class LocalRequests:
    """The requests of one server: each can be taken once it has arrived, in arrival order."""

    def __init__(self, arrivals: list[float]):
        self.arrivals = list(arrivals)
        self.next = 0

    def claim(self, now: float) -> int | None:
        if self.next < len(self.arrivals) and self.arrivals[self.next] <= now:
            self.next += 1
            return self.next - 1
        return None

    def exhausted(self) -> bool:
        return self.next >= len(self.arrivals)

    def wait_hint(self, now: float) -> float:
        """Seconds until the next request arrives (0 if one has, or none is left)."""
        return max(0.0, self.arrivals[self.next] - now) if self.next < len(self.arrivals) else 0.0


class SharedRequests:
    """The requests of several servers (one per GPU), dispatched as their slots free up: a server
    with room claims the next request in arrival order from a counter that every server shares
    (an atomic add on a torch.distributed store), and takes it when it arrives. Each request goes
    to exactly one server, the first to have room for it."""

    def __init__(self, store, arrivals: list[float], key: str = "ntr/serve/next"):
        self.store, self.key = store, key
        self.arrivals = list(arrivals)
        self.pending: int | None = None
        self.out = False

    def claim(self, now: float) -> int | None:
        if self.pending is None and not self.out:
            i = int(self.store.add(self.key, 1)) - 1
            if i >= len(self.arrivals):
                self.out = True
            else:
                self.pending = i
        if self.pending is not None and self.arrivals[self.pending] <= now:
            i, self.pending = self.pending, None
            return i
        return None

    def exhausted(self) -> bool:
        return self.out and self.pending is None

    def wait_hint(self, now: float) -> float:
        return max(0.0, self.arrivals[self.pending] - now) if self.pending is not None else 0.0


def serve(worlds, arrivals: list[float], steps: int, chunk: int = 4, max_scenes: int = 64, *, requests=None,
          build=None, build_threads: int = 8, batch_factory=None, clock=None) -> dict:
    """Continuous batching: a request enters the batch when it has arrived (and, with `build`,
    its scene has been built on a host thread, which its latency includes) and a slot and the
    device memory are free, runs `steps` steps among the others, and leaves. Latency = completion
    - arrival. Scenes are admitted by a thread of their own, in arrival order, while the batch
    steps: ntr_batch_admit creates a scene in a free slot beside a running batch step (its
    uploads on the slot's own stream), so admitting does not hold up the GPU.

    worlds         the requests' worlds, or their parameters when `build` (a function of them
                   returning a World, natray_b200.build_world) builds each on its arrival
    requests       where requests come from: LocalRequests(arrivals) by default, SharedRequests
                   when several servers share one stream
    batch_factory  makes the batch (natray_b200.batch.Batch); tests pass a stand-in"""
    import threading
    from collections import deque
    from concurrent.futures import ThreadPoolExecutor

    requests = requests or LocalRequests(arrivals)
    batch_factory = batch_factory or (lambda: Batch(max_scenes=max_scenes))
    clock = clock or time.perf_counter
    finish: dict[int, float] = {}
    slot_req: dict[int, int] = {}
    pool = ThreadPoolExecutor(max_workers=max(1, build_threads)) if build else None
    # The admission thread's queue (requests taken, in arrival order, with their worlds or the
    # builds of them) and its output (requests placed, with their slots); `room` wakes it when a
    # slot frees up.
    pending: deque = deque()
    placed: deque = deque()
    cv = threading.Condition()
    stop = [False]
    errors: list = []
    # Where the time goes: admitting scenes (on the admission thread), stepping, polling and
    # retiring, waiting with nothing to step; and how full the batch was, step call by step call.
    t_admit = [0.0]
    t_step = t_poll = t_idle = 0.0
    calls, occupancy = 0, 0

    def admitter(b):
        try:
            while True:
                with cv:
                    while not pending and not stop[0]:
                        cv.wait()
                    if not pending:
                        return
                    i, w = pending[0]
                if build:
                    w = w.result()
                while True:
                    ta = clock()
                    sl = b.admit(w, steps)
                    t_admit[0] += clock() - ta
                    if sl is not None:
                        break
                    with cv:  # no room: wait for a slot to free up
                        if stop[0]:
                            return
                        cv.wait(timeout=0.005)
                with cv:
                    pending.popleft()
                    placed.append((i, sl))
        except BaseException as e:  # surfaced on the serving thread
            errors.append(e)

    try:
        with batch_factory() as b:
            th = threading.Thread(target=admitter, args=(b,), daemon=True)
            th.start()
            t0 = clock()
            try:
                while True:
                    if errors:
                        raise errors[0]
                    now = clock() - t0
                    with cv:
                        while placed:
                            i, sl = placed.popleft()
                            slot_req[sl] = i
                        # Take requests while the batch has room for them (queued ones count).
                        while len(slot_req) + len(pending) < max_scenes:
                            i = requests.claim(now)
                            if i is None:
                                break
                            pending.append((i, pool.submit(build, worlds[i]) if build else worlds[i]))
                            cv.notify_all()
                        waiting = len(pending)
                    if not slot_req:
                        if requests.exhausted() and not waiting:
                            break
                        tb = clock()
                        time.sleep(min(requests.wait_hint(clock() - t0), 0.002) if not waiting else 0.0005)
                        t_idle += clock() - tb
                        continue
                    tb = clock()
                    b.step(chunk)
                    tc = clock()
                    t_step += tc - tb
                    calls += 1
                    occupancy += len(slot_req)
                    now = tc - t0
                    freed = False
                    for sl in list(slot_req):
                        if b.poll(sl)["finished"]:
                            finish[slot_req.pop(sl)] = now
                            b.retire(sl)
                            freed = True
                    if freed:
                        with cv:
                            cv.notify_all()
                    t_poll += clock() - tc
                makespan = clock() - t0
            finally:
                with cv:
                    stop[0] = True
                    cv.notify_all()
                th.join()
            info = b.info() if hasattr(b, "info") else {}
    finally:
        if pool:
            pool.shutdown(wait=True)
    served = sorted(finish)
    lat = np.array([finish[i] - arrivals[i] for i in served])
    out = {"requests": len(served), "seconds": makespan, "scenes_per_s": len(served) / makespan if makespan > 0 else 0.0,
           "latencies": [float(x) for x in lat], "requests_served": served,
           "loop": {"admit_s": t_admit[0], "step_s": t_step, "poll_s": t_poll, "idle_s": t_idle, "step_calls": calls,
                    "mean_scenes_per_call": occupancy / calls if calls else 0.0,
                    "graph_captures": info.get("captures"), "graph_instantiations": info.get("instantiations")}}
    if lat.size:
        out.update({"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean())})
    return out


def sequential_timeline(arrivals: list[float], durations: list[float]) -> dict:
    """One request at a time in arrival order (each taking its measured time alone)."""
    t = 0.0
    lat = []
    for a, d in zip(arrivals, durations):
        t = max(t, a) + d
        lat.append(t - a)
    lat = np.array(lat)
    return {"seconds": t, "scenes_per_s": len(arrivals) / t, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean())}


def poisson_arrivals(n: int, rate: float, seed: int) -> list[float]:
    rng = np.random.default_rng(seed)
    return list(np.cumsum(rng.exponential(1.0 / rate, n)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=16)
    ap.add_argument("--serve", type=int, default=0, help="requests of the serving loop (0: the batched run)")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--chunk", type=int, default=4)
    ap.add_argument("--rate", type=float, default=40.0, help="requests per second")
    ap.add_argument("--seed", type=int, default=7)
    args = ap.parse_args()
    import os
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        # Under torchrun: one process per GPU, each with its own batch; the requests go to the
        # ranks as their slots free up (natray_b200.replicas), each built by the rank that takes
        # it when it arrives, and the results are merged on rank 0.
        import torch
        import torch.distributed as dist
        from .replicas import serve_replicas
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl")
        n = args.serve or args.scenes
        ps = mixed_scenes(n, args.seed, lo=16_000, hi=2_000_000, lognormal_median=128_000)
        res = serve_replicas(ps, poisson_arrivals(n, args.rate, args.seed), args.steps, args.chunk, build=build_world)
        if res is not None:
            res.pop("latencies", None)
            print(json.dumps({"served": res}))
        dist.destroy_process_group()
        return
    if args.serve:
        ps = mixed_scenes(args.serve, args.seed, lo=16_000, hi=2_000_000, lognormal_median=128_000)
        arr = poisson_arrivals(args.serve, args.rate, args.seed)
        # Each request's scene is built when it arrives: its latency includes the build.
        out = {"served": serve(ps, arr, args.steps, args.chunk, build=build_world)}
        out["served"].pop("latencies", None)
        seq = run_sequential(ps, args.steps, args.chunk, build=build_world)
        # A request served alone pays for its scene's build and its simulation's creation too.
        out["sequential"] = sequential_timeline(arr, seq["per_scene_seconds_with_setup"])
    else:
        worlds = build_worlds(mixed_scenes(args.scenes, args.seed))
        out = {"batched": run_batched(worlds, args.steps, args.chunk)}
        seq = run_sequential(worlds, args.steps, args.chunk)
        seq.pop("per_scene_seconds"), seq.pop("per_scene_seconds_with_setup")
        out["sequential"] = seq
    print(json.dumps(out))


if __name__ == "__main__":
    main()
