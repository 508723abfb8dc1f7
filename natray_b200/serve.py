"""Batched runs and the serving loop over the batch engine (ntr_batch_*).

    python -m natray_b200.serve --scenes 64 --steps 500          # many mixed scenes in one batch
    python -m natray_b200.serve --serve 200 --steps 200 --rate 40 # Poisson arrivals, continuous batching

`mixed_scenes` draws seeded scenes of uneven size: particle counts log-uniform (or log-normal),
balloon diameter, projectile speed, and a membrane that is finer for bigger balloons. Worlds are
built on the host before timing; the timed part is the GPU work and the host loop around it.
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


def run_batched(worlds: list[World], steps: int, chunk: int = 4, max_scenes: int = 64) -> dict:
    """All scenes admitted into one batch and stepped together to `steps` steps each."""
    with Batch(max_scenes=max_scenes) as b:
        slots = [b.admit(w, steps) for w in worlds]
        if None in slots:
            raise RuntimeError("the batch could not hold every scene")
        t0 = time.perf_counter()
        while b.step(chunk):
            pass
        wall = time.perf_counter() - t0
        done = [b.poll(s)["steps_done"] for s in slots]
    n_ps = sum(w.h.n_particles * d for w, d in zip(worlds, done))
    return {"seconds": wall, "scenes_per_s": len(worlds) / wall, "particle_steps_per_s": n_ps / wall}


def run_sequential(worlds: list[World], steps: int, chunk: int = 4) -> dict:
    """The same scenes one after the other, each a Sim of its own."""
    times, with_setup = [], []
    t_all = time.perf_counter()
    n_ps = 0
    for w in worlds:
        t_setup = time.perf_counter()
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


def serve(worlds: list[World], arrivals: list[float], steps: int, chunk: int = 4, max_scenes: int = 64) -> dict:
    """Continuous batching: a request enters the batch at its arrival time or as soon as a slot
    and the device memory free up, runs `steps` steps, and leaves. Latency = completion - arrival."""
    n = len(worlds)
    finish = [0.0] * n
    queue: list[int] = []
    nxt = 0
    slot_req: dict[int, int] = {}
    with Batch(max_scenes=max_scenes) as b:
        t0 = time.perf_counter()
        while nxt < n or queue or slot_req:
            now = time.perf_counter() - t0
            while nxt < n and arrivals[nxt] <= now:
                queue.append(nxt)
                nxt += 1
            while queue:
                sl = b.admit(worlds[queue[0]], steps)
                if sl is None:
                    break
                slot_req[sl] = queue.pop(0)
            if not slot_req:
                if nxt < n:
                    time.sleep(max(0.0, arrivals[nxt] - (time.perf_counter() - t0)))
                continue
            b.step(chunk)
            now = time.perf_counter() - t0
            for sl in list(slot_req):
                if b.poll(sl)["finished"]:
                    finish[slot_req.pop(sl)] = now
                    b.retire(sl)
        makespan = time.perf_counter() - t0
    lat = np.array([f - a for f, a in zip(finish, arrivals)])
    return {"requests": n, "seconds": makespan, "scenes_per_s": n / makespan, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "latencies": [float(x) for x in lat]}


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
        # Under torchrun: one process per GPU, the request stream shared out by free device
        # memory (natray_b200.replicas), the results merged on rank 0.
        import torch
        import torch.distributed as dist
        from .replicas import serve_replicas
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl")
        n = args.serve or args.scenes
        ps = mixed_scenes(n, args.seed, lo=16_000, hi=2_000_000, lognormal_median=128_000)
        worlds = build_worlds(ps)
        res = serve_replicas(worlds, poisson_arrivals(n, args.rate, args.seed), args.steps, args.chunk)
        if res is not None:
            res.pop("plan", None)
            print(json.dumps({"served": res}))
        dist.destroy_process_group()
        return
    if args.serve:
        ps = mixed_scenes(args.serve, args.seed, lo=16_000, hi=2_000_000, lognormal_median=128_000)
        worlds = build_worlds(ps)
        arr = poisson_arrivals(args.serve, args.rate, args.seed)
        out = {"served": serve(worlds, arr, args.steps, args.chunk)}
        seq = run_sequential(worlds, args.steps, args.chunk)
        # A request served alone pays for its simulation's creation too, as in the batch.
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
