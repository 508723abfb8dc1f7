"""Per-kernel device time of the simulation step, the reference's NATRAY_PROF
(src/sim.rs:594-614, 670-689) as a command:

    python -m natray_b200.prof [--resolution 124] [--warmup 3] [--steps 5] [--graph-steps 10] [--keyframes 0]
    python -m natray_b200.prof --batch 64 [--warmup 8] [--graph-steps 16] [--steps 4]

Builds the 1M-particle scene of the benchmark (or another resolution), runs warm-up batches,
times `--graph-steps` steps through the step's CUDA graph, then runs `--steps` steps kernel by
kernel with events between them and prints each kernel's share. With `--keyframes N` it then
stores N keyframes (the reference's Cache, src/cache.rs) 4 us of simulated time apart and shows
the midpoint of each pair, printing their device times.
"""
from __future__ import annotations

import argparse

from .sim import Sim
from .world import Params, build_world


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--resolution", type=int, default=124)
    ap.add_argument("--mesh-level", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--graph-steps", type=int, default=10)
    ap.add_argument("--speed", type=float, default=350.0)
    ap.add_argument("--diameter", type=float, default=0.0, help="balloon diameter in cm (0: the scene default)")
    ap.add_argument("--thickness", type=float, default=0.0, help="rubber thickness in mm (0: the scene default)")
    ap.add_argument("--keyframes", type=int, default=0)
    ap.add_argument("--batch", type=int, default=0, help="profile a batch of this many mixed scenes instead")
    args = ap.parse_args()
    if args.batch:
        return batch_profile(args)
    extra = {}
    if args.diameter:
        extra["diameter"] = args.diameter
    if args.thickness:
        extra["thickness"] = args.thickness
    w = build_world(Params(resolution=args.resolution, mesh_level=args.mesh_level, dt_max=2e-6, bullet=6, caliber=8,
                           bullet_speed=args.speed, **extra))
    s = Sim(world=w)
    s.step(args.warmup)
    n = s.step(args.graph_steps)
    launches, ms = s.last_launches()
    st = s.state
    print(f"{w.h.n_particles} particles: graph {ms / max(n, 1):.3f} ms/step, {launches / max(n, 1):.0f} launches/step, "
          f"{st['n_blocks']} blocks, {st['solve_iters']} solver iterations")
    if args.steps:
        p = s.profile(args.steps)
        tot = sum(v[1] for v in p.values())
        print(f"kernel by kernel: {tot / args.steps:.3f} ms/step")
        for k, (c, t) in sorted(p.items(), key=lambda kv: -kv[1][1]):
            print(f"  {k:24s} {c:5d} launches {t / args.steps * 1e3:9.1f} us/step {100 * t / tot:5.1f}%")
    if args.keyframes:
        from .cache import Cache
        c = Cache(s)
        for _ in range(args.keyframes):
            s.advance(s._info().t + 4e-6, 16)
            c.store()
            i_ms, p_ms, _ = c.last_times()
            k = c.keys()[-1]
            print(f"keyframe at {k['t'] * 1e3:.4f} ms: {k['bytes']} B, {k['spray']} spray slots ({k['live']} live); "
                  f"index {i_ms * 1e3:.1f} us, pack {p_ms * 1e3:.1f} us")
        keys = c.keys()
        for a, b in zip(keys[1:], keys[2:]):
            c.show(0.5 * (a["t"] + b["t"]))
            print(f"show at {0.5 * (a['t'] + b['t']) * 1e3:.4f} ms: {c.last_times()[2] * 1e3:.1f} us")
        c.close()


def batch_profile(args):
    """The batch engine on the bench's mixed scenes: graph-timed batch steps, then one call of
    `--steps` steps kernel by kernel (ntr_batch_profile)."""
    import time

    from .batch import Batch
    from .serve import build_worlds, mixed_scenes
    worlds = build_worlds(mixed_scenes(args.batch, 7))
    n_p = sum(w.h.n_particles for w in worlds)
    with Batch(max_scenes=max(64, args.batch)) as b:
        for w in worlds:
            assert b.admit(w, 100000) is not None
        b.step(args.warmup)
        t0 = time.perf_counter()
        b.step(args.graph_steps)
        dt = time.perf_counter() - t0
        print(f"{len(worlds)} scenes, {n_p} particles: {dt / max(args.graph_steps, 1) * 1e3:.3f} ms per batch step (graph, "
              f"host-timed, states read back once)")
        if args.steps:
            p = b.profile(args.steps)
            tot = sum(v[1] for v in p.values())
            print(f"kernel by kernel: {tot / args.steps:.3f} ms per batch step")
            for k, (c, t) in sorted(p.items(), key=lambda kv: -kv[1][1]):
                print(f"  {k:24s} {c:5d} launches {t / args.steps * 1e3:9.1f} us/step {100 * t / tot:5.1f}%")


if __name__ == "__main__":
    main()
