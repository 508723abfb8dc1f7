"""Precision study of the 1M-particle scene: the product (FP32 state and grid arithmetic, FP64
solver inner products and residual norm, on the GPU) against the oracle with every real in FP64,
from the same start, with relative L2 errors every `--every` steps of positions, velocities,
particle pressure, membrane positions and the membrane's major principal stretch (per intact
triangle, from C = F^T F as shaders/membrane.wgsl:89-104 forms it).

It runs twice: with the solver's stopping tolerance of the scene (relative residual 1e-5, the
reference's, src/sim.rs:20) and with a tight one (1e-7) on both sides, which separates the FP32
arithmetic's own error from the difference the stopping tolerance leaves between two runs that
stop at different iterates.

    python tests/precision_study.py [--resolution 124] [--steps 1000] [--every 100] [--speed 350] [--out FILE]

Prints a table per tolerance and writes all figures as JSON to --out. Test infrastructure: it
drives the oracle. Needs a GPU.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path[:0] = [str(HERE.parent), str(HERE)]

from natray_b200 import Params, World, build_world  # noqa: E402
from natray_b200.sim import Sim  # noqa: E402
from oracle.py import Oracle  # noqa: E402


def rel(x, y) -> float:
    x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-30))


def major_stretch(w: World) -> np.ndarray:
    """Major principal stretch of every triangle (f64), from the current and rest shapes."""
    x = w.sec("MEM_X")[:, :3].astype(np.float64)
    t = w.sec("TRIS")
    v = t[:, :3].astype(np.int64)
    m = t[:, 4:8].view(np.float32).astype(np.float64).reshape(-1, 2, 2)
    e1, e2 = x[v[:, 1]] - x[v[:, 0]], x[v[:, 2]] - x[v[:, 0]]
    f0 = e1 * m[:, 0, 0:1] + e2 * m[:, 1, 0:1]
    f1 = e1 * m[:, 0, 1:2] + e2 * m[:, 1, 1:2]
    c00, c01, c11 = (f0 * f0).sum(1), (f0 * f1).sum(1), (f1 * f1).sum(1)
    mid = 0.5 * (c00 + c11)
    dev = np.sqrt(0.25 * (c00 - c11) ** 2 + c01 * c01)
    return np.sqrt(mid + dev)


def compare(a: World, b: World) -> dict:
    pa, pb = a.particles, b.particles
    alive = (a.sec("ALIVE") != 0) & (b.sec("ALIVE") != 0)
    return {"step": int(a.state["step"]), "t_us": a.state["t_ns"] * 1e-3,
            "x": rel(pa[:, :3], pb[:, :3]), "v": rel(pa[:, 4:7], pb[:, 4:7]), "p": rel(pa[:, 11], pb[:, 11]),
            "mem_x": rel(a.sec("MEM_X")[:, :3], b.sec("MEM_X")[:, :3]),
            "stretch": rel(major_stretch(a)[alive], major_stretch(b)[alive]),
            "torn": [int((a.sec("ALIVE") == 0).sum()), int((b.sec("ALIVE") == 0).sum())],
            "iters": [int(a.h.iters), int(b.h.iters)]}


def study(resolution: int, steps: int, every: int, tol: float, mesh_level: int = 6, speed: float = 350.0) -> list[dict]:
    params = Params(resolution=resolution, mesh_level=mesh_level, dt_max=2e-6, bullet=6, caliber=8, bullet_speed=speed,
                    solve_tol=tol)
    w = World(Oracle(build_world(params).blob).snapshot())  # the measuring substep on the CPU: both start alike
    sim, ref = Sim(world=w), Oracle(w.blob, real64=True)
    rows = []
    for k in range(steps // every):
        t0 = time.perf_counter()
        assert sim.step(every) == every
        assert ref.step(every) == every
        r = compare(sim.snapshot(), World(ref.snapshot()))
        r["oracle_s"] = time.perf_counter() - t0
        rows.append(r)
        print(f"  {r['step']:5d} {r['t_us']:8.1f}  {r['x']:.2e}  {r['v']:.2e}  {r['p']:.2e}  {r['mem_x']:.2e}  "
              f"{r['stretch']:.2e}  {r['torn']}", flush=True)
    sim.close()
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--resolution", type=int, default=124)
    ap.add_argument("--mesh-level", type=int, default=6)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--tols", default="1e-5,1e-7")
    ap.add_argument("--speed", type=float, default=350.0, help="the sphere's speed (1 m/s: it does not reach the balloon)")
    ap.add_argument("--out", default="")
    args = ap.parse_args()
    out = {"resolution": args.resolution, "mesh_level": args.mesh_level, "steps": args.steps, "speed": args.speed, "runs": {}}
    for tol in [float(t) for t in args.tols.split(",")]:
        print(f"solver tolerance {tol:g}: relative L2 against FP64")
        print("   step   t (us)      x          v          p        mem_x     stretch    torn (product, FP64)")
        out["runs"][f"{tol:g}"] = study(args.resolution, args.steps, args.every, tol, args.mesh_level, args.speed)
    if args.out:
        Path(args.out).write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
