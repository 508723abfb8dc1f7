"""Benchmark of natray's simulation step on B200: particle-substeps/s at ~1M particles.

A "step" here is one water step of the reference (one `Sim::run` step: begin_step .. g2p with
its rubber and air substeps and its pressure iterations, src/sim.rs:553-566), which the metric
calls a particle-substep. The workload is the full single scene at 1M particles: a 16 cm water
balloon on a lattice of resolution 124 (976,915 particles, spacing 1.29 mm, cell 2.58 mm), an
icosphere(6) latex membrane (40,962 vertices, 81,920 triangles), a rigid 8 mm steel sphere at
350 m/s, a fixed step of 2 us. Inputs are synthetic (the reference's seeded scene builder).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]

Prints one JSON line (rank 0). `--impl reference` times the CPU restatement of the reference's
step (the reference's own wgpu/WGSL path needs a graphics adapter, which this machine does
not have) on the same scene with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MEASURED_PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
METRIC = "particle-substeps/s @1M"
SCENE = dict(resolution=124, mesh_level=6, dt_max=2e-6, bullet=6, caliber=8, bullet_speed=350)
WORKLOAD = "single scene 1M particles: d=16 cm balloon, res 124 (976,915 particles), icosphere(6) 81,920 tris, 8 mm steel sphere at 350 m/s, dt=2 us"
# The small scene (d 8 cm, about 70k particles, 5,120 triangles, rubber 0.2 mm, 8 mm sphere at
# 300 m/s), timed over its 200 fixed steps of 2 us.
SMALL = dict(diameter=8, resolution=51, mesh_level=4, thickness=0.2, bullet=6, caliber=8, bullet_speed=300, dt_max=2e-6)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def hbm_peak() -> tuple[float, str]:
    try:
        d = json.loads(MEASURED_PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """SM clock and throttle reasons sampled during the timed region: NVML every millisecond
    from a thread (the region can be a few ms long), nvidia-smi every 25 ms if NVML is missing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*).
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown"}

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.samples: list[tuple[float, float, int]] = []
        self.t = None
        self.stop = threading.Event()
        self.nvml = None

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.nvml = (nv, h)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "25"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _poll(self):
        nv, h = self.nvml
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), self.max_mhz, int(get_reasons(h))))
            except Exception:
                pass
            time.sleep(0.001)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.t:
            self.t.join(timeout=2)

    def summary(self) -> dict:
        mhz, maxs, reasons = [], [], set()
        if self.nvml:
            for m, mx, r in self.samples:
                mhz.append(m)
                maxs.append(mx)
                reasons.update(n for bit, n in self.REASONS.items() if r & bit)
            src = "nvml, 1 ms"
        else:
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for ln in self.lines:
                f = [x.strip() for x in ln.split(",")]
                if len(f) < 9:
                    continue
                try:
                    mhz.append(float(f[1]))
                    maxs.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            src = "nvidia-smi, 25 ms"
        if not mhz:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": src}
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": max(maxs), "reasons": sorted(reasons), "samples": len(mhz),
                "source": src}


def algorithmic_bytes(kernel: str, st: dict, n_particles: int, iters: int) -> float:
    """Bytes a launch of `kernel` must move at the least, from the per-unit figures of the step:
    P2G reads a particle's 80 B and its index and writes its cells' particle counts (its tile of
    sums is this implementation's, not the algorithm's: the cells' sums are written by the tile
    gather); the solve reads d, z, diag, type, p, r, q and writes d', q, p, r, z per water cell
    and iteration (48 B) and sets up with 40 B per water cell; G2P reads a particle's 80 B, its
    index and its cells' 8 fields once (32 B per cell) and writes the particle's 80 B."""
    cells = st["n_blocks"] * 64
    if kernel.startswith("k_solve"):
        n_water = st.get("_n_water", cells)
        return 48.0 * n_water * max(iters, 1) + 40.0 * n_water
    if kernel == "k_p2g":
        return 84.0 * n_particles + 4.0 * cells
    if kernel.startswith("k_g2p"):
        return 164.0 * n_particles + 32.0 * cells
    return 0.0


def keyframe_bench(sim, reps: int, peak: float, wet_res: int) -> dict:
    """Keyframe store and show (the reference's Cache::bake / Cache::show) on the bench scene:
    `reps` keyframes 4 us of simulated time apart, then shows between them. A store's two device
    parts (spray index, packing) are timed with events on the simulation's stream; the shows are
    issued back to back (each call returns before its work is done) and timed as a run, so the
    device stays busy and host launch gaps do not count."""
    import numpy as np
    from natray_b200.cache import Cache

    info = sim.info
    n_p, n_v, n_t = info.n_particles, info.n_verts, info.n_tris
    c = Cache(sim)
    idx, pk, call, st_bytes = [], [], [], []
    for _ in range(reps):
        sim.advance(sim._info().t + 4e-6, 16)
        t0 = time.perf_counter()
        c.store()
        a, b, _ = c.last_times()
        call.append(time.perf_counter() - t0)
        idx.append(a * 1e-3)
        pk.append(b * 1e-3)
        k = c.keys()[-1]
        n, live = k["spray"], k["live"]
        # pack reads position (16 B) and the alive word (4 B) of a particle and writes 8 B; a vertex
        # 16 + 8; a triangle 4 + 1/8; a spray slot is read by the index (4 B) and the pack (24 B)
        # and its weights written (8 B); a live slot's 12 B and two words per 32 slots written.
        st_bytes.append(28 * n_p + 24 * n_v + 4.125 * n_t + 36 * n + 12 * live + 8 * ((n + 31) // 32))
    keys = c.keys()
    times = [0.5 * (a["t"] + b["t"]) for a, b in zip(keys[1:-1], keys[2:])]
    m = max(k["spray"] for k in keys)
    # two keyframes' particle words read (16 B) and the shown particle written (32 B); a vertex
    # 16 + 16; a triangle's flag written; a spray slot's words of both keys, its landing record
    # and weights read and 32 B written; the wet map cleared and the ground touch times read.
    sh_bytes = 48 * n_p + 32 * n_v + 4 * n_t + 80 * m + 8 * wet_res * wet_res
    c.show(times[-1])
    c.last_times()
    t0 = time.perf_counter()
    for tt in times[:-1]:
        c.show(tt)
    c.last_times()  # waits for the last show
    show_s = (time.perf_counter() - t0) / max(len(times) - 1, 1)
    c.close()
    med = lambda v: float(np.median(v))
    i_t, p_t, s_b = med(idx), med(pk), med(st_bytes)
    return {"workload": f"{reps} keyframes of the {n_p}-particle scene, 4 us apart, and a show between each pair",
            "key_bytes": int(keys[-1]["bytes"]), "spray_slots": int(keys[-1]["spray"]), "live_spray": int(keys[-1]["live"]),
            "index_us": i_t * 1e6, "pack_us": p_t * 1e6, "store_call_us": med(call) * 1e6,
            "pack_gbs": s_b / p_t / 1e9, "pack_frac": s_b / p_t / 1e9 / peak,
            "show_us": show_s * 1e6, "show_gbs": sh_bytes / show_s / 1e9, "show_frac": sh_bytes / show_s / 1e9 / peak,
            "peak_gbs": peak,
            "note": "store: events on the simulation's stream around each of its two device parts; the host's read of the "
                    "spray counts between them is in store_call_us only. show: back-to-back calls timed as a run"}


def run_native(args, rank, world, local):
    import numpy as np
    from natray_b200 import Params, build_world
    from natray_b200.sim import Sim

    params = Params(**SCENE)
    w = build_world(params)
    n_particles = w.h.n_particles
    sim = Sim(world=w, device=local)
    info = sim.info
    log(f"rank {rank}: {n_particles} particles, {info.n_verts} verts, {info.n_tris} tris, dx {info.dx*1e3:.3f} mm")
    import torch
    use_dist = world > 1
    if use_dist:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if use_dist:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(local)

    # Warm-up: W steps, one a batch: they size the solver's iterations and the substeps, and
    # build the step's graph. The timed steps are W + 1 .. W + K, as in the reference arm.
    for _ in range(args.warmup):
        sim.step(1)
    barrier()
    sim.work(reset=True)
    # Device-timed region: K steps in one batch, CUDA events on the simulation's stream.
    with Clocks(local) as clk:
        sim.step(args.steps)
    barrier()
    launches, ms = sim.last_launches()
    st = sim.state
    work = sim.work(reset=True)
    from natray_b200.replicas import max_over_ranks
    t_dev = max_over_ranks(ms * 1e-3)
    value = n_particles * args.steps * world / t_dev
    # The step-level roofline: the algorithmic bytes of the K timed steps, from the work the
    # steps counted on the device (blocks, water cells x iterations, gas cells x air substeps,
    # rubber substeps, spray), over their device time.
    step_bytes = sim.algorithmic_bytes(work)

    # End to end through the public API: one ntr_sim_step call per step, each uploading the
    # step's parameters from host memory and reading the state back.
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.step(1)
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e = n_particles * args.steps * world / t_e2e

    # Roofline of the dominant kernel: kernel-by-kernel event timing of a few steps.
    prof_steps = min(10, args.steps)
    prof = sim.profile(prof_steps)
    tot = sum(v[1] for v in prof.values())
    top, (cnt, kms) = max(prof.items(), key=lambda kv: kv[1][1])
    per_launch_s = kms / cnt * 1e-3
    st2 = sim.state
    cf_type = sim.download("CF", np.float32).reshape(11, -1)[10, : st2["n_blocks"] * 64]
    st2["_n_water"] = int((cf_type == 1.0).sum())
    iters = max(st2["solve_iters"], 1)
    alg = algorithmic_bytes(top, st2, n_particles, iters)
    peak, peak_kind = hbm_peak()
    achieved = alg / per_launch_s / 1e9 if alg > 0 else None
    # DRAM traffic of one launch of that kernel, from the ncu capture summarised in profiles/
    # (the file gives the command that made it; ncu's figures cannot be taken inside this run).
    traffic, traffic_src = None, None
    tf = ROOT / "profiles" / f"{top.split('<')[0]}.md"
    if tf.exists():
        for line in tf.read_text().splitlines():
            if line.startswith("traffic_per_launch_bytes:"):
                try:
                    traffic = float(line.split(":", 1)[1].strip())
                    traffic_src = f"profiles/{tf.name}"
                except ValueError:
                    pass

    # P2G's shared-memory atomics: 216 lane additions a particle (4 lattices x 27 nodes x value
    # and weight), against the device's measured rate for them at their best. Reported whichever
    # kernel has the largest share (P2G and the solve are within a point of each other).
    atomics = None
    p2g = prof.get("k_p2g")
    if p2g:
        import ctypes as C
        from natray_b200._abi import check, lib
        peak_at = C.c_double()
        check(lib().ntr_probe_shared_atomics(local, 16384, C.byref(peak_at)))
        p2g_s = p2g[1] / p2g[0] * 1e-3
        rate = 216.0 * n_particles / p2g_s
        atomics = {"kernel": "k_p2g", "achieved": rate, "peak": peak_at.value, "unit": "lane atomic adds/s",
                   "frac": rate / peak_at.value, "per_launch": 216 * n_particles, "launch_ms": p2g_s * 1e3,
                   "note": "peak: ntr_probe_shared_atomics, conflict-free adds in P2G's CTA shape on this GPU"}

    result = None
    if rank == 0:
        h2d = 192  # the Params uniform per call
        d2h = 176  # the device state read back per call
        shares = {k: round(v[1] / tot, 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])[:8]}
        result = {
            "metric": METRIC,
            "value": value,
            "unit": "particle-substeps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": t_dev * 1e3 / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded scene builder of the reference)",
            "config": {
                "workload": WORKLOAD,
                "n_particles": n_particles,
                "n_tris": int(info.n_tris),
                "dt_ns": st["dt_ns"],
                "n_blocks": st["n_blocks"],
                "solver_iters_last": st["solve_iters"],
                "substeps": [int(sim._info().substeps), int(sim._info().air_substeps)],
                "parallelism": f"replicas x{world}",
                "l2": "no flush: a step moves ~170 MB of particles, sort buffers, tiles and cell fields, above the 126 MB L2",
                "reductions": "fp64",
            },
            "e2e": {"value": e2e, "unit": "particle-substeps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "note": "one ntr_sim_step call per step from the host"},
            "gpu_launches": int(launches),
            "roofline": {"kernel": top, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind, "traffic": traffic,
                         "traffic_source": traffic_src, "algorithmic_bytes_per_launch": alg,
                         "launch_ms": per_launch_s * 1e3, "share": round(kms / tot, 4), "shared_atomics": atomics},
            "step_roofline": {"bound": "hbm", "achieved": step_bytes / t_dev / 1e9 * world, "peak": peak, "unit": "GB/s",
                              "frac": step_bytes / t_dev / 1e9 / peak, "peak_kind": peak_kind,
                              "algorithmic_bytes_per_step": step_bytes / max(work["steps"], 1), "work": work,
                              "note": "sum over the timed steps of 160 Np + 160 cells + 48 K Nw + (256 Nv + 32 Nt) Sm "
                                      "+ 44 Sa Na + 48 Nspray, counted on the device by the steps, over their device time"},
            "kernel_shares": shares,
            "clocks": clk.summary(),
        }
    if rank == 0 and world == 1 and args.keyframes:
        result["keyframes"] = keyframe_bench(sim, args.keyframes, peak, int(w.h.wet_res))
    sim.close()
    if use_dist:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return result


def cpu_baseline(sample_steps: int, threads: int | None = None, warmup: int = 1) -> dict:
    """The CPU restatement of the reference's step (FP32) on this host's cores, on a bounded
    sample of the same workload: `sample_steps` steps of the 1M scene after `warmup` untimed
    steps taken one a batch, as the native arm takes its warm-up. The world comes from the
    library's scene builder (CPU code, the reference's balloon.rs/bullet.rs/flight.rs restated):
    the only part of libnatray.so this arm uses, and it runs before the timed steps."""
    from natray_b200 import Params, World, build_world
    from oracle.py import Oracle, set_threads, threads as nthreads
    cores = threads or os.cpu_count() or 1
    set_threads(cores)
    w = build_world(Params(**SCENE))
    o = Oracle(w.blob, fp64_dots=False)
    for _ in range(max(warmup, 1)):
        o.step(1)
    t0 = time.perf_counter()
    n = o.step(sample_steps)
    dt = time.perf_counter() - t0
    return {"value": w.h.n_particles * n / dt, "unit": "particle-substeps/s", "cores": nthreads(), "kind": "port",
            "n_particles": int(w.h.n_particles),
            "sample": f"steps {max(warmup, 1) + 1}-{max(warmup, 1) + n} of the 1M-particle scene (after {max(warmup, 1)} untimed "
                      f"steps), oracle FP32 with the reference's FP32 sums, OpenMP; the scene built by the library's CPU "
                      f"scene builder before timing"}


def small_scene(steps: int = 200) -> dict:
    """The small scene's 200 fixed steps: device-timed in one call (CUDA events), and end to end
    with one ntr_sim_step call a step, after 5 warm-up steps of a separate simulation of it."""
    from natray_b200 import Params, build_world
    from natray_b200.sim import Sim
    w = build_world(Params(**SMALL))
    warm = Sim(world=w)
    for _ in range(5):
        warm.step(1)
    warm.close()
    s = Sim(world=w)
    assert s.step(steps) == steps
    _, ms = s.last_launches()
    s.close()
    s = Sim(world=w)
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step(1)
    e2e_s = time.perf_counter() - t0
    s.close()
    n = w.h.n_particles
    return {"workload": f"small scene: d=8 cm balloon, res 51 ({n} particles), icosphere(4) 5,120 tris, rubber 0.2 mm, "
                        f"8 mm steel sphere at 300 m/s, {steps} fixed steps of 2 us",
            "particle_steps_per_s": n * steps / (ms * 1e-3), "ms_per_step": ms / steps,
            "e2e_particle_steps_per_s": n * steps / e2e_s, "e2e_ms_per_step": e2e_s * 1e3 / steps}


def batch_and_serve(args) -> dict:
    """The batched workload (many mixed scenes stepped together, against the same scenes one at a
    time) and the serving loop (Poisson arrivals, continuous batching, against one request at a
    time in arrival order), on seeded synthetic scenes of the shapes the configs name, scaled
    down in count and steps so that the run stays within minutes."""
    from natray_b200 import serve as sv
    out = {}
    if args.batch_scenes:
        ws = sv.build_worlds(sv.mixed_scenes(args.batch_scenes, 7))
        b = sv.run_batched(ws, args.batch_steps, args.batch_chunk, max_scenes=max(64, args.batch_scenes), tune_steps=args.batch_tune)
        q = sv.run_sequential(ws, args.batch_steps, args.batch_chunk)
        out["batched"] = {
            "workload": f"{len(ws)} scenes, particles log-uniform 16k-512k (seeded; {sum(w.h.n_particles for w in ws)} in all), "
                        f"diameter 6.5-16 cm, 8 mm steel sphere at 150-400 m/s, membrane level 4-6 by size, "
                        f"{args.batch_steps} steps each, dt 2 us, FP64 solver sums",
            "scenes_per_s": b["scenes_per_s"], "particle_steps_per_s": b["particle_steps_per_s"], "seconds": b["seconds"],
            "sequential_scenes_per_s": q["scenes_per_s"], "sequential_seconds": q["seconds"],
            "speedup_vs_sequential": q["seconds"] / b["seconds"], "chunk": args.batch_chunk, "calls": b["calls"],
            "graph_captures": b["graph_captures"], "graph_instantiations": b["graph_instantiations"],
            "tuning": b["tuning"], "tuning_note": "launch shapes chosen by the batch autotuner on a throwaway batch of the same scenes"
                                                  if b["tuning"] else "default launch shapes"}
    if args.serve_requests:
        from natray_b200 import build_world
        ps = sv.mixed_scenes(args.serve_requests, 11, lo=16_000, hi=2_000_000, lognormal_median=128_000)
        arr = sv.poisson_arrivals(args.serve_requests, args.serve_rate, 11)
        # Each request's scene is built on a host thread when it arrives (its latency includes it).
        srv = sv.serve(ps, arr, args.serve_steps, args.batch_chunk, max_scenes=64, build=build_world)
        q = sv.run_sequential(ps, args.serve_steps, args.batch_chunk, build=build_world)
        seq = sv.sequential_timeline(arr, q["per_scene_seconds_with_setup"])
        out["serving"] = {
            "workload": f"{args.serve_requests} requests, Poisson arrivals at {args.serve_rate}/s (seeded), particles lognormal "
                        f"median 128k clipped 16k-2M, {args.serve_steps} steps each, each scene built when its request "
                        f"arrives (latency includes the build), admission by free HBM, 64 slots",
            "scenes_per_s": srv["scenes_per_s"], "p50_s": srv["p50_s"], "p99_s": srv["p99_s"], "seconds": srv["seconds"],
            "sequential": {"scenes_per_s": seq["scenes_per_s"], "p50_s": seq["p50_s"], "p99_s": seq["p99_s"], "seconds": seq["seconds"]}}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=30, help="steps of the CPU baseline sample")
    ap.add_argument("--batch-scenes", type=int, default=64, help="scenes of the batched run (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=500)
    ap.add_argument("--batch-chunk", type=int, default=8, help="steps per batch call (state read back between)")
    ap.add_argument("--batch-tune", type=int, default=4, help="timed steps per autotuner candidate before the batched run (0: default shapes)")
    ap.add_argument("--serve-requests", type=int, default=200, help="requests of the serving loop (0: skip)")
    ap.add_argument("--serve-steps", type=int, default=200)
    ap.add_argument("--serve-rate", type=float, default=15.0, help="request arrivals per second")
    ap.add_argument("--keyframes", type=int, default=16, help="keyframes stored and shown at the bench scene (0: skip)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()

    if args.impl == "reference":
        if rank != 0:
            return
        steps = max(1, min(args.steps, args.cpu_sample))
        cb = cpu_baseline(steps, warmup=args.warmup)
        line = {"metric": METRIC, "value": cb["value"], "unit": "particle-substeps/s", "n_gpus": args.gpus, "steps": steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded scene builder of the reference)", "impl": "reference",
                "config": {"workload": WORKLOAD, "parallelism": "host cores", "n_particles": cb["n_particles"]},
                "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "particle-substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference's wgpu/WGSL step needs a graphics adapter (none on this box, no Rust toolchain); this is the C++ restatement of its step kernels"}
        print(json.dumps(line), flush=True)
        return

    res = run_native(args, rank, world, local)
    if rank == 0 and res is not None:
        if world == 1:
            res["small"] = small_scene()
            res.update(batch_and_serve(args))
            res["cpu_baseline"] = cpu_baseline(args.cpu_sample, warmup=args.warmup)
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
