"""`Sim`: the reference's simulation surface (src/sim.rs:149-522) on one B200, through the C ABI.

    sim = Sim(Params(resolution=64))         # Sim::new
    sim.advance(t_target=0.001, budget=64)   # Sim::advance
    sim.step(n, stop_ns)                     # Sim::run: one batch
    sim.state                                # the State read back after a batch

The product path is the CUDA library only: there is no CPU fallback, and a machine without a
B200 gets NatrayError(NTR_E_NODEVICE).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import BUF, check, lib
from .world import Params, World, blob_arg, build_world


class Sim:
    def __init__(self, params: Params | None = None, *, world: World | bytes | None = None, device: int = 0,
                 fp64_reductions: bool = True):
        self._h = C.c_void_p()
        if world is None:
            world = build_world(params if params is not None else Params())
        blob, n = blob_arg(world)
        check(lib().ntr_sim_create_from_world(blob, n, device, C.byref(self._h)))
        if not fp64_reductions:
            check(lib().ntr_sim_set_precision(self._h, 0))
        self.info = self._info()

    # -- lifetime ---------------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().ntr_sim_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- stepping ---------------------------------------------------------------------------
    def step(self, n: int, stop_ns: int = 0xFFFFFFFF) -> int:
        """One batch of up to `n` steps that stops at `stop_ns` (Sim::run)."""
        taken = C.c_uint32()
        check(lib().ntr_sim_step(self._h, n, stop_ns, C.byref(taken)))
        return taken.value

    def stats(self) -> dict:
        """What the reference's debug_stats prints (src/sim.rs:691-863), computed on the device:
        see `natray_b200.sim.format_stats` for the printed form."""
        st = _abi.Stats()
        check(lib().ntr_sim_stats(self._h, C.byref(st)))
        out = {}
        for k, _ in st._fields_:
            if k.startswith("pad"):
                continue
            v = getattr(st, k)
            if k == "bullets":
                out[k] = [{f: (list(getattr(b, f)) if f == "x" else getattr(b, f)) for f, _ in b._fields_}
                          for b in v[: st.n_bullets]]
            elif k == "stretch":
                out[k] = [list(r) for r in v]
            elif hasattr(v, "__len__"):
                out[k] = list(v)
            else:
                out[k] = v
        return out

    def set_batch_steps(self, n: int) -> None:
        """Steps per batch of `advance` (0: the reference's 4 ms rule, which depends on the GPU's
        timing; a fixed count makes runs repeat bit for bit)."""
        check(lib().ntr_sim_set_batch_steps(self._h, n))

    def advance(self, t_target: float, budget: int) -> int:
        """Runs to `t_target` (s, the reference's timeline) in at most `budget` steps."""
        taken = C.c_uint32()
        check(lib().ntr_sim_advance(self._h, t_target, budget, C.byref(taken)))
        return taken.value

    # -- reading back -----------------------------------------------------------------------
    @property
    def state(self) -> dict:
        s = _abi.State()
        check(lib().ntr_sim_read_state(self._h, C.byref(s)))
        return s.as_dict()

    def _info(self) -> _abi.SimInfo:
        i = _abi.SimInfo()
        check(lib().ntr_sim_info_get(self._h, C.byref(i)))
        return i

    def snapshot(self) -> World:
        n = C.c_size_t()
        check(lib().ntr_sim_snapshot(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        check(lib().ntr_sim_snapshot(self._h, buf, n.value, C.byref(n)))
        return World(buf.raw[: n.value])

    def restore(self, world: World | bytes) -> None:
        blob, n = blob_arg(world)
        check(lib().ntr_sim_restore(self._h, blob, n))

    def buffer(self, name: str) -> tuple[int, int]:
        """(device pointer, bytes) of a lent buffer."""
        p, n = C.c_void_p(), C.c_size_t()
        check(lib().ntr_sim_buffer(self._h, BUF[name], C.byref(p), C.byref(n)))
        return p.value or 0, n.value

    def download(self, name: str, dtype=np.uint32, count: int | None = None) -> np.ndarray:
        _, n = self.buffer(name)
        if count is not None:
            n = min(n, count * np.dtype(dtype).itemsize)
        out = np.empty(n // np.dtype(dtype).itemsize, dtype=dtype)
        check(lib().ntr_sim_download(self._h, BUF[name], out.ctypes.data, out.nbytes))
        return out

    def grid(self) -> dict:
        """This step's grid in the layouts the oracle reports: block list, sorted particles,
        block starts, transfer sums and cell fields of the allocated blocks."""
        st = self.state
        nb = min(st["n_blocks"], self.info.block_cap)
        cap_cells = self.info.block_cap * 64
        cells = nb * 64
        bl = self.download("BLOCK_LIST", np.uint32, nb)
        bs = self.download("BLOCK_START", np.uint32, nb + 1)
        srt = self.download("SORTED", np.uint32, int(bs[-1]) if nb else 0)
        acc = self.download("ACC", np.int32).reshape(19, cap_cells)[:, :cells].copy()
        cf = self.download("CF", np.float32).reshape(11, cap_cells)[:, :cells].copy()
        nbt = self.download("BLOCK_NB", np.uint32, nb * 27)
        air = self.download("AIR", np.float32).reshape(5, cap_cells)[:, :cells].copy()
        return {"block_list": bl, "block_start": bs, "sorted": srt, "acc": acc.reshape(-1), "cf": cf.reshape(-1),
                "block_nb": nbt, "air": air.reshape(-1)}

    def profile(self, n: int, stop_ns: int = 0xFFFFFFFF) -> dict:
        """One batch launched kernel by kernel with events between them: {kernel: (launches, ms)}
        (the reference's NATRAY_PROF)."""
        buf = C.create_string_buffer(1 << 16)
        ln = C.c_size_t()
        check(lib().ntr_sim_profile(self._h, n, stop_ns, buf, len(buf), C.byref(ln)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, cnt, ms = line.rsplit(",", 2)
            out[name] = (int(cnt), float(ms))
        return out

    @property
    def tuning(self) -> dict:
        """The launch shapes (CTAs of the solve, per SM of the cell and transfer kernels)."""
        t = _abi.Tuning()
        check(lib().ntr_sim_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_ if k != "pad"}

    @tuning.setter
    def tuning(self, v: dict) -> None:
        t = _abi.Tuning(**{k: int(x) for k, x in v.items()})
        check(lib().ntr_sim_set_tuning(self._h, C.byref(t)))

    def autotune(self, steps: int = 4) -> tuple[dict, float]:
        """Times candidate launch shapes on this scene (its state is kept) and keeps the fastest;
        returns it and its ms per step."""
        t, ms = _abi.Tuning(), C.c_double()
        check(lib().ntr_sim_autotune(self._h, steps, C.byref(t), C.byref(ms)))
        return {k: getattr(t, k) for k, _ in t._fields_ if k != "pad"}, ms.value

    WORK = ("steps", "cells", "water_iters", "mem_substeps", "gas_substeps", "spray")

    def work(self, reset: bool = False) -> dict:
        """The steps' work counted on the device since creation, a restore or the last reset:
        steps, block cells, water cells x solver iterations, rubber substeps, gas cells x air
        substeps, spray slots (each summed over the steps)."""
        out = (C.c_uint64 * 6)()
        check(lib().ntr_sim_work(self._h, out, int(reset)))
        return dict(zip(self.WORK, list(out)))

    def algorithmic_bytes(self, work: dict) -> float:
        """Bytes the steps counted in `work` must move at the least: 160 per particle and step
        (its state read and written), 160 per block cell (transfer sums, cell fields, projection,
        the G2P read, the clear), 48 per water cell and solver iteration, 256 per vertex and 32
        per triangle and rubber substep, 44 per gas cell and air substep, 48 per spray slot."""
        i = self.info
        return (160.0 * i.n_particles * work["steps"] + 160.0 * work["cells"] + 48.0 * work["water_iters"]
                + (256.0 * i.n_verts + 32.0 * i.n_tris) * work["mem_substeps"] + 44.0 * work["gas_substeps"]
                + 48.0 * work["spray"])

    def last_launches(self) -> tuple[int, float]:
        n, ms = C.c_uint64(), C.c_double()
        check(lib().ntr_sim_last_launches(self._h, C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def conservation(self) -> np.ndarray:
        out = (C.c_double * 8)()
        check(lib().ntr_sim_conservation(self._h, out))
        return np.array(out[:])


__all__ = ["Sim"]


def format_stats(sim: Sim) -> str:
    """The lines the reference's Sim::debug_stats prints, from ntr_sim_stats and the state."""
    s, st, i = sim.stats(), sim.state, sim._info()
    f3 = lambda v, d=3: "[" + ", ".join(f"{x:.{d}f}" for x in v) + "]"
    lines = [
        f"t={i.t:.6f} dt={st['dt_ns']}ns steps {st['step']} | water {s['water']}/{s['n_particles']} bbox {f3(s['lo'])}.."
        f"{f3(s['hi'])} mean {f3(s['mean'], 4)} v {f3(s['vmean'])} vmax {s['vmax']:.2f} at {f3(s['fastest'], 4)} volume "
        f"{s['volume_l']:.3f} L | blocks {st['n_blocks']} solver {st['solve_iters']} iters (encoded {i.iters}) r "
        f"{st['r_norm']:.2e} of {st['b_norm']:.2e} | spray {st['spray_count']}"]
    for k in range(s["n_tension"]):
        l1, l2 = s["stretch"][k]
        lines.append(f"  tension {s['tension'][k]:.0f} N/m stretch {l1:.2f} x {l2:.3f} (triangle {s['tension_tri'][k]})")
    lines.append(
        f"  rubber: inside {s['inside_l']:.4f} L bbox {f3(s['mem_lo'], 4)}..{f3(s['mem_hi'], 4)} on water {s['on_water']}/"
        f"{s['free_verts']} fill min {s['fill_min']:.2f} mean {s['fill_mean']:.2f} torn {s['torn']} fastest "
        f"{s['rubber_vmax']:.1f} m/s | substep {st['mem_dt_seen'] * 1e6:.2f}us x{i.substeps} (step could be "
        f"{st['dt_flow'] * 1e6:.1f}us) capillary {st['cap_dt'] * 1e6:.1f}us")
    for k, b in enumerate(s["bullets"]):
        lines.append(f"  bullet {k}: state {b['state']} at {f3(b['x'], 4)} v {b['speed']:.1f} m/s yaw {b['yaw_deg']:.1f} deg "
                     f"spin {b['spin_rev_s']:.0f} rev/s, {b['sections']} sections")
    lines.append(f"  energy: water {s['water_j']:.2f} J, bullets {s['bullets_j']:.2f} J, vapour {s['vapour_cm3']:.1f} cm^3 "
                 f"(x 1 atm = {s['vapour_j']:.2f} J)")
    lines.append(f"  air: {s['air_cells']} cells, {s['vapour_cells']} of them vapour, gauge {s['gauge_lo']:.1f}.."
                 f"{s['gauge_hi']:.1f} Pa, fastest {s['air_umax']:.2f} m/s | substep {st['air_dt_seen'] * 1e6:.2f}us x"
                 f"{i.air_substeps}")
    return "\n".join(lines)
