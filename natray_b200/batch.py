"""`Batch`: many independent scenes on one GPU through the C ABI's ntr_batch_* calls.

    b = Batch(max_scenes=64)
    slot = b.admit(world, n_steps=500)     # None when no slot or device memory is free now
    b.step(4)                              # 4 steps of every unfinished scene, one joint solve per step
    b.poll(slot)                           # {"finished": ..., "steps_done": ..., "state": {...}}
    world = b.snapshot(slot); b.retire(slot)

A scene's results equal those of the same scene stepped alone by `Sim.step` with the same
chunk sizes. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

from . import _abi
from ._abi import NatrayError, check, lib
from .world import World, blob_arg

NTR_E_BUSY = 8


class Batch:
    def __init__(self, max_scenes: int = 64, *, device: int = 0, hbm_budget: int = 0):
        self._h = C.c_void_p()
        check(lib().ntr_batch_create(device, max_scenes, hbm_budget, C.byref(self._h)))
        self.max_scenes = max_scenes

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().ntr_batch_destroy(self._h)
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

    def admit(self, world: World | bytes, n_steps: int) -> int | None:
        """The scene's slot, or None when the batch has no room for it now."""
        blob, n = blob_arg(world)
        slot = C.c_uint32()
        st = lib().ntr_batch_admit(self._h, blob, n, n_steps, C.byref(slot))
        if st == NTR_E_BUSY:
            return None
        check(st)
        return slot.value

    def enqueue(self, world: World | bytes, n_steps: int) -> int:
        """Queues the scene from any thread; the stepping thread admits it at its next step.
        Returns the ticket."""
        blob, n = blob_arg(world)
        ticket = C.c_uint64()
        check(lib().ntr_batch_enqueue(self._h, blob, n, n_steps, C.byref(ticket)))
        return ticket.value

    def ticket(self, ticket: int) -> int | None:
        """The queued scene's slot once admitted, None while it waits."""
        slot = C.c_uint32()
        check(lib().ntr_batch_ticket(self._h, ticket, C.byref(slot)))
        return None if slot.value == _abi.BATCH_MAX else slot.value

    def step(self, n: int) -> int:
        """n steps of every unfinished scene; returns how many scenes stepped."""
        active = C.c_uint32()
        check(lib().ntr_batch_step(self._h, n, C.byref(active)))
        return active.value

    def profile(self, n: int) -> dict:
        """n steps of every unfinished scene launched kernel by kernel with events between them:
        {kernel: (launches, ms)} (ntr_batch_profile)."""
        buf = C.create_string_buffer(1 << 16)
        ln = C.c_size_t()
        check(lib().ntr_batch_profile(self._h, n, buf, len(buf), C.byref(ln)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, cnt, ms = line.rsplit(",", 2)
            out[name] = (int(cnt), float(ms))
        return out

    def poll(self, slot: int) -> dict:
        s = _abi.BatchSlot()
        check(lib().ntr_batch_poll(self._h, slot, C.byref(s)))
        return {"in_use": bool(s.in_use), "finished": bool(s.finished), "steps_done": s.steps_done,
                "steps_target": s.steps_target, "device_bytes": s.device_bytes, "state": s.state.as_dict()}

    def snapshot(self, slot: int) -> World:
        n = C.c_size_t()
        check(lib().ntr_batch_snapshot(self._h, slot, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        check(lib().ntr_batch_snapshot(self._h, slot, buf, n.value, C.byref(n)))
        return World(bytes(buf.raw[: n.value]))

    def retire(self, slot: int) -> None:
        check(lib().ntr_batch_retire(self._h, slot))

    def info(self) -> dict:
        i = _abi.BatchInfo()
        check(lib().ntr_batch_info_get(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in i._fields_ if k != "pad"}

    @property
    def tuning(self) -> dict:
        """The launch shapes of every scene's grids and of the joint solve."""
        t = _abi.Tuning()
        check(lib().ntr_batch_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_ if k != "pad"}

    @tuning.setter
    def tuning(self, v: dict) -> None:
        t = _abi.Tuning(**{k: int(x) for k, x in v.items()})
        check(lib().ntr_batch_set_tuning(self._h, C.byref(t)))

    def autotune(self, steps: int = 4) -> tuple[dict, float]:
        """Times candidate launch shapes on the batch's scenes (the tuning steps are steps of
        theirs) and keeps the fastest; returns it and its ms per batch step."""
        t, ms = _abi.Tuning(), C.c_double()
        check(lib().ntr_batch_autotune(self._h, steps, C.byref(t), C.byref(ms)))
        return {k: getattr(t, k) for k, _ in t._fields_ if k != "pad"}, ms.value


__all__ = ["Batch", "NatrayError"]
