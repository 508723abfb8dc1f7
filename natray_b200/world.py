"""Parameters and world blobs from Python.

`Params` mirrors the reference's `SimParams` (src/params.rs:266-314) with its `set_kv`
overrides and named presets; `build_world` runs the scene builder (src/balloon.rs:343-464,
src/sim.rs:208-441) and returns a `World`, whose sections are numpy views of the blob.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import SEC, SECTIONS, check, lib

# Element dtype and per-element width (in that dtype) of each section.
_SEC_DTYPE = {
    "PARTICLES": (np.float32, 20), "MEM_X": (np.float32, 4), "MEM_V": (np.float32, 4), "MEM_MASS": (np.float32, 1),
    "MEM_WATER": (np.float32, 4), "MEM_LAYER": (np.float32, 24), "MEM_PUSH": (np.float32, 2),
    "TRIS": (np.uint32, 8), "ALIVE": (np.uint32, 1), "VTRI_OFF": (np.uint32, 1), "VTRI": (np.uint32, 1),
    "BULLETS": (np.float32, 28), "PATCHES": (np.float32, 8), "OUTLINES": (np.float32, 2),
    "SECTIONS": (np.float32, 12), "BULLET_HIT": (np.int32, 1), "POSE_LOG": (np.float32, 12),
    "BLOCKS_PREV": (np.uint32, 1), "BLOCK_ACTIVE": (np.uint32, 1), "AIR": (np.float32, 1),
    "SPRAY": (np.float32, 12), "LANDED": (np.float32, 4), "TOUCH": (np.uint32, 1),
}


class Params:
    """SimParams with `set`, `preset` and attribute access to the C structure."""

    def __init__(self, **overrides):
        self.c = _abi.SimParams()
        check(lib().ntr_params_default(C.byref(self.c)))
        for k, v in overrides.items():
            self.set(k, v)

    @classmethod
    def preset(cls, name: str, **overrides) -> "Params":
        p = cls()
        check(lib().ntr_params_preset(C.byref(p.c), name.encode()))
        for k, v in overrides.items():
            p.set(k, v)
        return p

    def set(self, key: str, value) -> "Params":
        """`key=value` as the reference's `set_kv` takes it (src/params.rs:361-423)."""
        check(lib().ntr_params_set(C.byref(self.c), key.encode(), str(value).encode()))
        return self

    def __getattr__(self, name):
        return getattr(self.c, name)


def flights(params: Params) -> list[dict]:
    """Each shot's flight through the air to the balloon (the reference's Flight::new): the
    hand-over state, its time, and the speed, stability and yaw at impact. CPU only."""
    out = (_abi.Flight * _abi.MAX_SHOTS)()
    n = C.c_uint32()
    check(lib().ntr_shot_flights(C.byref(params.c), out, _abi.MAX_SHOTS, C.byref(n)))
    res = []
    for f in out[: n.value]:
        d = {}
        for k, _ in f._fields_:
            v = getattr(f, k)
            d[k] = list(v) if not isinstance(v, float) else v
        res.append(d)
    return res


def sized_for(n_particles: int, diameter_cm: float = 16.0) -> int:
    """Lattice resolution that fills a sphere of `diameter_cm` with about `n_particles`:
    N ~ pi/6 res^3 (src/balloon.rs:420 spacing = d / res)."""
    return max(16, int(round((6.0 * n_particles / np.pi) ** (1.0 / 3.0))))


class World:
    """A world blob and numpy views of its header and sections."""

    def __init__(self, blob: bytes | bytearray, copy: bool = True):
        self.blob = blob if not copy and isinstance(blob, bytearray) else bytearray(blob)
        self.h = _abi.WorldHeader.from_buffer_copy(bytes(self.blob[: C.sizeof(_abi.WorldHeader)]))
        if self.h.magic != _abi.WORLD_MAGIC:
            raise ValueError("not a world blob")

    def sec(self, name: str) -> np.ndarray:
        i = SEC[name]
        dt, w = _SEC_DTYPE[name]
        off, n = self.h.offset[i], self.h.bytes[i]
        a = np.frombuffer(self.blob, dtype=dt, count=n // np.dtype(dt).itemsize, offset=off)
        return a.reshape(-1, w) if w > 1 else a

    @property
    def state(self) -> dict:
        return self.h.state.as_dict()

    @property
    def particles(self) -> np.ndarray:
        return self.sec("PARTICLES")

    def air(self) -> np.ndarray:
        n = self.h.n_blocks_prev * 64
        return self.sec("AIR").reshape(5, n)

    def __len__(self) -> int:
        return len(self.blob)

    def summary(self) -> dict:
        h = self.h
        return {"n_particles": h.n_particles, "n_verts": h.n_verts, "n_tris": h.n_tris, "dx": h.dx,
                "spacing": h.params.fluid[3], "dims": list(h.params.dims[:3]), "block_cap": h.block_cap,
                "n_shots": h.n_shots, "bytes": len(self.blob)}


def blob_arg(world: "World | bytes | bytearray") -> tuple[object, int]:
    """A world blob as the library's (pointer, length) arguments. A World's bytearray is passed
    in place, not copied (93 MB at 1M particles): every entry point taking a blob reads it
    during the call and copies what it keeps."""
    if isinstance(world, World):
        world = world.blob
    if isinstance(world, bytearray):
        return (C.c_char * len(world)).from_buffer(world), len(world)
    b = bytes(world)
    return b, len(b)


def build_world(params: Params) -> World:
    """The initial world of `params`, built on the CPU."""
    p = C.c_void_p()
    n = C.c_size_t()
    check(lib().ntr_world_build(C.byref(params.c), C.byref(p), C.byref(n)))
    try:
        blob = bytearray(n.value)  # one copy, out of the library's buffer
        C.memmove((C.c_char * n.value).from_buffer(blob), p, n.value)
    finally:
        lib().ntr_free(p)
    return World(blob, copy=False)


__all__ = ["Params", "World", "blob_arg", "build_world", "sized_for", "SECTIONS"]
