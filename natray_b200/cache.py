"""`Cache`: the keyframe cache of the reference (src/cache.rs) on one B200, through the C ABI.

    sim = Sim(params)
    cache = Cache(sim, params)      # Cache::new: the first keyframe at the start
    cache.bake(500)                 # Cache::bake: up to 500 steps, keyframes when due
    cache.show(0.0004)              # Cache::show: the shown buffers for t = 0.4 ms
    cache.shown("PARTICLES")        # n_particles x 8 f32: position, 1, velocity, live

The cache borrows the simulation: keep `sim` alive while the cache is in use.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import SHOWN, SHOWN_COUNT, check, lib
from .world import Params

SHOWN_DTYPE = {"PARTICLES": np.float32, "SPRAY": np.float32, "MEM_POS": np.float32, "ALIVE": np.uint32,
               "WET": np.uint32, "SPRAY_W": np.float32}


def cache_params(params: Params | None = None, *, page_bytes: int | None = None, pages: int | None = None,
                 arrivals: list[float] | None = None, t_end: float | None = None) -> _abi.CacheParams:
    """The reference's pool (16 pages of 128 MiB) and timeline (1 s), with the shots' arrival
    times of `params` (src/sim.rs:280-291); each can be overridden."""
    cp = _abi.CacheParams()
    if params is not None:
        check(lib().ntr_cache_params_default(C.byref(params.c), C.byref(cp)))
    else:
        cp.page_bytes, cp.pages, cp.t_end, cp.n_arrivals = 128 << 20, 16, 1.0, 1
        cp.arrivals[0] = 0.0
    if page_bytes is not None:
        cp.page_bytes = page_bytes
    if pages is not None:
        cp.pages = pages
    if t_end is not None:
        cp.t_end = t_end
    if arrivals is not None:
        if len(arrivals) > _abi.MAX_SHOTS:
            raise ValueError("at most 4 arrivals")
        cp.n_arrivals = len(arrivals)
        for k, a in enumerate(arrivals):
            cp.arrivals[k] = a
    return cp


def key_bytes(n_particles: int, n_verts: int, n_tris: int, spray: int, live: int) -> int:
    return int(lib().ntr_key_bytes(n_particles, n_verts, n_tris, spray, live))


def key_next_time(t: float, arrivals: list[float], t_end: float, free_bytes: int, size: int) -> float:
    arr = (C.c_double * max(len(arrivals), 1))(*arrivals)
    return float(lib().ntr_key_next_time(t, arr, len(arrivals), t_end, free_bytes, size))


class Cache:
    def __init__(self, sim, params: Params | None = None, **kw):
        self.sim = sim
        self._h = C.c_void_p()
        self.params = cache_params(params, **kw)
        check(lib().ntr_cache_create(sim._h, C.byref(self.params), C.byref(self._h)))

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().ntr_cache_destroy(self._h)
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

    def rebuild(self, sim) -> None:
        """Starts over on `sim` (Cache::rebuild), reusing the pool."""
        check(lib().ntr_cache_rebuild(self._h, sim._h))
        self.sim = sim

    def bake(self, max_steps: int) -> int:
        n = C.c_uint32()
        check(lib().ntr_cache_bake(self._h, max_steps, C.byref(n)))
        return n.value

    def store(self) -> None:
        check(lib().ntr_cache_store(self._h))

    def show(self, t: float) -> bool:
        changed = C.c_int()
        check(lib().ntr_cache_show(self._h, t, C.byref(changed)))
        return bool(changed.value)

    @property
    def info(self) -> dict:
        i = _abi.CacheInfo()
        check(lib().ntr_cache_info_get(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in i._fields_}

    def last_times(self) -> tuple[float, float, float]:
        """Device ms of the last store's spray index and packing, and of the last show."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        check(lib().ntr_cache_last_times(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def end(self) -> float:
        return self.info["end"]

    def done(self) -> bool:
        return bool(self.info["done"])

    def keys(self) -> list[dict]:
        out = []
        for k in range(self.info["keys"]):
            r = _abi.KeyInfo()
            check(lib().ntr_cache_key(self._h, k, C.byref(r)))
            out.append({f: getattr(r, f) for f, _ in r._fields_ if f != "pad"})
        return out

    def key_words(self, k: int) -> np.ndarray:
        """Keyframe k's words (its whole 256-byte-rounded extent)."""
        r = _abi.KeyInfo()
        check(lib().ntr_cache_key(self._h, k, C.byref(r)))
        out = np.empty(r.bytes // 4, np.uint32)
        check(lib().ntr_cache_download(self._h, SHOWN_COUNT + k, out.ctypes.data, out.nbytes))
        return out

    def shown(self, name: str) -> np.ndarray:
        p, n = C.c_void_p(), C.c_size_t()
        check(lib().ntr_cache_buffer(self._h, SHOWN[name], C.byref(p), C.byref(n)))
        dt = np.dtype(SHOWN_DTYPE[name])
        out = np.empty(n.value // dt.itemsize, dt)
        check(lib().ntr_cache_download(self._h, SHOWN[name], out.ctypes.data, out.nbytes))
        return out
