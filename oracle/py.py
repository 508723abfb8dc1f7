"""ctypes wrapper of the oracle library (test infrastructure only: tests/, smoke(), and the
cpu_baseline leg of bench.py use it; the product never does)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        from . import build as _b  # noqa: F401  (oracle/build.py)
        path = HERE / "libntr_oracle.so"
        if not path.exists():
            _b.build()
        L = C.CDLL(str(path))
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.c_char_p, C.c_size_t, C.c_int, C.c_int, C.c_char_p, C.c_size_t]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_step.restype = C.c_int
        L.oracle_step.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        L.oracle_snapshot.restype = C.c_size_t
        L.oracle_snapshot.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.oracle_get.restype = C.c_size_t
        L.oracle_get.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
        L.oracle_solver.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_threads.restype = C.c_int
        _lib = L
    return _lib


GET = {"block_list": (0, np.uint32), "sorted": (1, np.uint32), "block_start": (2, np.uint32),
       "acc": (3, np.int32), "cf": (4, np.float32), "block_nb": (5, np.uint32), "air": (6, np.float32)}


class Oracle:
    """The CPU restatement of the step, created from a world blob."""

    def __init__(self, blob: bytes, real64: bool = False, fp64_dots: bool = True):
        err = C.create_string_buffer(512)
        b = bytes(blob)
        self.h = lib().oracle_create(b, len(b), int(real64), int(fp64_dots), err, 512)
        if not self.h:
            raise RuntimeError(f"oracle: {err.value.decode()}")

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int, stop_ns: int = 0xFFFFFFFF) -> int:
        r = lib().oracle_step(self.h, n, stop_ns)
        if r < 0:
            raise RuntimeError("oracle: the water needs more grid blocks than the capacity")
        return r

    def snapshot(self) -> bytes:
        n = lib().oracle_snapshot(self.h, None, 0)
        buf = C.create_string_buffer(n)
        lib().oracle_snapshot(self.h, buf, n)
        return buf.raw

    def get(self, what: str) -> np.ndarray:
        code, dt = GET[what]
        n = lib().oracle_get(self.h, code, None, 0)
        out = np.empty(n, dtype=dt)
        lib().oracle_get(self.h, code, out.ctypes.data, n)
        return out

    def solver(self) -> dict:
        a = (C.c_double * 6)()
        lib().oracle_solver(self.h, a)
        return dict(zip(["rz", "alpha", "beta", "b_norm", "r_norm", "iters"], list(a)))


def set_threads(n: int) -> None:
    lib().oracle_set_threads(n)


def threads() -> int:
    return lib().oracle_threads()
