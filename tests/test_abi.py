"""The C ABI boundary on a machine without a GPU: the library loads, exports every entry point
include/natray.h declares, the ctypes layouts match the header, and simulation calls fail
loudly (no CPU fallback)."""
import ctypes as C

import numpy as np
import pytest

from natray_b200 import Params, build_world
from natray_b200 import _abi
from natray_b200._abi import NatrayError, declared_symbols, lib
from tests.conftest import has_gpu


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 20
    L = lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_sizes_match_the_header():
    assert C.sizeof(_abi.State) == 96  # src/sim.rs:66-94, 24 words
    assert C.sizeof(_abi.GpuParams) == 192  # src/sim.rs:49-64, 12 vec4
    assert C.sizeof(_abi.Shot) == 48
    h = build_world(Params(resolution=16, mesh_level=1)).h
    assert h.offset[0] >= C.sizeof(_abi.WorldHeader) and h.offset[0] % 256 == 0


def test_version_and_errors():
    assert b"sm_100a" in lib().ntr_version()
    with pytest.raises(NatrayError) as e:
        Params().set("no_such_key", "1")
    assert e.value.status == 1 and "unknown parameter" in str(e.value)


def test_world_blob_rejects_garbage():
    h = C.c_void_p()
    bad = b"\0" * 4096
    st = lib().ntr_sim_create_from_world(bad, len(bad), 0, C.byref(h))
    assert st != 0


@pytest.mark.skipif(has_gpu(), reason="checks the behaviour without a GPU")
def test_no_silent_cpu_fallback():
    from natray_b200.sim import Sim
    with pytest.raises(NatrayError) as e:
        Sim(Params(resolution=16, mesh_level=1))
    assert e.value.status == 7  # NTR_E_NODEVICE
    from natray_b200.batch import Batch
    with pytest.raises(NatrayError) as e:
        Batch(max_scenes=4)
    assert e.value.status == 7


def test_batch_structs_and_null_handles():
    assert C.sizeof(_abi.BatchSlot) == 24 + 96
    assert C.sizeof(_abi.BatchInfo) == 56
    for name, args in [("ntr_batch_step", (None, 1, None)), ("ntr_batch_retire", (None, 0)),
                       ("ntr_batch_info_get", (None, None))]:
        assert getattr(lib(), name)(*args) == 1  # NTR_E_INVALID
    assert lib().ntr_batch_destroy(None) == 0


def test_oracle_float_math_error_bounds():
    """The oracle's float exp/log/sin/cos/asin/pow (the algorithms the CUDA build also uses)
    against float64 references: within a few float ulps over the ranges the step uses."""
    from oracle.py import lib as olib
    L = olib()
    L.oracle_math.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]
    rng = np.random.default_rng(0)

    def run(fn, x, y=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, dtype=np.float32)
        out = np.empty_like(x)
        L.oracle_math(fn, x.ctypes.data, y.ctypes.data, out.ctypes.data, x.size)
        return out

    def ulps(got, want):
        want32 = want.astype(np.float32)
        spacing = np.abs(np.spacing(want32)).astype(np.float64)
        return np.abs(got.astype(np.float64) - want) / np.maximum(spacing, 1e-45)

    x = rng.uniform(-87, 88, 200000)
    assert ulps(run(0, x), np.exp(x.astype(np.float32).astype(np.float64))).max() <= 2.0
    x = np.exp(rng.uniform(-80, 80, 200000))
    assert ulps(run(1, x), np.log(x.astype(np.float32).astype(np.float64))).max() <= 4.0
    x = rng.uniform(0.3, 3.0, 200000)  # near 1, where ln x is small
    assert ulps(run(1, x), np.log(x.astype(np.float32).astype(np.float64))).max() <= 4.0
    x = rng.uniform(-7, 7, 200000)
    xf = x.astype(np.float32).astype(np.float64)
    assert np.abs(run(2, x) - np.sin(xf)).max() < 2e-7
    assert np.abs(run(3, x) - np.cos(xf)).max() < 2e-7
    x = rng.uniform(-1, 1, 200000)
    assert np.abs(run(4, x) - np.arcsin(x.astype(np.float32).astype(np.float64))).max() < 4e-7
    x, y = np.exp(rng.uniform(-10, 12, 100000)), rng.uniform(-2, 2, 100000)
    xf, yf = x.astype(np.float32).astype(np.float64), y.astype(np.float32).astype(np.float64)
    want = np.power(xf, yf)
    assert (np.abs(run(5, x, y) - want) / want).max() < 4e-6
    # Edge cases the step can reach.
    assert run(0, np.array([0.0, -200.0, 100.0]))[0] == 1.0
    assert run(0, np.array([-200.0]))[0] == 0.0 and np.isinf(run(0, np.array([100.0]))[0])
    assert run(1, np.array([1.0]))[0] == 0.0
    assert run(5, np.array([2.0]), np.array([0.0]))[0] == 1.0
