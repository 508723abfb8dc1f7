"""ntr_sort_by_block_noalloc: the step's sort of particles by block, for callers that cannot
allocate device memory (a framework that has reserved the GPU's memory for its own pool, or a
frame loop that must not make the device-wide synchronising cudaMalloc/cudaFree calls). It
keeps its scratch in a fixed array inside the library instead of allocating.

Checked against the sort the simulation step itself does (read back through ntr_sim_download
after ntr_sim_step), on two calls in a row, so that the second call sees the scratch the first
one left behind. The arrays the call reads and writes are the test's own (allocated here by
torch, not by the library). This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from natray_b200 import Params, World, build_world
from natray_b200._abi import NatrayError, check, lib
from natray_b200.sim import Sim

pytestmark = pytest.mark.gpu

NONE = 0xFFFFFFFF


def keys_of(world: World, block_list: np.ndarray) -> np.ndarray:
    """Each live particle's block index among `block_list`, as the step computes it: the own
    cell floor((x - origin) / h) in float32, its block (cell >> 2), the block's index."""
    h = world.h
    org = np.array(h.params.origin[:3], dtype=np.float32)
    hh = np.float32(h.params.origin[3])
    bd = np.array(h.params.bdims[:3], dtype=np.int64)
    p = world.particles
    c = np.floor((p[:, :3] - org) / hh).astype(np.int64) >> 2
    slot = (c[:, 0] * bd[1] + c[:, 1]) * bd[2] + c[:, 2]
    idx = np.searchsorted(block_list, slot)
    idx_c = np.minimum(idx, len(block_list) - 1)
    ok = (p[:, 7] >= 0.5) & (block_list[idx_c] == slot) & np.all(c >= 0, axis=1) & np.all(c < bd, axis=1)
    return np.where(ok, idx_c, NONE).astype(np.uint32)


def sort_noalloc(keys: np.ndarray, n_blocks: int):
    import torch
    dev = torch.device("cuda:0")
    k = torch.from_numpy(keys.view(np.int32)).to(dev)
    srt = torch.empty(len(keys), dtype=torch.int32, device=dev)
    bs = torch.empty(n_blocks + 1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    check(lib().ntr_sort_by_block_noalloc(k.data_ptr(), len(keys), n_blocks, srt.data_ptr(), bs.data_ptr(), stream))
    torch.cuda.synchronize(dev)
    return srt.cpu().numpy().view(np.uint32), bs.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_the_step_twice():
    import torch
    torch.cuda.init()
    w = build_world(Params(resolution=28, mesh_level=3, block_cap=4096, spray_cap=100000))
    sim = Sim(world=w)
    for call in range(2):
        before = sim.snapshot()
        assert sim.step(1) == 1
        nb = sim.state["n_blocks"]
        bl = sim.download("BLOCK_LIST", np.uint32, nb)
        bs_step = sim.download("BLOCK_START", np.uint32, nb + 1)
        srt_step = sim.download("SORTED", np.uint32, int(bs_step[-1]))
        keys = keys_of(before, bl)
        srt, bs = sort_noalloc(keys, nb)
        assert np.array_equal(bs, bs_step), f"call {call}: block starts differ"
        assert np.array_equal(srt[: bs[-1]], srt_step), f"call {call}: sorted particles differ"
        assert bs[-1] == int((keys != NONE).sum())


def test_noalloc_sort_rejects_sizes_beyond_its_scratch():
    import torch
    dev = torch.device("cuda:0")
    small = torch.zeros(16, dtype=torch.int32, device=dev)
    with pytest.raises(NatrayError) as e:
        check(lib().ntr_sort_by_block_noalloc(small.data_ptr(), 1048577, 4, small.data_ptr(), small.data_ptr(), None))
    assert e.value.status == 1 and "at most 1048576" in str(e.value)
    with pytest.raises(NatrayError) as e:
        check(lib().ntr_sort_by_block_noalloc(small.data_ptr(), 4, 65536, small.data_ptr(), small.data_ptr(), None))
    assert e.value.status == 1 and "at most 65535" in str(e.value)


def expected_sort(keys: np.ndarray, n_blocks: int):
    """The stable sort by block of numpy: particle indices grouped by key (NONE last), and where
    each block's particles start."""
    order = np.argsort(keys.astype(np.int64), kind="stable").astype(np.uint32)
    valid = np.sort(keys[keys != NONE].astype(np.int64))
    starts = np.searchsorted(valid, np.arange(n_blocks + 1), side="left").astype(np.uint32)
    return order[: len(valid)], starts


@pytest.mark.parametrize("n,n_blocks", [(3 * 4096 + 17, 300), (1048576, 60000)])
def test_noalloc_sort_two_passes_up_to_the_key_limit(n, n_blocks):
    # More than 255 blocks: two 8-bit passes (through the scratch's alternate keys and values);
    # partial last tiles; about 5 % of the particles taking no part; the largest n it takes.
    import torch
    torch.cuda.init()
    rng = np.random.default_rng(n)
    keys = rng.integers(0, n_blocks, size=n, dtype=np.int64).astype(np.uint32)
    keys[rng.random(n) < 0.05] = NONE
    srt, bs = sort_noalloc(keys, n_blocks)
    want_srt, want_bs = expected_sort(keys, n_blocks)
    assert np.array_equal(bs, want_bs)
    assert np.array_equal(srt[: bs[-1]], want_srt)


def test_noalloc_sort_of_no_keys():
    import torch
    dev = torch.device("cuda:0")
    bs = torch.full((65,), -1, dtype=torch.int32, device=dev)
    check(lib().ntr_sort_by_block_noalloc(None, 0, 64, None, bs.data_ptr(), None))
    torch.cuda.synchronize(dev)
    assert np.array_equal(bs.cpu().numpy(), np.zeros(65, dtype=np.int32))
