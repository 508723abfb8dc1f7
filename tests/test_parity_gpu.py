"""Parity of the CUDA step with the oracle, through the C ABI, on the same seeded inputs.

Both sides run the canonical form of the reference's step (blocks by ascending slot,
particles by ascending index within a block, spray slots in that order), the same float
expressions without contraction, fixed-point i32 transfer sums, the same tree shapes for
the solver's inner products, and the same float transcendentals. So the comparison is bit for
bit: block sets, sort order and fixed-point sums as integers, every float field by its bits.
"""
import numpy as np
import pytest

from natray_b200 import Params, World, build_world
from natray_b200._abi import NatrayError
from natray_b200.sim import Sim
from oracle.py import Oracle

pytestmark = pytest.mark.gpu

SECTIONS_COMPARED = ["PARTICLES", "MEM_X", "MEM_V", "MEM_WATER", "MEM_LAYER", "MEM_PUSH", "ALIVE", "BULLETS",
                     "SECTIONS", "BULLET_HIT", "POSE_LOG", "BLOCKS_PREV", "BLOCK_ACTIVE", "AIR", "SPRAY", "LANDED", "TOUCH"]


def small(**kw):
    base = dict(resolution=24, mesh_level=3, block_cap=4096, spray_cap=200000)
    base.update(kw)
    return build_world(Params(**base))


def measured(w: World) -> World:
    """The world after the zero-length measuring substep, taken on the CPU so that both sides
    start from the same substep counts."""
    return World(Oracle(w.blob).snapshot())


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def first_diff(a, b):
    a, b = bits(a).reshape(-1), bits(b).reshape(-1)
    if a.shape != b.shape:
        return f"shape {a.shape} vs {b.shape}"
    d = np.nonzero(a != b)[0]
    if d.size == 0:
        return None
    return f"{d.size} of {a.size} differ, first at {d[:4]}"


def assert_worlds_equal(a: World, b: World, where: str):
    sa, sb = a.state, b.state
    bad = {k: (sa[k], sb[k]) for k in sa if not (sa[k] == sb[k] or (np.isnan(sa[k]) and np.isnan(sb[k])))}
    assert not bad, f"{where}: state differs {bad}"
    for sec in SECTIONS_COMPARED:
        d = first_diff(a.sec(sec), b.sec(sec))
        assert d is None, f"{where}: section {sec}: {d}"
    assert (a.h.iters, a.h.substeps, a.h.air_substeps) == (b.h.iters, b.h.substeps, b.h.air_substeps), where


def assert_grids_equal(o: Oracle, s: Sim, where: str):
    g = s.grid()
    for k in ["block_list", "block_start", "sorted", "block_nb", "acc", "cf", "air"]:
        d = first_diff(o.get(k), g[k])
        assert d is None, f"{where}: {k}: {d}"


@pytest.fixture(scope="module")
def w_small():
    return measured(small())


def test_first_step_is_bit_exact(w_small):
    o, s = Oracle(w_small.blob), Sim(world=w_small)
    assert o.step(1) == s.step(1) == 1
    assert_grids_equal(o, s, "step 1")
    assert_worlds_equal(World(o.snapshot()), s.snapshot(), "step 1")


def test_batches_stay_bit_exact(w_small):
    # Free running, through the impact: the bullet starts 5 cm out at 330 m/s.
    o, s = Oracle(w_small.blob), Sim(world=w_small)
    for k in range(6):
        assert o.step(4) == s.step(4)
        assert_worlds_equal(World(o.snapshot()), s.snapshot(), f"batch {k}")
    assert_grids_equal(o, s, "after 24 steps")
    st = s.state
    assert st["step"] == 24 and st["n_blocks"] > 0


def test_fixed_step_bb_shot_bit_exact():
    # The small fixed-step scene: d = 8 cm, a 5,120-triangle membrane, thickness 0.2 mm, a
    # steel sphere of 8 mm at 300 m/s, dt = 2 us. Scaled down in particle count to run in
    # seconds on the CPU side.
    w = measured(small(diameter=8, resolution=24, mesh_level=4, thickness=0.2, bullet=6, caliber=8,
                       bullet_speed=300, dt_max=2e-6))
    o, s = Oracle(w.blob), Sim(world=w)
    for k in range(5):
        o.step(8)
        s.step(8)
    a, b = World(o.snapshot()), s.snapshot()
    assert a.state["dt_ns"] == 2000
    assert_worlds_equal(a, b, "fixed step")


def test_solver_from_memory_bit_exact(oracle_threads):
    # More blocks than the persistent solver has warps (256 CTAs x 12): its warps own two blocks
    # or more, and keep the solver's values in memory instead of registers.
    w = measured(build_world(Params(resolution=132, mesh_level=4, block_cap=65535, spray_cap=100000)))
    o, s = Oracle(w.blob), Sim(world=w)
    assert o.step(2) == s.step(2) == 2
    assert s.state["n_blocks"] > 256 * 12 and s.state["solve_iters"] > 0
    assert_grids_equal(o, s, "step 2")
    assert_worlds_equal(World(o.snapshot()), s.snapshot(), "step 2")


def test_launch_shapes_do_not_change_results(oracle_threads):
    # One solver CTA for ~600 blocks: it owns all 256 residues, and its partial sums go to global
    # memory (more than fit in shared). Few and many CTAs for the other kernels. All bit-exact.
    w = measured(build_world(Params(resolution=64, mesh_level=4, block_cap=8192, spray_cap=100000)))
    o = Oracle(w.blob)
    assert o.step(2) == 2
    ref = World(o.snapshot())
    for tune in [dict(solve_ctas=1, cell_ctas_per_sm=2, block_ctas_per_sm=3),
                 dict(solve_ctas=37, cell_ctas_per_sm=16, block_ctas_per_sm=12)]:
        s = Sim(world=w)
        s.tuning = tune
        assert s.tuning["solve_ctas"] == tune["solve_ctas"]
        assert s.step(2) == 2
        assert s.state["n_blocks"] > 512
        assert_grids_equal(o, s, f"tuning {tune}")
        assert_worlds_equal(ref, s.snapshot(), f"tuning {tune}")


def test_autotune_keeps_the_state(w_small):
    s = Sim(world=w_small)
    s.step(2)
    before = s.snapshot()
    best, ms = s.autotune(steps=2)
    assert ms > 0 and best["block_ctas_per_sm"] > 0
    assert_worlds_equal(before, s.snapshot(), "after autotune")


def test_reference_fp32_sums_bit_exact(w_small):
    o = Oracle(w_small.blob, fp64_dots=False)
    s = Sim(world=w_small, fp64_reductions=False)
    for _ in range(3):
        o.step(4)
        s.step(4)
    assert_worlds_equal(World(o.snapshot()), s.snapshot(), "FP32 sums")


def test_snapshot_restore_roundtrip(w_small):
    s = Sim(world=w_small)
    s.step(5)
    a = s.snapshot()
    s2 = Sim(world=a)
    assert_worlds_equal(a, s2.snapshot(), "restore")
    s.step(3)
    s2.step(3)
    assert_worlds_equal(s.snapshot(), s2.snapshot(), "after restore")
    # Restoring a different state into a live simulation.
    s.restore(a)
    assert_worlds_equal(a, s.snapshot(), "restore into live")


def test_overflow_is_reported():
    w = measured(small(block_cap=16))
    s = Sim(world=w)
    with pytest.raises(NatrayError) as e:
        s.step(1)
    assert e.value.status == 3  # NTR_E_OVERFLOW


def test_advance_follows_the_reference_timeline(w_small):
    s = Sim(world=w_small)
    info = s.info
    taken = s.advance(info.t0 + 2e-4, 1000)
    st = s.state
    assert taken == st["step"] > 0
    assert st["t_ns"] == 200000  # lands exactly on the stop time
    assert s.advance(info.t0 + 2e-4, 1000) == 0


def test_conservation_sums(w_small):
    s = Sim(world=w_small)
    c = s.conservation()
    assert c[0] == w_small.h.n_particles
    p = w_small.particles.astype(np.float64)
    assert np.allclose(c[5:8], p[:, :3].sum(0), rtol=1e-6)
    s.step(2)
    launches, ms = s.last_launches()
    assert launches > 40 and ms > 0


def test_four_bullets_bit_exact(oracle_threads):
    # A 5.56 mm spitzer, a flat-nosed pellet, a .45 round nose and a steel BB from four sides,
    # 50 us apart (the reference's `shotN.key` parameters): every bullet branch of the step in
    # one scene, through their impacts, the tearing and the first spray.
    p = Params(resolution=24, mesh_level=3, block_cap=4096, spray_cap=200000)
    for k, (b, az, delay) in enumerate([(3, 0, 0.0), (5, 90, 0.05), (2, 180, 0.1), (6, 270, 0.15)], start=1):
        p.set(f"shot{k}.bullet", b)
        p.set(f"shot{k}.azimuth", az)
        p.set(f"shot{k}.delay", delay)
    w = measured(build_world(p))
    assert w.h.n_shots == 4
    o, s = Oracle(w.blob), Sim(world=w)
    for k in range(10):
        assert o.step(10) == s.step(10) == 10
        assert_worlds_equal(World(o.snapshot()), s.snapshot(), f"batch {k}")
    end = s.snapshot()
    assert end.state["spray_count"] > 0 and int((end.sec("ALIVE") == 0).sum()) > 0


def test_large_scene_bit_exact(oracle_threads):
    # From 300k particles G2P runs its many-block form (CTAs of 128 threads, six an SM), the one
    # the 1M-particle workload takes; the smaller scenes of the other tests take the 256-thread
    # form.
    w = measured(build_world(Params(resolution=88, mesh_level=5, block_cap=4096, spray_cap=200000)))
    assert w.h.n_particles >= 300000
    o, s = Oracle(w.blob), Sim(world=w)
    for k in range(2):
        assert o.step(2) == s.step(2) == 2
        assert_worlds_equal(World(o.snapshot()), s.snapshot(), f"batch {k}")


def test_long_run_to_the_ground_bit_exact(oracle_threads):
    # A low balloon (0.12 m) run for 1200 steps of the reference's adaptive dt, about 0.45 s:
    # the water and its spray fall, drops land (LANDED) and the ground gets wet (TOUCH), and
    # both sides still agree bit for bit.
    w = measured(build_world(Params(resolution=16, mesh_level=3, block_cap=4096, spray_cap=100000, height=0.12)))
    o, s = Oracle(w.blob), Sim(world=w)
    for k in range(12):
        assert o.step(100) == s.step(100) == 100
        if k % 4 == 3:
            assert_worlds_equal(World(o.snapshot()), s.snapshot(), f"after {100 * (k + 1)} steps")
    end = s.snapshot()
    assert int((end.sec("LANDED")[:, 3] > 0).sum()) > 100 and int((end.sec("TOUCH") != 0xFFFFFFFF).sum()) > 100


def test_pack_particles_gives_the_reference_layout(w_small):
    # ntr_sim_pack_particles: the five SoA arrays written as the reference's 20-float records
    # into a device buffer the caller owns (here torch's), on the caller's stream or not.
    import ctypes as C

    import torch
    from natray_b200._abi import lib
    s = Sim(world=w_small)
    s.step(6)
    want = s.snapshot().sec("PARTICLES")
    n = want.shape[0]
    buf = torch.zeros(n * 80, dtype=torch.uint8, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    assert lib().ntr_sim_pack_particles(s._h, C.c_void_p(buf.data_ptr()), n * 80, C.c_void_p(stream)) == 0
    got = buf.cpu().numpy().view(np.float32).reshape(n, 20)
    assert np.array_equal(bits(got), bits(want))
    buf.zero_()
    torch.cuda.synchronize()
    assert lib().ntr_sim_pack_particles(s._h, C.c_void_p(buf.data_ptr()), n * 80, None) == 0
    assert np.array_equal(bits(buf.cpu().numpy().view(np.float32).reshape(n, 20)), bits(want))
    assert lib().ntr_sim_pack_particles(s._h, C.c_void_p(buf.data_ptr()), n * 80 - 16, None) == 1  # too small
    s.close()
