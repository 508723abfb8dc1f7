"""Parity of the CUDA step with the oracle at the sizes the benchmark times.

The 1M-particle scene (`bench.py`'s workload: a 16 cm balloon at lattice resolution 124, 976,915
particles, an icosphere(6) membrane of 40,962 vertices and 81,920 triangles, an 8 mm steel
sphere at 350 m/s, a fixed step of 2 us) is run through the bullet's impact on the membrane
(the sphere starts 5 cm out, so it reaches the rubber after about 70 steps), and the small
fixed-step scene (d = 8 cm at resolution 51, about 70k particles, an icosphere(4) membrane of
thickness 0.2 mm, the sphere at 300 m/s) for its full 200 steps. Every section of the world and
the step's grid are compared bit for bit after each batch (src/sim.rs:553-566 is the step;
shaders/membrane.wgsl:283-400 the rubber substep whose contact search runs at the impact).
"""
import numpy as np
import pytest

from natray_b200 import Params, World, build_world
from natray_b200.sim import Sim
from oracle.py import Oracle

from test_parity_gpu import assert_grids_equal, assert_worlds_equal

pytestmark = pytest.mark.gpu

BENCH_SCENE = dict(resolution=124, mesh_level=6, dt_max=2e-6, bullet=6, caliber=8, bullet_speed=350)
SMALL_FIXED = dict(diameter=8, resolution=51, mesh_level=4, thickness=0.2, bullet=6, caliber=8, bullet_speed=300,
                   dt_max=2e-6)


def _measured(params: Params) -> World:
    return World(Oracle(build_world(params).blob).snapshot())


def _bullet_gap(w: World) -> float:
    """Distance from the bullet's centre to the nearest membrane vertex."""
    b = w.sec("BULLETS")[0]
    x = w.sec("MEM_X")[:, :3].astype(np.float64)
    return float(np.sqrt(((x - b[:3].astype(np.float64)) ** 2).sum(1)).min())


def test_bench_scene_through_the_impact(oracle_threads):
    w = _measured(Params(**BENCH_SCENE))
    assert w.h.n_particles == 976915 and w.h.n_tris == 81920 and w.h.n_verts == 40962
    gap0 = _bullet_gap(w)
    o, s = Oracle(w.blob), Sim(world=w)
    steps, touched = 0, False
    for k in range(10):
        assert o.step(10) == s.step(10) == 10
        steps += 10
        a, b = World(o.snapshot()), s.snapshot()
        assert_worlds_equal(a, b, f"1M scene after {steps} steps")
        touched = touched or int(a.sec("MEM_V")[:, 3].sum()) > 0
    assert_grids_equal(o, s, f"1M scene after {steps} steps")
    end = s.snapshot()
    assert end.state["dt_ns"] == 2000 and end.state["step"] == 100
    # The sphere has reached the rubber: vertices held on it (mem_v.w = 1) at some batch end,
    # and it is now inside the membrane's outer hull where it started 5 cm out.
    assert touched, "the bullet never held a membrane vertex: the run did not reach the impact"
    assert _bullet_gap(end) < gap0
    s.close()


def test_small_fixed_step_scene_at_full_size(oracle_threads):
    w = _measured(Params(**SMALL_FIXED))
    assert 60000 < w.h.n_particles < 80000 and w.h.n_tris == 5120
    o, s = Oracle(w.blob), Sim(world=w)
    for k in range(10):
        assert o.step(20) == s.step(20) == 20
        assert_worlds_equal(World(o.snapshot()), s.snapshot(), f"small fixed-step scene after {20 * (k + 1)} steps")
    assert_grids_equal(o, s, "small fixed-step scene after 200 steps")
    st = s.state
    assert st["step"] == 200 and st["dt_ns"] == 2000
    s.close()
