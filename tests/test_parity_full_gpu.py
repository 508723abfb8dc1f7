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


def _impact(w: World) -> tuple[int, int]:
    """Triangles torn, and the cavity sections the bullet has opened in the water (its info.w,
    bullet.wgsl:16-34)."""
    return int((w.sec("ALIVE") == 0).sum()), int(w.sec("BULLETS")[0, 24:28].view(np.uint32)[3])


def test_bench_scene_through_the_impact(oracle_threads):
    w = _measured(Params(**BENCH_SCENE))
    assert w.h.n_particles == 976915 and w.h.n_tris == 81920 and w.h.n_verts == 40962
    assert _impact(w) == (0, 0)
    o, s = Oracle(w.blob), Sim(world=w)
    steps = 0
    for k in range(10):
        assert o.step(10) == s.step(10) == 10
        steps += 10
        assert_worlds_equal(World(o.snapshot()), s.snapshot(), f"1M scene after {steps} steps")
    assert_grids_equal(o, s, f"1M scene after {steps} steps")
    end = s.snapshot()
    assert end.state["dt_ns"] == 2000 and end.state["step"] == 100
    # The sphere has gone through the rubber (it reaches it at about step 70 and tears it) and
    # is opening a cavity in the water behind.
    torn, sections = _impact(end)
    assert torn > 0 and sections > 0, (torn, sections)
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
