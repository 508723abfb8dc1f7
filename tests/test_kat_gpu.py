"""Known-answer tests of the CUDA step, through the C ABI: the cases of test_kat.py (Ogden
triangles against `Latex::stress`, the Sod shock tube against the exact Riemann solution, the
hydrostatic layer, the pressure solve against an f64 direct solve of the same system, uniform
translation), each also compared bit for bit with the oracle on the same world."""
import pytest

import kat_cases as K
from natray_b200 import World
from natray_b200.sim import Sim
from oracle.py import Oracle

from test_parity_gpu import assert_grids_equal, assert_worlds_equal

pytestmark = pytest.mark.gpu


def _run(w0, batches):
    s, o = Sim(world=w0), Oracle(w0.blob)
    for n in batches:
        assert s.step(n) == o.step(n) == n
    return s, o


def test_ogden_triangles_gpu():
    w0, info = K.ogden_world()
    s, o = _run(w0, [1])
    w1 = s.snapshot()
    assert_worlds_equal(World(o.snapshot()), w1, "ogden")
    errs = K.check_ogden(w0, info, w1)
    assert all(e < 1e-4 for e in errs.values()), errs
    s.close()


def test_sod_shock_tube_gpu():
    w0, info = K.sod_world()
    s, o = _run(w0, [1] * K.SOD_STEPS)
    w1 = s.snapshot()
    assert_worlds_equal(World(o.snapshot()), w1, "sod")
    r = K.check_sod(w1, info)
    assert r["core_spread"] < 1e-6
    assert r["plateau_p"] < 0.02 and r["plateau_u"] < 0.02 and r["plateau_cells"] >= 4
    assert r["shock_err_cells"] < 1.0
    assert r["l1_rho"] < 0.06 and r["l1_p"] < 0.06
    s.close()


def test_hydrostatic_layer_gpu():
    w0, _ = K.hydro_world()
    s, o = _run(w0, [1])
    assert_grids_equal(o, s, "hydrostatic")
    r = K.check_hydro(s.grid(), w0)
    assert r["rel_err"] < 1e-4 and r["max_v"] < 1e-6
    s.close()


def test_pressure_solve_against_direct_solve_gpu():
    w0, _ = K.pcg_world()
    s, o = _run(w0, [1])
    assert_grids_equal(o, s, "manufactured pressure")
    r = K.check_pressure_system(s.grid(), w0, s.state["dt_ns"] * 1e-9)
    assert r["n_water"] == 24 ** 3
    assert r["rel_err"] < 1e-4 and r["rel_residual"] < 1e-5
    s.close()


def test_uniform_block_translates_gpu():
    w0, info = K.advect_world()
    s, o = _run(w0, [1])
    assert_grids_equal(o, s, "uniform block")
    r = K.check_advect(s.snapshot(), info, s.grid())
    assert r["alive"] == r["n"]
    assert r["dv"] < 1e-4 and r["dx_f32"] == 0.0 and r["grid_du"] < 1e-4 and r["affine"] < 0.05
    assert s.step(K.ADV_STEPS - 1) == o.step(K.ADV_STEPS - 1) == K.ADV_STEPS - 1
    w1 = s.snapshot()
    assert_worlds_equal(World(o.snapshot()), w1, "uniform block, 20 steps")
    r = K.check_advect(w1, info)
    assert r["alive"] == r["n"] and r["dv"] < 1e-2
    s.close()
