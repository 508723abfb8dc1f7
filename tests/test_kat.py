"""Known-answer tests of the oracle (CPU): the restatement of the reference's kernels against
answers computed without it. The same cases run on the CUDA step in test_kat_gpu.py."""
import pytest

import kat_cases as K
from natray_b200 import World
from oracle.py import Oracle


def test_ogden_triangles_match_the_latex_closed_form():
    w0, info = K.ogden_world()
    o = Oracle(w0.blob)
    assert o.step(1) == 1
    errs = K.check_ogden(w0, info, World(o.snapshot()))
    print(errs)
    # FP32 stretches and stresses against f64: a few units in the last place of the forces.
    assert all(e < 1e-4 for e in errs.values()), errs


def test_sod_shock_tube_matches_the_exact_riemann_solution():
    w0, info = K.sod_world()
    o = Oracle(w0.blob)
    for _ in range(K.SOD_STEPS):
        assert o.step(1) == 1
    r = K.check_sod(World(o.snapshot()), info)
    print(r)
    assert r["core_spread"] < 1e-6  # the core of the tube is one-dimensional
    # A first-order HLL scheme smears the rarefaction, the contact and the shock over a few
    # cells each, but reaches the star state in between and moves the shock at its speed.
    assert r["plateau_p"] < 0.02 and r["plateau_u"] < 0.02 and r["plateau_cells"] >= 4
    assert r["shock_err_cells"] < 1.0
    assert r["l1_rho"] < 0.06 and r["l1_p"] < 0.06


def test_hydrostatic_layer_pressure_is_rho_g_depth():
    w0, _ = K.hydro_world()
    o = Oracle(w0.blob)
    assert o.step(1) == 1
    grid = {k: o.get(k) for k in ("block_list", "acc", "cf")}
    r = K.check_hydro(grid, w0)
    print(r)
    # Solver tolerance 1e-6, a system of condition about 100: 1e-4 with room to spare.
    assert r["rel_err"] < 1e-4 and r["max_v"] < 1e-6


def test_pressure_solve_matches_a_direct_solve_of_the_same_system():
    w0, _ = K.pcg_world()
    o = Oracle(w0.blob)
    assert o.step(1) == 1
    grid = {k: o.get(k) for k in ("block_list", "acc", "cf")}
    r = K.check_pressure_system(grid, w0, World(o.snapshot()).state["dt_ns"] * 1e-9)
    print({k: v for k, v in r.items() if not k.startswith("p_")})
    assert r["n_water"] == 24 ** 3
    assert r["rel_err"] < 1e-4 and r["rel_residual"] < 1e-5


def test_uniform_block_translates_unchanged():
    # One step: the transfers keep a uniform velocity to their fixed-point rounding (momentum
    # in steps of 2^-16 m/s, weights of 2^-24), and the positions move by exactly dt v. Later
    # steps see the still air outside push back on the moving block (about rho_air c_air |v|,
    # 150 Pa): the velocity then drifts, by 0.25 % after 20 steps, which the loose bound allows.
    w0, info = K.advect_world()
    o = Oracle(w0.blob)
    assert o.step(1) == 1
    grid = {k: o.get(k) for k in ("block_list", "acc", "cf")}
    r = K.check_advect(World(o.snapshot()), info, grid)
    print(r)
    assert r["alive"] == r["n"]
    assert r["dv"] < 1e-4 and r["dx_f32"] == 0.0 and r["grid_du"] < 1e-4 and r["affine"] < 0.05
    assert o.step(K.ADV_STEPS - 1) == K.ADV_STEPS - 1
    r = K.check_advect(World(o.snapshot()), info)
    assert r["alive"] == r["n"] and r["dv"] < 1e-2
