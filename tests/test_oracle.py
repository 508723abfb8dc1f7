"""The oracle (the CPU restatement of the step) against known answers and invariants that the
reference's kernels guarantee by construction. CPU only, small scenes.

The reference has no recorded outputs for its step kernels (no golden vectors, fixtures or
known answers for P2G/CG/G2P/membrane/air/bullet), so these tests pin the restatement by
properties: canonical block activation and sort order, partition of unity of the quadratic
B-spline weights, particle counts per cell, conservation, FP32 against FP64, and the regression
fixture in tests/golden/ that tests/golden/make_golden.py wrote from this oracle.
"""
import math

import numpy as np
import pytest

from natray_b200 import Params, World, build_world
from oracle.py import Oracle

FP_W = 16777216.0


def small(**kw):
    base = dict(resolution=20, mesh_level=3, block_cap=4096, spray_cap=100000)
    base.update(kw)
    return build_world(Params(**base))


@pytest.fixture(scope="module")
def stepped(oracle_threads):
    w = small()
    o = Oracle(w.blob)
    o.step(1)
    return w, o


def test_measure_sets_substeps(oracle_threads):
    o = Oracle(small().blob)
    w = World(o.snapshot())
    assert w.h.substeps >= 2 and w.h.substeps % 2 == 0
    assert w.h.air_substeps >= 2 and w.h.air_substeps % 2 == 0
    st = w.state
    assert 0 < st["mem_dt"] < 1e-3 and st["cap_dt"] > 0
    # The measuring substep writes each free vertex's area and moves nothing.
    assert (w.sec("MEM_PUSH")[:, 1] > 0).sum() > 0
    assert np.array_equal(w.sec("MEM_X"), small().sec("MEM_X"))


def test_block_activation_is_the_union_of_stencils(stepped):
    w, o = stepped
    bl = o.get("block_list")
    assert np.all(np.diff(bl.astype(np.int64)) > 0), "canonical order: ascending slots"
    h = w.h
    bd = np.array(h.params.bdims[:3], dtype=np.int64)
    org = np.array(h.params.origin[:3], dtype=np.float32)
    hh = np.float32(h.params.origin[3])
    p = w.particles[:, :3]
    c = np.floor((p - org) / hh).astype(np.int64)
    need = set()
    for dx in (-1, 2):
        for dy in (-1, 2):
            for dz in (-1, 2):
                b = np.clip((c + np.array([dx, dy, dz])) >> 2, 0, bd - 1)
                need.update(((b[:, 0] * bd[1] + b[:, 1]) * bd[2] + b[:, 2]).tolist())
    assert need <= set(bl.tolist())


def test_sort_is_canonical_and_counts_cells(stepped):
    w, o = stepped
    bl, bs, srt = o.get("block_list"), o.get("block_start"), o.get("sorted")
    n = len(bl)
    live = np.nonzero(w.particles[:, 7] >= 0.5)[0]
    assert np.array_equal(np.sort(srt), live)
    h = w.h
    bd = np.array(h.params.bdims[:3], dtype=np.int64)
    org = np.array(h.params.origin[:3], dtype=np.float32)
    hh = np.float32(h.params.origin[3])
    c = np.floor((w.particles[srt, :3] - org) / hh).astype(np.int64) >> 2
    slot = (c[:, 0] * bd[1] + c[:, 1]) * bd[2] + c[:, 2]
    idx = np.searchsorted(bl, slot)
    assert np.array_equal(bl[idx], slot)
    # Blocks ascending; particles ascending within a block.
    key = idx.astype(np.int64) * (1 << 32) + srt
    assert np.all(np.diff(key) > 0)
    assert bs[0] == 0 and bs[-1] == len(srt)
    acc = o.get("acc").reshape(19, n * 64)
    assert acc[8].sum() == len(srt)  # A_N counts each particle once


def test_weights_partition_unity(stepped):
    w, o = stepped
    n = len(o.get("block_list"))
    acc = o.get("acc").reshape(19, n * 64).astype(np.int64)
    npart = len(o.get("sorted"))
    for f in (1, 3, 5, 6):  # a_wt(0..2) and A_WC
        total = acc[f].sum() / FP_W
        # 27 rounded nodes per particle, each within half a unit of the last place.
        assert abs(total - npart) <= npart * 27 * 0.5 / FP_W + 1e-9


def test_momentum_transfer_at_rest(stepped):
    # Particles start at rest with zero affine matrices: every momentum sum is exactly zero.
    w, o = stepped
    n = len(o.get("block_list"))
    acc = o.get("acc").reshape(19, n * 64)
    for f in (0, 2, 4):
        assert np.all(acc[f] == 0)


def test_first_step_under_gravity(stepped):
    w, o = stepped
    s = World(o.snapshot())
    st = s.state
    assert st["step"] == 1 and st["dt_ns"] > 0
    live = s.particles[:, 7] >= 0.5
    assert live.sum() == w.h.n_particles
    v = s.particles[live, 4:7]
    # One step of gravity against the rubber and the pressure: the mean vertical velocity
    # is at most g dt and finite everywhere.
    dt = st["dt_ns"] * 1e-9
    assert np.isfinite(v).all()
    assert abs(v[:, 1].mean()) <= 9.81 * dt * 1.01


def test_snapshot_roundtrip_is_exact(oracle_threads):
    o = Oracle(small().blob)
    o.step(3)
    a = o.snapshot()
    b = Oracle(a).snapshot()
    assert a == b


def test_dead_step_changes_nothing(oracle_threads):
    o = Oracle(small().blob)
    o.step(2)
    a = World(o.snapshot())
    t = a.state["t_ns"]
    assert o.step(3, stop_ns=t) == 0
    b = World(o.snapshot())
    assert np.array_equal(a.particles, b.particles)
    assert b.state["t_ns"] == t


def test_fixed_step_is_dt_max(oracle_threads):
    o = Oracle(small(dt_max=2e-6).blob)
    o.step(4)
    st = World(o.snapshot()).state
    assert st["dt_ns"] == 2000 and st["t_ns"] == 8000


def test_fp32_tracks_fp64(oracle_threads):
    # The precision study in small: FP32 state with FP64 solver sums against an all-FP64 run.
    w = small(dt_max=2e-6)
    a, b = Oracle(w.blob), Oracle(w.blob, real64=True)
    for _ in range(3):
        a.step(4)
        b.step(4)
    pa, pb = World(a.snapshot()).particles.astype(np.float64), World(b.snapshot()).particles.astype(np.float64)
    rel_x = np.linalg.norm(pa[:, :3] - pb[:, :3]) / np.linalg.norm(pb[:, :3])
    rel_v = np.linalg.norm(pa[:, 4:7] - pb[:, 4:7]) / max(np.linalg.norm(pb[:, 4:7]), 1e-30)
    assert rel_x < 1e-6
    # Velocities 24 us after rest are a few mm/s; both runs stop the pressure solve at a
    # relative residual of 1e-5 of a right-hand side set by the rubber's pull (~1e5 Pa), so
    # their velocity fields agree to a few parts in 1e3, not to FP32 rounding.
    assert rel_v < 1e-2


def test_reference_sums_match_fp64_sums(oracle_threads):
    # The reference's FP32 tree for the solver's inner products and the FP64 one agree to the
    # solver tolerance.
    w = small(dt_max=2e-6)
    a, b = Oracle(w.blob, fp64_dots=True), Oracle(w.blob, fp64_dots=False)
    a.step(4)
    b.step(4)
    pa, pb = World(a.snapshot()).particles, World(b.snapshot()).particles
    rel_v = np.linalg.norm(pa[:, 4:7] - pb[:, 4:7]) / max(np.linalg.norm(pa[:, 4:7]), 1e-30)
    assert rel_v < 1e-3


def test_weightless_balloon_stays_put(oracle_threads):
    # No gravity and a balloon inflated without it: the water barely moves before the bullet
    # arrives (the shot is delayed beyond the steps run).
    w = small(gravity=0, dt_max=2e-6, delay=5)
    o = Oracle(w.blob)
    o.step(10)
    s = World(o.snapshot())
    d = np.abs(s.particles[:, :3] - w.particles[:, :3]).max()
    assert d < 1e-3 * w.h.params.origin[3]
    assert s.state["spray_count"] == 0
