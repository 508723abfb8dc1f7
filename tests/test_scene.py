"""Scene construction on the CPU, with the reference's own unit tests restated:
src/balloon.rs:479-514, src/bullet.rs:134-154, src/presets.rs:118-129, and set_kv
(src/params.rs:361-423)."""
import ctypes as C
import math

import numpy as np
import pytest

from natray_b200 import Params, build_world
from natray_b200._abi import NatrayError, Profile, check, lib

PRESETS = ["Backlit", "Tumbling rifle round", "Crossfire", "Four sides", "Moon gravity", "Weightless", "Slow pellet", "Bounce"]


def inflate(shear, thick, rest_r, volume, rho_g) -> Profile:
    p = Profile()
    check(lib().ntr_inflate(shear, thick, rest_r, volume, rho_g, C.byref(p)))
    return p


def samples(p: Profile) -> np.ndarray:
    return np.array(p.samples[: p.n_samples])


def r_at(p: Profile, z: float) -> float:
    """Profile::r_at (src/balloon.rs:91-100)."""
    s = samples(p)
    if z <= 0.0 or z >= p.z_neck:
        return 0.0
    i = int(np.searchsorted(s[:, 2], z, side="left"))
    i = min(max(i, 1), len(s) - 1)
    a, b = s[i - 1], s[i]
    return a[1] + (b[1] - a[1]) * (z - a[2]) / max(b[2] - a[2], 1e-15)


def test_inflation_holds_the_volume_and_hangs_pear_shaped():
    # balloon.rs:483-495
    d = 0.16
    v = math.pi / 6.0 * d ** 3
    p = inflate(0.42e6, 0.25e-3, 0.03, v, 1000.0 * 9.81)
    assert abs(p.volume - v) / v < 1e-6
    assert p.z_centroid < 0.5 * p.z_neck
    assert abs(samples(p)[-1, 1] - p.neck_r) < 1e-6 * p.neck_r


def test_weightless_balloon_is_round():
    # balloon.rs:497-506
    d = 0.16
    p = inflate(0.42e6, 0.25e-3, 0.03, math.pi / 6.0 * d ** 3, 0.0)
    rmax = samples(p)[:, 1].max()
    r = r_at(p, rmax)
    assert abs(r - rmax) / rmax < 0.02


def test_scene_builds():
    # balloon.rs:508-513 with the default parameters: icosphere(6) has 40,962 verts and
    # 81,920 triangles; the default lattice (resolution 64, d = 16 cm) about pi/6 64^3.
    w = build_world(Params())
    h = w.h
    assert h.n_verts == 40962 and h.n_tris == 81920
    assert abs(h.n_particles - math.pi / 6 * 64 ** 3) / (math.pi / 6 * 64 ** 3) < 0.05
    # The entry ray hits: the bullet starts on the -x side, moving +x at the shot's speed (plus
    # the few cm/s the air takes off it over the last 5 cm, src/flight.rs:404-471), its drop
    # and drift from the 10 m flight small.
    b = w.sec("BULLETS")[0]
    assert b[0] < -0.08 and abs(b[1] - 0.55) < 1e-3 and 330.0 < b[4] < 330.1
    assert abs(b[5]) < 1.0 and abs(b[6]) < 1.0
    # CSR of the triangles around each vertex covers every corner once.
    off, vt = w.sec("VTRI_OFF"), w.sec("VTRI")
    assert off[0] == 0 and off[-1] == len(vt) == 3 * h.n_tris
    tris = w.sec("TRIS")[:, :3]
    for v in [0, 123, 40961]:
        assert all(v in tris[t] for t in vt[off[v]:off[v + 1]])


def test_mesh_level_counts():
    for level, (nv, nt) in {2: (162, 320), 3: (642, 1280), 4: (2562, 5120)}.items():
        w = build_world(Params(resolution=16, mesh_level=level))
        assert (w.h.n_verts, w.h.n_tris) == (nv, nt)


@pytest.mark.parametrize("bullet", range(7))
def test_surfaces_are_closed(bullet):
    # bullet.rs:139-153
    w = build_world(Params(resolution=16, mesh_level=2, bullet=bullet))
    n = int(w.sec("BULLETS")[0, 24:].view(np.uint32)[1])
    assert 0 < n <= 576
    pt = w.sec("PATCHES")[:n]
    area = pt[:, 3].astype(np.float64)
    net = (pt[:, 4:7].astype(np.float64) * area[:, None]).sum(0)
    assert np.linalg.norm(net) < 1e-3 * area.sum()
    line = w.sec("OUTLINES")[:33]
    assert np.all(np.diff(line[:, 0]) >= 0), "contact needs z to rise along the outline"


def test_presets_fit_the_shot_limit():
    # presets.rs:123-128
    for name in PRESETS:
        p = Params.preset(name)
        assert 1 <= p.n_shots <= 4, name


def test_set_kv():
    p = Params()
    p.set("shot2.azimuth", 45)
    assert p.n_shots == 2 and abs(p.shots[1].azimuth_deg - 45) < 1e-6
    # A new shot is the last one a quarter turn further round (SimParams::add_shot).
    p = Params().set("shots", 3)
    assert [round(p.shots[k].azimuth_deg) for k in range(3)] == [0, 90, 180 - 360]
    p = Params().set("bullet", 6)
    assert abs(p.shots[0].caliber_mm - 4.4) < 1e-6 and p.shots[0].spin_rpm == 0.0
    for bad in [("shot0.speed", 1), ("shot5.speed", 1), ("bullet", 7), ("nope", 1), ("shots", 0), ("resolution", -3)]:
        with pytest.raises(NatrayError):
            Params().set(*bad)
    with pytest.raises(NatrayError):
        Params.preset("no such preset")
    # Look parameters are accepted and change nothing the simulation sees.
    a, b = Params(), Params().set("bloom", 0.5)
    assert bytes(a.c) == bytes(b.c)


def test_seeded_jitter_is_reproducible_and_seed_changes_it():
    a = build_world(Params(resolution=20, mesh_level=2))
    b = build_world(Params(resolution=20, mesh_level=2))
    c = build_world(Params(resolution=20, mesh_level=2, seed=7))
    assert np.array_equal(a.particles, b.particles)
    assert not np.array_equal(a.particles, c.particles)
    # Jitter is within 0.15 spacing of the staggered lattice (balloon.rs:433-442).
    s = a.h.params.fluid[3]
    y = a.particles[:, 1] - (a.particles[:, 1].min())
    assert a.particles[:, 3].min() == 1.0 and a.particles[:, 7].min() == 1.0
    assert np.isfinite(y).all() and s > 0


def test_world_header_and_sizes():
    w = build_world(Params(resolution=20, mesh_level=2, block_cap=4096, spray_cap=1000))
    h = w.h
    assert h.block_cap == 4096 and h.spray_cap == 1000 and h.params.bdims[3] == 4096
    assert h.substeps == 0  # not yet measured
    assert h.params.fluid[2] == np.float32(1e-3)
    assert all(d % 4 == 0 for d in h.params.dims[:3])
    assert h.params.dims[3] == h.n_particles
    st = w.state
    assert st["mem_dt"] == np.float32(3.4028235e38) and st["air_dt"] > 0


def test_fixed_step_configs_build():
    # The small scene at ~70k particles (d = 8 cm, resolution 51) with a 5,120-triangle mesh.
    p = Params(diameter=8, resolution=51, mesh_level=4, thickness=0.2, bullet=6, caliber=8, bullet_speed=300, dt_max=2e-6)
    w = build_world(p)
    assert 60000 < w.h.n_particles < 80000 and w.h.n_tris == 5120
    assert abs(w.h.params.fluid[2] - 2e-6) < 1e-12


_PROFILE_BITS = """
import ctypes as C, hashlib, math, sys
sys.path.insert(0, sys.argv[1])
from natray_b200._abi import Profile, check, lib
h = hashlib.sha256()
for d, g in ((0.065, 9.81), (0.16, 9.81), (0.12, 0.0)):
    p = Profile()
    check(lib().ntr_inflate(0.42e6, 0.25e-3, 0.03, math.pi / 6.0 * d ** 3, 1000.0 * g, C.byref(p)))
    h.update(bytes(p))
print(h.hexdigest())
"""


def test_inflation_on_threads_is_bit_identical_to_one_by_one():
    # The search runs its likely next shots together on a pool; with NATRAY_BUILD_THREADS=1 it
    # runs them one at a time in the reference's order. The profiles must agree to the bit.
    import os
    import subprocess
    import sys
    from pathlib import Path

    root = str(Path(__file__).resolve().parents[1])
    out = []
    for n in ("1", "8"):
        env = dict(os.environ, NATRAY_BUILD_THREADS=n)
        r = subprocess.run([sys.executable, "-c", _PROFILE_BITS, root], env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        out.append(r.stdout.strip())
    assert out[0] == out[1] and len(out[0]) == 64


def test_world_blob_is_passed_in_place():
    # A World's bytearray reaches the library without a copy; bytes are passed as they are.
    import ctypes as C

    from natray_b200.replicas import device_bytes
    from natray_b200.world import blob_arg

    w = build_world(Params(resolution=20, mesh_level=2))
    arg, n = blob_arg(w)
    assert n == len(w.blob)
    assert C.addressof(arg) == C.addressof((C.c_char * n).from_buffer(w.blob))
    raw, n2 = blob_arg(bytes(w.blob))
    assert isinstance(raw, bytes) and n2 == n
    assert device_bytes(w) == device_bytes(bytes(w.blob)) > 0
