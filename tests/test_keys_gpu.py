"""The keyframe cache on the GPU (ntr_cache_*) against the oracle (oracle/keys.py), bit for bit:
keyframes packed from the simulation's state, the shown buffers blended from two keyframes, and
the keyframe table a bake builds (times, pool pages and offsets, sizes, spray counts) against
the reference's bake loop and schedule restated over an identical simulation."""
import numpy as np
import pytest

from natray_b200 import Params, World, build_world
from natray_b200.cache import Cache
from natray_b200.sim import Sim
from oracle import keys as K

pytestmark = pytest.mark.gpu

SCENE = dict(resolution=20, mesh_level=3, block_cap=4096, spray_cap=20000)


@pytest.fixture(scope="module")
def world():
    return build_world(Params(**SCENE))


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a).view(np.uint32)


def step_until_spray(sim: Sim, max_steps: int = 3000) -> int:
    done = 0
    while sim.state["spray_count"] == 0 and done < max_steps:
        done += sim.step(20)
    return done


def test_pack_matches_the_oracle(world):
    with Sim(world=world) as sim, Cache(sim) as c:
        shots = [sim.snapshot()]  # keyframe 0: the start
        step_until_spray(sim)
        for _ in range(3):
            sim.step(15)
            c.store()
            shots.append(sim.snapshot())
        assert shots[-1].state["spray_count"] > 0, "the scene threw no spray"
        for k, w in enumerate(shots):
            want, sw = K.pack_world(w)
            got = c.key_words(k)
            info = c.keys()[k]
            assert (info["spray"], info["live"]) == (int(want[0]), int(want[1]))
            assert info["bytes"] == K.key_bytes(w.h.n_particles, w.h.n_verts, w.h.n_tris, int(want[0]), int(want[1]))
            assert np.array_equal(got[: len(want)], want), f"keyframe {k}: first word differing " \
                f"{int(np.flatnonzero(got[: len(want)] != want)[0])}"
        n = len(sw)
        assert np.array_equal(bits(c.shown("SPRAY_W").reshape(-1, 2)[:n]), bits(sw))


def shown_by_oracle(c: Cache, sim: Sim, w0: World, t: float) -> dict:
    keys = c.keys()
    t_sel, a, b, (tf, f, inv, ta, tb) = K.show_select([k["t"] for k in keys], sim._info().t_start, t)
    ka, kb = c.key_words(a), c.key_words(b)
    i = sim.info
    return K.show(ka, kb, i.n_particles, i.n_verts, i.n_tris, c.shown("SPRAY_W"), sim.download("LANDED", np.float32),
                  sim.download("TOUCH", np.uint32), tf, f, inv, ta, tb, np.float32(w0.h.params.wet[0]), w0.h.wet_res)


def test_show_matches_the_oracle(world):
    with Sim(world=world) as sim, Cache(sim) as c:
        step_until_spray(sim)
        c.bake(120)
        keys = c.keys()
        assert len(keys) >= 4 and keys[-1]["spray"] > 0
        t = [k["t"] for k in keys]
        times = [t[0] - 1.0, t[0], 0.3 * t[1] + 0.7 * t[2], 0.8 * t[-2] + 0.2 * t[-1], t[-2], t[-1] + 1.0]
        for when in times:
            assert c.show(when)
            want = shown_by_oracle(c, sim, world, when)
            m = want["SPRAY"].shape[0]
            got = {"PARTICLES": c.shown("PARTICLES").reshape(-1, 8), "MEM_POS": c.shown("MEM_POS").reshape(-1, 4),
                   "ALIVE": c.shown("ALIVE"), "SPRAY": c.shown("SPRAY").reshape(-1, 8)[:m], "WET": c.shown("WET")}
            for name, g in got.items():
                assert np.array_equal(bits(g), bits(want[name])), f"t={when}: {name}"
        assert not c.show(times[-1])  # the same time again: nothing to do
        assert c.info["shown_spray"] == max(keys[-2]["spray"], keys[-1]["spray"])


def test_bake_builds_the_reference_keyframe_table(world):
    h = world.h
    page = K.key_bytes(h.n_particles, h.n_verts, h.n_tris, h.spray_cap, h.spray_cap)
    kw = dict(page_bytes=page, pages=3, t_hits=[0.0])
    # Batches of a fixed length on both sides: with the default, batches end where 4 ms of the
    # measured step time does, and the host's adaptation between batches changes the results.
    s1 = Sim(world=world)
    s1.set_batch_steps(8)
    with s1, Cache(s1, page_bytes=page, pages=3, arrivals=[0.0]) as c:
        steps = c.bake(400)
        got, info = c.keys(), c.info
    with Sim(world=world) as s2:
        s2.set_batch_steps(8)
        o = K.BakeOracle(s2, **kw)
        want_steps = o.bake(400)
    assert steps == want_steps
    assert len(got) == len(o.keys) and len(got) > 3
    for g, w in zip(got, o.keys):
        assert g == w
    assert (bool(info["done"]), bool(info["full"])) == (o.done, o.full)
    assert info["next_t"] == o.next_t
    assert len({k["page"] for k in got}) > 1  # keyframes filled more than one page


def test_a_full_pool_ends_the_timeline(world):
    h = world.h
    page = K.key_bytes(h.n_particles, h.n_verts, h.n_tris, h.spray_cap, h.spray_cap)
    with Sim(world=world) as sim, Cache(sim, page_bytes=page, pages=1, arrivals=[0.0]) as c:
        c.bake(100000)
        info = c.info
        assert info["full"] and info["done"]
        assert info["used_bytes"] <= page
        assert c.bake(10) == 0


def test_rebuild_starts_over(world):
    with Sim(world=world) as s1, Sim(world=world) as s2, Cache(s1) as c:
        c.bake(60)
        assert c.info["keys"] > 1
        c.show(c.end())
        c.rebuild(s2)
        info = c.info
        assert info["keys"] == 1 and info["shown"] != info["shown"]  # NaN: nothing shown yet
        w = s2.snapshot()
        want, _ = K.pack_world(w)
        assert np.array_equal(c.key_words(0)[: len(want)], want)
