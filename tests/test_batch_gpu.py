"""The batch engine (ntr_batch_*): scenes of uneven size stepped together, with one joint
pressure solve per step, give bit for bit the results of each scene stepped alone with the same
chunks of steps, also when scenes arrive and leave while others run (continuous batching)."""
import numpy as np
import pytest

from natray_b200 import Params, World, build_world
from natray_b200.batch import Batch
from natray_b200.sim import Sim
from oracle.py import Oracle

pytestmark = pytest.mark.gpu


def scene(**kw):
    base = dict(resolution=20, mesh_level=3, block_cap=4096, spray_cap=100000)
    base.update(kw)
    w = build_world(Params(**base))
    return World(Oracle(w.blob).snapshot())  # the measuring substep taken once, on the CPU


def solo(w: World, target: int, chunk: int) -> World:
    s = Sim(world=w)
    done = 0
    while done < target:
        done += s.step(min(chunk, target - done))
    out = s.snapshot()
    s.close()
    return out


def first_difference(a: World, b: World):
    from natray_b200._abi import SECTIONS
    if a.state != b.state:
        return "state " + str({k: (a.state[k], b.state[k]) for k in a.state if a.state[k] != b.state[k]})
    for name in SECTIONS:
        x, y = a.sec(name), b.sec(name)
        if x.tobytes() != y.tobytes():
            return f"section {name}"
    if bytes(a.blob) != bytes(b.blob):
        return "header"
    return None


@pytest.fixture(scope="module")
def worlds():
    return [scene(resolution=20), scene(resolution=28, bullet_speed=250), scene(resolution=14, diameter=10)]


def test_batch_equals_each_scene_alone(worlds):
    targets = [12, 8, 16]
    with Batch(max_scenes=4) as b:
        slots = [b.admit(w, t) for w, t in zip(worlds, targets)]
        assert None not in slots
        while b.step(4):
            pass
        for w, t, sl in zip(worlds, targets, slots):
            p = b.poll(sl)
            assert p["finished"] and p["steps_done"] == t
            d = first_difference(solo(w, t, 4), b.snapshot(sl))
            assert d is None, f"slot {sl}: {d}"


def test_uneven_targets_end_as_alone(worlds):
    # Targets that are not multiples of the call's steps: in a scene's last call it takes fewer
    # steps than the others and is parked for the rest of the call; its state is that of the
    # scene alone after the same chunks.
    targets = [10, 6, 13]
    with Batch(max_scenes=4) as b:
        slots = [b.admit(w, t) for w, t in zip(worlds, targets)]
        while b.step(4):
            pass
        for w, t, sl in zip(worlds, targets, slots):
            assert b.poll(sl)["steps_done"] == t
            d = first_difference(solo(w, t, 4), b.snapshot(sl))
            assert d is None, f"slot {sl}: {d}"


def test_scenes_arrive_and_leave(worlds):
    # Two scenes start; a third arrives after two batch steps; the first leaves when done and a
    # fourth takes its slot. Each ends as it would alone.
    w4 = scene(resolution=18, bullet_speed=300)
    with Batch(max_scenes=2) as b:
        s0 = b.admit(worlds[0], 8)
        s1 = b.admit(worlds[1], 16)
        assert b.admit(worlds[2], 8) is None  # both slots taken
        b.step(4)
        b.step(4)
        assert b.poll(s0)["finished"]
        r0 = b.snapshot(s0)
        b.retire(s0)
        s2 = b.admit(worlds[2], 8)
        assert s2 == s0
        b.step(4)
        b.step(4)
        r1, r2 = b.snapshot(s1), b.snapshot(s2)
        b.retire(s1)
        s3 = b.admit(w4, 4)
        b.step(4)
        r3 = b.snapshot(s3)
        info = b.info()
        assert info["in_use"] == 2 and info["active"] == 0
    for w, t, r in [(worlds[0], 8, r0), (worlds[1], 16, r1), (worlds[2], 8, r2), (w4, 4, r3)]:
        d = first_difference(solo(w, t, 4), r)
        assert d is None, d


def test_admission_respects_the_budget(worlds):
    with Batch(max_scenes=4, hbm_budget=1) as b:
        assert b.admit(worlds[0], 4) is None
        assert b.info()["in_use"] == 0


def test_serving_loop_finishes_every_request(worlds):
    from natray_b200.serve import poisson_arrivals, serve
    ws = worlds * 2
    out = serve(ws, poisson_arrivals(len(ws), 200.0, 3), steps=8, chunk=4, max_scenes=3)
    assert out["requests"] == len(ws) and out["p99_s"] >= out["p50_s"] > 0.0


def test_serving_builds_each_scene_on_arrival():
    # The requests are parameters; each scene is built on a host thread when its request
    # arrives, and its latency includes the build.
    from natray_b200.serve import poisson_arrivals, serve
    ps = [Params(resolution=r, mesh_level=3, block_cap=4096, spray_cap=100000) for r in (14, 16, 18, 16)]
    out = serve(ps, poisson_arrivals(len(ps), 100.0, 5), steps=6, chunk=3, max_scenes=2, build=build_world)
    assert out["requests"] == len(ps) and sorted(out["requests_served"]) == list(range(len(ps)))
    assert out["p99_s"] >= out["p50_s"] > 0.0


def test_queue_from_other_threads(worlds):
    # Three host threads queue scenes while the main thread steps the batch (every call takes
    # the batch's lock); each scene is admitted at a step in queue order and ends as it would
    # alone.
    import threading
    with Batch(max_scenes=2) as b:
        tickets = {}

        def submit(k):
            tickets[k] = b.enqueue(worlds[k], 8)

        threads = [threading.Thread(target=submit, args=(k,)) for k in range(3)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        assert sorted(tickets.values()) == [1, 2, 3]
        order = sorted(tickets, key=tickets.get)
        got = {}
        for _ in range(12):
            b.step(4)
            for k in order:
                sl = b.ticket(tickets[k])
                if sl is not None and k not in got and b.poll(sl)["finished"]:
                    got[k] = b.snapshot(sl)
                    b.retire(sl)
            if len(got) == 3:
                break
        assert len(got) == 3
    for k, r in got.items():
        d = first_difference(solo(worlds[k], 8, 4), r)
        assert d is None, f"scene {k}: {d}"


def test_launch_shapes_do_not_change_results(worlds):
    # The same scenes and calls under the default shapes, under odd ones (3 and 5 CTAs an SM,
    # the joint solve on one CTA a scene) and after the autotuner's search: the same bits.
    targets = [12, 8, 16]
    runs = []
    for tuning in (None, {"cell_ctas_per_sm": 3, "block_ctas_per_sm": 5, "solve_ctas": 3}):
        with Batch(max_scenes=4) as b:
            if tuning:
                b.tuning = tuning
                got = b.tuning
                assert (got["cell_ctas_per_sm"], got["block_ctas_per_sm"], got["solve_ctas"]) == (3, 5, 3)
            slots = [b.admit(w, t) for w, t in zip(worlds, targets)]
            while b.step(4):
                pass
            runs.append([b.snapshot(sl) for sl in slots])
    for a, c in zip(*runs):
        assert first_difference(a, c) is None
    with Batch(max_scenes=4) as b:
        slots = [b.admit(w, 200) for w in worlds]
        best, ms = b.autotune(steps=2)
        assert ms > 0 and 1 <= best["cell_ctas_per_sm"] <= 64 and 1 <= best["block_ctas_per_sm"] <= 64
        assert best["solve_ctas"] >= 3 and b.tuning == best
        assert all(b.poll(sl)["steps_done"] == 12 * 3 for sl in slots)  # 12 candidates, 1 + 2 steps each


def test_admission_beside_a_running_step(worlds):
    # One scene steps while another thread admits the other two (ntr_batch_admit lets the
    # step run: it creates the scene outside the batch's lock); every scene still ends as alone.
    import threading
    import time
    targets = [40, 12, 16]
    with Batch(max_scenes=4) as b:
        slots = {0: b.admit(worlds[0], targets[0])}

        def admit_rest():
            for k in (1, 2):
                time.sleep(0.01)
                slots[k] = b.admit(worlds[k], targets[k])

        th = threading.Thread(target=admit_rest)
        th.start()
        while True:
            active = b.step(4)
            if not active and not th.is_alive():
                break
        th.join()
        while b.step(4):
            pass
        for k, (w, t) in enumerate(zip(worlds, targets)):
            p = b.poll(slots[k])
            assert p["finished"] and p["steps_done"] == t
            d = first_difference(solo(w, t, 4), b.snapshot(slots[k]))
            assert d is None, f"scene {k}: {d}"
