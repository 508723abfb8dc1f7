"""The bullet's flight through the air to the balloon (the reference's Flight::new,
src/flight.rs:404-471), which sets where and how the simulation takes each bullet over. CPU
only. Pinned by the reference's own test of it (src/flight.rs:905-919, the air part: every
preset arrives within 2 m/s of its speed and rifled bullets are gyroscopically stable; a rifle
bullet fired without spin is tumbling by the time it arrives), and by what the hand-over must
satisfy by construction."""
import math

import numpy as np
import pytest

from natray_b200 import Params
from natray_b200.world import flights

SPEEDS = [330.0, 360.0, 255.0, 940.0, 860.0, 240.0, 150.0]  # src/params.rs:193-201
TWIST = [16.0, 10.0, 16.0, 7.0, 10.0, 16.0, 0.0]


def one(k: int, **kw) -> dict:
    return flights(Params(bullet=k, **kw))[0]


@pytest.mark.parametrize("k", range(7))
def test_presets_arrive_at_their_speed(k):
    f = one(k)
    assert abs(f["v_impact"] - SPEEDS[k]) < 2.0
    assert f["sg_air"] > 1.0 or TWIST[k] == 0.0


def test_no_spin_tumbles_before_it_arrives():
    assert one(3, spin=0)["yaw_impact_deg"] > 10.0
    assert one(3)["yaw_impact_deg"] < 10.0


@pytest.mark.parametrize("k", [0, 3, 6])
def test_hand_over_is_lookahead_short_of_the_balloon(k):
    # The tip at the hand-over lies 5 cm before the plane where it meets the balloon, about
    # 5 cm / v before the arrival, travelling along the line of fire.
    f = one(k)
    u = np.array(f["u"])
    v = np.linalg.norm(u)
    assert abs(v - SPEEDS[k]) < 3.0
    assert 0.05 / v * 0.98 < f["t_hit"] - f["t_read"] < 0.05 / v * 1.02
    assert u[0] > 0.999 * v  # azimuth 0, elevation 0: along +x
    n = np.array(f["n"])
    assert abs(np.linalg.norm(n) - 1.0) < 1e-12


def test_range_and_yaw_change_the_launch_not_the_arrival():
    a, b = one(1), one(1, range=40, yaw=2.0)
    assert abs(a["v_impact"] - b["v_impact"]) < 2.0
    assert np.linalg.norm(np.array(b["muzzle_u"])) > np.linalg.norm(np.array(a["muzzle_u"]))  # more drag to make up
    assert b["muzzle_x"][0] < a["muzzle_x"][0] - 25.0


def test_shots_arrive_in_delay_order():
    p = Params(bullet=1)
    p.set("shots", 2)
    p.c.shots[1] = p.c.shots[0]
    p.c.shots[1].delay_ms = 3.0
    f = flights(p)
    assert len(f) == 2 and f[0]["t_hit"] == 0.0 and math.isclose(f[1]["t_hit"], 3e-3, rel_tol=1e-6)
