"""ntr_sim_stats: the reference's debug statistics (src/sim.rs:691-863) computed on the device,
against the same quantities computed here with numpy, the reference's way, from the
simulation's state read back (its snapshot and its grid). Counts, minima, maxima and which
particle or triangle is picked are exact; FP64 sums agree to their rounding."""
import numpy as np
import pytest

from natray_b200 import Params, build_world
from natray_b200.sim import Sim, format_stats

pytestmark = pytest.mark.gpu
F = np.float32


@pytest.fixture(scope="module")
def run():
    w0 = build_world(Params(resolution=28, mesh_level=3, block_cap=4096, spray_cap=100000))
    sim = Sim(world=w0)
    done = 0
    while sim.state["spray_count"] == 0 and done < 3000:  # through the impact
        done += sim.step(20)
    sim.step(10)
    stats = sim.stats()
    yield sim, sim.snapshot(), sim.grid(), stats
    sim.close()


def test_water(run):
    sim, w, g, s = run
    p = w.sec("PARTICLES")
    live = p[:, 7] > F(0.5)
    x, v = p[live, 0:3], p[live, 4:7]
    assert s["water"] == int(live.sum()) > 0 and s["n_particles"] == len(p)
    assert np.array_equal(np.array(s["lo"], F), x.min(0)) and np.array_equal(np.array(s["hi"], F), x.max(0))
    assert np.allclose(s["mean"], x.astype(np.float64).sum(0) / len(x), rtol=1e-12, atol=1e-15)
    assert np.allclose(s["vmean"], v.astype(np.float64).sum(0) / len(x), rtol=1e-9, atol=1e-12)
    lsq = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]
    speed = np.sqrt(lsq)
    ke = (0.5 * lsq.astype(np.float64)).sum()
    assert s["vmax"] == speed.max()
    assert np.array_equal(np.array(s["fastest"], F), x[int(np.argmax(speed))])
    h = w.h
    dx = h.dx
    assert np.isclose(s["water_j"], ke * 1000.0 * (0.5 * dx) ** 3, rtol=1e-12)
    # cells holding 4 or more particles (floor((x - origin) / h) in f32, as the reference)
    org = np.array(h.params.origin[:3], F)
    c = np.floor((x - org) / F(h.params.origin[3])).astype(np.int64)
    _, counts = np.unique(c, axis=0, return_counts=True)
    assert np.isclose(s["volume_l"], (counts >= 4).sum() * dx ** 3 * 1e3, rtol=1e-12)


def test_rubber(run):
    sim, w, g, s = run
    mx = w.sec("MEM_X")[:, :3]
    mw, mm, mv = w.sec("MEM_WATER"), w.sec("MEM_MASS"), w.sec("MEM_V")[:, :3]
    alive = w.sec("ALIVE")
    tris = w.sec("TRIS")
    idx = tris[:, :3].astype(np.int64)
    a, b, c = (mx[idx[:, k]].astype(np.float64) for k in range(3))
    inside = (a * np.cross(b, c)).sum(1) / 6.0
    assert np.isclose(s["inside_l"], inside.sum() * 1e3, rtol=1e-9)
    assert s["torn"] == int((alive == 0).sum())
    free = mm > 0.0
    fill = mw[free, 3]
    assert s["free_verts"] == int(free.sum()) and s["on_water"] == int((fill >= F(0.05)).sum())
    assert s["fill_min"] == fill.min() and np.isclose(s["fill_mean"], fill.astype(np.float64).mean(), rtol=1e-6)
    assert np.array_equal(np.array(s["mem_lo"], F), mx.min(0)) and np.array_equal(np.array(s["mem_hi"], F), mx.max(0))
    rv = np.sqrt((mv[:, 0] * mv[:, 0] + mv[:, 1] * mv[:, 1]) + mv[:, 2] * mv[:, 2])
    assert s["rubber_vmax"] == rv.max()
    # the most tense intact triangles: Ogden (alpha 1.3, 5, -2) with the moduli the step uses
    mu = np.array(w.h.params.rubber[:3], np.float64)
    thick = float(w.h.params.rubber[3])
    dm = tris[:, 4:8].view(np.float32).astype(np.float64)
    e1, e2 = b - a, c - a
    f0 = e1 * dm[:, 0:1] + e2 * dm[:, 2:3]
    f1 = e1 * dm[:, 1:2] + e2 * dm[:, 3:4]
    c00, c01, c11 = (f0 * f0).sum(1), (f0 * f1).sum(1), (f1 * f1).sum(1)
    mid = 0.5 * (c00 + c11)
    dev = np.sqrt(0.25 * (c00 - c11) ** 2 + c01 * c01)
    l1, l2 = np.sqrt(mid + dev), np.sqrt(np.maximum(mid - dev, 0.0))
    al = np.array([1.3, 5.0, -2.0])
    sig = lambda p, q: sum(mu[i] * (p ** al[i] - q ** al[i]) for i in range(3))
    nat = l1 ** -0.5
    s1 = np.where(l1 <= 1.0, 0.0, np.where(l2 < nat, sig(l1, nat), sig(l1, 1.0 / (l1 * l2))))
    ten = s1 * thick / np.maximum(l1 * l2, 1e-9)
    order = [t for t in np.argsort(-ten, kind="stable") if alive[t] != 0][:3]
    assert s["n_tension"] == 3 and s["tension_tri"] == [int(t) for t in order]
    assert np.allclose(s["tension"], ten[order], rtol=1e-9)
    assert np.allclose(np.array(s["stretch"]), np.stack([l1[order], l2[order]], 1), rtol=1e-6)


def test_air_and_bullets(run):
    sim, w, g, s = run
    cells = len(g["block_list"]) * 64
    ty = g["cf"].reshape(11, cells)[10]
    air = g["air"].reshape(5, cells)
    sel = ty == 0.0
    rho, m, e = air[0, sel], air[1:4, sel], air[4, sel]
    lsq = (m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]
    p = F(0.4) * (e - F(0.5) * lsq / rho) - F(101325.0)
    assert s["air_cells"] == int(sel.sum()) > 0 and s["vapour_cells"] == int((p < F(-90e3)).sum())
    assert s["gauge_lo"] == p.min() and s["gauge_hi"] == p.max() and s["air_umax"] == (np.sqrt(lsq) / rho).max()
    assert np.isclose(s["vapour_cm3"], s["vapour_cells"] * w.h.dx ** 3 * 1e6, rtol=1e-12)
    bl = w.sec("BULLETS")
    assert len(s["bullets"]) == 1
    v = bl[0, 4:7].astype(np.float64)
    assert np.isclose(s["bullets"][0]["speed"], np.linalg.norm(v), rtol=1e-6)
    assert np.isclose(s["bullets_j"], 0.5 * float(bl[0, 3]) * float((bl[0, 4:7] ** 2).sum()), rtol=1e-6)
    text = format_stats(sim)
    assert text.startswith("t=") and "rubber: inside" in text and "bullet 0:" in text and "air:" in text
