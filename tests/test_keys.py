"""Keyframe cache on the CPU: the oracle's packing and playback against answers that follow from
the keyframe layout (shaders/keys.wgsl:1-10), and the library's host functions (keyframe sizes,
the keyframe schedule of src/cache.rs:22-46 and 249-264, the shots' arrival times) against the
oracle's restatement, bit for bit."""
import ctypes as C
import math

import numpy as np

from natray_b200 import Params, _abi
from natray_b200._abi import lib
from natray_b200.cache import cache_params, key_bytes, key_next_time
from oracle import keys as K

F = np.float32


def test_pack_pos_known_answers():
    p = np.array([[-4.0, -0.5, -4.0], [4.0, 7.5, 4.0], [-9.0, -3.0, 9.0], [0.0, 3.5, 0.0]], F)
    w = K.pack_pos(p, np.array([True, False, True, False]))
    assert w[0].tolist() == [0, 0x80000000]  # the low corner, flagged
    assert w[1].tolist() == [0xFFFFFFFF, 0x7FFFFFFF]  # the high corner: 21 ones per axis
    assert w[2].tolist() == [0, 0x7FFFFC00 | 0x80000000]  # clamped to (lo, lo, hi)
    q = (F(0.5) * K.Q_MAX + F(0.5)).astype(np.uint32)  # the centre: 1048576 steps per axis
    assert w[3].tolist() == [int(q) | ((int(q) << 21) & 0xFFFFFFFF), (int(q) >> 11) | (int(q) << 10)]
    assert K.flagged(w).tolist() == [True, False, True, False]


def test_unpack_round_trip_within_half_a_step():
    rng = np.random.default_rng(7)
    p = (rng.random((20000, 3)) * np.array([8.0, 8.0, 8.0]) + np.array([-4.0, -0.5, -4.0])).astype(F)
    back = K.unpack_pos(K.pack_pos(p))
    assert np.abs(back - p).max() <= 0.5 * float(K.Q_STEP) * 1.001 + 1e-6
    again = K.pack_pos(back)
    assert np.array_equal(again, K.pack_pos(p))  # packing is idempotent on unpacked positions


def test_pack_layout():
    rng = np.random.default_rng(3)
    n, nv, nt, ns = 100, 40, 70, 77
    pos = rng.random((n, 3)).astype(F)
    vel_w = (rng.random(n) > 0.3).astype(F)
    mem = rng.random((nv, 3)).astype(F)
    alive = (rng.random(nt) > 0.2).astype(np.uint32)
    spray = rng.random((ns, 12)).astype(F)
    spray[rng.random(ns) > 0.5, 3] = 0.0
    words, w = K.pack(pos, vel_w, mem, alive, spray, ns)
    live = spray[:, 3] > 0
    L = K.Layout(n, nv, nt)
    assert words[:4].tolist() == [ns, int(live.sum()), 0, 0]
    assert len(words) == K.key_words_count(n, nv, nt, ns, int(live.sum()))
    for t in range(nt):
        assert ((words[L.alive_word + t // 32] >> (t % 32)) & 1) == alive[t]
    nw = K.bit_words(ns)
    run = 0
    for j in range(nw):
        assert words[L.spray_word + nw + j] == run
        run += bin(int(words[L.spray_word + j])).count("1")
    back = K.spray_slots(words, L, ns)
    assert np.array_equal(back[:, 3], np.where(live, spray[:, 3], 0.0).astype(F))
    assert np.abs(back[live, :3] - spray[live, :3]).max() <= float(K.Q_STEP)
    assert np.array_equal(w, spray[:, [7, 11]])


def test_show_between_equal_keys_is_the_key():
    rng = np.random.default_rng(5)
    n, nv, nt = 64, 16, 40
    pos = rng.random((n, 3)).astype(F)
    words, w = K.pack(pos, np.ones(n, F), rng.random((nv, 3)).astype(F), np.ones(nt, np.uint32), np.zeros((0, 12), F), 0)
    out = K.show(words, words, n, nv, nt, w, np.zeros((0, 4), F), np.full(16, 0xFFFFFFFF, np.uint32),
                 F(0.1), F(0.3), F(100.0), F(0.0), F(0.2), F(1.2), 4)
    assert np.array_equal(out["PARTICLES"][:, :3], K.unpack_pos(words[4: 4 + 2 * n]))
    assert not out["PARTICLES"][:, 4:7].any() and (out["PARTICLES"][:, 7] == 1).all()
    assert (out["ALIVE"] == 1).all() and not out["WET"].any()


def test_show_select_clamps_and_brackets():
    ts = [0.0, 1e-5, 3e-5]
    assert K.show_select(ts, -1.0, -5.0)[:3] == (-1.0, 0, 1)
    t, a, b, u = K.show_select(ts, -1.0, 2e-5)
    assert (a, b) == (1, 2) and u[1] == F(0.5)
    t, a, b, u = K.show_select(ts, -1.0, 9.0)
    assert (t, a, b) == (3e-5, 2, 2) and u[1] == 0.0 and u[2] == 0.0


def test_key_bytes_match_the_oracle():
    rng = np.random.default_rng(11)
    for _ in range(200):
        a = [int(x) for x in rng.integers(0, 2_000_000, 5)]
        a[4] = min(a[4], a[3])
        assert key_bytes(*a) == K.key_bytes(*a)
    assert key_bytes(0, 0, 0, 0, 0) == 256


def test_schedule_matches_the_oracle():
    rng = np.random.default_rng(13)
    for _ in range(500):
        hits = [float(x) for x in rng.choice([0.0, 1e-4, 2e-3, 0.05, 0.3, -1e-3], rng.integers(0, 4))]
        t = float(rng.choice([0.0, 5e-6, 3e-4, 0.01, 0.2, 0.7, 0.999, 1.2])) * float(rng.random() + 0.5)
        free = int(rng.integers(1, 1 << 31))
        size = int(rng.integers(256, 1 << 26))
        got = key_next_time(t, hits, 1.0, free, size)
        want = K.next_time(t, hits, 1.0, free, size)
        assert got == want or (math.isnan(got) and math.isnan(want)), (t, hits, free, size, got, want)
    assert K.spacing(0.0) == 10e-6 and K.spacing(10.0) == 4e-3
    assert K.keys_after(0.0) == 0.0


def test_arrivals_follow_the_shots():
    p = Params()
    p.c.n_shots = 3
    for k, d in enumerate([5.0, 2.5, 7.25]):
        p.c.shots[k].delay_ms = d
    cp = cache_params(p)
    assert cp.n_arrivals == 3 and cp.pages == 16 and cp.page_bytes == 128 << 20 and cp.t_end == 1.0
    want = [float(F(d) - F(2.5)) * 1e-3 for d in [5.0, 2.5, 7.25]]
    assert list(cp.arrivals)[:3] == want


def test_cache_calls_reject_null_handles():
    h = C.c_void_p()
    cp = cache_params()
    assert lib().ntr_cache_create(None, C.byref(cp), C.byref(h)) == 1  # NTR_E_INVALID
    assert lib().ntr_cache_destroy(None) == 0
    info = _abi.CacheInfo()
    assert lib().ntr_cache_info_get(None, C.byref(info)) == 1
    assert lib().ntr_cache_show(None, 0.0, None) == 1


def test_struct_sizes():
    assert C.sizeof(_abi.CacheParams) == 56 and C.sizeof(_abi.KeyInfo) == 40 and C.sizeof(_abi.CacheInfo) == 64
