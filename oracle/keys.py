"""CPU restatement of the reference's keyframe cache: test infrastructure only (tests/ use it as
the checker of the CUDA keyframe kernels and of the cache's host logic; the product never does).

Follows shaders/keys.wgsl (layout, 21-bit position packing), shaders/pack.wgsl (packing),
shaders/show.wgsl (playback between two keyframes) and src/cache.rs (keyframe sizes, the
keyframe schedule, placement in the pool, the bake loop and the choice of the two keyframes a
time is shown from). numpy float32 arithmetic rounds once per operation, as the WGSL does when
no operation is contracted; `mix(a, b, f)` is a * (1 - f) + b * f, the WGSL definition.

Parity unpinned: the reference has no tests, fixtures or recorded output for its cache, so
this restatement is checked against known answers that follow from the layout itself
(tests/test_keys.py) and against the CUDA kernels on the same inputs.
"""
from __future__ import annotations

import bisect
import math

import numpy as np

F = np.float32
U = np.uint32
KEY_HEAD = 4            # src/cache.rs:20
SPRAY_WORDS = 3         # src/cache.rs:21
Q_LO = np.array([-4.0, -0.5, -4.0], F)  # shaders/keys.wgsl:18
Q_SIZE = F(8.0)         # :19
Q_MAX = F(2097151.0)    # :20
Q_STEP = F(8.0) / F(2097151.0)  # the f32 constant Q_SIZE / Q_MAX of :31
T_END = 1.0             # src/cache.rs:14
PAGE_BYTES = 128 << 20  # :16
PAGES = 16              # :17


def bit_words(n: int) -> int:  # shaders/keys.wgsl:52-54
    return (n + 31) // 32


class Layout:  # shaders/keys.wgsl:38-49
    def __init__(self, np_: int, nv: int, nt: int):
        self.np, self.nv, self.nt = np_, nv, nt
        self.mem_word = KEY_HEAD + 2 * np_
        self.alive_word = KEY_HEAD + 2 * (np_ + nv)
        self.spray_word = self.alive_word + (nt + 31) // 32


def pack_pos(p: np.ndarray, flag: np.ndarray | None = None) -> np.ndarray:
    """shaders/keys.wgsl:22-25: (n, 3) f32 positions -> (n, 2) u32 words."""
    p = np.asarray(p, F).reshape(-1, 3)
    u = (p - Q_LO) / Q_SIZE
    u = np.minimum(np.maximum(u, F(0.0)), F(1.0))
    q = (u * Q_MAX + F(0.5)).astype(U)
    w0 = q[:, 0] | (q[:, 1] << U(21))
    w1 = (q[:, 1] >> U(11)) | (q[:, 2] << U(10))
    if flag is not None:
        w1 = w1 | np.where(np.asarray(flag, bool), U(0x80000000), U(0))
    return np.stack([w0, w1], 1).astype(U)


def unpack_pos(w: np.ndarray) -> np.ndarray:
    """shaders/keys.wgsl:27-32: (n, 2) u32 -> (n, 3) f32."""
    w = np.asarray(w, U).reshape(-1, 2)
    x = w[:, 0] & U(0x1FFFFF)
    y = (w[:, 0] >> U(21)) | ((w[:, 1] & U(0x3FF)) << U(11))
    z = (w[:, 1] >> U(10)) & U(0x1FFFFF)
    return Q_LO + np.stack([x, y, z], 1).astype(F) * Q_STEP


def flagged(w: np.ndarray) -> np.ndarray:
    return (np.asarray(w, U).reshape(-1, 2)[:, 1] >> U(31)) != 0


def bits_of(live: np.ndarray) -> np.ndarray:
    """One bit per element, 32 to a word, bit k of word w for element 32 w + k."""
    live = np.asarray(live, bool)
    n = bit_words(live.size)
    pad = np.zeros(n * 32, np.uint8)
    pad[: live.size] = live
    return np.packbits(pad, bitorder="little").view("<u4").astype(U)


def key_words_count(np_: int, nv: int, nt: int, spray: int, live: int) -> int:
    return KEY_HEAD + 2 * (np_ + nv) + (nt + 31) // 32 + 2 * bit_words(spray) + SPRAY_WORDS * live


def key_bytes(np_: int, nv: int, nt: int, spray: int, live: int) -> int:
    """src/cache.rs:412-421: rounded up to 256 bytes."""
    return (key_words_count(np_, nv, nt, spray, live) * 4 + 255) // 256 * 256


def pack(pos: np.ndarray, vel_w: np.ndarray, mem_pos: np.ndarray, alive: np.ndarray, spray: np.ndarray,
         spray_count: int):
    """A keyframe of the state (shaders/pack.wgsl): water positions (n, 3) with the alive word
    vel.w (n,), membrane positions (nv, 3), triangle alive flags (nt,), the spray slots
    (>= spray_count, 12) f32 and the slot count. Returns (key words, spray weights (n, 2))."""
    np_, nv, nt = len(pos), len(mem_pos), len(alive)
    sp = np.asarray(spray, F).reshape(-1, 12)[:spray_count]
    live = sp[:, 3] > F(0.0)
    n_live = int(live.sum())
    L = Layout(np_, nv, nt)
    out = np.zeros(key_words_count(np_, nv, nt, spray_count, n_live), U)
    out[0], out[1] = spray_count, n_live
    out[KEY_HEAD: L.mem_word] = pack_pos(pos, np.asarray(vel_w, F) > F(0.5)).reshape(-1)  # pack_water :38-44
    out[L.mem_word: L.alive_word] = pack_pos(mem_pos).reshape(-1)  # pack_mem :46-51
    out[L.alive_word: L.spray_word] = bits_of(np.asarray(alive) != 0)  # pack_alive :53-63
    nw = bit_words(spray_count)  # index_bits, index_scan, pack_spray :65-124
    bits = bits_of(live)
    counts = np.bitwise_count(bits).astype(np.int64)
    before = (np.cumsum(counts) - counts).astype(U)
    s0 = L.spray_word
    out[s0: s0 + nw] = bits
    out[s0 + nw: s0 + 2 * nw] = before
    ent = np.zeros((n_live, 3), U)
    ent[:, :2] = pack_pos(sp[live, :3])
    ent[:, 2] = sp[live, 3].view(U)
    out[s0 + 2 * nw:] = ent.reshape(-1)
    spray_w = np.stack([sp[:, 7], sp[:, 11]], 1).astype(F)
    return out, spray_w


def pack_world(world) -> tuple[np.ndarray, np.ndarray]:
    """pack() of a world blob's state (natray_b200.World)."""
    p = world.sec("PARTICLES")
    st = world.state
    n = min(st["spray_count"], world.h.spray_cap)
    return pack(p[:, 0:3], p[:, 7], world.sec("MEM_X")[:, :3], world.sec("ALIVE"), world.sec("SPRAY"), n)


# ---- playback (shaders/show.wgsl) ------------------------------------------------------------------

def mix(a, b, f):
    return a * (F(1.0) - f) + b * f


def spray_slots(key: np.ndarray, L: Layout, m: int) -> np.ndarray:
    """Position and radius of spray slots 0..m-1 of a keyframe, 0 where empty (:28-39)."""
    out = np.zeros((m, 4), F)
    n = int(key[0])
    k = min(n, m)
    if k == 0:
        return out
    nw = bit_words(n)
    i = np.arange(k)
    w = i // 32
    bits = key[L.spray_word + w]
    bit = (U(1) << (i % 32).astype(U)).astype(U)
    live = (bits & bit) != 0
    rank = np.bitwise_count(bits & (bit - U(1))).astype(np.int64)
    base = L.spray_word + 2 * nw + SPRAY_WORDS * (key[L.spray_word + nw + w].astype(np.int64) + rank)
    base = base[live]
    out[i[live], :3] = unpack_pos(np.stack([key[base], key[base + 1]], 1))
    out[i[live], 3] = key[base + 2].view(F)
    return out


def show(ka: np.ndarray, kb: np.ndarray, np_: int, nv: int, nt: int, spray_w: np.ndarray, landed: np.ndarray,
         touch: np.ndarray, t: F, f: F, inv: F, ta: F, tb: F, wet_half: F, wet_res: int) -> dict:
    """The shown buffers for the f32 uniform values the host passes (src/cache.rs:286-289).
    Spray covers slots below max(ka[0], kb[0]), the slots show_spray writes."""
    t, f, inv, ta, tb, h = F(t), F(f), F(inv), F(ta), F(tb), F(wet_half)
    L = Layout(np_, nv, nt)
    out = {}
    # show_water :41-60
    wa = ka[KEY_HEAD: L.mem_word].reshape(-1, 2)
    wb = kb[KEY_HEAD: L.mem_word].reshape(-1, 2)
    pa, pb = unpack_pos(wa), unpack_pos(wb)
    fa, fb = flagged(wa), flagged(wb)
    first = f < F(0.5)
    pos = np.where(first, pa, pb)
    live = np.where(first, fa, fb)
    vel = np.zeros_like(pa)
    both = fa & fb
    pos[both] = mix(pa, pb, f)[both]
    vel[both] = ((pb - pa) * inv)[both]
    P = np.zeros((np_, 8), F)
    P[:, :3], P[:, 3], P[:, 4:7], P[:, 7] = pos, F(1.0), vel, np.where(live, F(1.0), F(0.0))
    out["PARTICLES"] = P
    # show_mem :62-68
    M = np.zeros((nv, 4), F)
    M[:, :3] = mix(unpack_pos(ka[L.mem_word: L.alive_word]), unpack_pos(kb[L.mem_word: L.alive_word]), f)
    out["MEM_POS"] = M
    # show_alive :70-77
    words = (ka if first else kb)[L.alive_word: L.spray_word]
    t_idx = np.arange(nt)
    out["ALIVE"] = ((words[t_idx // 32] >> (t_idx % 32).astype(U)) & U(1)).astype(U)
    # show_spray :79-112
    m = max(int(ka[0]), int(kb[0]))
    sa, sb = spray_slots(ka, L, m), spray_slots(kb, L, m)
    pa, pb, ra, rb = sa[:, :3], sb[:, :3], sa[:, 3], sb[:, 3]
    pos = np.where(first, pa, pb)
    r = np.where(first, ra, rb)
    vel = np.zeros_like(pa)
    l = np.asarray(landed, F).reshape(-1, 4)[:m]
    both = (ra > F(0.0)) & (rb > F(0.0))
    lands = ~both & (ra > F(0.0)) & (l[:, 2] > F(0.0)) & (l[:, 3] <= tb)
    pos[both] = mix(pa, pb, f)[both]
    r[both] = mix(ra, rb, f)[both]
    vel[both] = ((pb - pa) * inv)[both]
    hit = np.stack([l[:, 0], l[:, 2], l[:, 1]], 1)
    span = np.maximum(l[:, 3] - ta, F(1e-9))
    s = np.minimum(np.maximum((t - ta) / span, F(0.0)), F(1.0))
    pos[lands] = mix(pa, hit, s[:, None])[lands]
    r[lands] = np.where(t < l[:, 3], ra, F(0.0))[lands]
    vel[lands] = ((hit - pa) / span[:, None])[lands]
    w = np.asarray(spray_w, F).reshape(-1, 2)[:m]
    S = np.zeros((m, 8), F)
    S[:, :3], S[:, 3], S[:, 4:7], S[:, 7] = pos, r, vel, np.where(t < w[:, 1], -w[:, 0], w[:, 0])
    out["SPRAY"] = S
    # show_wet_drops :114-136, then show_wet_touch :138-146
    res = int(wet_res)
    wet = np.zeros(res * res, U)
    nb = int(kb[0])
    l = np.asarray(landed, F).reshape(-1, 4)[:nb]
    ok = ~(l[:, 2] <= F(0.0)) & ~(l[:, 3] > t)
    l = l[ok]
    cell = (F(2.0) * h) / F(res)
    r = l[:, 2]
    k = np.minimum(np.maximum((F(3.0) * r) / cell, F(0.0)), F(2.0)).astype(np.int32)
    n = ((2 * k + 1) * (2 * k + 1)).astype(F)
    amt = ((((F(4.18879) * r) * r) * r) * F(1e12)) / n
    amount = np.where(amt >= F(4294967296.0), np.uint64(0xFFFFFFFF), amt.astype(np.uint64)).astype(U)
    two_h = F(2.0) * h
    for y in range(-2, 3):
        for x in range(-2, 3):
            sel = (abs(x) <= k) & (abs(y) <= k)
            u = ((l[:, 0] + F(x) * cell) + h) / two_h
            v = ((l[:, 1] + F(y) * cell) + h) / two_h
            sel &= (u >= F(0.0)) & (v >= F(0.0)) & (u < F(1.0)) & (v < F(1.0))
            cx = np.minimum((u[sel] * F(res)).astype(U).astype(np.int64), res - 1)
            cy = np.minimum((v[sel] * F(res)).astype(U).astype(np.int64), res - 1)
            np.add.at(wet, cy * res + cx, amount[sel])
    if not (t < F(0.0)):
        tb_bits = np.array([t], F).view(U)[0]
        soaked = np.asarray(touch, U)[: res * res] <= tb_bits
        wet = np.where(soaked, np.maximum(wet, U(4000000)), wet).astype(U)
    out["WET"] = wet
    return out


def show_select(key_times: list[float], t_start: float, t: float):
    """The host side of show (src/cache.rs:269-290): the time shown (clamped), the two
    keyframes (a, b) and the f32 uniform values (t, f, inv, ta, tb)."""
    end = key_times[-1]
    t = t_start if t < t_start else end if t > end else t
    b = bisect.bisect_right(key_times, t)
    b = min(max(b, 1), len(key_times))
    a = b - 1
    b = min(b, len(key_times) - 1)
    ta, tb = key_times[a], key_times[b]
    if b > a:
        f = min(max((t - ta) / (tb - ta), 0.0), 1.0)
        inv = 1.0 / (tb - ta)
    else:
        f, inv = 0.0, 0.0
    return t, a, b, (F(t), F(f), F(inv), F(ta), F(tb))


# ---- schedule and placement (src/cache.rs:22-46, 231-265) -----------------------------------------

def spacing(tau: float) -> float:
    v = 0.02 * tau
    return 10e-6 if v < 10e-6 else 4e-3 if v > 4e-3 else v


def keys_after(tau: float) -> float:
    a, b = 10e-6 / 0.02, 4e-3 / 0.02
    c = a if tau < a else b if tau > b else tau
    return min(tau, a) / 10e-6 + 50.0 * math.log(c / a) + max(tau - b, 0.0) / 4e-3


def keys_left(t: float, arrivals: list[float], t_end: float = T_END) -> float:
    n = 0.0
    for i, a in enumerate(arrivals):
        end = arrivals[i + 1] if i + 1 < len(arrivals) else t_end
        if end > t:
            n += keys_after(end - a) - keys_after(max(t, a) - a)
    return n


def next_time(t: float, t_hits: list[float], t_end: float, free: int, size: int) -> float:
    arr = sorted(set([max(a, 0.0) for a in t_hits] + [0.0]))
    last = max([a for a in arr if a <= t], default=0.0)
    nxt = min([a for a in arr if a > t], default=t_end)
    overrun = 1.2 * keys_left(t, arr, t_end) * size / free
    return min(min(t + spacing(t - last) * max(overrun, 1.0), nxt), t_end)


class BakeOracle:
    """Cache::restart / bake / store_key (src/cache.rs:161-265) over a natray_b200.Sim, with the
    keyframe's spray counts taken from the simulation's own buffers: the keyframe table
    (time, page, offset, bytes, spray, live) the cache should build."""

    def __init__(self, sim, page_bytes: int = PAGE_BYTES, pages: int = PAGES, t_hits=(0.0,), t_end: float = T_END):
        self.sim, self.page_bytes, self.pages, self.t_hits, self.t_end = sim, page_bytes, pages, list(t_hits), t_end
        i = sim._info()
        self.np, self.nv, self.nt, self.cap = i.n_particles, i.n_verts, i.n_tris, i.spray_cap
        assert key_bytes(self.np, self.nv, self.nt, self.cap, self.cap) <= page_bytes
        sim.advance(0.0, 0)
        self.keys, self.cursor, self.next_t, self.done, self.full = [], (0, 0), 0.0, False, False
        self.store()

    def t(self) -> float:
        return self.sim._info().t

    def end(self) -> float:
        return self.keys[-1]["t"] if self.keys else 0.0

    def store(self) -> None:
        n = min(self.sim.state["spray_count"], self.cap)
        sp = self.sim.download("SPRAY", np.float32, n * 12).reshape(-1, 12)
        live = int((sp[:, 3] > 0).sum())
        size = key_bytes(self.np, self.nv, self.nt, n, live)
        page, off = self.cursor
        if off + size > self.page_bytes:
            page, off = page + 1, 0
        self.cursor = (page, off)
        if page >= self.pages:
            self.full = self.done = True
            return
        t = self.t()
        self.keys.append({"t": t, "page": page, "offset": off, "bytes": size, "spray": n, "live": live})
        self.cursor = (page, off + size)
        if self.next_t >= self.t_end:
            self.done = True
        else:
            used = sum(k["bytes"] for k in self.keys)
            free = max(self.page_bytes * self.pages - used, 0) or 1
            self.next_t = next_time(t, self.t_hits, self.t_end, free, size)

    def bake(self, max_steps: int) -> int:
        steps = 0
        while not self.done and steps < max_steps:
            left = max_steps - steps
            n = self.sim.advance(self.next_t, left)
            steps += n
            if n == left:
                continue
            if self.t() > self.end():
                self.store()
            else:
                steps += self.sim.advance(float("inf"), 1)
        return steps
