// Keyframe cache (include/natray.h, ntr_cache_*): `Cache` of src/cache.rs with the keyframe
// layout of shaders/keys.wgsl, the packing of shaders/pack.wgsl and the playback of
// shaders/show.wgsl.
//
// Storing a keyframe is two launches on the simulation's stream and one 8-byte read back:
// k_key_index (live spray slots per tile of 256, from one warp ballot per 32 slots; the CTA
// that finishes last scans the tiles and writes the slot and live counts), the read back that
// sizes and places the keyframe, then k_key_pack, one launch whose CTA ranges pack
// the water particles, the membrane vertices, the triangles' alive bits (a ballot per 32) and
// the spray (bits, per-word prefixes and the live slots' words). Showing one is a clear of the
// wet map, k_key_drops (the landed drops' additions, when key b has spray) and k_key_show
// (ranges for water, vertices, triangles, spray and the ground touch, a max over the drops'
// sums, so after them).
//
// Every float operation is written as the reference's expression with one rounding per
// operation (no contraction; this file is built with -fmad=false): `mix(a, b, f)` is
// a * (1 - f) + b * f, the definition the WGSL specification gives.
//
// Included at the end of sim.cu (it uses the Sim internals there).
#pragma once

#include <cmath>
#include <limits>

namespace ntr {

constexpr uint32_t KEY_HEAD = NTR_KEY_HEAD, KEY_SPRAY_WORDS = NTR_KEY_SPRAY_WORDS;
constexpr float Q_SIZE = 8.0f, Q_MAX = 2097151.0f;
constexpr float Q_STEP = Q_SIZE / Q_MAX;  // the WGSL constant Q_SIZE / Q_MAX, one f32 division
constexpr uint32_t KEY_T = 256;           // threads per CTA of the keyframe kernels
constexpr uint32_t KEY_TILE = 256;        // spray slots per tile (8 words of live bits)
constexpr uint32_t KEY_PER = 4;           // water particles per thread in the pack and show kernels

// Word offsets of a keyframe's parts (shaders/keys.wgsl:38-54).
struct KeyLayout {
    uint32_t np, nv, nt;
    __host__ __device__ uint32_t mem_word() const { return KEY_HEAD + 2u * np; }
    __host__ __device__ uint32_t alive_word() const { return KEY_HEAD + 2u * (np + nv); }
    __host__ __device__ uint32_t spray_word() const { return alive_word() + (nt + 31u) / 32u; }
};
__host__ __device__ __forceinline__ uint32_t bit_words(uint32_t n) { return (n + 31u) / 32u; }

// One axis of pack_pos (shaders/keys.wgsl:22-25): clamp((p - lo) / 8, 0, 1) * Q_MAX + 0.5,
// truncated.
__device__ __forceinline__ uint32_t q_axis(float p, float lo) {
    float u = __fdiv_rn(__fsub_rn(p, lo), Q_SIZE);
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    return __float2uint_rz(__fadd_rn(__fmul_rn(u, Q_MAX), 0.5f));
}

__device__ __forceinline__ uint2 pack_pos(float x, float y, float z, bool flag) {
    const uint32_t qx = q_axis(x, -4.0f), qy = q_axis(y, -0.5f), qz = q_axis(z, -4.0f);
    return make_uint2(qx | (qy << 21), (qy >> 11) | (qz << 10) | (flag ? 0x80000000u : 0u));
}

// unpack_pos (shaders/keys.wgsl:27-32): lo + f32(q) * (Q_SIZE / Q_MAX).
__device__ __forceinline__ V3 unpack_pos(uint2 w) {
    const uint32_t x = w.x & 0x1fffffu, y = (w.x >> 21) | ((w.y & 0x3ffu) << 11), z = (w.y >> 10) & 0x1fffffu;
    return {__fadd_rn(-4.0f, __fmul_rn((float)x, Q_STEP)), __fadd_rn(-0.5f, __fmul_rn((float)y, Q_STEP)),
            __fadd_rn(-4.0f, __fmul_rn((float)z, Q_STEP))};
}

__device__ __forceinline__ bool flagged(uint2 w) { return (w.y >> 31) != 0u; }

__device__ __forceinline__ float mixf(float a, float b, float f) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, f)), __fmul_rn(b, f));
}
__device__ __forceinline__ V3 mix3(V3 a, V3 b, float f) { return {mixf(a.x, b.x, f), mixf(a.y, b.y, f), mixf(a.z, b.z, f)}; }

// ---- storing ------------------------------------------------------------------------------------

// The live spray index: live slots (radius > 0) of the first n = min(spray_count, spray_cap)
// counted per tile of KEY_TILE slots (one ballot per 32), then, in the CTA that finishes last
// (a counter taken after a fence; no CTA waits for another), the tiles' exclusive prefix and
// counts = {n, live}. The live bits themselves are taken again by k_key_pack from the same data.
// counts[2] is the finish counter: zero before the launch, zero again after it.
__global__ void __launch_bounds__(KEY_T) k_key_index(Dev D, uint32_t* tile_tot, uint32_t* tile_pre, uint32_t* counts) {
    __shared__ uint32_t s_w[KEY_T / 32];
    __shared__ uint32_t s_last;
    const uint32_t n = min(D.st->s.spray_count, D.spray_cap);
    const uint32_t nt = (n + KEY_TILE - 1) / KEY_TILE;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t t = blockIdx.x; t < nt; t += gridDim.x) {
        const uint32_t i = t * KEY_TILE + threadIdx.x;
        const bool live = i < n && D.spray[3 * (size_t)i].w > 0.0f;
        const uint32_t bits = __ballot_sync(0xffffffffu, live);
        if (lane == 0) s_w[warp] = __popc(bits);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t sum = 0;
            for (uint32_t w = 0; w < KEY_T / 32; w++) sum += s_w[w];
            tile_tot[t] = sum;
        }
        __syncthreads();
    }
    __threadfence();
    if (threadIdx.x == 0) s_last = atomicAdd(counts + 2, 1u) == gridDim.x - 1u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nt; base += KEY_T) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nt ? __ldcg(tile_tot + i) : 0u;
        uint32_t total;
        const uint32_t ex = cta_scan256(v, &total);
        if (i < nt) tile_pre[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) {
        counts[0] = n;
        counts[1] = carry;
        counts[2] = 0u;
    }
}

// CTA ranges of k_key_pack: [0, b_mem) particles (KEY_PER a thread), [b_mem, b_alive) vertices, [b_alive, b_spray)
// alive words (a warp per word), [b_spray, b_end) spray tiles.
struct PackRanges {
    uint32_t b_mem, b_alive, b_spray, b_end;
    uint32_t n, live;  // spray slots, live ones
};

__global__ void __launch_bounds__(KEY_T) k_key_pack(Dev D, uint32_t* __restrict__ key, float2* __restrict__ spray_w,
                                                    const uint32_t* __restrict__ tile_pre, PackRanges R) {
    const KeyLayout K{D.Np, D.Nv, D.Nt};
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t b = blockIdx.x;
    if (b == 0 && threadIdx.x < KEY_HEAD) key[threadIdx.x] = threadIdx.x == 0 ? R.n : threadIdx.x == 1 ? R.live : 0u;
    if (b < R.b_mem) {  // pack_water (shaders/pack.wgsl:38-44), KEY_PER particles a thread
        const uint32_t i0 = b * KEY_T * KEY_PER + threadIdx.x;
        float4 p[KEY_PER];
        float alive[KEY_PER];
#pragma unroll
        for (uint32_t k = 0; k < KEY_PER; k++) {  // every load first: KEY_PER in flight
            const uint32_t i = i0 + k * KEY_T;
            p[k] = i < D.Np ? D.pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            alive[k] = i < D.Np ? D.vel[i].w : 0.f;
        }
#pragma unroll
        for (uint32_t k = 0; k < KEY_PER; k++) {
            const uint32_t i = i0 + k * KEY_T;
            if (i < D.Np) reinterpret_cast<uint2*>(key + KEY_HEAD)[i] = pack_pos(p[k].x, p[k].y, p[k].z, alive[k] > 0.5f);
        }
        return;
    }
    if (b < R.b_alive) {  // pack_mem (:46-51)
        const uint32_t i = (b - R.b_mem) * KEY_T + threadIdx.x;
        if (i >= D.Nv) return;
        const float4 p = D.mem_x[0][i];
        reinterpret_cast<uint2*>(key + K.mem_word())[i] = pack_pos(p.x, p.y, p.z, false);
        return;
    }
    if (b < R.b_spray) {  // pack_alive (:53-63), one warp per word
        const uint32_t w = (b - R.b_alive) * (KEY_T / 32) + warp;
        if (w * 32u >= D.Nt) return;
        const uint32_t t = w * 32u + lane;
        const uint32_t bits = __ballot_sync(0xffffffffu, t < D.Nt && D.alive[t] != 0u);
        if (lane == 0) key[K.alive_word() + w] = bits;
        return;
    }
    // pack_spray (:106-124): tile of KEY_TILE slots, a warp per word of live bits.
    __shared__ uint32_t s_cnt[KEY_T / 32];
    const uint32_t tile = b - R.b_spray;
    const uint32_t wd = tile * (KEY_TILE / 32) + warp;
    const uint32_t i = wd * 32u + lane;
    const uint32_t nw = bit_words(R.n);
    const bool in = i < R.n;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
    float ww = 0.f, wt = 0.f;
    if (in) {
        p = D.spray[3 * (size_t)i];
        ww = D.spray[3 * (size_t)i + 1].w;
        wt = D.spray[3 * (size_t)i + 2].w;
    }
    const uint32_t bits = __ballot_sync(0xffffffffu, in && p.w > 0.0f);
    if (lane == 0) s_cnt[warp] = __popc(bits);
    __syncthreads();
    uint32_t before = tile_pre[tile];
    for (uint32_t v = 0; v < warp; v++) before += s_cnt[v];
    if (!in) return;
    const uint32_t sw = K.spray_word();
    if (lane == 0) {
        key[sw + wd] = bits;
        key[sw + nw + wd] = before;
    }
    // A slot keeps its weight and tear time for life: the latest values serve every keyframe.
    spray_w[i] = make_float2(ww, wt);
    if (!(bits & (1u << lane))) return;
    const uint32_t base = sw + 2u * nw + KEY_SPRAY_WORDS * (before + __popc(bits & ((1u << lane) - 1u)));
    const uint2 q = pack_pos(p.x, p.y, p.z, false);
    key[base] = q.x;
    key[base + 1] = q.y;
    key[base + 2] = __float_as_uint(p.w);
}

// ---- showing ------------------------------------------------------------------------------------

// The uniform of shaders/show.wgsl (`CacheU`, src/cache.rs:48-54), as the host fills it.
struct ShowArgs {
    const uint32_t* ka;
    const uint32_t* kb;
    const float2* spray_w;
    float4* out_p;
    float4* out_spray;
    float4* out_mem;
    uint32_t* out_alive;
    uint32_t* out_wet;
    float t, f, inv, ta, tb;  // shown time, blend towards b, 1 / (tb - ta), key times (f32)
    float wet_half;
    uint32_t wet_res;
    uint32_t b_mem, b_alive, b_spray, b_drops, b_end;  // CTA ranges
};

// Position and radius of spray slot i in a keyframe, radius 0 where the slot is empty
// (shaders/show.wgsl:28-39).
__device__ __forceinline__ float4 spray_slot(const uint32_t* key, const KeyLayout& K, uint32_t i) {
    const uint32_t n = key[0];
    if (i >= n) return make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t nw = bit_words(n), w = i / 32u, sw = K.spray_word();
    const uint32_t bits = key[sw + w];
    const uint32_t bit = 1u << (i % 32u);
    if (!(bits & bit)) return make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t base = sw + 2u * nw + KEY_SPRAY_WORDS * (key[sw + nw + w] + __popc(bits & (bit - 1u)));
    const V3 p = unpack_pos(make_uint2(key[base], key[base + 1]));
    return make_float4(p.x, p.y, p.z, __uint_as_float(key[base + 2]));
}

__device__ __forceinline__ void show_water_one(const ShowArgs& A, uint32_t i, uint2 wa, uint2 wb) {
    const V3 pa = unpack_pos(wa), pb = unpack_pos(wb);
    V3 pos = A.f < 0.5f ? pa : pb;
    const bool live = A.f < 0.5f ? flagged(wa) : flagged(wb);
    V3 vel{0.f, 0.f, 0.f};
    if (flagged(wa) && flagged(wb)) {
        pos = mix3(pa, pb, A.f);
        vel = {__fmul_rn(__fsub_rn(pb.x, pa.x), A.inv), __fmul_rn(__fsub_rn(pb.y, pa.y), A.inv),
               __fmul_rn(__fsub_rn(pb.z, pa.z), A.inv)};
    }
    A.out_p[2 * (size_t)i] = make_float4(pos.x, pos.y, pos.z, 1.0f);
    A.out_p[2 * (size_t)i + 1] = make_float4(vel.x, vel.y, vel.z, live ? 1.0f : 0.0f);
}

// CTA ranges: [0, b_mem) water (KEY_PER particles a thread), [b_mem, b_alive) vertices,
// [b_alive, b_spray) triangles, [b_spray, b_drops) spray slots, [b_drops, b_end) wet-map cells
// (the ground touch, after k_key_drops has added the landed drops).
__global__ void __launch_bounds__(KEY_T) k_key_show(Dev D, ShowArgs A) {
    const KeyLayout K{D.Np, D.Nv, D.Nt};
    const uint32_t b = blockIdx.x;
    if (b < A.b_mem) {  // show_water (shaders/show.wgsl:41-60)
        const uint32_t i0 = b * KEY_T * KEY_PER + threadIdx.x;
        uint2 wa[KEY_PER], wb[KEY_PER];
#pragma unroll
        for (uint32_t k = 0; k < KEY_PER; k++) {  // every load first
            const uint32_t i = i0 + k * KEY_T;
            wa[k] = i < D.Np ? reinterpret_cast<const uint2*>(A.ka + KEY_HEAD)[i] : make_uint2(0u, 0u);
            wb[k] = i < D.Np ? reinterpret_cast<const uint2*>(A.kb + KEY_HEAD)[i] : make_uint2(0u, 0u);
        }
#pragma unroll
        for (uint32_t k = 0; k < KEY_PER; k++) {
            const uint32_t i = i0 + k * KEY_T;
            if (i < D.Np) show_water_one(A, i, wa[k], wb[k]);
        }
        return;
    }
    if (b < A.b_alive) {  // show_mem (:62-68)
        const uint32_t i = (b - A.b_mem) * KEY_T + threadIdx.x;
        if (i >= D.Nv) return;
        const uint2 wa = reinterpret_cast<const uint2*>(A.ka + K.mem_word())[i];
        const uint2 wb = reinterpret_cast<const uint2*>(A.kb + K.mem_word())[i];
        const V3 p = mix3(unpack_pos(wa), unpack_pos(wb), A.f);
        A.out_mem[i] = make_float4(p.x, p.y, p.z, 0.0f);
        return;
    }
    if (b < A.b_spray) {  // show_alive (:70-77)
        const uint32_t t = (b - A.b_alive) * KEY_T + threadIdx.x;
        if (t >= D.Nt) return;
        const uint32_t w = K.alive_word() + t / 32u;
        const uint32_t bits = A.f < 0.5f ? A.ka[w] : A.kb[w];
        A.out_alive[t] = (bits >> (t % 32u)) & 1u;
        return;
    }
    if (b < A.b_drops) {  // show_spray (:79-112)
        const uint32_t i = (b - A.b_spray) * KEY_T + threadIdx.x;
        if (i >= max(A.ka[0], A.kb[0])) return;
        const float4 sa = spray_slot(A.ka, K, i), sb = spray_slot(A.kb, K, i);
        const V3 pa{sa.x, sa.y, sa.z}, pb{sb.x, sb.y, sb.z};
        const float ra = sa.w, rb = sb.w, f = A.f, t = A.t;
        V3 pos = f < 0.5f ? pa : pb;
        float r = f < 0.5f ? ra : rb;
        V3 vel{0.f, 0.f, 0.f};
        const float4 l = D.landed[i];
        if (ra > 0.0f && rb > 0.0f) {
            pos = mix3(pa, pb, f);
            r = mixf(ra, rb, f);
            vel = {__fmul_rn(__fsub_rn(pb.x, pa.x), A.inv), __fmul_rn(__fsub_rn(pb.y, pa.y), A.inv),
                   __fmul_rn(__fsub_rn(pb.z, pa.z), A.inv)};
        } else if (ra > 0.0f && l.z > 0.0f && l.w <= A.tb) {
            // A drop that lands between the keys flies to its landing point and vanishes there.
            const V3 hit{l.x, l.z, l.y};
            const float span = fmaxf(__fsub_rn(l.w, A.ta), 1e-9f);
            const float s = fminf(fmaxf(__fdiv_rn(__fsub_rn(t, A.ta), span), 0.0f), 1.0f);
            pos = mix3(pa, hit, s);
            r = t < l.w ? ra : 0.0f;
            vel = {__fdiv_rn(__fsub_rn(hit.x, pa.x), span), __fdiv_rn(__fsub_rn(hit.y, pa.y), span),
                   __fdiv_rn(__fsub_rn(hit.z, pa.z), span)};
        }
        const float2 w = A.spray_w[i];
        A.out_spray[2 * (size_t)i] = make_float4(pos.x, pos.y, pos.z, r);
        A.out_spray[2 * (size_t)i + 1] = make_float4(vel.x, vel.y, vel.z, t < w.y ? -w.x : w.x);
        return;
    }
    {  // show_wet_touch (:138-146): where the water body touched down by now the ground is soaked
        const uint32_t i = (b - A.b_drops) * KEY_T + threadIdx.x;
        const uint32_t res = A.wet_res;
        if (i >= res * res || A.t < 0.0f) return;
        if (D.touch[i] <= __float_as_uint(A.t)) atomicMax(A.out_wet + i, 4000000u);
    }
}

// show_wet_drops (shaders/show.wgsl:114-136): a landed drop spreads over up to 5 x 5 cells of
// the cleared wet map. Runs before k_key_show, whose ground-touch range takes a max over these
// sums; launched only when key b has spray slots.
__global__ void __launch_bounds__(KEY_T) k_key_drops(Dev D, ShowArgs A) {
    const uint32_t i = blockIdx.x * KEY_T + threadIdx.x;
    if (i >= A.kb[0]) return;
    const float4 l = D.landed[i];
    if (l.z <= 0.0f || l.w > A.t) return;
    const float h = A.wet_half;
    const uint32_t res = A.wet_res;
    const float cell = __fdiv_rn(__fmul_rn(2.0f, h), (float)res);
    const float r = l.z;
    const int k = (int)fminf(fmaxf(__fdiv_rn(__fmul_rn(3.0f, r), cell), 0.0f), 2.0f);
    const float n = (float)((2 * k + 1) * (2 * k + 1));
    const uint32_t amount =
        __float2uint_rz(__fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(4.18879f, r), r), r), 1e12f), n));
    const float two_h = __fmul_rn(2.0f, h);
    for (int y = -k; y <= k; y++) {
        for (int x = -k; x <= k; x++) {
            const float u = __fdiv_rn(__fadd_rn(__fadd_rn(l.x, __fmul_rn((float)x, cell)), h), two_h);
            const float v = __fdiv_rn(__fadd_rn(__fadd_rn(l.y, __fmul_rn((float)y, cell)), h), two_h);
            if (u < 0.0f || v < 0.0f || u >= 1.0f || v >= 1.0f) continue;
            // u, v < 1 keep the cell inside the map for a power-of-two resolution (the
            // reference's 1024); the min guards any other.
            const uint32_t cx = min(__float2uint_rz(__fmul_rn(u, (float)res)), res - 1u);
            const uint32_t cy = min(__float2uint_rz(__fmul_rn(v, (float)res)), res - 1u);
            atomicAdd(A.out_wet + (size_t)cy * res + cx, amount);
        }
    }
}

// ---- host: sizes and the keyframe schedule (src/cache.rs:22-46, 249-264, 410-421) ---------------

static uint64_t key_bytes_of(uint32_t np, uint32_t nv, uint32_t nt, uint32_t spray, uint32_t live) {
    const uint64_t words = KEY_HEAD + 2ull * ((uint64_t)np + nv) + ((uint64_t)nt + 31u) / 32u + 2ull * ((spray + 31ull) / 32u) +
                           (uint64_t)KEY_SPRAY_WORDS * live;
    return (words * 4u + 255u) / 256u * 256u;
}

// Keyframe spacing: 2% of the time since the last arrival, between 10 us and 4 ms.
static double key_spacing(double tau) { return std::clamp(0.02 * tau, 10e-6, 4e-3); }

// Keys the spacing asks for in the first tau after an arrival: the integral of 1 / spacing.
static double keys_after(double tau) {
    const double a = 10e-6 / 0.02, b = 4e-3 / 0.02;
    return std::fmin(tau, a) / 10e-6 + 50.0 * std::log(std::clamp(tau, a, b) / a) + std::fmax(tau - b, 0.0) / 4e-3;
}

// Keys still to come from t to t_end, the spacing starting over at every arrival.
static double keys_left(double t, const std::vector<double>& arr, double t_end) {
    double n = 0.0;
    for (size_t i = 0; i < arr.size(); i++) {
        const double a = arr[i], end = i + 1 < arr.size() ? arr[i + 1] : t_end;
        if (end > t) n += keys_after(end - a) - keys_after(std::fmax(t, a) - a);
    }
    return n;
}

// The arrivals, each at least 0, with 0 itself, ascending and without repeats.
static std::vector<double> arrival_list(const double* arrivals, uint32_t n) {
    std::vector<double> v;
    for (uint32_t k = 0; k < n; k++) v.push_back(std::fmax(arrivals[k], 0.0));
    v.push_back(0.0);
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    return v;
}

static double key_next_time(double t, const double* arrivals, uint32_t n_arrivals, double t_end, uint64_t free_bytes,
                            uint64_t size) {
    const std::vector<double> arr = arrival_list(arrivals, n_arrivals);
    double last = 0.0, next = t_end;
    for (double a : arr)
        if (a <= t) last = a;
    for (double a : arr)
        if (a > t) {
            next = a;
            break;
        }
    // Fast bullets throw far more spray, and at the usual spacing their keys would fill the pool
    // long before the end: the spacing stretches by however much the rest would overrun.
    const double overrun = 1.2 * keys_left(t, arr, t_end) * (double)size / (double)free_bytes;
    return std::fmin(std::fmin(t + key_spacing(t - last) * std::fmax(overrun, 1.0), next), t_end);
}

// ---- host: the cache ------------------------------------------------------------------------------

struct KeyRec {
    double t;
    uint64_t offset, bytes;
    uint32_t page, spray, live;
};

struct Cache {
    ntr_sim* handle = nullptr;
    Sim* S = nullptr;
    int device = 0;
    ntr_cache_params P{};
    uint8_t* pool = nullptr;
    uint64_t pool_bytes = 0;
    std::vector<KeyRec> keys;
    double next_t = 0.0;
    bool done = false, full = false;
    uint32_t cur_page = 0;
    uint64_t cur_off = 0;
    // What the shown buffers are sized for.
    uint32_t np = 0, nv = 0, nt = 0, spray_cap = 0, wet_res = 0;
    float4 *shown_p = nullptr, *shown_drops = nullptr, *shown_mem = nullptr;
    uint32_t *shown_alive = nullptr, *shown_wet = nullptr;
    float2* spray_w = nullptr;
    uint32_t *tile_tot = nullptr, *tile_pre = nullptr, *counts = nullptr;
    uint32_t* h_counts = nullptr;  // pinned
    double shown = std::numeric_limits<double>::quiet_NaN();
    uint64_t shown_id = 0;
    uint32_t shown_spray = 0;
    // Device time of the last store (the index launches, then the pack launch: the host's read
    // of the counts between them is not counted) and of the last show, from events on the
    // simulation's stream.
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    bool stored = false, showed = false;

    void free_shown() {
        for (void* p : {(void*)shown_p, (void*)shown_drops, (void*)shown_mem, (void*)shown_alive, (void*)shown_wet,
                        (void*)spray_w, (void*)tile_tot, (void*)tile_pre, (void*)counts})
            if (p) cudaFree(p);
        shown_p = shown_drops = shown_mem = nullptr;
        shown_alive = shown_wet = tile_tot = tile_pre = counts = nullptr;
        spray_w = nullptr;
    }
    ~Cache() {
        DeviceScope scope(device);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        free_shown();
        if (pool) cudaFree(pool);
        if (h_counts) cudaFreeHost(h_counts);
    }
    uint64_t used() const {
        uint64_t u = 0;
        for (const KeyRec& k : keys) u += k.bytes;
        return u;
    }
    double end() const { return keys.empty() ? 0.0 : keys.back().t; }
    uint32_t* key_ptr(const KeyRec& k) const { return (uint32_t*)(pool + (size_t)k.page * P.page_bytes + k.offset); }
};

// The shown buffers (src/cache.rs:393-408) and the spray index's scratch, zeroed, for the
// simulation's sizes; kept when the sizes are those already allocated.
static ntr_status cache_size_for(Cache& C, const Sim& S) {
    const Dev& D = S.D;
    if (C.shown_p && C.np == D.Np && C.nv == D.Nv && C.nt == D.Nt && C.spray_cap == D.spray_cap && C.wet_res == D.wet_res)
        return NTR_OK;
    C.free_shown();
    C.np = D.Np, C.nv = D.Nv, C.nt = D.Nt, C.spray_cap = D.spray_cap, C.wet_res = D.wet_res;
    const size_t tiles = ((size_t)D.spray_cap + KEY_TILE - 1) / KEY_TILE + 1;
    struct {
        void** p;
        size_t bytes;
    } want[] = {{(void**)&C.shown_p, (size_t)D.Np * 32}, {(void**)&C.shown_drops, (size_t)D.spray_cap * 32},
                {(void**)&C.shown_mem, (size_t)D.Nv * 16}, {(void**)&C.shown_alive, (size_t)D.Nt * 4},
                {(void**)&C.shown_wet, (size_t)D.wet_res * D.wet_res * 4}, {(void**)&C.spray_w, (size_t)D.spray_cap * 8},
                {(void**)&C.tile_tot, tiles * 4}, {(void**)&C.tile_pre, tiles * 4}, {(void**)&C.counts, 16}};
    for (auto& w : want) {
        const size_t bytes = std::max<size_t>(w.bytes, 16);
        if (cudaMalloc(w.p, bytes) != cudaSuccess) {
            cudaGetLastError();
            C.free_shown();
            return fail(NTR_E_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes for the keyframe cache failed");
        }
        CU(cudaMemset(*w.p, 0, bytes));
    }
    return NTR_OK;
}

// store_key (src/cache.rs:231-265): index the live spray, read the slot and live counts back so
// the keyframe gets exactly the space it needs, place it, pack it, and schedule the next one.
static ntr_status cache_store(Cache& C) {
    Sim& S = *C.S;
    const Dev& D = S.D;
    cudaStream_t s = S.stream;
    // The grid is sized from the host's copy of the spray count (read back with the state after
    // every batch); the kernel strides over the device's own count, so a stale copy only changes
    // how the work is spread.
    const uint32_t hint = std::min(S.h_state->s.spray_count, D.spray_cap);
    const uint32_t g_count = std::max(1u, std::min((hint + KEY_TILE - 1) / KEY_TILE, (uint32_t)S.sms * 8u));
    CU(cudaEventRecord(C.ev[0], s));
    k_key_index<<<g_count, KEY_T, 0, s>>>(D, C.tile_tot, C.tile_pre, C.counts);
    CU(cudaGetLastError());
    CU(cudaEventRecord(C.ev[1], s));
    CU(cudaMemcpyAsync(C.h_counts, C.counts, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const uint32_t n = C.h_counts[0], live = C.h_counts[1];
    const uint64_t size = key_bytes_of(D.Np, D.Nv, D.Nt, n, live);
    if (C.cur_off + size > C.P.page_bytes) C.cur_page++, C.cur_off = 0;
    if (C.cur_page >= C.P.pages) {
        C.full = C.done = true;
        return NTR_OK;
    }
    KeyRec k{S.host.h.t, C.cur_off, size, C.cur_page, n, live};
    PackRanges R{};
    R.b_mem = (D.Np + KEY_T * KEY_PER - 1) / (KEY_T * KEY_PER);
    R.b_alive = R.b_mem + (D.Nv + KEY_T - 1) / KEY_T;
    R.b_spray = R.b_alive + (bit_words(D.Nt) + KEY_T / 32 - 1) / (KEY_T / 32);
    R.b_end = R.b_spray + (n + KEY_TILE - 1) / KEY_TILE;
    R.n = n, R.live = live;
    CU(cudaEventRecord(C.ev[2], s));
    k_key_pack<<<std::max(R.b_end, 1u), KEY_T, 0, s>>>(D, C.key_ptr(k), C.spray_w, C.tile_pre, R);
    CU(cudaGetLastError());
    CU(cudaEventRecord(C.ev[3], s));
    C.stored = true;
    C.cur_off += size;
    C.keys.push_back(k);
    if (C.next_t >= C.P.t_end) {
        C.done = true;
    } else {
        const uint64_t u = C.used();
        const uint64_t free_b = std::max<uint64_t>(C.pool_bytes > u ? C.pool_bytes - u : 0, 1);
        C.next_t = key_next_time(k.t, C.P.arrivals, C.P.n_arrivals, C.P.t_end, free_b, size);
    }
    return NTR_OK;
}

// restart (src/cache.rs:161-173).
static ntr_status cache_restart(Cache& C) {
    const Dev& D = C.S->D;
    const uint64_t largest = key_bytes_of(D.Np, D.Nv, D.Nt, D.spray_cap, D.spray_cap);
    if (largest > C.P.page_bytes)
        return fail(NTR_E_INVALID, "a keyframe (" + std::to_string(largest) + " bytes) must fit in one pool page");
    ntr_status r = ntr_sim_advance(C.handle, 0.0, 0, nullptr);
    if (r != NTR_OK) return r;
    C.keys.clear();
    C.cur_page = 0, C.cur_off = 0;
    C.next_t = 0.0;
    C.done = C.full = false;
    C.shown = std::numeric_limits<double>::quiet_NaN();
    C.shown_id++;
    return cache_store(C);
}

// bake (src/cache.rs:196-216).
static ntr_status cache_bake(Cache& C, uint32_t max_steps, uint32_t* steps_out) {
    uint32_t steps = 0;
    ntr_status r = NTR_OK;
    while (!C.done && steps < max_steps) {
        const uint32_t left = max_steps - steps;
        uint32_t n = 0;
        if ((r = ntr_sim_advance(C.handle, C.next_t, left, &n)) != NTR_OK) break;
        steps += n;
        if (n == left) continue;
        if (C.S->host.h.t > C.end()) {
            if ((r = cache_store(C)) != NTR_OK) break;
        } else {
            // The next step is longer than the keyframe spacing: take it anyway, the keyframe
            // lands right after.
            if ((r = ntr_sim_advance(C.handle, std::numeric_limits<double>::infinity(), 1, &n)) != NTR_OK) break;
            steps += n;
        }
    }
    if (steps_out) *steps_out = steps;
    return r;
}

// show (src/cache.rs:269-332).
static ntr_status cache_show(Cache& C, double t, int* changed) {
    if (changed) *changed = 0;
    if (C.keys.empty()) return fail(NTR_E_INVALID, "the cache holds no keyframe");
    Sim& S = *C.S;
    const Dev& D = S.D;
    const double lo = S.host.h.t_start, hi = C.end();
    t = t < lo ? lo : t > hi ? hi : t;
    if (t == C.shown) return NTR_OK;
    size_t b = std::partition_point(C.keys.begin(), C.keys.end(), [&](const KeyRec& k) { return k.t <= t; }) - C.keys.begin();
    b = std::clamp<size_t>(b, 1, C.keys.size());
    const size_t a = b - 1;
    b = std::min(b, C.keys.size() - 1);
    const KeyRec &ka = C.keys[a], &kb = C.keys[b];
    const uint32_t spray = std::max(ka.spray, kb.spray);
    double f = 0.0, inv = 0.0;
    if (b > a) f = std::clamp((t - ka.t) / (kb.t - ka.t), 0.0, 1.0), inv = 1.0 / (kb.t - ka.t);
    ShowArgs A{};
    A.ka = C.key_ptr(ka), A.kb = C.key_ptr(kb), A.spray_w = C.spray_w;
    A.out_p = C.shown_p, A.out_spray = C.shown_drops, A.out_mem = C.shown_mem, A.out_alive = C.shown_alive, A.out_wet = C.shown_wet;
    A.t = (float)t, A.f = (float)f, A.inv = (float)inv, A.ta = (float)ka.t, A.tb = (float)kb.t;
    A.wet_half = S.U.wet[0], A.wet_res = D.wet_res;
    const size_t cells = (size_t)D.wet_res * D.wet_res;
    A.b_mem = (D.Np + KEY_T * KEY_PER - 1) / (KEY_T * KEY_PER);
    A.b_alive = A.b_mem + (D.Nv + KEY_T - 1) / KEY_T;
    A.b_spray = A.b_alive + (D.Nt + KEY_T - 1) / KEY_T;
    A.b_drops = A.b_spray + (spray + KEY_T - 1) / KEY_T;
    A.b_end = A.b_drops + (uint32_t)((cells + KEY_T - 1) / KEY_T);
    cudaStream_t s = S.stream;
    CU(cudaEventRecord(C.ev[4], s));
    CU(cudaMemsetAsync(C.shown_wet, 0, cells * 4, s));
    if (kb.spray > 0) k_key_drops<<<(kb.spray + KEY_T - 1) / KEY_T, KEY_T, 0, s>>>(D, A);
    k_key_show<<<std::max(A.b_end, 1u), KEY_T, 0, s>>>(D, A);
    CU(cudaGetLastError());
    CU(cudaEventRecord(C.ev[5], s));
    C.showed = true;
    C.shown = t;
    C.shown_id++;
    C.shown_spray = spray;
    if (changed) *changed = 1;
    return NTR_OK;
}

}  // namespace ntr
