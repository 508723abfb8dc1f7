// Grid to particle and the spray (shaders/fluid.wgsl:676-901, bullet.wgsl:395-424).
//
// Break-ups get their spray slots in a canonical order: block by block, and in sorted order
// within a block. g2p writes each block's break-ups, ranked in that order, into scratch at the
// block's own range of sorted positions; a scan over the blocks' counts then gives every one
// its slots, and k_spray_emit writes the drops. The reference hands slots out with atomicAdd
// (fluid.wgsl:726), whose order is the hardware's.
#pragma once

#include "kernels_grid.cuh"
#include "kernels_mem.cuh"

namespace ntr {

__device__ __forceinline__ float drag_cd(float re) {
    if (re < 1e-4f) return 24.0f / 1e-4f;
    return 24.0f / re * (1.0f + 0.15f * nt_pow(re, 0.687f)) + 0.42f / (1.0f + 42500.0f * nt_pow(re, -1.16f));
}

template <class CT>
__device__ __forceinline__ void spray_update_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t n = min(st->s.spray_count, D.spray_cap);
    const float step = dt_of(st), now = now_of(st);
    const ntr_gpu_params* U = D.U;
    const V3 grav = {U->gravity[0], U->gravity[1], U->gravity[2]};
    const float rhow = U->fluid[0];
    for (uint32_t i = C.x() * blockDim.x + threadIdx.x; i < n; i += C.nx() * blockDim.x) {
        float4 pos = D.spray[3 * (size_t)i], vel = D.spray[3 * (size_t)i + 1];
        float r = pos.w;
        if (r <= 0.0f) continue;
        float sp = length(xyz(vel));
        float re = 2.0f * r * sp * RHO_AIR / MU_AIR;
        float k = 3.0f * RHO_AIR * drag_cd(re) * sp / (8.0f * rhow * r);
        V3 v = (xyz(vel) + step * grav) / (1.0f + k * step);
        r = sqrtf(mx(r * r - EVAPORATION * step, 0.0f));
        if (r < 2.5e-6f) r = 0.0f;
        V3 p = xyz(pos) + step * v;
        if (p.y <= r) {
            D.landed[i] = make_float4(p.x, p.z, r * nt_pow(vel.w, 1.0f / 3.0f), now);
            r = 0.0f;
        }
        D.spray[3 * (size_t)i] = f4(p, r);
        D.spray[3 * (size_t)i + 1] = f4(v, vel.w);
    }
}
__global__ void k_spray_update(Dev D) { spray_update_body(D, HwCta{}); }
__global__ void k_spray_update_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    spray_update_body(sD, c);
}

__device__ __forceinline__ void ground_touch(const Dev& D, V3 p, float now) {
    const float hw = D.U->wet[0];
    const uint32_t res = D.U->limits[0];
    float ux = (p.x + hw) / (2.0f * hw), uz = (p.z + hw) / (2.0f * hw);
    if (ux < 0.0f || uz < 0.0f || ux >= 1.0f || uz >= 1.0f) return;
    uint32_t cx = f2u(ux * (float)res), cz = f2u(uz * (float)res);
    atomicMin(D.touch + (size_t)cz * res + cx, __float_as_uint(now));
}

// `reach`: the bullets' reach spheres (DBullet::reach), `n_shots` of them, read once per CTA.
__device__ void carve(const Dev& D, const float4* reach_of, uint32_t n_shots, V3& x, V3& v, uint32_t id, float t, float hh,
                      uint32_t step_no) {
    const float hand2 = R_HAND * R_HAND * hh * hh;
    for (uint32_t bi = 0; bi < n_shots; bi++) {
        const float4 reach = reach_of[bi];
        if (reach.w <= 0.0f || distance(x, xyz(reach)) > reach.w) continue;
        for (uint32_t k = 0; k < NTR_N_SEC; k++) {
            const DSection s = D.sections[bi * NTR_N_SEC + k];
            float r2 = section_r2(s, t);
            if (s.b.w <= 0.0f || r2 >= hand2) continue;
            V3 ab = xyz(s.b) - xyz(s.a);
            float f = dot(x - xyz(s.a), ab) / mx(dot(ab, ab), 1e-20f);
            if (f < 0.0f || f > 1.0f) continue;
            V3 on = xyz(s.a) + f * ab;
            V3 d = x - on;
            if (dot(d, d) >= r2) continue;
            if (dot(d, d) < 1e-14f) {
                uint32_t seed = hash3(id, step_no, k);
                float g0 = rnd_gauss(seed);
                float g1 = rnd_gauss(seed);
                float g2 = rnd_gauss(seed);
                d = cross(ab + 1e-9f, v3(g0, g1, g2));
            }
            V3 dir = normalize(d);
            float r = sqrtf(r2);
            x = on + dir * r;
            float wall = s.b.w / (2.0f * r);
            v = v + dir * mx(wall - dot(v, dir), 0.0f);
        }
    }
}

struct Gathered {
    float s;
    V3 g;
    float w;
};

__device__ __forceinline__ Gathered gather(const float* tg, V3 X, V3 o, I3 corner, uint32_t fa, uint32_t fw, float hh) {
    I3 base = vi(vfloor(X - o - 0.5f));
    V3 fx = X - o - vf(base);
    V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    I3 tq = base - corner;
    uint32_t t0 = (uint32_t)tq.x * 49u + (uint32_t)tq.y * 7u + (uint32_t)tq.z;
    Gathered r = {0.0f, {0.0f, 0.0f, 0.0f}, 0.0f};
#pragma unroll
    for (uint32_t a = 0; a < 3; a++)
#pragma unroll
        for (uint32_t b = 0; b < 3; b++)
#pragma unroll
            for (uint32_t c = 0; c < 3; c++) {
                float weight = wx[a] * wy[b] * wz[c];
                uint32_t t = t0 + a * 49u + b * 7u + c;
                float u = weight * tg[fa * TILE + t];
                r.s += u;
                // The gradient's and the weight's sums are fused multiply-adds (the oracle's
                // gather does the same), one rounding a term instead of two.
                const V3 d = v3((float)a, (float)b, (float)c) - fx;
                r.g = {__fmaf_rn(u, d.x, r.g.x), __fmaf_rn(u, d.y, r.g.y), __fmaf_rn(u, d.z, r.g.z)};
                r.w = __fmaf_rn(weight, tg[fw * TILE + t], r.w);
            }
    r.g = r.g * hh;
    return r;
}

// Asynchronous 4-byte copies global -> shared (cp.async; a source of size 0 fills zeros), in
// groups a thread commits and later waits for.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool valid) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(sa), "l"(gmem), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The raw fields of a block's 7^3 tile on their way to shared memory: per node the three
// velocities and the three weight sums, the cell type and the pressure (zeros where no block
// is), and the block's own 64 cells' rubber area sums.
constexpr uint32_t G2P_RAW = 8;
__device__ __forceinline__ void g2p_stage(const Dev& D, uint32_t b, uint32_t* links, uint32_t* raw, uint32_t* raw_cov, uint32_t nthreads) {
    if (threadIdx.x < 27) links[threadIdx.x] = D.block_nb[b * 27u + threadIdx.x];
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < TILE; t += nthreads) {
        const uint32_t cell = tile_cell(links, t);
        const bool ok = cell != NONE;
        const uint32_t c = ok ? cell : 0u;
#pragma unroll
        for (uint32_t d = 0; d < 3; d++) {
            cp_async4(raw + d * TILE + t, D.cf + (size_t)(F_U + d) * D.cap_cells + c, ok);
            cp_async4(raw + (3 + d) * TILE + t, D.acc + (size_t)a_wt(d) * D.cap_cells + c, ok);
        }
        cp_async4(raw + 6 * TILE + t, D.cf + (size_t)F_TYPE * D.cap_cells + c, ok);
        cp_async4(raw + 7 * TILE + t, D.cf + (size_t)F_P * D.cap_cells + c, ok);
    }
    if (threadIdx.x < 64) cp_async4(raw_cov + threadIdx.x, D.acc + (size_t)A_MA * D.cap_cells + b * 64u + threadIdx.x, true);
    cp_async_commit();
}

// The break-ups of one segment of a block's particles (sorted positions seg .. seg + G2P_SEG),
// written at their own positions and flagged in `bits`, moved to their ranks: after the block's
// earlier ones (`brk`), in sorted order. One warp moves them a word (up to 32) at a time in
// ascending order, so a move never lands on a break-up still to be moved (a rank is at most its
// position, and the positions still to come are above it). `any`: this thread flagged one in the
// segment. Every thread of the CTA calls it (it has barriers).
constexpr uint32_t G2P_SEG = 1024;
__device__ __forceinline__ void g2p_rank_breakups(const Dev& D, uint32_t first, uint32_t seg, uint32_t* bits, uint32_t& brk,
                                                  bool any, uint32_t warp, uint32_t lane) {
    if (!__syncthreads_or(any)) return;  // most segments have none
    if (warp == 0) {
        uint32_t n = brk;
        for (uint32_t w0 = 0; w0 < G2P_SEG / 32; w0++) {
            const uint32_t word = bits[w0];
            if (!word) continue;
            const uint32_t cnt = (uint32_t)__popc(word);
            const uint32_t at = lane < cnt ? (uint32_t)__fns(word, 0u, (int)lane + 1) : 0u;
            float4 x = make_float4(0.0f, 0.0f, 0.0f, 0.0f), v = x;
            if (lane < cnt) {
                x = D.brk_x[first + seg + w0 * 32u + at];
                v = D.brk_v[first + seg + w0 * 32u + at];
            }
            __syncwarp();
            if (lane < cnt) {
                D.brk_x[first + n + lane] = x;
                D.brk_v[first + n + lane] = v;
            }
            __syncwarp();
            n += cnt;
            bits[w0] = 0u;
        }
        if (lane == 0) brk = n;
    }
    __syncthreads();
}

// G2P_T threads a CTA, 768 / G2P_T CTAs an SM. With many blocks (the 1M-particle scene: 128
// threads, six CTAs an SM) a block's few hundred particles take 3 rounds with a short last one,
// and the SM has more CTAs to switch to while one waits on its loads or barriers. With few
// blocks (small scenes: 256 threads) every block runs at once and its chain of rounds is the
// time. The result does not depend on the CTA's size.
template <int G2P_T, class CT>
__device__ __forceinline__ void g2p_body(const Dev& D, const CT& C) {
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    const ntr_gpu_params* U = D.U;
    const uint32_t nb = min(st->s.n_blocks, D.cap_blocks);
    const float hh = g.h, step = dt_of(st), now = now_of(st);
    const float spacing = U->fluid[3];
    const V3 lo = g.org + 3.5f * hh;
    const V3 hi = g.org + (v3((float)g.dims[0], (float)g.dims[1], (float)g.dims[2]) - 4.5f) * hh;
    const float r_thin = 0.75f * spacing;
    const float t_thin = 3.0f * sqrtf(U->fluid[0] * r_thin * r_thin * r_thin / SIGMA_W);
    const float cs = 4.0f / (hh * hh);
    const uint32_t step_no = st->s.step;
    __shared__ float tg[8 * TILE];
    __shared__ uint32_t raw[G2P_RAW * TILE];  // the next block's fields, arriving (g2p_stage)
    __shared__ uint32_t raw_cov[64];
    __shared__ uint32_t s_links[2][27];       // the current block's neighbours, and the next's
    __shared__ uint8_t s_cov[64];  // the block's own cells: rubber over them (A_MA > 0)
    __shared__ uint32_t s_bits[G2P_SEG / 32];  // the segment's break-up flags, a bit per particle
    __shared__ uint32_t s_brk;
    __shared__ float4 s_reach[NTR_MAX_SHOTS];
    const uint32_t n_shots = min(U->mem[3], (uint32_t)NTR_MAX_SHOTS);
    if (threadIdx.x < n_shots) s_reach[threadIdx.x] = D.bullets[threadIdx.x].reach;  // barriers follow before its use
    float fastest = 0.0f;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    // The CTA's blocks that hold particles, in turn (an empty one only gets its count of break-ups).
    auto next_full = [&](uint32_t x) {
        while (x < nb && D.block_start[x + 1] == D.block_start[x]) {
            if (threadIdx.x == 0) D.brk_count[x] = 0;
            x += C.nx();
        }
        return x;
    };
    // A one-scene launch hands the blocks out from a counter as CTAs come free (thread 0 takes
    // them, the empty ones in passing); a CTA takes its next block at the start of this one, in
    // time to stage it, into the slot of its turn's parity.
    __shared__ uint32_t s_next[2];
    auto take = [&]() {
        uint32_t x = atomicAdd(&D.st->next_block[1], 1u);
        while (x < nb && D.block_start[x + 1] == D.block_start[x]) {
            D.brk_count[x] = 0;
            x = atomicAdd(&D.st->next_block[1], 1u);
        }
        return x;
    };
    uint32_t turn = 0;
    if constexpr (CT::dynamic) {
        if (threadIdx.x == 0) s_next[0] = take();
        __syncthreads();
    }
    // Each block's tile is staged while the block before it is processed: its fields come in by
    // asynchronous copies behind that block's particles, and only the first block's wait is bare.
    uint32_t b = CT::dynamic ? s_next[0] : next_full(C.x()), cur = 0;
    if (b < nb) g2p_stage(D, b, s_links[0], raw, raw_cov, G2P_T);
    while (b < nb) {
        turn++;
        if (CT::dynamic && threadIdx.x == 0) s_next[turn & 1u] = take();
        const uint32_t* links = s_links[cur];
        const uint32_t first = D.block_start[b];
        const uint32_t count = D.block_start[b + 1] - first;
        // This thread's particle of the first round, loaded before the tile is made so that the
        // waits overlap; each round then loads the next round's particle before its gathers.
        uint32_t i_next = 0u;
        float4 pos_next = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float c1w_next = 0.0f;
        if (threadIdx.x < count) {
            i_next = D.sorted[first + threadIdx.x];
            pos_next = D.pos[i_next];
            c1w_next = D.c1[i_next].w;
        }
        cp_async_wait_all();
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < TILE; t += G2P_T) {
            const float ty = __uint_as_float(raw[6 * TILE + t]);
            const bool water = ty == WATER_T;  // zeros (gas) where no block is
#pragma unroll
            for (uint32_t d = 0; d < 3; d++) {
                tg[a_mom(d) * TILE + t] = __uint_as_float(raw[d * TILE + t]);
                tg[a_wt(d) * TILE + t] = from_fp((int32_t)raw[(3 + d) * TILE + t], FP_W);
            }
            tg[A_PC * TILE + t] = water ? mx(__uint_as_float(raw[7 * TILE + t]), P_VAPOUR - P_ATM) : 0.0f;
            tg[A_WC * TILE + t] = water ? 1.0f : 0.0f;
        }
        if (threadIdx.x < 64) s_cov[threadIdx.x] = (int32_t)raw_cov[threadIdx.x] > 0 ? 1 : 0;
        if (threadIdx.x == 0) s_brk = 0;
        for (uint32_t w = threadIdx.x; w < G2P_SEG / 32; w += G2P_T) s_bits[w] = 0u;
        __syncthreads();
        const uint32_t nxt = CT::dynamic ? s_next[turn & 1u] : next_full(b + C.nx());
        if (nxt < nb) g2p_stage(D, nxt, s_links[cur ^ 1u], raw, raw_cov, G2P_T);
        const I3 corner = slot_coord(g, g.list[b]) * 4 - I3{1, 1, 1};
        // Rounds of G2P_T particles; the break-ups are ranked in sorted order per segment.
        uint32_t seg = 0;
        bool seg_any = false;
        for (uint32_t base = 0; base < count; base += G2P_T) {
            const uint32_t k = base + threadIdx.x;
            bool brk = false;
            V3 bx = {0.0f, 0.0f, 0.0f}, bv = bx;
            uint32_t bid = 0;
            const uint32_t i = i_next;
            const float4 pos = pos_next;
            const float c1w = c1w_next;
            if (k + G2P_T < count) {
                i_next = D.sorted[first + k + G2P_T];
                pos_next = D.pos[i_next];
                c1w_next = D.c1[i_next].w;
            }
            if (k < count) {
                V3 X = (xyz(pos) - g.org) / hh;
                Gathered gu = gather(tg, X, v3(0.0f, 0.5f, 0.5f), corner, 0, 1, hh);
                Gathered gv = gather(tg, X, v3(0.5f, 0.0f, 0.5f), corner, 2, 3, hh);
                Gathered gw = gather(tg, X, v3(0.5f, 0.5f, 0.0f), corner, 4, 5, hh);
                Gathered gp = gather(tg, X, v3(0.5f, 0.5f, 0.5f), corner, A_PC, A_WC, hh);
                V3 v = {gu.s, gv.s, gw.s};
                float m_near = gu.w + gv.w + gw.w;
                V3 x = xyz(pos) + step * v;
                if (n_shots > 0u) carve(D, s_reach, n_shots, x, v, i, now, hh, step_no);
                bool escaped = x.x < lo.x || x.z < lo.z || x.x > hi.x || x.z > hi.z || x.y > hi.y;
                float fill = m_near / 24.0f;
                bool on_ground = x.y < 1.5f * spacing;
                // The particle's own cell, in this block (tile coordinates 1-4) as a rule: its rubber
                // flag is in shared memory; elsewhere it is looked up.
                const I3 oc = vi(vfloor(X)) - corner;
                bool covered;
                if ((uint32_t)(oc.x - 1) < 4u && (uint32_t)(oc.y - 1) < 4u && (uint32_t)(oc.z - 1) < 4u) {
                    covered = s_cov[(oc.x - 1) * 16 + (oc.y - 1) * 4 + (oc.z - 1)] != 0;
                } else {
                    const uint32_t own_t = tile_cell(links, (uint32_t)oc.x * 49u + (uint32_t)oc.y * 7u + (uint32_t)oc.z);
                    covered = own_t != NONE && accv(D, A_MA, own_t) > 0;
                }
                float thin_age = (fill < 0.45f && !on_ground && !covered) ? c1w + step : 0.0f;
                if (escaped || (!covered && fill < 0.2f) || thin_age > t_thin) {
                    if (on_ground) {
                        ground_touch(D, x, now);
                    } else {
                        brk = true;
                        bx = x, bv = v, bid = i;
                    }
                    D.vel[i] = f4(v, 0.0f);
                } else {
                    V3 xx = x, vv = v;
                    if (xx.y < 0.3f * spacing) {
                        xx.y = 0.3f * spacing;
                        vv.y = mx(vv.y, 0.0f);
                    }
                    if (xx.y < 0.7f * spacing) ground_touch(D, xx, now);
                    D.pos[i] = f4(xx, pos.w);
                    D.vel[i] = f4(vv, 1.0f);
                    D.c0[i] = f4(gu.g * cs, gp.w > 1e-6f ? gp.s / gp.w : 0.0f);
                    D.c1[i] = f4(gv.g * cs, thin_age);
                    D.c2[i] = f4(gw.g * cs, 0.0f);
                    fastest = mx(fastest, length(vv));
                }
            }
            // A break-up goes to scratch at its own sorted position and is flagged, a bit per
            // particle; the flags are ranked (in sorted order) a segment of G2P_SEG particles at a
            // time, so that the rounds need no barrier.
            const uint32_t bal = __ballot_sync(0xffffffffu, brk);
            if (lane == 0) s_bits[((base - seg) >> 5) + warp] = bal;
            if (brk) {
                D.brk_x[first + k] = f4(bx, __uint_as_float(bid));
                D.brk_v[first + k] = f4(bv, 0.0f);
            }
            seg_any = seg_any || brk;
            if (base + G2P_T >= count || base + G2P_T - seg >= G2P_SEG) {
                g2p_rank_breakups(D, first, seg, s_bits, s_brk, seg_any, warp, lane);
                seg = base + G2P_T;
                seg_any = false;
            }
        }
        if (threadIdx.x == 0) D.brk_count[b] = s_brk;
        __syncthreads();
        b = nxt;
        cur ^= 1u;
    }
    for (int o = 16; o > 0; o >>= 1) fastest = fmaxf(fastest, __shfl_down_sync(0xffffffffu, fastest, o));
    if (lane == 0 && fastest > 0.0f) atomicMax((unsigned int*)&st->s.max_speed, __float_as_uint(fastest));
}
template <int G2P_T>
__global__ void __launch_bounds__(G2P_T, 768 / G2P_T) k_g2p(Dev D) { g2p_body<G2P_T>(D, HwCta{}); }
template <int G2P_T>
__global__ void __launch_bounds__(G2P_T, 768 / G2P_T) k_g2p_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    g2p_body<G2P_T>(sD, c);
}

// The step's last bookkeeping (what the reference's break_up leaves in its counters): the spray
// count advanced by the step's break-ups (5 slots each), and the step's work, whose algorithmic
// bytes are counted from these: blocks, water cells times solver iterations, rubber substeps,
// free-gas cells times air substeps, spray slots in use. By k_spray_scan, once it has the
// step's break-ups; k_spray_emit takes its first slot as the count less those.
__device__ __forceinline__ void spray_commit(const Dev& D, DevState* st) {
    st->s.spray_count += 5u * st->nbrk;
    const ntr_gpu_params* U = D.U;
    st->work[0] += 1ull;
    st->work[1] += 64ull * min(st->s.n_blocks, D.cap_blocks);
    st->work[2] += (unsigned long long)st->n_water * st->s.solve_iters;
    st->work[3] += U->mem[1];
    st->work[4] += (unsigned long long)st->n_gas * U->mem[2];
    st->work[5] += min(st->s.spray_count, D.spray_cap);
    st->n_water = st->n_gas = 0u;
}

// Exclusive scan of the blocks' break-up counts (one CTA); advances the spray count.
template <class CT>
__device__ __forceinline__ void spray_scan_body(const Dev& D, const CT& C) {
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t n = min(st->s.n_blocks, D.cap_blocks);
    const uint32_t per = (n + 1023u) / 1024u;
    const uint32_t lo = min(threadIdx.x * per, n), hi = min(lo + per, n);
    uint32_t s = 0;
    for (uint32_t i = lo; i < hi; i++) s += D.brk_count[i];
    __shared__ uint32_t ws[32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = s;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += v;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t v = ws[lane], x = v;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        ws[lane] = x;  // inclusive
    }
    __syncthreads();
    uint32_t run = (warp > 0 ? ws[warp - 1] : 0u) + inc - s;
    for (uint32_t i = lo; i < hi; i++) {
        D.brk_off[i] = run;
        run += D.brk_count[i];
    }
    if (threadIdx.x == 0) {
        uint32_t total = ws[31];
        st->nbrk = total;
        spray_commit(D, st);
    }
}
__global__ void __launch_bounds__(1024) k_spray_scan(Dev D) { spray_scan_body(D, HwCta{}); }
__global__ void __launch_bounds__(1024) k_spray_scan_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    spray_scan_body(sD, c);
}

// Writes the drops of every break-up (fluid.wgsl:718-765): 4 drops and a parcel of finer ones.
template <class CT>
__device__ __forceinline__ void spray_emit_body(const Dev& D, const CT& C) {
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t nb = min(st->s.n_blocks, D.cap_blocks);
    const uint32_t cap = D.spray_cap;
    const uint32_t base_count = st->s.spray_count - 5u * st->nbrk;  // k_spray_scan advanced it
    const float hs = D.U->fluid[3], rhow = D.U->fluid[0];
    const float now = now_of(st);
    const uint32_t step_no = st->s.step;
    const float vol = hs * hs * hs;
    // One warp per block, lanes over its break-ups.
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gw = (C.x() * blockDim.x + threadIdx.x) >> 5, nw = (C.nx() * blockDim.x) >> 5;
    for (uint32_t b = gw; b < nb; b += nw) {
        const uint32_t cnt = D.brk_count[b];
        if (cnt == 0) continue;
        const uint32_t first_pos = D.block_start[b];
        for (uint32_t r = lane; r < cnt; r += 32) {
            const uint32_t grank = D.brk_off[b] + r;
            const uint32_t firsts = base_count + 5u * grank;
            if (firsts >= cap) continue;
            const float4 ex = D.brk_x[first_pos + r], ev = D.brk_v[first_pos + r];
            const V3 x = xyz(ex), v = xyz(ev);
            const uint32_t id = __float_as_uint(ex.w);
            uint32_t seed = hash3(step_no, id, 0xb4eau);
            float speed = length(v);
            float bd2 = WE_CRIT * SIGMA_W / (RHO_AIR * mx(speed * speed, 1e-4f));
            float d_med = mn(0.55f * hs, 0.5f * bd2);
            float dd[4];
            float used = 0.0f;
            for (int k = 0; k < 4; k++) {
                dd[k] = clampf_(d_med * nt_exp(0.5f * rnd_gauss(seed)), 2e-5f, 1.24f * hs);
                used += 0.5236f * dd[k] * dd[k] * dd[k];
            }
            float df = 0.5f * d_med;
            bool fine = df < 1e-4f;
            float fit = nt_pow(vol / used, 1.0f / 3.0f);
            float scale = fine ? mn(1.0f, fit) : fit;
            bool stop = false;
            for (uint32_t k = 0; k < 4; k++) {
                uint32_t slot = firsts + k;
                if (slot >= cap) {
                    stop = true;
                    break;
                }
                float dk = dd[k] * scale;
                float spread = sqrtf(SIGMA_W / (rhow * dk)) + 0.05f * speed;
                float g0 = rnd_gauss(seed);
                float g1 = rnd_gauss(seed);
                float g2 = rnd_gauss(seed);
                V3 u = normalize(v3(g0, g1, g2) + 1e-6f);
                float o0 = rnd(seed);
                float o1 = rnd(seed);
                float o2 = rnd(seed);
                V3 off = (v3(o0, o1, o2) - 0.5f) * hs;
                float rr = rnd(seed);
                D.spray[3 * (size_t)slot] = f4(x + off, 0.5f * dk);
                D.spray[3 * (size_t)slot + 1] = f4(v + u * spread * rr, 1.0f);
                D.spray[3 * (size_t)slot + 2] = make_float4(0.0f, 0.0f, 0.0f, now);
            }
            if (stop) continue;
            uint32_t slot = firsts + 4;
            if (slot >= cap) continue;
            float nn = (vol - used * scale * scale * scale) / (0.5236f * df * df * df);
            D.spray[3 * (size_t)slot] = f4(x, (fine && nn >= 2.0f) ? 0.5f * df : 0.0f);
            D.spray[3 * (size_t)slot + 1] = f4(v, mx(nn, 2.0f));
            D.spray[3 * (size_t)slot + 2] = make_float4(0.0f, 0.0f, 0.0f, now);
        }
    }
}
__global__ void k_spray_emit(Dev D) { spray_emit_body(D, HwCta{}); }
__global__ void k_spray_emit_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    spray_emit_body(sD, c);
}

// The spray count moves on by five slots per break-up, capacity or not (fluid.wgsl:726).
// ---- the zero-length measuring substep and diagnostics --------------------------------------------
// Conservation sums over live particles in FP64: count, momentum, kinetic energy (per particle
// mass) and the sum of positions.
// The particles in the reference's layout (`Particle`, sim_defs.wgsl:61): 20 floats each, the
// five float4 of the SoA arrays in order. One thread per output float4: coalesced writes.
__global__ void k_pack_particles(Dev D, float4* __restrict__ dst) {
    const size_t n = (size_t)D.Np * 5;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
        const size_t i = o / 5;
        const uint32_t k = (uint32_t)(o - i * 5);
        const float4* src = k == 0 ? D.pos : k == 1 ? D.vel : k == 2 ? D.c0 : k == 3 ? D.c1 : D.c2;
        dst[o] = src[i];
    }
}

__global__ void k_conservation(Dev D, double* out) {
    __shared__ double red[8][8];
    double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < D.Np; i += gridDim.x * blockDim.x) {
        float4 v = D.vel[i];
        if (v.w < 0.5f) continue;
        float4 p = D.pos[i];
        a[0] += 1.0;
        a[1] += v.x, a[2] += v.y, a[3] += v.z;
        a[4] += 0.5 * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
        a[5] += p.x, a[6] += p.y, a[7] += p.z;
    }
    for (int k = 0; k < 8; k++)
        for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 8; k++) red[warp][k] = a[k];
    __syncthreads();
    if (threadIdx.x < 8) {
        double s = 0;
        for (uint32_t w = 0; w < blockDim.x / 32; w++) s += red[w][threadIdx.x];
        atomicAdd(out + threadIdx.x, s);
    }
}

}  // namespace ntr
