// Kernels of the step up to the transfer to the grid: the step clock, block activation over a
// bitmask, the stable radix sort of particles by block, and APIC P2G in a shared-memory tile.
//
// Reference: shaders/fluid.wgsl:33-303 (begin_step .. p2g), membrane.wgsl:164-180
// (mark_rubber), air.wgsl:271-277 (keep_blocks).
#pragma once

#include "dev.cuh"

namespace ntr {

// ---- begin_step, fluid.wgsl:33-89 ------------------------------------------------------------
template <class CT>
__device__ __forceinline__ void begin_step_body(const Dev& D, const CT& C) {
    if (threadIdx.x != 0 || C.x() != 0) return;
    const ntr_gpu_params* U = D.U;
    ntr_state& s = D.st->s;
    if (D.st->step_budget == 0u) {  // a batch scene that has taken its steps of the call
        if (!D.st->parked) D.st->parked = 1u, D.st->parked_dt = s.dt_ns;
        s.dt_ns = 0;
        return;
    }
    float vmax = s.max_speed;
    uint32_t arrive = U->limits[3];
    for (uint32_t k = 0; k < U->mem[3]; k++) {
        const DBullet& b = D.bullets[k];
        if (b.info.z == 1u) {
            vmax = mx(vmax, b.l.w);
        } else if (b.info.z == 0u) {
            if (b.info.x > s.t_ns)
                arrive = min(arrive, b.info.x);
            else
                vmax = mx(vmax, length(xyz(b.v)));
        }
    }
    float mem_dt = s.mem_dt, air_dt = s.air_dt;
    float dt_s = mn(U->fluid[2], s.cap_dt);
    if (vmax > 0.0f) dt_s = mn(dt_s, U->fluid[1] * U->origin[3] / vmax);
    s.dt_flow = dt_s;
    s.mem_dt_seen = mem_dt;
    s.air_dt_seen = air_dt;
    dt_s = mn(dt_s, mn((float)U->mem[1] * mem_dt, (float)U->mem[2] * air_dt));
    if (s.free_dt_ns > 0u) dt_s = mn(dt_s, 1.25f * (float)s.free_dt_ns * 1e-9f);
    uint32_t free_ns = max(f2u(dt_s * 1e9f), 20u);
    uint32_t stop = U->limits[3];
    const uint32_t budget = D.st->step_budget;
    bool live = s.t_ns < stop;
    uint32_t dt_ns = 0;
    if (live) {
        if (budget != 0xFFFFFFFFu) D.st->step_budget = budget - 1u;
        dt_ns = min(free_ns, min(stop, arrive) - s.t_ns);
        s.free_dt_ns = free_ns;
        s.t_ns += dt_ns;
        s.step += 1;
        s.max_speed = 0.0f;
        s.mem_dt = __uint_as_float(FLT_MAX_BITS);
        s.cap_dt = __uint_as_float(FLT_MAX_BITS);
        s.air_dt = __uint_as_float(FLT_MAX_BITS);
        s.mem_ticket = 0;
        s.n_blocks_prev = min(s.n_blocks, U->bdims[3]);
        s.n_blocks = 0;
        D.st->nbrk = 0;
    }
    s.dt_ns = dt_ns;
}
__global__ void k_begin_step(Dev D) { begin_step_body(D, HwCta{}); }
__global__ void k_begin_step_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    begin_step_body(sD, c);
}

// ---- clear: the last step's transfer sums, and this step's bitmask ----------------------------
// Fields 0..7 of the sums are written whole by k_p2g_gather and A_N by k_p2g; the rest
// accumulate atomically and start from zero. The two clears run on different streams.
template <class CT>
__device__ __forceinline__ void clear_acc_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t ncell = st->s.n_blocks_prev * 64u;
    const size_t stride = (size_t)C.nx() * blockDim.x;
    const size_t tid = (size_t)C.x() * blockDim.x + threadIdx.x;
    constexpr uint32_t F0 = A_MF, NF = NTR_ACC_FIELDS - A_MF;
    for (size_t i = tid; i < (size_t)ncell * NF; i += stride) {
        size_t f = i / ncell, c = i - f * ncell;
        D.acc[(F0 + f) * D.cap_cells + c] = 0;
    }
}
__global__ void k_clear_acc(Dev D) { clear_acc_body(D, HwCta{}); }
__global__ void k_clear_acc_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    clear_acc_body(sD, c);
}

template <class CT>
__device__ __forceinline__ void clear_mask_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    uint32_t* m = D.mask[cur_of(st)];
    for (size_t w = (size_t)C.x() * blockDim.x + threadIdx.x; w < D.nwords; w += (size_t)C.nx() * blockDim.x) m[w] = 0u;
}
__global__ void k_clear_mask(Dev D) { clear_mask_body(D, HwCta{}); }
__global__ void k_clear_mask_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    clear_mask_body(sD, c);
}

// Sets the bits of the blocks `slot` of the lanes where `valid`: one atomicOr per distinct
// word of the bitmask in the warp, with the bits of all its lanes. All 32 lanes call it.
__device__ __forceinline__ void set_block_bits(uint32_t* mask, uint32_t slot, bool valid) {
    const uint32_t word = valid ? slot >> 5 : NONE;
    const uint32_t peers = __match_any_sync(0xffffffffu, word);
    const uint32_t bits = __reduce_or_sync(peers, valid ? 1u << (slot & 31u) : 0u);
    if (valid && (__ffs(peers) - 1) == (int)(threadIdx.x & 31u)) atomicOr(mask + word, bits);
}

__host__ __device__ __forceinline__ uint32_t warp_round(uint32_t n) { return (n + 31u) & ~31u; }

// ---- mark: particles' stencils, active air, dry rubber (fluid.wgsl:131-150, air.wgsl:271-277,
// membrane.wgsl:164-180). Three ranges of threads, each a whole number of warps: one thread per
// particle, per last-step block (up to the block capacity), per vertex. Every lane of a warp
// runs the same loop, so the bits are merged per warp before they go out.
template <class CT>
__device__ __forceinline__ void mark_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const int cur = cur_of(st);
    const Grid g = grid_of(D, cur);
    const uint32_t n_prev = st->s.n_blocks_prev;
    uint32_t* mask = D.mask[cur];
    const uint32_t i = C.x() * blockDim.x + threadIdx.x;
    const I3 bmax = {(int32_t)g.bd[0] - 1, (int32_t)g.bd[1] - 1, (int32_t)g.bd[2] - 1};
    auto clampb = [&](I3 b) {
        return I3{min(max(b.x, 0), bmax.x), min(max(b.y, 0), bmax.y), min(max(b.z, 0), bmax.z)};
    };
    const uint32_t np_w = warp_round(D.Np), nb_w = warp_round(D.cap_blocks);
    if (i < np_w) {
        // The up to 2x2x2 blocks of a particle's stencil.
        const bool isp = i < D.Np;
        bool alive = false;
        I3 lo = {0, 0, 0}, hi = {-1, -1, -1};
        if (isp) {
            float4 p = D.pos[i];
            alive = D.vel[i].w >= 0.5f;
            I3 c = own_cell(g, xyz(p));
            lo = clampb(shr2(c - I3{1, 1, 1}));
            hi = clampb(shr2(c + I3{2, 2, 2}));
            I3 ob = shr2(c);
            D.pslot[i] = (alive && in_bd(g, ob)) ? block_slot(g, ob) : NONE;
        }
        for (int k = 0; k < 8; k++) {
            I3 b = {lo.x + (k & 1), lo.y + ((k >> 1) & 1), lo.z + ((k >> 2) & 1)};
            bool valid = alive && b.x <= hi.x && b.y <= hi.y && b.z <= hi.z;
            set_block_bits(mask, valid ? block_slot(g, b) : 0u, valid);
        }
        return;
    }
    uint32_t j = i - np_w;
    if (j < nb_w) {
        const bool valid = j < n_prev && D.block_active[j] != 0u;
        set_block_bits(mask, valid ? D.block_list[cur ^ 1][j] : 0u, valid);
        return;
    }
    j -= nb_w;
    if (j >= warp_round(D.Nv)) return;
    // Dry rubber: the blocks within two cells of the vertex (at most 3 per axis).
    bool dry = false;
    I3 lo = {0, 0, 0}, hi = {-1, -1, -1};
    if (j < D.Nv) {
        float2 push = D.mem_push[j];
        bool on_water = D.mem_mass[j] > 0.0f && D.mem_water[j].w >= CONTACT_F;
        dry = !(push.y <= 0.0f || on_water);
        if (dry) {
            I3 c = own_cell(g, xyz(D.mem_x[0][j]));
            lo = clampb(shr2(c - I3{2, 2, 2}));
            hi = clampb(shr2(c + I3{3, 3, 3}));
        }
    }
    if (!__any_sync(0xffffffffu, dry)) return;
    for (int k = 0; k < 27; k++) {
        I3 b = {lo.x + k / 9, lo.y + (k / 3) % 3, lo.z + k % 3};
        bool valid = dry && b.x <= hi.x && b.y <= hi.y && b.z <= hi.z;
        set_block_bits(mask, valid ? block_slot(g, b) : 0u, valid);
    }
}
__global__ void k_mark(Dev D) { mark_body(D, HwCta{}); }
__global__ void k_mark_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    mark_body(sD, c);
}

// ---- compaction of the bitmask: blocks numbered in ascending slot order ----------------------
constexpr int SCAN_T = 256, SCAN_W = 8;  // 2048 words per CTA

template <class CT>
__device__ __forceinline__ void scan_words_a_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t* m = D.mask[cur_of(st)];
    uint32_t base = C.x() * SCAN_T * SCAN_W;
    uint32_t s = 0;
    for (int k = 0; k < SCAN_W; k++) {
        uint32_t w = base + k * SCAN_T + threadIdx.x;
        if (w < D.nwords) s += __popc(m[w]);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ uint32_t ws[SCAN_T / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < SCAN_T / 32; k++) t += ws[k];
        D.cta_sum[C.x()] = t;
    }
}
__global__ void __launch_bounds__(SCAN_T) k_scan_words_a(Dev D) { scan_words_a_body(D, HwCta{}); }
__global__ void __launch_bounds__(SCAN_T) k_scan_words_a_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    scan_words_a_body(sD, c);
}

template <class CT>
__device__ __forceinline__ void scan_words_b_body(const Dev& D, const CT& C) {
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const int cur = cur_of(st);
    const uint32_t* m = D.mask[cur];
    uint32_t* prefix = D.prefix[cur];
    uint32_t* list = D.block_list[cur];
    __shared__ uint32_t s_base, ws[SCAN_T / 32];
    if (threadIdx.x < 32) {
        uint32_t t = 0;
        for (uint32_t k = threadIdx.x; k < C.x(); k += 32) t += D.cta_sum[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) s_base = t;
    }
    // Each thread owns SCAN_W consecutive words.
    uint32_t w0 = C.x() * SCAN_T * SCAN_W + threadIdx.x * SCAN_W;
    uint32_t words[SCAN_W], cnt = 0;
    for (int k = 0; k < SCAN_W; k++) {
        words[k] = (w0 + k < D.nwords) ? m[w0 + k] : 0u;
        cnt += __popc(words[k]);
    }
    uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += v;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    uint32_t wbase = 0;
    for (uint32_t k = 0; k < warp; k++) wbase += ws[k];
    uint32_t run = s_base + wbase + inc - cnt;
    const uint32_t cap = D.cap_blocks;
    for (int k = 0; k < SCAN_W; k++) {
        uint32_t w = w0 + k;
        if (w >= D.nwords) break;
        prefix[w] = run;
        uint32_t bits = words[k];
        while (bits) {
            uint32_t b = __ffs(bits) - 1;
            bits &= bits - 1;
            if (run < cap) list[run] = w * 32u + b;
            run++;
        }
    }
    if (C.x() == C.nx() - 1 && threadIdx.x == SCAN_T - 1) {
        st->s.n_blocks = run;
        if (run > cap) st->s.overflow = 1u;
    }
}
__global__ void __launch_bounds__(SCAN_T) k_scan_words_b(Dev D) { scan_words_b_body(D, HwCta{}); }
__global__ void __launch_bounds__(SCAN_T) k_scan_words_b_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    scan_words_b_body(sD, c);
}

// ---- keys: each live particle's block index ---------------------------------------------------
// ---- stable LSD radix sort of (block index, particle index), 8 bits per pass ------------------
// Pass p orders the elements stably by digit (key >> 8p) & 255, in tiles of RADIX_TILE: a
// digit-major histogram of every tile's digits, a scan of it (each tile's offset in each
// digit's run, and the digits' totals), then the scatter. The keys are each particle's block
// index (NONE, a particle in no block, sorts last); pass 0's values are the particle indices.
constexpr int RADIX_T = 256, RADIX_ITEMS = 16, RADIX_TILE = RADIX_T * RADIX_ITEMS;
// Threads per tile of the keys-and-histogram kernel and of the scatter (more threads than the
// histogram's 256 keep more of a tile's loads in flight).
constexpr int KEYS_T = 1024, KEYS_ITEMS = RADIX_TILE / KEYS_T;
constexpr int SCAT_T = 512, SCAT_WARPS = SCAT_T / 32, SCAT_ITEMS = RADIX_TILE / SCAT_T, SCAT_WARP_ITEMS = RADIX_TILE / SCAT_WARPS;

// Exclusive scan over the first 256 threads of a CTA of NT >= 256 (every thread calls it; the
// others pass 0). Returns the thread's exclusive prefix and sets *total.
template <int NT>
__device__ __forceinline__ uint32_t cta_scan_first256(uint32_t v, uint32_t* total) {
    __shared__ uint32_t ws[NT / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += y;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    uint32_t before = 0, all = 0;
    for (uint32_t w = 0; w < 8; w++) {
        if (w < warp) before += ws[w];
        all += ws[w];
    }
    __syncthreads();
    *total = all;
    return before + inc - v;
}

// Adds one digit per lane to a tile's histogram in shared memory: the lanes holding a digit
// agree on it (match) and the lowest of them adds their count. Digit 256: nothing.
__device__ __forceinline__ void tile_hist_add(uint32_t* h, uint32_t d) {
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (d < 256u && (__ffs(peers) - 1) == (int)(threadIdx.x & 31u)) atomicAdd(&h[d], (uint32_t)__popc(peers));
}

// The sort keys and pass 0's histogram in one read of the particles' block slots: each
// particle's block index (fluid.wgsl:109-125's claim, canonical: the slot's rank in the block
// bitmask) and its tile's count of each low digit. Also zeroes the tile's column of pass 1's
// histogram, which pass 0's scatter fills.
template <class CT>
__device__ __forceinline__ void keys_hist_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const int cur = cur_of(st);
    __shared__ uint32_t h[256];
    if (threadIdx.x < 256) {
        h[threadIdx.x] = 0;
        if (D.radix_passes > 1) D.hist2[threadIdx.x * D.n_tiles + C.x()] = 0u;
    }
    __syncthreads();
    const uint32_t base = C.x() * RADIX_TILE;
    uint32_t slot[KEYS_ITEMS];
#pragma unroll
    for (int r = 0; r < KEYS_ITEMS; r++) {  // every load first
        const uint32_t i = base + r * KEYS_T + threadIdx.x;
        slot[r] = i < D.Np ? D.pslot[i] : NONE;
    }
    uint32_t key[KEYS_ITEMS];
#pragma unroll
    for (int r = 0; r < KEYS_ITEMS; r++)
        key[r] = slot[r] == NONE ? NONE : lookup(D.mask[cur], D.prefix[cur], slot[r], D.cap_blocks);
#pragma unroll
    for (int r = 0; r < KEYS_ITEMS; r++) {
        const uint32_t i = base + r * KEYS_T + threadIdx.x;
        if (i < D.Np) D.key[i] = key[r];
        tile_hist_add(h, i < D.Np ? (key[r] & 255u) : 256u);
    }
    __syncthreads();
    if (threadIdx.x < 256) D.hist[threadIdx.x * D.n_tiles + C.x()] = h[threadIdx.x];
}
__global__ void __launch_bounds__(KEYS_T) k_keys_hist(Dev D) { keys_hist_body(D, HwCta{}); }
__global__ void __launch_bounds__(KEYS_T) k_keys_hist_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    keys_hist_body(sD, c);
}

// A pass's histogram from its input keys (the passes no earlier kernel counted).
template <class CT>
__device__ __forceinline__ void radix_hist_body(const Dev& D, const CT& C, uint32_t* hist, const uint32_t* keys, uint32_t shift) {
    if (D.st->s.dt_ns == 0) return;
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = C.x() * RADIX_TILE;
    for (int r = 0; r < RADIX_ITEMS; r++) {
        const uint32_t i = base + r * RADIX_T + threadIdx.x;
        tile_hist_add(h, i < D.Np ? (keys[i] >> shift) & 255u : 256u);
    }
    __syncthreads();
    hist[threadIdx.x * D.n_tiles + C.x()] = h[threadIdx.x];
}
__global__ void __launch_bounds__(RADIX_T) k_radix_hist(Dev D, uint32_t* hist, const uint32_t* keys, uint32_t shift) { radix_hist_body(D, HwCta{}, hist, keys, shift); }

// Exclusive scan of 256 values held one per thread of a 256-thread CTA; returns the thread's
// exclusive prefix and sets *total.
__device__ __forceinline__ uint32_t cta_scan256(uint32_t v, uint32_t* total) {
    __shared__ uint32_t ws[8];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += y;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    uint32_t before = 0, all = 0;
    for (uint32_t w = 0; w < 8; w++) {
        if (w < warp) before += ws[w];
        all += ws[w];
    }
    __syncthreads();
    *total = all;
    return before + inc - v;
}

// The digit-major histogram (digit, then tile): CTA d scans its digit's column of tile
// counts into offsets within the digit, and records the digit's total.
template <class CT>
__device__ __forceinline__ void radix_scan_body(const Dev& D, const CT& C, uint32_t* hist) {
    if (D.st->s.dt_ns == 0) return;
    const uint32_t d = C.x(), nt = D.n_tiles;
    uint32_t* col = hist + (size_t)d * nt;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nt; base += 256) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nt ? col[i] : 0u;
        uint32_t total;
        const uint32_t ex = cta_scan256(v, &total);
        if (i < nt) col[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) D.coltot[d] = carry;
}
__global__ void __launch_bounds__(256) k_radix_scan(Dev D, uint32_t* hist) { radix_scan_body(D, HwCta{}, hist); }

// One tile of a pass. Warp w takes the tile's elements [512 w, 512 w + 512) in 16 rounds of 32
// and ranks each among the warp's earlier elements of its digit (a match per round and a
// running count per digit in shared memory; no block-wide barrier in the loop). The warps'
// offsets within each digit's run and the runs' starts give every element its place in the
// tile's stable digit order; the tile is reordered in shared memory and written out run by
// run, consecutive threads to consecutive addresses. With hist_next, the same write-out counts
// the next pass's digit per destination tile (a match on (tile, digit) and one global atomic
// per group), which spares that pass its histogram kernel; hist_next must be zero before.
template <class CT>
__device__ __forceinline__ void radix_scatter_body(const Dev& D, const CT& C, const uint32_t* hist, const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out, uint32_t shift, uint32_t* hist_next) {
    if (D.st->s.dt_ns == 0) return;
    __shared__ uint16_t s_wc[SCAT_WARPS][256];  // per warp and digit: the running count, then the warp's offset
    __shared__ uint32_t s_dstart[256];          // where each digit's run starts in the tile
    __shared__ uint32_t s_gbase[256];           // where it starts in the output
    __shared__ uint32_t s_k[RADIX_TILE], s_v[RADIX_TILE];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t base = C.x() * RADIX_TILE;
    const uint32_t n_here = D.Np > base ? min((uint32_t)RADIX_TILE, D.Np - base) : 0u;
    for (uint32_t e = threadIdx.x; e < SCAT_WARPS * 256; e += SCAT_T) (&s_wc[0][0])[e] = 0;
    const uint32_t wbase = base + warp * SCAT_WARP_ITEMS;
    uint32_t key[SCAT_ITEMS], val[SCAT_ITEMS], rank[SCAT_ITEMS];
#pragma unroll
    for (int r = 0; r < SCAT_ITEMS; r++) {  // every load first
        const uint32_t i = wbase + r * 32 + lane;
        const bool in = i < D.Np;
        key[r] = in ? keys_in[i] : NONE;
        val[r] = in ? (vals_in ? vals_in[i] : i) : 0u;
    }
    __syncthreads();
    const uint32_t lower_mask = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < SCAT_ITEMS; r++) {
        const bool in = wbase + r * 32 + lane < D.Np;
        const uint32_t d = in ? (key[r] >> shift) & 255u : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t lower = __popc(peers & lower_mask);
        const uint32_t cnt = in ? s_wc[warp][d] : 0u;
        __syncwarp();
        if (in && lower == 0) s_wc[warp][d] = (uint16_t)(cnt + __popc(peers));
        __syncwarp();
        rank[r] = cnt + lower;
    }
    __syncthreads();
    uint32_t run = 0, cold = 0;
    if (threadIdx.x < 256) {
        const uint32_t d = threadIdx.x;
#pragma unroll
        for (int w = 0; w < SCAT_WARPS; w++) {
            const uint32_t c = s_wc[w][d];
            s_wc[w][d] = (uint16_t)run;
            run += c;
        }
        cold = D.coltot[d];
    }
    uint32_t total;
    const uint32_t dstart = cta_scan_first256<SCAT_T>(run, &total);
    const uint32_t digit_base = cta_scan_first256<SCAT_T>(cold, &total);
    if (threadIdx.x < 256) {
        s_dstart[threadIdx.x] = dstart;
        s_gbase[threadIdx.x] = digit_base + hist[threadIdx.x * D.n_tiles + C.x()];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SCAT_ITEMS; r++) {
        if (wbase + r * 32 + lane >= D.Np) continue;
        const uint32_t d = (key[r] >> shift) & 255u;
        const uint32_t p = s_dstart[d] + s_wc[warp][d] + rank[r];
        s_k[p] = key[r];
        s_v[p] = val[r];
    }
    __syncthreads();
    for (uint32_t j0 = 0; j0 < n_here; j0 += SCAT_T) {
        const uint32_t j = j0 + threadIdx.x;
        const bool in = j < n_here;
        uint32_t k = 0u, g = 0u;
        if (in) {
            k = s_k[j];
            const uint32_t d = (k >> shift) & 255u;
            g = s_gbase[d] + (j - s_dstart[d]);
            keys_out[g] = k;
            vals_out[g] = s_v[j];
        }
        if (hist_next) {
            const uint32_t dn = (k >> (shift + 8u)) & 255u;
            const uint32_t combo = in ? ((g / (uint32_t)RADIX_TILE) << 8) | dn : 0xFFFFFFFFu;
            const uint32_t peers = __match_any_sync(0xffffffffu, combo);
            if (in && (__ffs(peers) - 1) == (int)lane)
                atomicAdd(hist_next + dn * D.n_tiles + (g / (uint32_t)RADIX_TILE), (uint32_t)__popc(peers));
        }
    }
}
__global__ void __launch_bounds__(SCAT_T) k_radix_scatter(Dev D, const uint32_t* hist, const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out, uint32_t shift, uint32_t* hist_next) { radix_scatter_body(D, HwCta{}, hist, keys_in, vals_in, keys_out, vals_out, shift, hist_next); }

// The buffers of pass p of the step's sort, as the host's loop of a one-scene step passes
// them: keys and values in (the particle indices on pass 0) and out (the last pass writes the
// final arrays), the pass's histogram, and the next pass's when this pass's scatter counts it.
struct RadixPass {
    const uint32_t *kin, *vin;
    uint32_t *kout, *vout, *hist, *next;
    uint32_t shift;
};
__device__ __forceinline__ bool radix_to_final(const Dev& D, uint32_t p) { return ((D.radix_passes - 1u - p) % 2u) == 0u; }
__device__ __forceinline__ RadixPass radix_pass(const Dev& D, uint32_t p) {
    RadixPass r;
    r.kin = p == 0 ? D.key : (radix_to_final(D, p - 1) ? D.key_sorted : D.key_alt);
    r.vin = p == 0 ? nullptr : (radix_to_final(D, p - 1) ? D.sorted : D.val_alt);
    r.kout = radix_to_final(D, p) ? D.key_sorted : D.key_alt;
    r.vout = radix_to_final(D, p) ? D.sorted : D.val_alt;
    r.hist = (p % 2u == 0u) ? D.hist : D.hist2;
    r.next = (p == 0 && D.radix_passes > 1) ? D.hist2 : nullptr;
    r.shift = 8u * p;
    return r;
}
// The sort's kernels over many scenes, pass p (a scene with fewer passes skips it).
__global__ void __launch_bounds__(RADIX_T) k_radix_hist_m(Multi M, uint32_t p) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    if (p >= sD.radix_passes) return;
    const RadixPass r = radix_pass(sD, p);
    radix_hist_body(sD, c, r.hist, r.kin, r.shift);
}
__global__ void __launch_bounds__(256) k_radix_scan_m(Multi M, uint32_t p) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    if (p >= sD.radix_passes) return;
    radix_scan_body(sD, c, radix_pass(sD, p).hist);
}
__global__ void __launch_bounds__(SCAT_T) k_radix_scatter_m(Multi M, uint32_t p) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    if (p >= sD.radix_passes) return;
    const RadixPass r = radix_pass(sD, p);
    radix_scatter_body(sD, c, r.hist, r.kin, r.vin, r.kout, r.vout, r.shift, r.next);
}

// block_start from the sorted keys: block b starts at the first position whose key is >= b.
template <class CT>
__device__ __forceinline__ void block_bounds_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t nb = min(st->s.n_blocks, D.cap_blocks);
    const uint32_t* ks = D.key_sorted;
    for (uint32_t p = C.x() * blockDim.x + threadIdx.x; p <= D.Np; p += C.nx() * blockDim.x) {
        int64_t k = p < D.Np ? (int64_t)min(ks[p], nb) : (int64_t)nb;
        int64_t kp = p > 0 ? (int64_t)min(ks[p - 1], nb) : -1;
        for (int64_t b = kp + 1; b <= k; b++) D.block_start[b] = p;
    }
}
__global__ void k_block_bounds(Dev D) { block_bounds_body(D, HwCta{}); }
__global__ void k_block_bounds_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    block_bounds_body(sD, c);
}

// ---- P2G, fluid.wgsl:198-303 -----------------------------------------------------------------
// One block per iteration of a CTA: the block's particles add into a 7^3 x 8-field tile of i32
// fixed-point sums in shared memory, which then goes out to the grid with one atomic add per
// nonzero tile entry. Fixed-point sums do not depend on the order of the adds.
constexpr int P2G_T = 256;
// The P2G tile in shared memory: 7 x 7 x 7 nodes per field with strides (68, 8, 1) and 476
// words per field instead of (49, 7, 1) and 343. The 32 lanes of an atomic are 32 particles in
// 32 cells of one half of the block (the layered order below): with these strides their nodes
// at any one stencil offset fall in 32 different banks (x strides 0, 4, 8, 12 mod 32, y 0, 8,
// 16, 24, z 0-3), where the packed strides put pairs of them in one bank.
constexpr uint32_t TPX = 68, TPY = 8, TPF = 7 * TPX;

__device__ __forceinline__ void splat(int32_t* tile, V3 x, V3 o, I3 corner, uint32_t fa, float val, V3 grad, uint32_t fw, float scale, float hh) {
    I3 base = vi(vfloor(x - o - 0.5f));
    V3 fx = x - o - vf(base);
    V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    I3 t = base - corner;
    uint32_t t0 = (uint32_t)t.x * TPX + (uint32_t)t.y * TPY + (uint32_t)t.z;
    V3 hg = grad * hh;
    // The weights are products of three B-spline factors in [0, 0.75], and a node's value is at
    // most |val| + 1.5 |hg|_1 in size (every node - fx is within 1.5 per axis). When that bound
    // times the scale is well below 2^22 (and nothing is infinite or NaN), every to_fp of the
    // stencil is the rounding by addition (weight * 2^24 < 2^23 as well); otherwise convert.
    const float bound = fabsf(val) + 1.5f * (fabsf(hg.x) + fabsf(hg.y) + fabsf(hg.z));
    if (bound * scale < 4.0e6f && fabsf(fx.x) + fabsf(fx.y) + fabsf(fx.z) < 8.0f) {
#pragma unroll
        for (uint32_t a = 0; a < 3; a++)
#pragma unroll
            for (uint32_t b = 0; b < 3; b++)
#pragma unroll
                for (uint32_t c = 0; c < 3; c++) {
                    float weight = wx[a] * wy[b] * wz[c];
                    uint32_t tt = t0 + a * TPX + b * TPY + c;
                    float node = val + dot(hg, v3((float)a, (float)b, (float)c) - fx);
                    atomicAdd(&tile[fa * TPF + tt], fp_round(__fmul_rn(weight * node, scale)));
                    atomicAdd(&tile[fw * TPF + tt], fp_round_pos(__fmul_rn(weight, FP_W)));
                }
    } else {
#pragma unroll 1
        for (uint32_t a = 0; a < 3; a++)
            for (uint32_t b = 0; b < 3; b++)
                for (uint32_t c = 0; c < 3; c++) {
                    float weight = wx[a] * wy[b] * wz[c];
                    uint32_t tt = t0 + a * TPX + b * TPY + c;
                    float node = val + dot(hg, v3((float)a, (float)b, (float)c) - fx);
                    atomicAdd(&tile[fa * TPF + tt], to_fp(weight * node, scale));
                    atomicAdd(&tile[fw * TPF + tt], to_fp(weight, FP_W));
                }
    }
}

__device__ __forceinline__ uint32_t tile_cell(const uint32_t* links, uint32_t t) {
    I3 rel = {(int32_t)(t / 49u) - 1, (int32_t)((t / 7u) % 7u) - 1, (int32_t)(t % 7u) - 1};
    I3 nb = {(rel.x + 4) / 4 - 1, (rel.y + 4) / 4 - 1, (rel.z + 4) / 4 - 1};
    uint32_t b = links[(uint32_t)((nb.x + 1) * 9 + (nb.y + 1) * 3 + nb.z + 1)];
    if (b == NONE) return NONE;
    I3 l = rel - nb * 4;
    return b * 64u + (uint32_t)l.x * 16u + (uint32_t)l.y * 4u + (uint32_t)l.z;
}

// P2G by stencil groups. Particles of one cell whose stencils on a lattice start at the same
// node add to the same 27 nodes of the tile: for a face lattice these are the particles of the
// cell on one side of its middle along that lattice's axis (the half decides whether the
// stencil starts at the cell below or at the cell itself); the cell-centred lattice's stencil is
// the same for the whole cell, which is split in two by its x half. A thread owns one such group
// (a lattice, a cell, a half) and sums its particles' rounded i32 contributions to the 27 nodes
// in registers, then adds each node's sum to the tile with one shared atomic, instead of one
// atomic per particle and node. Integer sums do not depend on the order of the adds, so the tile
// is the same as the particle-by-particle splat's, bit for bit.
//
// A block's particles are taken in chunks of P2G_CHUNK. Each chunk's particles are counted by
// (cell, octant) (octant = the particle's half of its cell along each axis, from the same float
// expressions as the stencils' first nodes), the counts scanned, and the particles' values
// staged in shared memory in (cell, x half, y half, z half) order: position in cells and the
// cell-centred value, and per face lattice the velocity component and h times the affine row.
// Two lists of staged indices put the same particles in (cell, y half, x half, z half) and
// (cell, z half, x half, y half) order, so that every group is one contiguous run: in the staged
// order for the x faces and the cell centres, in those lists for the y and z faces. Each
// lattice's non-empty groups are listed most particles first, and its threads take them in that
// order: the lanes of a warp, all on one lattice, loop over similar counts. A particle whose
// values would leave the range in which the rounding by addition is exact on any lattice (or that
// are not finite) takes the particle-by-particle splat instead.
constexpr uint32_t P2G_CHUNK = 2 * P2G_T;
constexpr uint32_t P2G_KEYS = 64 * 8;  // (cell, octant)
constexpr uint16_t P2G_ODD = 0xffffu;
constexpr uint32_t P2G_BUCKETS = 16;   // groups sorted by min(particles, 15), most first

struct P2GShared {
    float4 x[P2G_CHUNK];      // position in cells, w = the cell-centred value (pressure / 1e6)
    float4 g[3][P2G_CHUNK];   // per face lattice: h * affine row, w = velocity component
    int32_t tile[8 * TPF];
    uint32_t start[P2G_KEYS + 1];         // key counts, then where each key's run starts
    uint16_t lst[2][P2G_CHUNK];           // staged indices in y-half and in z-half order
    uint8_t pre[2][64][8];                // per cell and octant: where its run starts in those orders, in the cell
    uint16_t items[4][128];               // per lattice: its groups (cell * 2 + half), most particles first
    uint32_t bucket[4][P2G_BUCKETS + 1];  // per lattice: groups per count, then where they start
    uint32_t odd[P2G_CHUNK];
    uint32_t own[64];
    uint32_t warp_sum[P2G_T / 32];
    uint32_t n_odd;
};
constexpr size_t P2G_SMEM = sizeof(P2GShared);

// The fast-path test of splat() for one lattice: the rounding by addition is exact when every
// node value times the scale is well inside 2^22 and nothing is infinite or NaN.
__device__ __forceinline__ bool p2g_fast(float val, V3 hg, V3 fx, float scale) {
    const float bound = fabsf(val) + 1.5f * (fabsf(hg.x) + fabsf(hg.y) + fabsf(hg.z));
    return bound * scale < 4.0e6f && fabsf(fx.x) + fabsf(fx.y) + fabsf(fx.z) < 8.0f;
}

// Octant o = (x half, y half, z half) as bits 2, 1, 0; its place in the y-half and z-half orders.
__device__ __forceinline__ uint32_t oct_y_first(uint32_t o) { return ((o >> 1) & 1u) << 2 | (o >> 2) << 1 | (o & 1u); }
__device__ __forceinline__ uint32_t oct_z_first(uint32_t o) { return (o & 1u) << 2 | (o >> 2) << 1 | ((o >> 1) & 1u); }

// One group's sums. Lattice L: 0, 1, 2 the faces along x, y, z (offset 0 along that axis, 0.5
// along the others), 3 the cell centres. The group is the run [lo, hi) of the staged order (x
// faces, cell centres) or of the y-half or z-half list; `b` is the stencil's first node
// (domain cells, as floats), `t0` its tile index.
template <int L>
__device__ __forceinline__ void p2g_group(P2GShared& S, uint32_t lo, uint32_t hi, V3 b, uint32_t t0) {
    int32_t sv[27], sw[27];
#pragma unroll
    for (int k = 0; k < 27; k++) sv[k] = 0, sw[k] = 0;
#pragma unroll 1
    for (uint32_t q = lo; q < hi; q++) {
        const uint32_t j = (L == 1 || L == 2) ? (uint32_t)S.lst[L - 1][q] : q;
        const float4 X = S.x[j];
        // x - o per axis (x - 0 is x), then the offset from the stencil's first node.
        const V3 xo = {L == 0 ? X.x : X.x - 0.5f, L == 1 ? X.y : X.y - 0.5f, L == 2 ? X.z : X.z - 0.5f};
        const V3 fx = xo - b;
        const V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
        // The fixed-point scales are powers of two, so scaling is exact: weight16 = weight * 2^16
        // (wx taken times 2^16 first), its value t = weight16 * node = (weight * node) * 2^16, and
        // weight16 * 2^8 = weight * 2^24, bit for bit the splat's products. Pairs of them go
        // through the packed FP32 instructions (each lane rounds as the scalar one would).
        const float wx16[3] = {wx[0] * FP_M, wx[1] * FP_M, wx[2] * FP_M};
        const float2 mag = make_float2(12582912.0f, 8388608.0f);
        if (L < 3) {
            const float4 G = S.g[L][j];
            // hg . ((a, b, c) - fx) as the splat sums it: (x term + y term) + z term.
            const float px[3] = {G.x * (0.0f - fx.x), G.x * (1.0f - fx.x), G.x * (2.0f - fx.x)};
            const float py[3] = {G.y * (0.0f - fx.y), G.y * (1.0f - fx.y), G.y * (2.0f - fx.y)};
            const float pz[3] = {G.z * (0.0f - fx.z), G.z * (1.0f - fx.z), G.z * (2.0f - fx.z)};
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int bb = 0; bb < 3; bb++) {
                    const float wab16 = wx16[a] * wy[bb];
                    const float sab = px[a] + py[bb];
                    const float2 w01 = __fmul2_rn(make_float2(wab16, wab16), make_float2(wz[0], wz[1]));
                    const float2 n01 = __fadd2_rn(make_float2(G.w, G.w), __fadd2_rn(make_float2(sab, sab), make_float2(pz[0], pz[1])));
                    const float w2 = wab16 * wz[2];
                    const float n2 = G.w + (sab + pz[2]);
                    const float2 r0 = __fadd2_rn(__fmul2_rn(make_float2(w01.x, w01.x), make_float2(n01.x, 256.0f)), mag);
                    const float2 r1 = __fadd2_rn(__fmul2_rn(make_float2(w01.y, w01.y), make_float2(n01.y, 256.0f)), mag);
                    const float2 r2 = __fadd2_rn(__fmul2_rn(make_float2(w2, w2), make_float2(n2, 256.0f)), mag);
                    const int k = a * 9 + bb * 3;
                    sv[k] += __float_as_int(r0.x), sw[k] += __float_as_int(r0.y);
                    sv[k + 1] += __float_as_int(r1.x), sw[k + 1] += __float_as_int(r1.y);
                    sv[k + 2] += __float_as_int(r2.x), sw[k + 2] += __float_as_int(r2.y);
                }
        } else {
            // No affine term: the node value is the particle's (adding the dot product of a
            // zero gradient changes at most the sign of a zero, which rounds to 0 either way).
            const float2 val = make_float2(X.w, 256.0f);
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int bb = 0; bb < 3; bb++) {
                    const float wab16 = wx16[a] * wy[bb];
                    const float2 w01 = __fmul2_rn(make_float2(wab16, wab16), make_float2(wz[0], wz[1]));
                    const float w2 = wab16 * wz[2];
                    const float2 r0 = __fadd2_rn(__fmul2_rn(make_float2(w01.x, w01.x), val), mag);
                    const float2 r1 = __fadd2_rn(__fmul2_rn(make_float2(w01.y, w01.y), val), mag);
                    const float2 r2 = __fadd2_rn(__fmul2_rn(make_float2(w2, w2), val), mag);
                    const int k = a * 9 + bb * 3;
                    sv[k] += __float_as_int(r0.x), sw[k] += __float_as_int(r0.y);
                    sv[k + 1] += __float_as_int(r1.x), sw[k + 1] += __float_as_int(r1.y);
                    sv[k + 2] += __float_as_int(r2.x), sw[k + 2] += __float_as_int(r2.y);
                }
        }
    }
    const uint32_t n = hi - lo;
    if (n == 0) return;
    // Each sum carries n times the rounding constant's bits; take them off (mod 2^32).
    const int32_t ov = (int32_t)(n * 0x4B400000u), ow = (int32_t)(n * 0x4B000000u);
    const uint32_t fa = L < 3 ? 2u * L : (uint32_t)A_PC, fw = L < 3 ? 2u * L + 1u : (uint32_t)A_WC;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int bb = 0; bb < 3; bb++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const uint32_t t = t0 + a * TPX + bb * TPY + c;
                const int k = a * 9 + bb * 3 + c;
                atomicAdd(&S.tile[fa * TPF + t], sv[k] - ov);
                atomicAdd(&S.tile[fw * TPF + t], sw[k] - ow);
            }
}

// Particles of group (lattice L, cell, half h) in its run: the particle count and the run's start.
__device__ __forceinline__ void p2g_run(const P2GShared& S, uint32_t L, uint32_t cell, uint32_t h, uint32_t& lo, uint32_t& hi) {
    const uint32_t k0 = cell * 8u, base = S.start[k0];
    if (L == 0 || L == 3) {  // x half: octants 4h .. 4h + 3 of the staged order
        lo = S.start[k0 + 4u * h], hi = S.start[k0 + 4u * h + 4u];
    } else {  // y or z half: the cell's run in that order, up to the first octant of the upper half
        // (octant 2 = y half 1 alone, octant 1 = z half 1 alone, where that order starts it)
        const uint32_t n = S.start[k0 + 8u] - base;
        const uint32_t lower = S.pre[L - 1][cell][L == 1 ? 2 : 1];
        lo = base + (h ? lower : 0u);
        hi = base + (h ? n : lower);
    }
}

// One block per iteration of a CTA; the tile is stored whole and k_p2g_gather sums the tiles
// that overlap each cell.
template <class CT>
__device__ __forceinline__ void p2g_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    extern __shared__ __align__(16) unsigned char p2g_smem[];
    P2GShared& S = *reinterpret_cast<P2GShared*>(p2g_smem);
    const Grid g = grid_of(D, cur_of(st));
    const uint32_t nb = min(st->s.n_blocks, D.cap_blocks);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const float hh = g.h;
    for (uint32_t b = C.x(); b < nb; b += C.nx()) {
        const I3 bc = slot_coord(g, g.list[b]);
        if (tid < 27) {
            I3 n = bc + I3{(int32_t)(tid / 9u), (int32_t)((tid / 3u) % 3u), (int32_t)(tid % 3u)} - I3{1, 1, 1};
            D.block_nb[b * 27u + tid] = block_at(g, n);
        }
        if (tid < 64) S.own[tid] = 0;
        const uint32_t first = D.block_start[b];
        const uint32_t count = D.block_start[b + 1] - first;
        if (count == 0) {
            if (tid < 64) D.acc[(size_t)A_N * D.cap_cells + b * 64u + tid] = 0;
            if (tid == 0) D.tile_ok[b] = 0u;
            __syncthreads();
            continue;
        }
        for (uint32_t t = tid; t < 8 * TPF; t += P2G_T) S.tile[t] = 0;
        const I3 corner = bc * 4 - I3{1, 1, 1};
        for (uint32_t chunk = 0; chunk < count; chunk += P2G_CHUNK) {
            const uint32_t n = min(P2G_CHUNK, count - chunk);
            for (uint32_t k = tid; k < P2G_KEYS; k += P2G_T) S.start[k] = 0;
            if (tid < 4 * (P2G_BUCKETS + 1)) (&S.bucket[0][0])[tid] = 0;
            if (tid == 0) S.n_odd = 0;
            __syncthreads();
            // Each thread's two particles: key, rank in its key, and the staged values, kept in
            // registers until the keys' starts are known.
            uint32_t key[2], rank[2];
            float4 vx[2], vg[2][3];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const uint32_t j = tid + q * P2G_T;
                key[q] = P2G_ODD;
                if (j >= n) continue;
                const uint32_t i = D.sorted[first + chunk + j];
                const float4 pos = D.pos[i], vel = D.vel[i], c0 = D.c0[i], c1 = D.c1[i], c2 = D.c2[i];
                const V3 x = (xyz(pos) - g.org) / hh;
                const I3 own = vi(vfloor(x)) - bc * 4;  // own_cell, in the block
                if ((uint32_t)own.x < 4u && (uint32_t)own.y < 4u && (uint32_t)own.z < 4u)
                    atomicAdd(&S.own[(uint32_t)(own.x * 16 + own.y * 4 + own.z)], 1u);
                // First stencil nodes: offset 0 along an axis gives A, offset 0.5 gives B.
                const V3 xh = {x.x - 0.5f, x.y - 0.5f, x.z - 0.5f};
                const I3 A = vi(vfloor(xh));
                const I3 B = vi(vfloor(xh - 0.5f));
                const I3 l = B - corner;
                const I3 o = A - B;
                // fx of the two offsets: (x - 0) - A and (x - 0.5) - B.
                const V3 fa3 = x - vf(A), fb3 = xh - vf(B);
                const V3 hu = xyz(c0) * hh, hv = xyz(c1) * hh, hw = xyz(c2) * hh;
                const float pc = c0.w * 1e-6f;
                bool ok = l.x == own.x && l.y == own.y && l.z == own.z && (uint32_t)own.x < 4u && (uint32_t)own.y < 4u &&
                          (uint32_t)own.z < 4u && (uint32_t)o.x <= 1u && (uint32_t)o.y <= 1u && (uint32_t)o.z <= 1u;
                ok = ok && p2g_fast(vel.x, hu, V3{fa3.x, fb3.y, fb3.z}, FP_M) && p2g_fast(vel.y, hv, V3{fb3.x, fa3.y, fb3.z}, FP_M) &&
                     p2g_fast(vel.z, hw, V3{fb3.x, fb3.y, fa3.z}, FP_M) && p2g_fast(pc, V3{0.0f, 0.0f, 0.0f}, fb3, FP_P);
                if (!ok) {
                    S.odd[atomicAdd(&S.n_odd, 1u)] = i;
                    continue;
                }
                key[q] = (uint32_t)(l.x * 16 + l.y * 4 + l.z) * 8u + (uint32_t)(o.x * 4 + o.y * 2 + o.z);
                rank[q] = atomicAdd(&S.start[key[q]], 1u);
                vx[q] = make_float4(x.x, x.y, x.z, pc);
                vg[q][0] = make_float4(hu.x, hu.y, hu.z, vel.x);
                vg[q][1] = make_float4(hv.x, hv.y, hv.z, vel.y);
                vg[q][2] = make_float4(hw.x, hw.y, hw.z, vel.z);
            }
            __syncthreads();
            // Each cell's octant counts in the y-half and z-half orders (threads 0-63), before
            // the counts become starts.
            uint32_t cnt8[8];
            if (tid < 64) {
#pragma unroll
                for (int o = 0; o < 8; o++) cnt8[o] = S.start[tid * 8 + o];
                uint32_t py = 0, pz = 0;
#pragma unroll
                for (int r = 0; r < 8; r++)
#pragma unroll
                    for (int o = 0; o < 8; o++) {
                        if (oct_y_first(o) == (uint32_t)r) S.pre[0][tid][o] = (uint8_t)py, py += cnt8[o];
                        if (oct_z_first(o) == (uint32_t)r) S.pre[1][tid][o] = (uint8_t)pz, pz += cnt8[o];
                    }
            }
            // Exclusive scan of the 512 key counts: two a thread, warp scans, then the warps'.
            {
                const uint32_t c0n = S.start[2 * tid], c1n = S.start[2 * tid + 1];
                uint32_t inc = c0n + c1n;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xffffffffu, inc, off);
                    if (lane >= (uint32_t)off) inc += v;
                }
                if (lane == 31) S.warp_sum[warp] = inc;
                __syncthreads();
                uint32_t before = 0;
                for (uint32_t w = 0; w < warp; w++) before += S.warp_sum[w];
                const uint32_t ex = before + inc - c0n - c1n;
                S.start[2 * tid] = ex;
                S.start[2 * tid + 1] = ex + c0n;
                if (tid == P2G_T - 1) S.start[P2G_KEYS] = ex + c0n + c1n;
            }
            __syncthreads();
            // Stage the values; the two lists; count each lattice's groups by size.
#pragma unroll
            for (int q = 0; q < 2; q++) {
                if (key[q] == P2G_ODD) continue;
                const uint32_t at = S.start[key[q]] + rank[q];
                S.x[at] = vx[q];
                S.g[0][at] = vg[q][0];
                S.g[1][at] = vg[q][1];
                S.g[2][at] = vg[q][2];
                const uint32_t cell = key[q] >> 3, o = key[q] & 7u, base = S.start[cell * 8u];
                S.lst[0][base + S.pre[0][cell][o] + rank[q]] = (uint16_t)at;
                S.lst[1][base + S.pre[1][cell][o] + rank[q]] = (uint16_t)at;
            }
            uint32_t gsz[2], gslot[2];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const uint32_t it = tid + q * P2G_T, L = it >> 7, cell = (it >> 1) & 63u, h = it & 1u;
                uint32_t lo, hi;
                p2g_run(S, L, cell, h, lo, hi);
                gsz[q] = hi - lo;
                if (gsz[q]) gslot[q] = atomicAdd(&S.bucket[L][P2G_BUCKETS - 1 - min(gsz[q], P2G_BUCKETS - 1)], 1u);
            }
            __syncthreads();
            if (tid < 4) {
                uint32_t at = 0;
                for (uint32_t k = 0; k < P2G_BUCKETS; k++) {
                    const uint32_t c = S.bucket[tid][k];
                    S.bucket[tid][k] = at;
                    at += c;
                }
                S.bucket[tid][P2G_BUCKETS] = at;
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const uint32_t it = tid + q * P2G_T, L = it >> 7;
                if (gsz[q]) S.items[L][S.bucket[L][P2G_BUCKETS - 1 - min(gsz[q], P2G_BUCKETS - 1)] + gslot[q]] = (uint16_t)(it & 127u);
            }
            __syncthreads();
            // Two rounds of groups: warps 0-3 take a lattice's groups and warps 4-7 another's,
            // x faces with y faces, then z faces with the cell centres.
#pragma unroll 1
            for (uint32_t round = 0; round < 2; round++) {
                const uint32_t L = round * 2u + (tid >> 7), k = tid & 127u;
                if (k >= S.bucket[L][P2G_BUCKETS]) continue;
                const uint32_t grp = S.items[L][k], cell = grp >> 1, h = grp & 1u;
                uint32_t lo, hi;
                p2g_run(S, L, cell, h, lo, hi);
                I3 t = {(int32_t)(cell >> 4), (int32_t)((cell >> 2) & 3u), (int32_t)(cell & 3u)};
                if (L == 0) t.x += (int32_t)h;
                else if (L == 1) t.y += (int32_t)h;
                else if (L == 2) t.z += (int32_t)h;
                const V3 base = vf(corner + t);
                const uint32_t t0 = (uint32_t)t.x * TPX + (uint32_t)t.y * TPY + (uint32_t)t.z;
                switch (L) {
                    case 0: p2g_group<0>(S, lo, hi, base, t0); break;
                    case 1: p2g_group<1>(S, lo, hi, base, t0); break;
                    case 2: p2g_group<2>(S, lo, hi, base, t0); break;
                    default: p2g_group<3>(S, lo, hi, base, t0); break;
                }
            }
            // Particles outside the exact fast range: splatted one by one.
            for (uint32_t k = tid; k < S.n_odd; k += P2G_T) {
                const uint32_t i = S.odd[k];
                float4 pos = D.pos[i], vel = D.vel[i], c0 = D.c0[i], c1 = D.c1[i], c2 = D.c2[i];
                V3 x = (xyz(pos) - g.org) / hh;
                splat(S.tile, x, v3(0.0f, 0.5f, 0.5f), corner, 0, vel.x, xyz(c0), 1, FP_M, hh);
                splat(S.tile, x, v3(0.5f, 0.0f, 0.5f), corner, 2, vel.y, xyz(c1), 3, FP_M, hh);
                splat(S.tile, x, v3(0.5f, 0.5f, 0.0f), corner, 4, vel.z, xyz(c2), 5, FP_M, hh);
                splat(S.tile, x, v3(0.5f, 0.5f, 0.5f), corner, A_PC, c0.w * 1e-6f, v3(0.0f, 0.0f, 0.0f), A_WC, FP_P, hh);
            }
            __syncthreads();
        }
        // Stored in the packed layout (8 fields x 343, strides 49, 7, 1) k_p2g_gather reads.
        int32_t* dst = D.tiles + (size_t)b * 8 * TILE;
        for (uint32_t e = tid; e < 8 * TILE; e += P2G_T) {
            const uint32_t f = e / TILE, r = e - f * TILE, x = r / 49u, y = (r - x * 49u) / 7u, z = r - x * 49u - y * 7u;
            dst[e] = S.tile[f * TPF + x * TPX + y * TPY + z];
        }
        if (tid < 64) D.acc[(size_t)A_N * D.cap_cells + b * 64u + tid] = (int32_t)S.own[tid];
        if (tid == 0) D.tile_ok[b] = 1u;
        __syncthreads();
    }
}
__global__ void __launch_bounds__(P2G_T, 2) k_p2g(Dev D) { p2g_body(D, HwCta{}); }
__global__ void __launch_bounds__(P2G_T, 2) k_p2g_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    p2g_body(sD, c);
}

template <class CT>
__device__ __forceinline__ void p2g_gather_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t n_cells = min(st->s.n_blocks, D.cap_blocks) * 64u;
    for (uint32_t cell = C.x() * blockDim.x + threadIdx.x; cell < n_cells; cell += C.nx() * blockDim.x) {
        const uint32_t b = cell >> 6;
        const I3 l = local_coord(cell);
        // The up to 2 x 2 x 2 tiles over the cell: per axis its own block (offset 0) and the one
        // below (l <= 1) or above (l == 3). Their indices, then whether they hold sums, then all
        // their entries, each step's loads in flight together.
        const int ax[2] = {0, l.x <= 1 ? -1 : 1}, ay[2] = {0, l.y <= 1 ? -1 : 1}, az[2] = {0, l.z <= 1 ? -1 : 1};
        const int nx = l.x == 2 ? 1 : 2, ny = l.y == 2 ? 1 : 2, nz = l.z == 2 ? 1 : 2;
        const uint32_t* nbt = D.block_nb + (size_t)b * 27u;
        uint32_t src[8], tix[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int ix = i & 1, iy = (i >> 1) & 1, iz = i >> 2;
            const int ox = ax[ix], oy = ay[iy], oz = az[iz];
            src[i] = (ix < nx && iy < ny && iz < nz) ? nbt[(ox + 1) * 9 + (oy + 1) * 3 + oz + 1] : NONE;
            tix[i] = (uint32_t)(l.x + 1 - 4 * ox) * 49u + (uint32_t)(l.y + 1 - 4 * oy) * 7u + (uint32_t)(l.z + 1 - 4 * oz);
        }
        bool ok[8];
#pragma unroll
        for (int i = 0; i < 8; i++) ok[i] = src[i] != NONE && D.tile_ok[src[i] != NONE ? src[i] : b] != 0u;
        // Integer sums: the same in any order.
        uint32_t s[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int32_t* tp = D.tiles + (size_t)(ok[i] ? src[i] : b) * 8 * TILE + (ok[i] ? tix[i] : 0u);
#pragma unroll
            for (int f = 0; f < 8; f++) s[f] += ok[i] ? (uint32_t)tp[f * TILE] : 0u;
        }
#pragma unroll
        for (int f = 0; f < 8; f++) D.acc[(size_t)f * D.cap_cells + cell] = (int32_t)s[f];
    }
}
__global__ void k_p2g_gather(Dev D) { p2g_gather_body(D, HwCta{}); }
__global__ void k_p2g_gather_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    p2g_gather_body(sD, c);
}

}  // namespace ntr
