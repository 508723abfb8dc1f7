// Kernels of the step up to the transfer to the grid: the step clock, block activation over a
// bitmask, the stable radix sort of particles by block, and APIC P2G in a shared-memory tile.
//
// Reference: shaders/fluid.wgsl:33-303 (begin_step .. p2g), membrane.wgsl:164-180
// (mark_rubber), air.wgsl:271-277 (keep_blocks).
#pragma once

#include "dev.cuh"
#include "kernels_cells.cuh"

namespace ntr {

// ---- begin_step, fluid.wgsl:33-89 ------------------------------------------------------------
template <class CT>
__device__ __forceinline__ void begin_step_body(const Dev& D, const CT& C) {
    if (threadIdx.x != 0 || C.x() != 0) return;
    D.st->next_block[0] = D.st->next_block[1] = 0u;
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
    // Each thread owns SCAN_W consecutive words (two 16-byte loads where all are in range).
    static_assert(SCAN_W == 8, "two uint4 per thread");
    uint32_t w0 = C.x() * SCAN_T * SCAN_W + threadIdx.x * SCAN_W;
    uint32_t words[SCAN_W], cnt = 0;
    if (w0 + SCAN_W <= D.nwords) {
        const uint4 a = *reinterpret_cast<const uint4*>(m + w0), b = *reinterpret_cast<const uint4*>(m + w0 + 4);
        words[0] = a.x, words[1] = a.y, words[2] = a.z, words[3] = a.w;
        words[4] = b.x, words[5] = b.y, words[6] = b.z, words[7] = b.w;
    } else {
        for (int k = 0; k < SCAN_W; k++) words[k] = (w0 + k < D.nwords) ? m[w0 + k] : 0u;
    }
#pragma unroll
    for (int k = 0; k < SCAN_W; k++) cnt += __popc(words[k]);
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
        // lookup() reads a word's prefix only for a set bit of it: the empty words (nearly all
        // of the domain) are not written.
        uint32_t bits = words[k];
        if (bits) prefix[w] = run;
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
// Four CTAs of 256 threads an SM (64 registers, a few spilled): 118 us a step at 1M particles
// against 124 with three CTAs at 80 registers; five: 121.
constexpr int P2G_T = 256;
// The P2G tile in shared memory: 7 x 7 x 7 nodes per field with strides (68, 8, 1) and 476
// words per field instead of (49, 7, 1) and 343. The 32 lanes of an atomic are 32 particles in
// 32 cells of one half of the block (the layered order below): with these strides their nodes
// at any one stencil offset fall in 32 different banks (x strides 0, 4, 8, 12 mod 32, y 0, 8,
// 16, 24, z 0-3), where the packed strides put pairs of them in one bank.
constexpr uint32_t TPX = 68, TPY = 8, TPF = 7 * TPX;

static_assert(FP_M == 65536.0f && FP_P == 65536.0f && FP_W == 16777216.0f, "splat's fused rounding needs power-of-two scales");
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
                    // The scales are powers of two (FP_M, FP_P, FP_W), so the scaling is exact and
                    // one fused multiply-add with the rounding constant rounds once, as the add
                    // after the multiply does: fp_round(x * scale) in one instruction fewer.
                    atomicAdd(&tile[fa * TPF + tt], __float_as_int(__fmaf_rn(weight * node, scale, 12582912.0f)) - 0x4B400000);
                    atomicAdd(&tile[fw * TPF + tt], __float_as_int(__fmaf_rn(weight, FP_W, 8388608.0f)) - 0x4B000000);
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

constexpr uint32_t P2G_CAP = 1024;  // particles of a block ordered at a time
constexpr uint32_t P2G_LAYERS = 64;  // ranks within a cell that get the interleaved order

// One block per iteration of a CTA. Its particles add into a 7^3 x 8-field tile of i32 sums in
// shared memory, in an order that spreads the 32 lanes of an atomic over 32 different cells:
// a counting sort by cell gives each particle its rank in its cell, and the particles are
// taken rank layer by rank layer, cell by cell within a layer (layer r holds the cells with
// more than r particles). Lanes in different cells add to different nodes of the tile, mostly
// in different banks; neighbours in the particle list share a cell and would collide. Integer
// sums do not depend on the order of the adds. The tile is stored whole; k_p2g_gather sums the
// tiles that overlap each cell.
template <class CT>
__device__ __forceinline__ void p2g_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    const uint32_t nb = min(st->s.n_blocks, D.cap_blocks);
    const uint32_t lane = threadIdx.x & 31u;
    __shared__ __align__(16) int32_t tile[8 * TPF];
    __shared__ uint32_t own[64], s_cnt[64];
    __shared__ uint32_t s_pid[P2G_CAP];
    __shared__ uint8_t s_cell[P2G_CAP];
    __shared__ uint16_t s_rank[P2G_CAP];
    __shared__ uint32_t s_mlo[P2G_LAYERS], s_mhi[P2G_LAYERS];  // layer r: cells 0-31, 32-63 with > r particles
    __shared__ uint32_t s_start[P2G_LAYERS + 1], s_over;
    __shared__ uint32_t s_next[2];  // the block after this one, by the parity of the CTA's turn
    const float hh = g.h;
    // A one-scene launch hands the blocks out from a counter as CTAs come free (their particle
    // counts differ, and a fixed stride leaves some CTAs a block more than others); a CTA takes
    // its next block at the start of this one, so the fetch is off the critical path.
    uint32_t turn = 0;
    if constexpr (CT::dynamic) {
        if (threadIdx.x == 0) s_next[0] = atomicAdd(&D.st->next_block[0], 1u);
        __syncthreads();
    }
    for (uint32_t b = CT::dynamic ? s_next[0] : C.x(); b < nb; b = CT::dynamic ? s_next[turn & 1u] : b + C.nx()) {
        turn++;
        if (CT::dynamic && threadIdx.x == 0) s_next[turn & 1u] = atomicAdd(&D.st->next_block[0], 1u);
        const I3 bc = slot_coord(g, g.list[b]);
        if (threadIdx.x < 27) {
            uint32_t li = threadIdx.x;
            I3 n = bc + I3{(int32_t)(li / 9u), (int32_t)((li / 3u) % 3u), (int32_t)(li % 3u)} - I3{1, 1, 1};
            D.block_nb[b * 27u + li] = block_at(g, n);
        }
        if (threadIdx.x < 64) own[threadIdx.x] = 0;
        const uint32_t first = D.block_start[b];
        const uint32_t count = D.block_start[b + 1] - first;
        if (count == 0) {
            if (threadIdx.x < 64) D.acc[(size_t)A_N * D.cap_cells + b * 64u + threadIdx.x] = 0;
            if (threadIdx.x == 0) D.tile_ok[b] = 0u;
            __syncthreads();
            continue;
        }
        for (uint32_t t = threadIdx.x; t < 8 * TPF; t += P2G_T) tile[t] = 0;
        const I3 corner = bc * 4 - I3{1, 1, 1};
        for (uint32_t chunk = 0; chunk < count; chunk += P2G_CAP) {
            const uint32_t n = min(P2G_CAP, count - chunk);
            if (threadIdx.x < 64) s_cnt[threadIdx.x] = 0, s_mlo[threadIdx.x] = 0u, s_mhi[threadIdx.x] = 0u;
            if (threadIdx.x == 0) s_over = 0;
            __syncthreads();
            // Each particle's cell and rank in its cell.
            for (uint32_t j = threadIdx.x; j < n; j += P2G_T) {
                const uint32_t i = D.sorted[first + chunk + j];
                const I3 l = own_cell(g, xyz(D.pos[i])) - bc * 4;
                const uint32_t c = (uint32_t)(l.x * 16 + l.y * 4 + l.z);
                s_cell[j] = (uint8_t)c;
                s_rank[j] = (uint16_t)atomicAdd(&s_cnt[c], 1u);
            }
            __syncthreads();
            // The layers' cell masks (a ballot per layer by the two warps of the 64 cells), then
            // where each layer starts (a scan by one warp).
            if (threadIdx.x < 64) {
                const uint32_t cnt = s_cnt[threadIdx.x];
                own[threadIdx.x] += cnt;
                uint32_t* m = threadIdx.x < 32 ? s_mlo : s_mhi;
                for (uint32_t r = 0; r < P2G_LAYERS; r++) {
                    const uint32_t bits = __ballot_sync(0xffffffffu, cnt > r);
                    if (bits == 0u) break;
                    if (lane == 0) m[r] = bits;
                }
            }
            __syncthreads();
            if (threadIdx.x < 32) {
                const uint32_t p = __popc(s_mlo[2 * lane]) + __popc(s_mhi[2 * lane]);
                const uint32_t q = __popc(s_mlo[2 * lane + 1]) + __popc(s_mhi[2 * lane + 1]);
                uint32_t inc = p + q;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= (uint32_t)o) inc += v;
                }
                s_start[2 * lane] = inc - p - q, s_start[2 * lane + 1] = inc - q;
                if (lane == 31) s_start[P2G_LAYERS] = inc;
            }
            __syncthreads();
            for (uint32_t j = threadIdx.x; j < n; j += P2G_T) {
                const uint32_t c = s_cell[j], r = s_rank[j];
                uint32_t pos;
                if (r < P2G_LAYERS)
                    pos = s_start[r] + (c < 32u ? __popc(s_mlo[r] & ((1u << c) - 1u)) : __popc(s_mlo[r]) + __popc(s_mhi[r] & ((1u << (c - 32u)) - 1u)));
                else
                    pos = s_start[P2G_LAYERS] + atomicAdd(&s_over, 1u);
                s_pid[pos] = D.sorted[first + chunk + j];
            }
            __syncthreads();
            for (uint32_t j = threadIdx.x; j < n; j += P2G_T) {
                const uint32_t i = s_pid[j];
                float4 pos = D.pos[i], vel = D.vel[i], c0 = D.c0[i], c1 = D.c1[i], c2 = D.c2[i];
                V3 x = (xyz(pos) - g.org) / hh;
                splat(tile, x, v3(0.0f, 0.5f, 0.5f), corner, 0, vel.x, xyz(c0), 1, FP_M, hh);
                splat(tile, x, v3(0.5f, 0.0f, 0.5f), corner, 2, vel.y, xyz(c1), 3, FP_M, hh);
                splat(tile, x, v3(0.5f, 0.5f, 0.0f), corner, 4, vel.z, xyz(c2), 5, FP_M, hh);
                splat(tile, x, v3(0.5f, 0.5f, 0.5f), corner, A_PC, c0.w * 1e-6f, v3(0.0f, 0.0f, 0.0f), A_WC, FP_P, hh);
            }
            __syncthreads();
        }
        // Stored in the packed layout (8 fields x 343, strides 49, 7, 1) gather_cell reads.
        int32_t* dst = D.tiles + (size_t)b * 8 * TILE;
        for (uint32_t e = threadIdx.x; e < 8 * TILE; e += P2G_T) {
            const uint32_t f = e / TILE, r = e - f * TILE, x = r / 49u, y = (r - x * 49u) / 7u, z = r - x * 49u - y * 7u;
            dst[e] = tile[f * TPF + x * TPX + y * TPY + z];
        }
        if (threadIdx.x < 64) D.acc[(size_t)A_N * D.cap_cells + b * 64u + threadIdx.x] = (int32_t)own[threadIdx.x];
        if (threadIdx.x == 0) D.tile_ok[b] = 1u;
        __syncthreads();
    }
}
__global__ void __launch_bounds__(P2G_T, 4) k_p2g(Dev D) { p2g_body(D, HwCta{}); }
__global__ void __launch_bounds__(P2G_T, 4) k_p2g_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    p2g_body(sD, c);
}

// The transfer sums of fields 0-7 of `cell`: the entries of the tiles over it, added.
__device__ __forceinline__ void gather_cell(const Dev& D, uint32_t cell, int32_t (&out)[8]) {
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
    for (int f = 0; f < 8; f++) out[f] = (int32_t)s[f];
}

// The tiles' flush and grid_prep (fluid.wgsl:305-356) in one pass over the cells: grid_prep
// reads only the cell's own sums, so each cell's are used as they are gathered. The rubber's
// splat (fields A_MF and up) must be complete.
template <class CT>
__device__ __forceinline__ void gather_prep_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    const ntr_gpu_params* U = D.U;
    const V3 knot = {U->knot[0], U->knot[1], U->knot[2]};
    const float kr = U->knot[3] + 0.5f * g.h;
    const float dt = dt_of(st);
    const float grav[3] = {U->gravity[0], U->gravity[1], U->gravity[2]};
    const uint32_t n_cells = min(st->s.n_blocks, D.cap_blocks) * 64u;
    for (uint32_t cell = C.x() * blockDim.x + threadIdx.x; cell < n_cells; cell += C.nx() * blockDim.x) {
        int32_t s8[8];
        gather_cell(D, cell, s8);
#pragma unroll
        for (int f = 0; f < 8; f++) D.acc[(size_t)f * D.cap_cells + cell] = s8[f];
        grid_prep_cell(D, g, knot, kr, dt, grav, cell, s8);
    }
}
__global__ void k_gather_prep(Dev D) { gather_prep_body(D, HwCta{}); }
__global__ void k_gather_prep_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    gather_prep_body(sD, c);
}

}  // namespace ntr
