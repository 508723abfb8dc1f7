// The pressure solve (shaders/fluid.wgsl:381-578) as one persistent kernel per step.
//
// The reference dispatches solve_init, solve_start, then the encoded number of iterations of
// solve_q, solve_alpha, solve_update and solve_beta, every reduction a dispatch of its own, and
// keeps dispatching no-ops once the solver has switched itself off. Here one cooperative
// launch runs the whole solve and stops at convergence.
//
// Layout of the work:
//   - one warp per 4^3 block, each lane two cells of opposite red-black colour (solve_cell),
//     so the block-local Gauss-Seidel sweeps and the block's 64-wide sum tree need only warp
//     synchronisation, and every lane has a cell to update in every half-sweep;
//   - the reference sums the per-block partials with 256 strided running sums (lane l adds
//     blocks l, l + 256, ...) and then a 256-wide tree (fluid.wgsl:426-439). CTA c owns the
//     blocks b = c (mod 256) (with G < 256 CTAs, the residues c, c + G, ...), so it forms lane
//     c's running sum from its own blocks and publishes it; after a grid barrier every
//     warp reads the 256 values and runs the same tree. All CTAs agree on alpha, beta and
//     convergence bit for bit, and the result equals the reference's order of summation;
//   - a warp that owns at most SOLVE_R blocks keeps their cells' solver values (type, diagonal,
//     water neighbours, p, r, z, d, q) in registers for the whole solve, and writes to memory
//     only what other warps read (d and z, for their neighbours) and, at the end, the final
//     fields. Otherwise it loads and stores them per phase. Either way every load of a phase is
//     issued before its first store, so the latencies overlap;
//   - the grid barrier is a counter that only grows during the launch (reset before it): the
//     k-th barrier waits for k * (CTAs) arrivals. One atomic per CTA and a poll of the same word;
//   - one launch can solve several simulations' systems (a batch): the CTAs split over them
//     (solve_split), each simulation's CTAs with their own barrier and sums.
// The barrier spins a bounded number of times; when it gives up it sets an error bit that the
// host reports as NTR_E_TIMEOUT, and the kernel returns.
#pragma once

#include "kernels_cells.cuh"

namespace ntr {

constexpr int SOLVE_W = 12;                 // warps per CTA
constexpr int SOLVE_T = SOLVE_W * 32;       // 384 threads
constexpr int SOLVE_R = 1;                  // blocks per warp kept in registers
constexpr uint32_t BARRIER_SPINS = 1u << 24;
constexpr int SOLVE_XQ = 3;                 // quantities per exchange, at most

__device__ __forceinline__ uint32_t atom_add_release(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <bool FP64>
struct SolveMath {
    using A = typename std::conditional<FP64, double, float>::type;
    static __device__ __forceinline__ A prod(float a, float b) { return FP64 ? (A)((double)a * (double)b) : (A)(a * b); }
    static __device__ __forceinline__ bool converged(double rr, double b_norm, float tol) {
        if (FP64) return sqrt(rr) <= (double)tol * fmax(b_norm, 1.0);
        return sqrtf((float)rr) <= tol * mx((float)b_norm, 1.0f);
    }
    static __device__ __forceinline__ double root(double x) { return FP64 ? sqrt(x) : (double)sqrtf((float)x); }
    static __device__ __forceinline__ double ratio(double a, double b) { return FP64 ? a / b : (double)((float)a / (float)b); }
};

// The 64-wide tree of block_sum (fluid.wgsl:414-422) over a warp whose lane l holds the
// values of its cells (solve_cell): the first level adds cells l and l + 32 (the latter held by
// lane l ^ 1), the rest are shuffles. Valid in lane 0.
template <class A>
__device__ __forceinline__ A warp_tree64(A v0, A v1) {
    A x = v0 + __shfl_xor_sync(0xffffffffu, v1, 1);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x = x + __shfl_down_sync(0xffffffffu, x, off);
    return x;
}

// A lane's two cells of a block: cell `lane` and cell (lane ^ 1) + 32. They have opposite
// red-black colours (the second is two layers up in x and one step over in z), so in every
// half-sweep of the block's Gauss-Seidel each lane updates exactly one cell.
__device__ __forceinline__ uint32_t solve_cell(int lane, int k) { return k == 0 ? (uint32_t)lane : (uint32_t)(lane ^ 1) + 32u; }

// Symmetric red-black Gauss-Seidel, two sweeps inside the block (fluid.wgsl:390-410), by one
// warp. zl, wl: the warp's 64 cells in shared memory. The cells of one colour do not touch each
// other, so the order in which a half-sweep visits them does not matter.
__device__ __forceinline__ void warp_precondition(float* zl, uint8_t* wl, int lane, const float r[2], const float diag[2],
                                                  const bool water[2], float z[2]) {
    const int li0 = (int)solve_cell(lane, 0), li1 = (int)solve_cell(lane, 1);
    zl[li0] = 0.0f, zl[li1] = 0.0f;
    wl[li0] = water[0], wl[li1] = water[1];
    __syncwarp();
    // Which of the block's face neighbours are water, in the order the sum visits them:
    // -x, +x, -y, +y, -z, +z (local index steps 16, 4, 1).
    uint32_t nm[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int li = c ? li1 : li0;
        const int lx = li >> 4, ly = (li >> 2) & 3, lz = li & 3;
        nm[c] = (lx > 0 && wl[li - 16] ? 1u : 0u) | (lx < 3 && wl[li + 16] ? 2u : 0u) | (ly > 0 && wl[li - 4] ? 4u : 0u) |
                (ly < 3 && wl[li + 4] ? 8u : 0u) | (lz > 0 && wl[li - 1] ? 16u : 0u) | (lz < 3 && wl[li + 1] ? 32u : 0u);
    }
    const uint32_t colour0 = (uint32_t)((li0 >> 4) + ((li0 >> 2) & 3) + (li0 & 3)) % 2u;
    for (uint32_t k = 0; k < 5; k++) {
        const bool first = colour0 == k % 2u;  // this half-sweep's cell is the lane's first
        if (first ? water[0] : water[1]) {
            const int li = first ? li0 : li1;
            const uint32_t m = first ? nm[0] : nm[1];
            float s = first ? r[0] : r[1];
            if (m & 1u) s += zl[li - 16];
            if (m & 2u) s += zl[li + 16];
            if (m & 4u) s += zl[li - 4];
            if (m & 8u) s += zl[li + 4];
            if (m & 16u) s += zl[li - 1];
            if (m & 32u) s += zl[li + 1];
            zl[li] = s / (first ? diag[0] : diag[1]);
        }
        __syncwarp();
    }
    z[0] = zl[li0], z[1] = zl[li1];
    __syncwarp();
}

// The 256-wide tree over the running sums (fluid.wgsl:434-438) of one quantity, by one warp:
// lane l loads sums l, l + 32, ..., l + 224, does the levels 128, 64 and 32 in registers and
// the rest with shuffles. Valid in lane 0.
template <class A>
__device__ __forceinline__ A warp_tree256(const double* sums, int q, int lane) {
    A v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = (A)__ldcg(sums + (size_t)(lane + 32 * i) * SOLVE_XQ + q);
    // Level 128: positions l, l + 32, l + 64, l + 96 add l + 128, ... ; level 64; level 32.
    const A a0 = v[0] + v[4], a1 = v[1] + v[5], a2 = v[2] + v[6], a3 = v[3] + v[7];
    const A b0 = a0 + a2, b1 = a1 + a3;
    A x = b0 + b1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x = x + __shfl_down_sync(0xffffffffu, x, off);
    return x;
}

// Where a CTA keeps its blocks' partial sums: its blocks are those of residues c, c + G,
// c + 2 G, ... (below 256), in that order and by ascending block within a residue; residue k's
// blocks are the CTA's E[k] .. E[k + 1] - 1. Quantity q of the CTA's e-th block, block b, is at
// part[q * stride + e] in shared memory, or part[q * stride + b] in the job's global array.
template <class A>
struct SolveParts {
    A* part;
    uint32_t stride;
    bool by_block;
    const uint32_t* E;
    uint32_t n_res;
    __device__ __forceinline__ A& at(uint32_t q, uint32_t e, uint32_t b) const { return part[q * stride + (by_block ? b : e)]; }
};

// Publishes this CTA's running sums (fluid.wgsl:429-431) of quantities 0..NQ-1 of `P`, waits at
// the grid barrier, and returns the 256-wide trees in `out`. The sums are double-buffered by
// the barrier's parity: a CTA writes the next-but-one sums only after every CTA has passed the
// next barrier, that is, has read these. False (in every thread) if the wait gave up.
template <class A, int NQ>
__device__ __forceinline__ bool exchange(const Dev& D, DevState* st, uint32_t& gen, const SolveParts<A>& P, uint32_t c, uint32_t G,
                                         A (&out)[NQ]) {
    __shared__ uint32_t s_ok;
    gen++;
    double* sums = D.xsum + (size_t)(gen & 1u) * 256u * SOLVE_XQ;
    __syncthreads();  // every warp's partials and cell writes of this phase are done
    for (uint32_t t = threadIdx.x; t < P.n_res * NQ; t += blockDim.x) {
        const uint32_t k = t / NQ, q = t % NQ, r = c + k * G;
        A s = A(0);
        for (uint32_t e = P.E[k], b = r; e < P.E[k + 1]; e++, b += 256u) s = s + P.at(q, e, b);
        sums[r * SOLVE_XQ + q] = (double)s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // Release: this CTA's writes (ordered before by the barrier above) before the arrival.
        const uint32_t target = gen * G;
        if (!(gen == 1u && c == D.bar_skip)) atom_add_release(&st->bar_count, 1u);
        uint32_t ok = 1u;
        for (uint32_t spins = 0; ld_acquire(&st->bar_count) < target;) {
            // Give up after a bounded wait, or at once when another CTA of the solve has.
            if (++spins > D.bar_spins || ((spins & 1023u) == 0u && *(volatile uint32_t*)&st->err != 0u)) {
                atomicOr(&st->err, 1u);
                ok = 0u;
                break;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) return false;
    // One warp forms the trees; every CTA gets the same values.
    __shared__ A s_out[SOLVE_XQ];
    if (threadIdx.x < 32)
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            const A x = warp_tree256<A>(sums, q, (int)threadIdx.x);
            if (threadIdx.x == 0) s_out[q] = x;
        }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NQ; q++) out[q] = s_out[q];
    return true;
}

// A lane's two cells of one block (solve_cell): the solver's values for them.
struct SolveCells {
    float diag[2], z[2], d[2], r[2], p[2], q[2];
    uint32_t wn[2][6];  // water neighbours in solve_q's order (-x, +x, -y, +y, -z, +z), or NONE
    bool water[2];
};

constexpr uint32_t SOLVE_MAX_JOBS = 128;  // systems solved by one launch, at most
constexpr uint32_t SOLVE_PART_SH = 512;   // partial sums per quantity kept in shared memory

// The CTAs of a launch split over its jobs (independent systems, each a simulation's step):
// every job that steps gets one CTA and the rest go by expected work, its blocks times its last
// solve's iterations, at most 256 each. Every CTA computes the same split. c0[j] .. c0[j + 1]
// are job j's CTAs. (A job's result does not depend on how many CTAs it gets.)
__device__ __forceinline__ void solve_split(const Dev* jobs, uint32_t n_jobs, uint32_t* w, uint32_t* c0) {
    for (uint32_t j = threadIdx.x; j < n_jobs; j += blockDim.x) {
        const DevState* st = jobs[j].st;
        w[j] = st->s.dt_ns == 0u ? NONE : min(st->s.n_blocks, jobs[j].cap_blocks) * max(min(st->iters_prev, 4096u), 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t live = 0;
        uint64_t total = 0;
        for (uint32_t j = 0; j < n_jobs; j++)
            if (w[j] != NONE) live++, total += w[j];
        const uint32_t spare = gridDim.x > live ? gridDim.x - live : 0u;
        uint32_t at = 0;
        for (uint32_t j = 0; j < n_jobs; j++) {
            c0[j] = at;
            if (w[j] == NONE || at >= gridDim.x) continue;
            const uint32_t extra = total ? (uint32_t)((uint64_t)spare * w[j] / total) : 0u;
            at += min(1u + extra, min(256u, gridDim.x - at));
        }
        c0[n_jobs] = at;
    }
    __syncthreads();
}

// The solve of one system by CTAs c = 0 .. G - 1 of a cooperative launch (k_solve for one
// simulation, k_solve_batch for several). A job's result does not depend on G: the sums are the
// reference's 256 running sums and tree either way.
template <bool FP64>
__device__ __forceinline__ void solve_body(const Dev& D, uint32_t c, uint32_t G) {
    using M = SolveMath<FP64>;
    using A = typename M::A;
    __shared__ uint32_t s_E[257];
    __shared__ A s_part[3 * SOLVE_PART_SH];
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    uint32_t gen = 0;
    const Grid g = grid_of(D, cur_of(st));
    const ntr_gpu_params* U = D.U;
    const uint32_t nb = min(st->s.n_blocks, D.cap_blocks);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float tol = U->solve[0];
    const uint32_t limit = U->limits[2];
    const float hh = g.h, dt = dt_of(st);
    const float rho = U->fluid[0];
    __shared__ float zl[SOLVE_W][64];
    __shared__ uint8_t wl[SOLVE_W][64];
    // Read before the first barrier: CTA 0 writes them back at the end. alpha keeps the last
    // step's value when the solver does not run, as the reference's state does.
    uint32_t iters_max = st->s.iters_max, unconverged = st->s.unconverged;
    double alpha = st->alpha;
    // This CTA's residues c, c + G, ... and their blocks.
    auto count_of = [&](uint32_t r) -> uint32_t { return r < nb ? (nb - r + 255u) / 256u : 0u; };
    const uint32_t n_res = c < 256u ? (256u - c + G - 1u) / G : 0u;
    if (threadIdx.x == 0) {
        uint32_t e = 0;
        for (uint32_t k = 0; k < n_res; k++) s_E[k] = e, e += count_of(c + k * G);
        s_E[n_res] = e;
    }
    __syncthreads();
    const uint32_t n_mine = s_E[n_res];
    // The partial sums: in shared memory, or in the job's own array when the CTA has too many
    // blocks for that.
    SolveParts<A> P;
    P.by_block = n_mine > SOLVE_PART_SH;
    P.part = P.by_block ? reinterpret_cast<A*>(D.spart) : s_part;
    P.stride = P.by_block ? D.cap_blocks : SOLVE_PART_SH;
    P.E = s_E;
    P.n_res = n_res;
    // The CTA's e-th block: residue k (the last with E[k] <= e), its (e - E[k])-th block.
    auto block_of = [&](uint32_t e) -> uint32_t {
        uint32_t lo = 0, hi = n_res;  // E[lo] <= e < E[hi]
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) / 2u;
            if (s_E[mid] <= e) lo = mid; else hi = mid;
        }
        return c + lo * G + 256u * (e - s_E[lo]);
    };
    const uint32_t n_warp = n_mine > (uint32_t)warp ? (n_mine - 1u - (uint32_t)warp) / SOLVE_W + 1u : 0u;
    const bool in_regs = (n_mine + SOLVE_W - 1) / SOLVE_W <= (uint32_t)SOLVE_R;
    SolveCells R[SOLVE_R];

    // ---- solve_init (fluid.wgsl:445-491): diagonal, right-hand side, residual, preconditioned
    // residual, and the block's (r.z, r.r, b.b).
    auto init_block = [&](SolveCells& C, uint32_t b, uint32_t e) {
        uint32_t cell[2];
        float bq[2];
        // One cell after the other (to bound the registers), each with all its loads first.
#pragma unroll
        for (int k = 0; k < 2; k++) {
            cell[k] = b * 64u + solve_cell(lane, k);
            uint32_t nbr[6];
            float nty[6], np[6], nu[3], uc[3];
#pragma unroll
            for (int j = 0; j < 6; j++) nbr[j] = neighbour(g, cell[k], ed(j >> 1, (j & 1) ? 1 : -1));
            const float ty = cfv(D, F_TYPE, cell[k]);
            const float pc = cfv(D, F_P, cell[k]);
            const float dold = cfv(D, F_D, cell[k]);
            const int32_t src = accv(D, A_SRC, cell[k]);
#pragma unroll
            for (int d = 0; d < 3; d++) uc[d] = cfv(D, F_U + d, cell[k]);
#pragma unroll
            for (int j = 0; j < 6; j++) {
                nty[j] = GAS_T, np[j] = 0.0f;
                if (nbr[j] != NONE) nty[j] = cfv(D, F_TYPE, nbr[j]), np[j] = cfv(D, F_P, nbr[j]);
            }
#pragma unroll
            for (int d = 0; d < 3; d++) nu[d] = nbr[2 * d + 1] != NONE ? cfv(D, F_U + d, nbr[2 * d + 1]) : 0.0f;
            C.water[k] = ty == WATER_T;
            C.diag[k] = 1.0f, C.r[k] = 0.0f, C.p[k] = pc, C.d[k] = dold, bq[k] = 0.0f;
#pragma unroll
            for (int j = 0; j < 6; j++) C.wn[k][j] = NONE;
            if (!C.water[k]) continue;
            float cs = U->gravity[3] * dt;
            float kc = hh * hh / (cs * cs);
            float div = 0.0f, off = 0.0f;
            float dg = kc, bb = kc * pc;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                // face_u of the face above (its cell the neighbour, below it this cell) minus
                // the face below (this cell over the neighbour below).
                const float fu_hi = nbr[2 * d + 1] == NONE ? 0.0f : bounded(nu[d], nty[2 * d + 1], ty);
                const float fu_lo = bounded(uc[d], ty, nty[2 * d]);
                div += fu_hi - fu_lo;
#pragma unroll
                for (int s = 0; s < 2; s++) {
                    const int j = 2 * d + s;
                    if (nty[j] == SOLID_T) continue;
                    dg += 1.0f;
                    if (nty[j] == WATER_T) {
                        off -= np[j];
                        C.wn[k][j] = nbr[j];
                    } else {
                        bb += np[j];  // pressure_of: 0 outside the grid, p of a non-water cell
                    }
                }
            }
            div -= from_fp(src, FP_Q) / (hh * hh);
            bb -= rho * hh / dt * div;
            C.r[k] = bb - dg * pc - off;
            C.diag[k] = dg, bq[k] = bb;
        }
        for (int k = 0; k < 2; k++) {
            if (!C.water[k]) continue;
            *cfp(D, F_DIAG, cell[k]) = C.diag[k];
            *cfp(D, F_R, cell[k]) = C.r[k];
            if (!in_regs) {
                uint4* wp = reinterpret_cast<uint4*>(D.wnb + (size_t)cell[k] * 8);
                wp[0] = make_uint4(C.wn[k][0], C.wn[k][1], C.wn[k][2], C.wn[k][3]);
                wp[1] = make_uint4(C.wn[k][4], C.wn[k][5], NONE, NONE);
            }
        }
        warp_precondition(zl[warp], wl[warp], lane, C.r, C.diag, C.water, C.z);
        for (int k = 0; k < 2; k++)
            if (C.water[k]) *cfp(D, F_Z, cell[k]) = C.z[k];
        A sx = warp_tree64(M::prod(C.r[0], C.z[0]), M::prod(C.r[1], C.z[1]));
        A sy = warp_tree64(M::prod(C.r[0], C.r[0]), M::prod(C.r[1], C.r[1]));
        A sz = warp_tree64(M::prod(bq[0], bq[0]), M::prod(bq[1], bq[1]));
        if (lane == 0) P.at(0, e, b) = sx, P.at(1, e, b) = sy, P.at(2, e, b) = sz;
    };

    // ---- solve_q (fluid.wgsl:513-534): the new search direction and A d. `old` is the parity
    // of the direction field the last iteration wrote.
    auto q_block = [&](SolveCells& C, uint32_t b, uint32_t e, uint32_t old, float fbeta) {
        uint32_t cell[2];
        for (int k = 0; k < 2; k++) cell[k] = b * 64u + solve_cell(lane, k);
        if (!in_regs) {
#pragma unroll
            for (int k = 0; k < 2; k++) {
                C.water[k] = cfv(D, F_TYPE, cell[k]) == WATER_T;
                C.z[k] = cfv(D, F_Z, cell[k]);
                C.d[k] = cfv(D, F_D + old, cell[k]);
                C.diag[k] = cfv(D, F_DIAG, cell[k]);
                const uint4* wp = reinterpret_cast<const uint4*>(D.wnb + (size_t)cell[k] * 8);
                const uint4 w0 = wp[0], w1 = wp[1];
                C.wn[k][0] = w0.x, C.wn[k][1] = w0.y, C.wn[k][2] = w0.z, C.wn[k][3] = w0.w;
                C.wn[k][4] = w1.x, C.wn[k][5] = w1.y;
            }
        }
        // The neighbours' z and old d were written by other warps and CTAs earlier in this
        // launch: read through L2.
        float zn[2][6], dnb[2][6];
#pragma unroll
        for (int k = 0; k < 2; k++)
#pragma unroll
            for (int j = 0; j < 6; j++) {
                zn[k][j] = 0.0f, dnb[k][j] = 0.0f;
                const uint32_t n = C.wn[k][j];
                if (C.water[k] && n != NONE) zn[k][j] = __ldcg(cfp(D, F_Z, n)), dnb[k][j] = __ldcg(cfp(D, F_D + old, n));
            }
        A v[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            v[k] = A(0);
            if (!C.water[k]) continue;
            const float dn = C.z[k] + fbeta * C.d[k];
            float q = C.diag[k] * dn;
#pragma unroll
            for (int j = 0; j < 6; j++)
                if (C.wn[k][j] != NONE) q -= zn[k][j] + fbeta * dnb[k][j];
            *cfp(D, F_D + 1 - old, cell[k]) = dn;
            if (!in_regs) *cfp(D, F_Q, cell[k]) = q;
            C.d[k] = dn, C.q[k] = q;
            v[k] = M::prod(dn, q);
        }
        A s = warp_tree64(v[0], v[1]);
        if (lane == 0) P.at(0, e, b) = s;
    };

    // ---- solve_update (fluid.wgsl:543-559): p, r, and the preconditioned residual. `nw` is
    // the parity of the direction field this iteration's solve_q wrote.
    auto update_block = [&](SolveCells& C, uint32_t b, uint32_t e, uint32_t nw, float a) {
        uint32_t cell[2];
        for (int k = 0; k < 2; k++) cell[k] = b * 64u + solve_cell(lane, k);
        if (!in_regs) {
#pragma unroll
            for (int k = 0; k < 2; k++) {
                C.water[k] = cfv(D, F_TYPE, cell[k]) == WATER_T;
                C.p[k] = cfv(D, F_P, cell[k]);
                C.d[k] = cfv(D, F_D + nw, cell[k]);
                C.r[k] = cfv(D, F_R, cell[k]);
                C.q[k] = cfv(D, F_Q, cell[k]);
                C.diag[k] = cfv(D, F_DIAG, cell[k]);
            }
        }
        float r[2], diag[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            diag[k] = 1.0f, r[k] = 0.0f;
            if (!C.water[k]) continue;
            C.p[k] = C.p[k] + a * C.d[k];
            C.r[k] = C.r[k] - a * C.q[k];
            if (!in_regs) {
                *cfp(D, F_P, cell[k]) = C.p[k];
                *cfp(D, F_R, cell[k]) = C.r[k];
            }
            r[k] = C.r[k], diag[k] = C.diag[k];
        }
        warp_precondition(zl[warp], wl[warp], lane, r, diag, C.water, C.z);
        for (int k = 0; k < 2; k++)
            if (C.water[k]) *cfp(D, F_Z, cell[k]) = C.z[k];
        A sx = warp_tree64(M::prod(r[0], C.z[0]), M::prod(r[1], C.z[1]));
        A sy = warp_tree64(M::prod(r[0], r[0]), M::prod(r[1], r[1]));
        if (lane == 0) P.at(0, e, b) = sx, P.at(1, e, b) = sy;
    };

    // Runs `body(C, b, e)` over the warp's blocks (the CTA's warp-th, (warp + SOLVE_W)-th, ...).
    auto each_block = [&](auto&& body) {
        if (in_regs) {
#pragma unroll
            for (int j = 0; j < SOLVE_R; j++)
                if ((uint32_t)j < n_warp) {
                    const uint32_t e = (uint32_t)warp + (uint32_t)j * SOLVE_W;
                    body(R[j], block_of(e), e);
                }
        } else {
            for (uint32_t j = 0; j < n_warp; j++) {
                const uint32_t e = (uint32_t)warp + j * SOLVE_W;
                body(R[0], block_of(e), e);
            }
        }
    };

    each_block([&](SolveCells& C, uint32_t b, uint32_t e) { init_block(C, b, e); });

    // solve_start (fluid.wgsl:493-506).
    double rz, beta = 0.0, b_norm, r_norm;
    uint32_t iters = 0;
    bool on;
    {
        A s3[3];
        if (!exchange<A, 3>(D, st, gen, P, c, G, s3)) return;
        const A sx = s3[0], sy = s3[1], sz = s3[2];
        rz = (double)sx;
        b_norm = M::root((double)sz);
        r_norm = M::root((double)sy);
        on = (double)sx > 0.0 && !M::converged((double)sy, b_norm, tol);
    }
    while (on) {
        const uint32_t old = iters % 2u;
        const float fbeta = (float)beta;
        each_block([&](SolveCells& C, uint32_t b, uint32_t e) { q_block(C, b, e, old, fbeta); });
        // solve_alpha (fluid.wgsl:536-541).
        {
            A s1[1];
            if (!exchange<A, 1>(D, st, gen, P, c, G, s1)) return;
            alpha = (double)s1[0] > 0.0 ? M::ratio(rz, (double)s1[0]) : 0.0;
        }
        const float a = (float)alpha;
        each_block([&](SolveCells& C, uint32_t b, uint32_t e) { update_block(C, b, e, 1u - old, a); });
        // solve_beta (fluid.wgsl:561-578).
        {
            A s2[2];
            if (!exchange<A, 2>(D, st, gen, P, c, G, s2)) return;
            const A sx = s2[0], sy = s2[1];
            iters += 1;
            r_norm = M::root((double)sy);
            beta = rz > 0.0 ? M::ratio((double)sx, rz) : 0.0;
            rz = (double)sx;
            bool done = M::converged((double)sy, b_norm, tol);
            if (done || iters >= limit) {
                iters_max = max(iters_max, iters);
                unconverged += done ? 0u : 1u;
                on = false;
            }
        }
    }
    // The fields kept in registers go to memory once, as the iterations would have left them.
    if (in_regs && iters > 0)
        each_block([&](SolveCells& C, uint32_t b, uint32_t) {
            for (int k = 0; k < 2; k++) {
                if (!C.water[k]) continue;
                const uint32_t cell = b * 64u + solve_cell(lane, k);
                *cfp(D, F_P, cell) = C.p[k];
                *cfp(D, F_R, cell) = C.r[k];
                *cfp(D, F_Q, cell) = C.q[k];
            }
        });
    if (c == 0 && threadIdx.x == 0) {
        st->rz = rz, st->alpha = alpha, st->beta = beta, st->b_norm = b_norm, st->r_norm = r_norm;
        st->solver_on = 0u;
        st->s.solve_iters = iters, st->s.iters_max = iters_max, st->s.unconverged = unconverged;
        st->s.rz = (float)rz, st->s.alpha = (float)alpha, st->s.beta = (float)beta;
        st->s.b_norm = (float)b_norm, st->s.r_norm = (float)r_norm;
    }
}

template <bool FP64>
__global__ void __launch_bounds__(SOLVE_T, 2) k_solve(Dev D) {
    solve_body<FP64>(D, blockIdx.x, gridDim.x);
}

// One launch for the systems of `n_jobs` simulations (their pointer tables at `jobs`): the CTAs
// split over them (solve_split) and each group solves its own.
template <bool FP64>
__global__ void __launch_bounds__(SOLVE_T, 2) k_solve_batch(const Dev* __restrict__ jobs, uint32_t n_jobs) {
    __shared__ uint32_t s_w[SOLVE_MAX_JOBS], s_c0[SOLVE_MAX_JOBS + 1];
    __shared__ Dev s_dev;
    solve_split(jobs, n_jobs, s_w, s_c0);
    uint32_t job = NONE;
    for (uint32_t j = 0; j < n_jobs; j++)
        if (blockIdx.x >= s_c0[j] && blockIdx.x < s_c0[j + 1]) job = j;
    if (job == NONE) return;
    for (uint32_t k = threadIdx.x; k < sizeof(Dev) / 4; k += blockDim.x)
        reinterpret_cast<uint32_t*>(&s_dev)[k] = reinterpret_cast<const uint32_t*>(jobs + job)[k];
    __syncthreads();
    solve_body<FP64>(s_dev, blockIdx.x - s_c0[job], s_c0[job + 1] - s_c0[job]);
}

// Every scene's grid barrier counter back to zero before the joint solve (a one-scene step
// clears its own with a memset), and its last solve's iterations set aside for the split: the
// solve itself rewrites them, and every CTA must compute the same split.
__global__ void k_solve_reset_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (threadIdx.x == 0) sD.st->bar_count = 0u, sD.st->iters_prev = sD.st->s.solve_iters;
}

}  // namespace ntr
