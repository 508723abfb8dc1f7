// The pressure solve (shaders/fluid.wgsl:381-578) as one persistent kernel per step.
//
// The reference dispatches solve_init, solve_start, then the encoded number of iterations of
// solve_q, solve_alpha, solve_update and solve_beta, every reduction a dispatch of its own, and
// keeps dispatching no-ops once the solver has switched itself off. Here one cooperative
// launch runs the whole solve and stops at convergence.
//
// Layout of the work:
//   - one warp per 4^3 block, each lane two cells (l and l + 32, which have the same
//     red-black colour), so the block-local Gauss-Seidel sweeps and the block's 64-wide sum
//     tree need only warp synchronisation;
//   - the reference sums the per-block partials with 256 strided running sums (lane l adds
//     blocks l, l + 256, ...) and then a 256-wide tree (fluid.wgsl:426-439). CTA c owns the
//     blocks b = c (mod 256) (with fewer than 256 CTAs, several residues), so it forms lane
//     c's running sum from its own blocks and publishes one value; after a grid barrier every
//     CTA reads the 256 values and runs the same tree. All CTAs agree on alpha, beta and
//     convergence bit for bit, and the result equals the reference's order of summation.
// The grid barrier spins a bounded number of times; when it gives up it sets an error bit
// that the host reports as NTR_E_TIMEOUT, and the kernel returns.
#pragma once

#include "kernels_cells.cuh"

namespace ntr {

constexpr int SOLVE_W = 12;                 // warps per CTA
constexpr int SOLVE_T = SOLVE_W * 32;       // 384 threads
constexpr uint32_t SOLVE_MAX_M = 256;       // blocks per residue: 65536 blocks / 256
constexpr uint32_t BARRIER_SPINS = 1u << 24;

// Grid-wide barrier of a cooperative launch. Returns false in every thread of the CTA if the
// wait gave up; the error bit is then set in the state.
__device__ __forceinline__ uint32_t atom_add_release(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Thread 0 arrives with release semantics (after the CTA's barrier, so the whole CTA's writes
// are ordered before it) and waits with acquire semantics; the last to arrive resets the
// count and releases the next generation.
__device__ __forceinline__ bool grid_sync(DevState* st, uint32_t& gen) {
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t target = gen + 1u;
        uint32_t ok = 1u;
        const uint32_t t = atom_add_release(&st->bar_count, 1u);
        if (t == gridDim.x - 1) {
            atomicExch(&st->bar_count, 0u);
            st_release(&st->bar_gen, target);
        } else {
            uint32_t spins = 0;
            while (ld_acquire(&st->bar_gen) != target) {
                if (++spins > BARRIER_SPINS) {
                    atomicOr(&st->err, 1u);
                    ok = 0u;
                    break;
                }
                if (spins > 64) __nanosleep(32);
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    gen++;
    return s_ok != 0;
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

// The 64-wide tree of block_sum (fluid.wgsl:414-422) over a warp whose lane l holds cells l
// and l + 32: the first level adds those two, the rest are shuffles. Valid in lane 0.
template <class A>
__device__ __forceinline__ A warp_tree64(A v0, A v1) {
    A x = v0 + v1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x = x + __shfl_down_sync(0xffffffffu, x, off);
    return x;
}

// Symmetric red-black Gauss-Seidel, two sweeps inside the block (fluid.wgsl:390-410), by one
// warp. zl, wl: the warp's 64 cells in shared memory.
__device__ __forceinline__ void warp_precondition(float* zl, uint8_t* wl, int lane, const float r[2], const float diag[2],
                                                  const bool water[2], float z[2]) {
    zl[lane] = 0.0f, zl[lane + 32] = 0.0f;
    wl[lane] = water[0], wl[lane + 32] = water[1];
    __syncwarp();
    const int ly = (lane / 4) % 4, lz = lane % 4;
    const int lx0 = lane / 16;  // the second cell is at lx0 + 2
    const uint32_t colour = (uint32_t)(lx0 + ly + lz) % 2u;
    for (uint32_t k = 0; k < 5; k++) {
        if (colour == k % 2u) {
#pragma unroll
            for (int c = 0; c < 2; c++) {
                if (!water[c]) continue;
                const int li = lane + 32 * c, lx = lx0 + 2 * c;
                float s = r[c];
                if (lx > 0 && wl[li - 16]) s += zl[li - 16];
                if (lx < 3 && wl[li + 16]) s += zl[li + 16];
                if (ly > 0 && wl[li - 4]) s += zl[li - 4];
                if (ly < 3 && wl[li + 4]) s += zl[li + 4];
                if (lz > 0 && wl[li - 1]) s += zl[li - 1];
                if (lz < 3 && wl[li + 1]) s += zl[li + 1];
                zl[li] = s / diag[c];
            }
        }
        __syncwarp();
    }
    z[0] = zl[lane], z[1] = zl[lane + 32];
    __syncwarp();
}

// The 256-wide tree over the published running sums (fluid.wgsl:434-438). All threads of the
// CTA call it; every CTA gets the same value.
template <class A>
__device__ __forceinline__ A tree256(const double* rs, A* red) {
    if (threadIdx.x < 256) red[threadIdx.x] = (A)__ldcg(rs + threadIdx.x);
    __syncthreads();
    for (int off = 128; off >= 32; off >>= 1) {
        if ((int)threadIdx.x < off) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x < 32) {
        A x = red[threadIdx.x];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x = x + __shfl_down_sync(0xffffffffu, x, off);
        if (threadIdx.x == 0) red[0] = x;
    }
    __syncthreads();
    A r = red[0];
    __syncthreads();
    return r;
}

template <bool FP64>
__global__ void __launch_bounds__(SOLVE_T) k_solve(Dev D) {
    using M = SolveMath<FP64>;
    using A = typename M::A;
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    uint32_t gen = *(volatile uint32_t*)&st->bar_gen;
    const Grid g = grid_of(D, cur_of(st));
    const ntr_gpu_params* U = D.U;
    const uint32_t nb = min(st->s.n_blocks, D.cap_blocks);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t G = gridDim.x, c = blockIdx.x;
    const float tol = U->solve[0];
    const uint32_t limit = U->limits[2];
    const float hh = g.h, dt = dt_of(st);
    const float rho = U->fluid[0];
    // Per-block partial sums of this CTA's blocks, by (residue slot, m), three quantities.
    __shared__ A part[3][2][SOLVE_MAX_M];
    __shared__ float zl[SOLVE_W][64];
    __shared__ uint8_t wl[SOLVE_W][64];
    __shared__ A red[256];
    // Read before the first barrier: CTA 0 writes them back at the end. alpha keeps the last
    // step's value when the solver does not run, as the reference's state does.
    uint32_t iters_max = st->s.iters_max, unconverged = st->s.unconverged;
    double alpha = st->alpha;
    // Residues of this CTA: c, c + G (G >= 128 keeps it to two).
    const uint32_t n_res = (c + G < 256u) ? 2u : 1u;
    auto count_of = [&](uint32_t r) -> uint32_t { return r < nb ? (nb - r + 255u) / 256u : 0u; };

    // Runs `body(b, ri, m)` for every block this CTA owns, one warp per block.
    auto for_my_blocks = [&](auto&& body) {
        uint32_t e = 0;
        for (uint32_t ri = 0; ri < n_res; ri++) {
            const uint32_t r = c + ri * G;
            const uint32_t cnt = count_of(r);
            for (uint32_t m = 0; m < cnt; m++, e++)
                if ((int)(e % SOLVE_W) == warp) body(r + 256u * m, ri, m);
        }
    };
    // Lane r's running sum (fluid.wgsl:429-431) of quantity q, into rs[r].
    auto publish = [&](int q, double* rs) {
        __syncthreads();
        if (threadIdx.x < n_res) {
            const uint32_t ri = threadIdx.x, r = c + ri * G;
            A s = A(0);
            const uint32_t cnt = count_of(r);
            for (uint32_t m = 0; m < cnt; m++) s = s + part[q][ri][m];
            rs[r] = (double)s;
        }
    };

    // solve_init (fluid.wgsl:445-491): diagonal, right-hand side, residual, preconditioned
    // residual, and the block's (r.z, r.r, b.b).
    for_my_blocks([&](uint32_t b, uint32_t ri, uint32_t m) {
        float r[2], diag[2], bq[2], z[2];
        bool water[2];
        for (int k = 0; k < 2; k++) {
            const uint32_t cell = b * 64u + lane + 32u * k;
            water[k] = cfv(D, F_TYPE, cell) == WATER_T;
            diag[k] = 1.0f, r[k] = 0.0f, bq[k] = 0.0f;
            if (!water[k]) continue;
            float cs = U->gravity[3] * dt;
            float kc = hh * hh / (cs * cs);
            float div = 0.0f, off = 0.0f;
            float dg = kc, bb = kc * cfv(D, F_P, cell);
            uint32_t wn[8] = {NONE, NONE, NONE, NONE, NONE, NONE, NONE, NONE};
            for (uint32_t d = 0; d < 3; d++) {
                div += face_u(D, neighbour(g, cell, ed(d, 1)), cell, d) - face_u(D, cell, neighbour(g, cell, ed(d, -1)), d);
                for (int s = -1; s <= 1; s += 2) {
                    uint32_t nbc = neighbour(g, cell, ed(d, s));
                    float nt = cell_type(D, nbc);
                    if (nt == SOLID_T) continue;
                    dg += 1.0f;
                    if (nt == WATER_T) {
                        off -= cfv(D, F_P, nbc);
                        wn[2 * d + (s > 0 ? 1 : 0)] = nbc;
                    } else {
                        bb += pressure_of(D, nbc);
                    }
                }
            }
            // The water neighbours, in the order solve_q visits them, for the iterations.
            uint4* wp = reinterpret_cast<uint4*>(D.wnb + (size_t)cell * 8);
            wp[0] = make_uint4(wn[0], wn[1], wn[2], wn[3]);
            wp[1] = make_uint4(wn[4], wn[5], NONE, NONE);
            div -= from_fp(accv(D, A_SRC, cell), FP_Q) / (hh * hh);
            bb -= rho * hh / dt * div;
            float rr = bb - dg * cfv(D, F_P, cell) - off;
            *cfp(D, F_DIAG, cell) = dg;
            *cfp(D, F_R, cell) = rr;
            diag[k] = dg, r[k] = rr, bq[k] = bb;
        }
        warp_precondition(zl[warp], wl[warp], lane, r, diag, water, z);
        for (int k = 0; k < 2; k++)
            if (water[k]) *cfp(D, F_Z, b * 64u + lane + 32u * k) = z[k];
        A sx = warp_tree64(M::prod(r[0], z[0]), M::prod(r[1], z[1]));
        A sy = warp_tree64(M::prod(r[0], r[0]), M::prod(r[1], r[1]));
        A sz = warp_tree64(M::prod(bq[0], bq[0]), M::prod(bq[1], bq[1]));
        if (lane == 0) part[0][ri][m] = sx, part[1][ri][m] = sy, part[2][ri][m] = sz;
    });
    publish(0, D.px);
    publish(1, D.py);
    publish(2, D.pz);
    if (!grid_sync(st, gen)) return;

    // solve_start (fluid.wgsl:493-506).
    double rz, beta = 0.0, b_norm, r_norm;
    uint32_t iters = 0;
    bool on;
    {
        A sx = tree256<A>(D.px, red);
        A sy = tree256<A>(D.py, red);
        A sz = tree256<A>(D.pz, red);
        rz = (double)sx;
        b_norm = M::root((double)sz);
        r_norm = M::root((double)sy);
        on = (double)sx > 0.0 && !M::converged((double)sy, b_norm, tol);
    }
    while (on) {
        // solve_q (fluid.wgsl:513-534): the new search direction and A d.
        const uint32_t old = iters % 2u;
        const float fbeta = (float)beta;
        for_my_blocks([&](uint32_t b, uint32_t ri, uint32_t m) {
            A v[2];
            for (int k = 0; k < 2; k++) {
                const uint32_t cell = b * 64u + lane + 32u * k;
                v[k] = A(0);
                if (cfv(D, F_TYPE, cell) != WATER_T) continue;
                float dn = cfv(D, F_Z, cell) + fbeta * cfv(D, F_D + old, cell);
                float q = cfv(D, F_DIAG, cell) * dn;
                const uint4* wp = reinterpret_cast<const uint4*>(D.wnb + (size_t)cell * 8);
                const uint4 w0 = wp[0], w1 = wp[1];
                const uint32_t wn[6] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y};
                // All neighbour loads first (written by other CTAs earlier in this launch:
                // read through L2), then the sum in the reference's order.
                float zn[6], dnb[6];
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    zn[k] = 0.0f, dnb[k] = 0.0f;
                    if (wn[k] != NONE) zn[k] = __ldcg(cfp(D, F_Z, wn[k])), dnb[k] = __ldcg(cfp(D, F_D + old, wn[k]));
                }
#pragma unroll
                for (int k = 0; k < 6; k++)
                    if (wn[k] != NONE) q -= zn[k] + fbeta * dnb[k];
                *cfp(D, F_D + 1 - old, cell) = dn;
                *cfp(D, F_Q, cell) = q;
                v[k] = M::prod(dn, q);
            }
            A s = warp_tree64(v[0], v[1]);
            if (lane == 0) part[0][ri][m] = s;
        });
        publish(0, D.pq);
        if (!grid_sync(st, gen)) return;
        // solve_alpha (fluid.wgsl:536-541).
        {
            A s = tree256<A>(D.pq, red);
            alpha = (double)s > 0.0 ? M::ratio(rz, (double)s) : 0.0;
        }
        // solve_update (fluid.wgsl:543-559): p, r, and the preconditioned residual.
        const float a = (float)alpha;
        for_my_blocks([&](uint32_t b, uint32_t ri, uint32_t m) {
            float r[2], diag[2], z[2];
            bool water[2];
            for (int k = 0; k < 2; k++) {
                const uint32_t cell = b * 64u + lane + 32u * k;
                water[k] = cfv(D, F_TYPE, cell) == WATER_T;
                diag[k] = 1.0f, r[k] = 0.0f;
                if (!water[k]) continue;
                *cfp(D, F_P, cell) = cfv(D, F_P, cell) + a * cfv(D, F_D + 1 - old, cell);
                r[k] = cfv(D, F_R, cell) - a * cfv(D, F_Q, cell);
                *cfp(D, F_R, cell) = r[k];
                diag[k] = cfv(D, F_DIAG, cell);
            }
            warp_precondition(zl[warp], wl[warp], lane, r, diag, water, z);
            for (int k = 0; k < 2; k++)
                if (water[k]) *cfp(D, F_Z, b * 64u + lane + 32u * k) = z[k];
            A sx = warp_tree64(M::prod(r[0], z[0]), M::prod(r[1], z[1]));
            A sy = warp_tree64(M::prod(r[0], r[0]), M::prod(r[1], r[1]));
            if (lane == 0) part[0][ri][m] = sx, part[1][ri][m] = sy;
        });
        publish(0, D.px);
        publish(1, D.py);
        if (!grid_sync(st, gen)) return;
        // solve_beta (fluid.wgsl:561-578).
        {
            A sx = tree256<A>(D.px, red);
            A sy = tree256<A>(D.py, red);
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
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->rz = rz, st->alpha = alpha, st->beta = beta, st->b_norm = b_norm, st->r_norm = r_norm;
        st->solver_on = 0u;
        st->s.solve_iters = iters, st->s.iters_max = iters_max, st->s.unconverged = unconverged;
        st->s.rz = (float)rz, st->s.alpha = (float)alpha, st->s.beta = (float)beta;
        st->s.b_norm = (float)b_norm, st->s.r_norm = (float)r_norm;
    }
}

}  // namespace ntr
