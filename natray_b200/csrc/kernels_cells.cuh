// Per-cell and per-vertex kernels of the step: air carry/fill/substep (shaders/air.wgsl),
// rubber splat/sample/substep (shaders/membrane.wgsl, bullet.wgsl:426-611), grid prep,
// projection and velocity extension (shaders/fluid.wgsl:305-674), and the PCG solve
// (fluid.wgsl:381-578).
//
// Cell kernels run a grid-stride loop over this step's cells (64 per block, field-major
// storage, so a warp touches 128 contiguous bytes of a field). Kernels that need a block's 64
// cells together (the block-local preconditioner and the per-block partial sums) run 4 blocks
// per 256-thread CTA.
#pragma once

#include "dev.cuh"

namespace ntr {

#define CELL_LOOP(D, st)                                                                  \
    const uint32_t n_cells_ = min((st)->s.n_blocks, (D).cap_blocks) * 64u;                \
    for (uint32_t cell = C.x() * blockDim.x + threadIdx.x; cell < n_cells_; cell += C.nx() * blockDim.x)

__device__ __forceinline__ float* cfp(const Dev& D, uint32_t f, uint32_t cell) { return D.cf + (size_t)f * D.cap_cells + cell; }
__device__ __forceinline__ float cfv(const Dev& D, uint32_t f, uint32_t cell) { return D.cf[(size_t)f * D.cap_cells + cell]; }
__device__ __forceinline__ int32_t accv(const Dev& D, uint32_t f, uint32_t cell) { return D.acc[(size_t)f * D.cap_cells + cell]; }
__device__ __forceinline__ int32_t* accp(const Dev& D, uint32_t f, uint32_t cell) { return D.acc + (size_t)f * D.cap_cells + cell; }
__device__ __forceinline__ float cell_type(const Dev& D, uint32_t cell) { return cell == NONE ? GAS_T : cfv(D, F_TYPE, cell); }
__device__ __forceinline__ float dt_of(const DevState* st) { return (float)st->s.dt_ns * 1e-9f; }
__device__ __forceinline__ float now_of(const DevState* st) { return (float)st->s.t_ns * 1e-9f; }

// ---- gas, air.wgsl:34-83, 150-235 ----------------------------------------------------------------
struct Gas {
    float rho;
    V3 m;
    float e;
};
__device__ __forceinline__ Gas read_gas(const Dev& D, int buf, uint32_t cell) {
    const float* a = D.air[buf];
    size_t cc = D.cap_cells;
    return {a[cell], {a[cc + cell], a[2 * cc + cell], a[3 * cc + cell]}, a[4 * cc + cell]};
}
__device__ __forceinline__ void write_gas(const Dev& D, int buf, uint32_t cell, const Gas& g) {
    float* a = D.air[buf];
    size_t cc = D.cap_cells;
    a[cell] = g.rho, a[cc + cell] = g.m.x, a[2 * cc + cell] = g.m.y, a[3 * cc + cell] = g.m.z, a[4 * cc + cell] = g.e;
}
__device__ __forceinline__ Gas gas_at_rest(float rho, float p) { return {rho, {0.0f, 0.0f, 0.0f}, p / (GAMMA_F - 1.0f)}; }
__device__ __forceinline__ Gas ambient() { return gas_at_rest(RHO_ATM, P_ATM); }
__device__ __forceinline__ Gas no_gas() { return {0.0f, {0.0f, 0.0f, 0.0f}, 0.0f}; }
__device__ __forceinline__ float gas_p(const Gas& g) { return (GAMMA_F - 1.0f) * (g.e - 0.5f * dot(g.m, g.m) / g.rho); }
__device__ __forceinline__ Gas floored(Gas o) {
    o.rho = mx(o.rho, RHO_VAPOUR);
    o.e = mx(o.e, P_VAPOUR / (GAMMA_F - 1.0f) + 0.5f * dot(o.m, o.m) / o.rho);
    return o;
}
__device__ __forceinline__ bool free_gas(const Dev& D, uint32_t cell) { return cell == NONE || cfv(D, F_TYPE, cell) == GAS_T; }

__device__ __forceinline__ Gas hll(const Gas& l, const Gas& r, uint32_t d) {
    float pl = gas_p(l), pr = gas_p(r);
    float ul = l.m[d] / l.rho, ur = r.m[d] / r.rho;
    float cl = sqrtf(GAMMA_F * pl / l.rho), cr = sqrtf(GAMMA_F * pr / r.rho);
    float sl = mn(ul - cl, ur - cr), sr = mx(ul + cl, ur + cr);
    V3 ml = l.m * ul;
    ml[d] += pl;
    V3 mr = r.m * ur;
    mr[d] += pr;
    Gas fl = {l.rho * ul, ml, (l.e + pl) * ul};
    Gas fr = {r.rho * ur, mr, (r.e + pr) * ur};
    if (sl >= 0.0f) return fl;
    if (sr <= 0.0f) return fr;
    float k = 1.0f / (sr - sl);
    float a = sr * k, b = -sl * k, c = sl * sr * k;
    return {a * fl.rho + b * fr.rho + c * (r.rho - l.rho), a * fl.m + b * fr.m + c * (r.m - l.m), a * fl.e + b * fr.e + c * (r.e - l.e)};
}

// The state across face (d, hi) of `cell` (air.wgsl:150-200): the outside air, the neighbour's
// gas, or a ghost mirrored at a moving wall. `nb` is the neighbour, `nty` its type and `ng` its
// gas (loaded by the caller; meaningless when nb is NONE).
__device__ __forceinline__ Gas across(const Dev& D, uint32_t cell, const Gas& own, uint32_t d, bool hi, uint32_t nb, float nty, const Gas& ng) {
    if (nb == NONE) return ambient();
    if (nty == GAS_T) return ng;
    float w = cfv(D, F_U + d, hi ? nb : cell);
    if (nty == RUBBER_T) w = from_fp(accv(D, A_MV + d, nb), FP_A) / from_fp(accv(D, A_MW, nb), FP_A);
    Gas gg = own;
    float u = own.m[d] / own.rho;
    gg.m[d] = own.rho * (2.0f * w - u);
    gg.e = own.e + 0.5f * (gg.m[d] * gg.m[d] - own.m[d] * own.m[d]) / own.rho;
    return gg;
}

__device__ float gas_pressure_at(const Dev& D, const Grid& g, int buf, V3 x) {
    I3 base = vi(vfloor((x - g.org) / g.h - 1.0f));
    V3 fx = (x - g.org) / g.h - 0.5f - vf(base);
    V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    const Stencil27 sc = stencil_of(g, near_of(g, base), base);
    float sx = 0.0f, sy = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                uint32_t cell = sc.cell(a, b, c);
                float w = wx[a] * wy[b] * wz[c];
                if (cell == NONE) {
                    sx = sx + w * P_ATM;
                    sy = sy + w;
                } else if (free_gas(D, cell)) {
                    sx = sx + w * gas_p(read_gas(D, buf, cell));
                    sy = sy + w;
                }
            }
    return sy > 1e-6f ? sx / sy : P_ATM;
}

// ---- air_carry, air.wgsl:85-99 --------------------------------------------------------------------
template <class CT>
__device__ __forceinline__ void air_carry_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const int cur = cur_of(st);
    const uint32_t* list = D.block_list[cur];
    CELL_LOOP(D, st) {
        uint32_t b = cell >> 6, li = cell & 63u;
        uint32_t o = lookup(D.mask[cur ^ 1], D.prefix[cur ^ 1], list[b], D.cap_blocks);
        Gas g = ambient();
        if (o != NONE && o < st->s.n_blocks_prev) g = read_gas(D, 0, o * 64u + li);
        write_gas(D, 1, cell, g);
        if (li == 0) D.block_active[b] = 0u;
    }
}
__global__ void k_air_carry(Dev D) { air_carry_body(D, HwCta{}); }
__global__ void k_air_carry_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    air_carry_body(sD, c);
}

// ---- mem_splat, membrane.wgsl:182-217 -------------------------------------------------------------
// Sums of runs of equal keys among the lanes of a warp: the lanes of a run (consecutive lanes
// with the same key) hold their run's sum in its last lane, which `last` tells. Every lane takes
// part; the shuffles are uniform (a segmented scan over the run boundaries from a ballot).
struct WarpRuns {
    uint32_t start;  // first lane of this lane's run
    bool last;       // this lane ends its run
    __device__ __forceinline__ WarpRuns(uint32_t key, uint32_t lane) {
        const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1), next = __shfl_down_sync(0xffffffffu, key, 1);
        const uint32_t heads = __ballot_sync(0xffffffffu, lane == 0 || prev != key);
        start = 31u - __clz(heads & (0xffffffffu >> (31u - lane)));
        last = lane == 31 || next != key;
    }
    __device__ __forceinline__ int32_t sum(int32_t x, uint32_t lane) const {
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= start + o) x += y;
        }
        return x;
    }
};

// The rubber's splat: per vertex its area-weighted velocity into its own
// cell, and where it touches water its push and area over the 27 cells around it. Vertices are
// in the mesh's spatial order, so neighbouring lanes of a warp mostly add to the same cells: each
// run of lanes with one target cell sums its i32 terms across the lanes and its last lane adds
// the sums with one atomic each. Integer sums: the same as an atomic per term, in any grouping.
template <class CT>
__device__ __forceinline__ void mem_splat_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    const uint32_t i = C.x() * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    bool valid = i < D.Nv && D.mem_mass[i] != 0.0f;
    float2 pa = make_float2(0.0f, 0.0f);
    float4 x4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (valid) {
        pa = D.mem_push[i];
        valid = pa.y > 0.0f;
        x4 = D.mem_x[0][i];
    }
    if (!__any_sync(0xffffffffu, valid)) return;  // warp-uniform
    const uint32_t own = valid ? cell_at(g, own_cell(g, xyz(x4))) : NONE;
    {
        const WarpRuns r(own, lane);
        int32_t vw = 0, vx = 0, vy = 0, vz = 0;
        if (own != NONE) {
            const float a = pa.y * 1e6f;
            const float4 mv = D.mem_v[0][i];
            vw = to_fp(a, FP_A), vx = to_fp(a * mv.x, FP_A), vy = to_fp(a * mv.y, FP_A), vz = to_fp(a * mv.z, FP_A);
        }
        vw = r.sum(vw, lane), vx = r.sum(vx, lane), vy = r.sum(vy, lane), vz = r.sum(vz, lane);
        if (r.last && own != NONE) {
            atomicAdd(accp(D, A_MW, own), vw);
            atomicAdd(accp(D, A_MV + 0, own), vx);
            atomicAdd(accp(D, A_MV + 1, own), vy);
            atomicAdd(accp(D, A_MV + 2, own), vz);
        }
    }
    const bool on_water = valid && D.mem_water[i].w >= CONTACT_F;
    if (!__any_sync(0xffffffffu, on_water)) return;  // warp-uniform
    V3 x = (xyz(x4) - g.org) / g.h - 0.5f;
    I3 base = vi(vfloor(x - 0.5f));
    V3 fx = x - vf(base);
    V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    const Stencil27 sc = stencil_of(g, near_of(g, on_water ? base : I3{0, 0, 0}), on_water ? base : I3{0, 0, 0});
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const uint32_t cell = on_water ? sc.cell(a, b, c) : NONE;
                const WarpRuns r(cell, lane);
                int32_t sf = 0, sa = 0;
                if (cell != NONE) {
                    const float w = wx[a] * wy[b] * wz[c];
                    sf = to_fp(w * pa.x, FP_F), sa = to_fp(w * pa.y * 1e6f, FP_A);
                }
                sf = r.sum(sf, lane), sa = r.sum(sa, lane);
                if (r.last && cell != NONE) {
                    atomicAdd(accp(D, A_MF, cell), sf);
                    atomicAdd(accp(D, A_MA, cell), sa);
                }
            }
}
__global__ void k_mem_splat(Dev D) { mem_splat_body(D, HwCta{}); }
__global__ void k_mem_splat_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    mem_splat_body(sD, c);
}

// ---- grid_prep, fluid.wgsl:305-356 -----------------------------------------------------------------
// One cell: its type, velocities and pressure from the transfer sums. `s8`: its sums of fields
// 0-7 (momenta and weights of the three face lattices, A_WC, A_PC); the rest are read here.
__device__ __forceinline__ void grid_prep_cell(const Dev& D, const Grid& g, V3 knot, float kr, float dt, const float (&grav)[3], uint32_t cell,
                                               const int32_t (&s8)[8]) {
    const float hh = g.h;
    float ty = GAS_T;
    I3 c = cell_coord(g, cell);
    bool ground = g.org.y + ((float)c.y + 0.5f) * hh < 0.0f;
    V3 p = g.org + (vf(c) + 0.5f) * hh - knot;
    bool knot_c = p.y > 0.0f && p.y < 2.0f * kr && sqrtf(p.x * p.x + p.z * p.z) < kr;
    if (ground || knot_c)
        ty = SOLID_T;
    else if (accv(D, A_N, cell) > 0)
        ty = WATER_T;
#pragma unroll
    for (uint32_t d = 0; d < 3; d++) {
        float w = from_fp(s8[a_wt(d)], FP_W);
        float u = 0.0f;
        if (w > 1e-6f) u = from_fp(s8[a_mom(d)], FP_M) / w + dt * grav[d];
        *cfp(D, F_U + d, cell) = u;
    }
    float wc = from_fp(s8[A_WC], FP_W);
    float ma = from_fp(accv(D, A_MA, cell), FP_A);
    if (ty == GAS_T && accv(D, A_MW, cell) > 0) ty = RUBBER_T;
    float pr = 0.0f;
    if (ty == WATER_T && wc > 1e-6f) {
        pr = from_fp(s8[A_PC], FP_P) / wc * 1e6f;
    } else if (ty != WATER_T && ty != SOLID_T && ma > 0.0f) {
        ty = COVERED_T;
        pr = from_fp(accv(D, A_MF, cell), FP_F) / ma * 1e6f;
    }
    *cfp(D, F_TYPE, cell) = ty;
    *cfp(D, F_P, cell) = pr;
}

__constant__ int8_t E6[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
__device__ __forceinline__ I3 e6(int k) { return {E6[k][0], E6[k][1], E6[k][2]}; }
__device__ __forceinline__ I3 ed(uint32_t d, int s) { return {d == 0 ? s : 0, d == 1 ? s : 0, d == 2 ? s : 0}; }

// ---- air_fill (reads the second air buffer, writes the first), air.wgsl:101-148 ---------------
template <class CT>
__device__ __forceinline__ void air_fill_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    CELL_LOOP(D, st) {
        float ty = cfv(D, F_TYPE, cell);
        if (ty == WATER_T || ty == SOLID_T) {
            write_gas(D, 0, cell, no_gas());
            continue;
        }
        Gas gg = read_gas(D, 1, cell);
        if (gg.rho <= 0.0f) {
            Gas sum = no_gas();
            float cnt = 0.0f;
            for (int k = 0; k < 6; k++) {
                uint32_t nb = neighbour(g, cell, e6(k));
                if (nb == NONE) continue;
                Gas q = read_gas(D, 1, nb);
                if (q.rho > 0.0f) {
                    sum = {sum.rho + q.rho, sum.m + q.m, sum.e + q.e};
                    cnt += 1.0f;
                }
            }
            if (cnt > 0.0f)
                gg = {sum.rho / cnt, sum.m / cnt, sum.e / cnt};
            else
                gg = gas_at_rest(RHO_VAPOUR, P_VAPOUR);
        }
        write_gas(D, 0, cell, gg);
        if (ty == GAS_T) *cfp(D, F_P, cell) = gas_p(gg) - P_ATM;
        if (ty == RUBBER_T) {
            float p = BIG_F;
            for (int k = 0; k < 6; k++) {
                uint32_t nb = neighbour(g, cell, e6(k));
                if (nb == NONE || !free_gas(D, nb)) continue;
                Gas q = read_gas(D, 1, nb);
                if (q.rho > 0.0f) p = mn(p, gas_p(q));
            }
            *cfp(D, F_P, cell) = (p < BIG_F ? p : gas_p(gg)) - P_ATM;
        }
    }
}
__global__ void k_air_fill(Dev D) { air_fill_body(D, HwCta{}); }
__global__ void k_air_fill_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    air_fill_body(sD, c);
}

// ---- bullet_apply, bullet.wgsl:385-393 ---------------------------------------------------------------
template <class CT>
__device__ __forceinline__ void bullet_apply_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    CELL_LOOP(D, st) {
#pragma unroll
        for (uint32_t d = 0; d < 3; d++) {
            int32_t du = accv(D, A_BU + d, cell);
            if (du != 0) *cfp(D, F_U + d, cell) = cfv(D, F_U + d, cell) + from_fp(du, FP_M);
        }
    }
}
// A one-scene step's: CTA 0 also starts the pressure solve's grid barrier counter from zero
// (one graph node fewer than a memset; a many-scene step has k_solve_reset_m).
__global__ void k_bullet_apply(Dev D) {
    if (blockIdx.x == 0 && threadIdx.x == 0) D.st->bar_count = 0u;
    bullet_apply_body(D, HwCta{});
}
__global__ void k_bullet_apply_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    bullet_apply_body(sD, c);
}

// ---- the pressure solve -----------------------------------------------------------------------------
__device__ __forceinline__ float bounded(float u, float hi, float lo) {
    if (lo == SOLID_T && hi == SOLID_T) return 0.0f;
    if (lo == SOLID_T) return mx(u, 0.0f);
    if (hi == SOLID_T) return mn(u, 0.0f);
    return u;
}
__device__ __forceinline__ float face_u(const Dev& D, uint32_t cell, uint32_t lo, uint32_t d) {
    if (cell == NONE) return 0.0f;
    return bounded(cfv(D, F_U + d, cell), cfv(D, F_TYPE, cell), cell_type(D, lo));
}
__device__ __forceinline__ float pressure_of(const Dev& D, uint32_t cell) {
    if (cell == NONE) return 0.0f;
    float p = cfv(D, F_P, cell);
    return cfv(D, F_TYPE, cell) == WATER_T ? mx(p, P_VAPOUR - P_ATM) : p;
}

// ---- project, extend, fluid.wgsl:580-674 -------------------------------------------------------------
template <class CT>
__device__ __forceinline__ void project_body(const Dev& D, const CT& C) {
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    const float k = dt_of(st) / (D.U->fluid[0] * g.h);
    __shared__ uint32_t s_cnt[2];
    if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    uint32_t n_water = 0, n_gas = 0;  // the step's cells by type, for its work counts
    CELL_LOOP(D, st) {
        float ty = cfv(D, F_TYPE, cell);
        n_water += ty == WATER_T;
        n_gas += ty == GAS_T;
#pragma unroll
        for (uint32_t d = 0; d < 3; d++) {
            uint32_t nb = neighbour(g, cell, ed(d, -1));
            float nt = cell_type(D, nb);
            float u = bounded(cfv(D, F_U + d, cell), ty, nt);
            if (ty != SOLID_T && nt != SOLID_T && (ty == WATER_T || nt == WATER_T)) u -= k * (pressure_of(D, cell) - pressure_of(D, nb));
            *cfp(D, F_U + d, cell) = u;
        }
    }
    n_water = __reduce_add_sync(0xffffffffu, n_water);
    n_gas = __reduce_add_sync(0xffffffffu, n_gas);
    if ((threadIdx.x & 31u) == 0) {
        atomicAdd(&s_cnt[0], n_water);
        atomicAdd(&s_cnt[1], n_gas);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&st->n_water, s_cnt[0]);
        atomicAdd(&st->n_gas, s_cnt[1]);
    }
}
__global__ void k_project(Dev D) { project_body(D, HwCta{}); }
__global__ void k_project_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    project_body(sD, c);
}

// Velocity extension in two passes (fluid.wgsl:604-674). Each cell loads everything its pass
// reads first, all loads in flight together, then decides in the reference's order.
__device__ __forceinline__ uint32_t cube_at(int x, int y, int z) { return (uint32_t)((x + 1) * 9 + (y + 1) * 3 + (z + 1)); }

template <class CT>
__device__ __forceinline__ void extend_1_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    CELL_LOOP(D, st) {
        // A water cell has all three of its faces set (face_set at offset 0 is true on every
        // axis): it keeps its velocities and needs nothing around it.
        if (cfv(D, F_TYPE, cell) == WATER_T) {
#pragma unroll
            for (int d = 0; d < 3; d++) *cfp(D, F_EXT + d, cell) = cfv(D, F_U + d, cell);
            *cfp(D, F_EXT_SET, cell) = 7.0f;
            continue;
        }
        // Types of the 3^3 cells around (GAS outside the grid), of the cells two down each axis,
        // and the face velocities of the cell and its six neighbours.
        // face_set below reads 16 of the 27: the cell, its 6 face neighbours and the 9 edge
        // neighbours with a step down along some axis (o - e_d for a face offset o); the 8
        // corners and the 3 edges up along both axes are neither looked up nor loaded.
        auto read = [](int k) {
            const int x = k / 9 - 1, y = (k / 3) % 3 - 1, z = k % 3 - 1;
            const int nnz = (x != 0) + (y != 0) + (z != 0);
            return nnz <= 1 || (nnz == 2 && (x < 0 || y < 0 || z < 0));
        };
        uint32_t nc[27], n2[3];
#pragma unroll
        for (int k = 0; k < 27; k++) nc[k] = k == 13 ? cell : (read(k) ? neighbour(g, cell, I3{k / 9 - 1, (k / 3) % 3 - 1, k % 3 - 1}) : NONE);
#pragma unroll
        for (int d = 0; d < 3; d++) n2[d] = neighbour(g, cell, ed((uint32_t)d, -2));
        float T[27], T2[3], un[6][3], uo[3];
#pragma unroll
        for (int k = 0; k < 27; k++) T[k] = nc[k] != NONE ? cfv(D, F_TYPE, nc[k]) : GAS_T;
#pragma unroll
        for (int d = 0; d < 3; d++) T2[d] = n2[d] != NONE ? cfv(D, F_TYPE, n2[d]) : GAS_T;
#pragma unroll
        for (int d = 0; d < 3; d++) uo[d] = cfv(D, F_U + d, cell);
#pragma unroll
        for (int j = 0; j < 6; j++) {
            const I3 o = e6(j);
            const uint32_t nb = nc[cube_at(o.x, o.y, o.z)];
#pragma unroll
            for (int d = 0; d < 3; d++) un[j][d] = nb != NONE ? cfv(D, F_U + d, nb) : 0.0f;
        }
        // face_set (fluid.wgsl:604-610) of the cell at offset o: it exists, and it or the cell
        // below it along d is water.
        auto face_set = [&](I3 o, int d) -> bool {
            if (nc[cube_at(o.x, o.y, o.z)] == NONE) return false;
            if (T[cube_at(o.x, o.y, o.z)] == WATER_T) return true;
            const I3 b = o - ed((uint32_t)d, 1);
            const float tb = (b.x < -1 || b.y < -1 || b.z < -1) ? T2[d] : T[cube_at(b.x, b.y, b.z)];
            return tb == WATER_T;
        };
        uint32_t done = 0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            float u = uo[d];
            if (face_set(I3{0, 0, 0}, d)) {
                done |= 1u << d;
            } else {
                float sum = 0.0f, cnt = 0.0f;
#pragma unroll
                for (int j = 0; j < 6; j++) {
                    if (face_set(e6(j), d)) {
                        sum += un[j][d];
                        cnt += 1.0f;
                    }
                }
                if (cnt > 0.0f) {
                    u = sum / cnt;
                    done |= 1u << d;
                }
            }
            *cfp(D, F_EXT + d, cell) = u;
        }
        *cfp(D, F_EXT_SET, cell) = (float)done;
    }
}
__global__ void k_extend_1(Dev D) { extend_1_body(D, HwCta{}); }
__global__ void k_extend_1_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    extend_1_body(sD, c);
}

template <class CT>
__device__ __forceinline__ void extend_2_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    CELL_LOOP(D, st) {
        const float ty = cfv(D, F_TYPE, cell);
        const uint32_t set = f2u(cfv(D, F_EXT_SET, cell));
        // All three faces set (water cells among them): each takes its extended value, bounded
        // by the types of the cell and the one below it; the neighbours' values are not needed.
        if (set == 7u) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const uint32_t lo = neighbour(g, cell, ed((uint32_t)d, -1));
                *cfp(D, F_U + d, cell) = bounded(cfv(D, F_EXT + d, cell), ty, lo != NONE ? cfv(D, F_TYPE, lo) : GAS_T);
            }
            continue;
        }
        uint32_t nb[6], lo[3];
#pragma unroll
        for (int j = 0; j < 6; j++) nb[j] = neighbour(g, cell, e6(j));
#pragma unroll
        for (int d = 0; d < 3; d++) lo[d] = nb[2 * d];  // e6 order: -x, +x, -y, +y, -z, +z
        float uo[3], eo[3], tlo[3], en[6][3];
        uint32_t sn[6];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            uo[d] = cfv(D, F_U + d, cell);
            eo[d] = cfv(D, F_EXT + d, cell);
            tlo[d] = lo[d] != NONE ? cfv(D, F_TYPE, lo[d]) : GAS_T;
        }
#pragma unroll
        for (int j = 0; j < 6; j++) {
            sn[j] = nb[j] != NONE ? f2u(cfv(D, F_EXT_SET, nb[j])) : 0u;
#pragma unroll
            for (int d = 0; d < 3; d++) en[j][d] = nb[j] != NONE ? cfv(D, F_EXT + d, nb[j]) : 0.0f;
        }
#pragma unroll
        for (int d = 0; d < 3; d++) {
            float u = uo[d];
            if ((set >> d) & 1u) {
                u = eo[d];
            } else {
                float sum = 0.0f, cnt = 0.0f;
#pragma unroll
                for (int j = 0; j < 6; j++) {
                    if (nb[j] != NONE && ((sn[j] >> d) & 1u)) {
                        sum += en[j][d];
                        cnt += 1.0f;
                    }
                }
                if (cnt > 0.0f) u = sum / cnt;
            }
            *cfp(D, F_U + d, cell) = bounded(u, ty, tlo[d]);
        }
    }
}
__global__ void k_extend_2(Dev D) { extend_2_body(D, HwCta{}); }
__global__ void k_extend_2_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    extend_2_body(sD, c);
}

// ---- sampling the grid at a point, membrane.wgsl:219-239, bullet.wgsl:113-158 ---------------------------
__device__ __forceinline__ float2 sample_grid(const Dev& D, const Grid& g, V3 x, uint32_t fu, uint32_t fw) {
    I3 base = vi(vfloor(x - 0.5f));
    V3 fx = x - vf(base);
    V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    const Stencil27 sc = stencil_of(g, near_of(g, base), base);
    float sx = 0.0f, sy = 0.0f;
    // A plane of 9 cells at a time: its 18 loads go out together, then the sums in order.
#pragma unroll
    for (int a = 0; a < 3; a++) {
        uint32_t cells[9];
        int32_t wv[9];
        float uv[9];
#pragma unroll
        for (int k = 0; k < 9; k++) {
            cells[k] = sc.cell(a, k / 3, k % 3);
            wv[k] = cells[k] != NONE ? accv(D, fw, cells[k]) : 0;
            uv[k] = cells[k] != NONE ? cfv(D, fu, cells[k]) : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < 9; k++) {
            if (cells[k] == NONE) continue;
            float w = wx[a] * wy[k / 3] * wz[k % 3] * from_fp(wv[k], FP_W);
            sx = sx + w * uv[k];
            sy = sy + w;
        }
    }
    return make_float2(sx, sy);
}

// ---- 3^3 stencils taken by a warp: lane c < 27 has cell base + (c / 9, (c / 3) % 3, c % 3) --------
__device__ __forceinline__ float wsel(V3 w, int i) { return i == 0 ? w.x : (i == 1 ? w.y : w.z); }

// The sums of the lanes' `vx` and `vy` where `present`, added in lane order, which is the order
// of the single-thread stencil loops (a, b, c). Every lane gets them.
__device__ __forceinline__ float2 fold27(bool present, float vx, float vy) {
    const uint32_t pm = __ballot_sync(0xffffffffu, present);
    float sx = 0.0f, sy = 0.0f;
#pragma unroll
    for (int c = 0; c < 27; c++) {
        const float a = __shfl_sync(0xffffffffu, vx, c), b = __shfl_sync(0xffffffffu, vy, c);
        if ((pm >> c) & 1u) sx = sx + a, sy = sy + b;
    }
    return make_float2(sx, sy);
}

// sample_grid by a warp.
__device__ __forceinline__ float2 warp_sample_grid(const Dev& D, const Grid& g, V3 x, uint32_t fu, uint32_t fw, int lane) {
    I3 base = vi(vfloor(x - 0.5f));
    V3 fx = x - vf(base);
    V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    const int a = lane / 9, b = (lane / 3) % 3, c = lane % 3;
    bool present = false;
    float wu = 0.0f, w = 0.0f;
    if (lane < 27) {
        const uint32_t cell = cell_at(g, base + I3{a, b, c});
        if (cell != NONE) {
            present = true;
            w = wsel(wx, a) * wsel(wy, b) * wsel(wz, c) * from_fp(accv(D, fw, cell), FP_W);
            wu = w * cfv(D, fu, cell);
        }
    }
    return fold27(present, wu, w);
}

// Four lanes per vertex, one per stencil (the three velocity lattices and the cell centres).
template <class CT>
__device__ __forceinline__ void mem_sample_body(const Dev& D, const CT& C) {
    const DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    const uint32_t t = C.x() * blockDim.x + threadIdx.x;
    const uint32_t i = t >> 2, q = t & 3u;
    const bool act = i < D.Nv && D.mem_mass[i] != 0.0f;
    float r = 0.0f;
    if (act) {
        V3 x = (xyz(D.mem_x[0][i]) - g.org) / g.h;
        // One call for the four lanes of a vertex (three face lattices and the fill, whose
        // lattice offset is 0.5 on every axis), so that they do not run one after the other.
        const bool fill = q == 3u;
        const float2 s = sample_grid(D, g, x - lattice_offset(q), fill ? (uint32_t)F_TYPE : F_U + q, fill ? (uint32_t)A_WC : a_wt(q));
        r = fill ? s.y / 8.0f : (s.y > 1e-6f ? s.x / s.y : 0.0f);
    }
    const int l0 = (int)(threadIdx.x & 28u);
    const float v0 = __shfl_sync(0xffffffffu, r, l0), v1 = __shfl_sync(0xffffffffu, r, l0 + 1);
    const float v2 = __shfl_sync(0xffffffffu, r, l0 + 2), v3 = __shfl_sync(0xffffffffu, r, l0 + 3);
    if (act && q == 0u) D.mem_water[i] = make_float4(v0, v1, v2, v3);
}
// CTAs of 128 threads, nine an SM (at most 56 registers): the 40,962 x 4 threads of a 1M-particle
// scene's membrane fit in one wave (four CTAs of 256 an SM at 62 registers left a second wave of
// 49 CTAs): 22.8 -> 20.5 us.
__global__ void __launch_bounds__(128, 9) k_mem_sample(Dev D) { mem_sample_body(D, HwCta{}); }
__global__ void k_mem_sample_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    mem_sample_body(sD, c);
}

// ---- air_substep, air.wgsl:237-269 --------------------------------------------------------------------
// Three CTAs an SM (80 registers, from 84 and two CTAs): 38.5 -> 34.8 us a step at 1M particles
// (the many-scene kernel's shape; the one-scene kernel's is below).
template <class CT>
__device__ __forceinline__ void air_substep_body(const Dev& D, const CT& C, int par) {
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const Grid g = grid_of(D, cur_of(st));
    const float hh = g.h;
    const float k = dt_of(st) / (float)max(D.U->mem[2], 1u) / hh;
    float lim = BIG_F;
    CELL_LOOP(D, st) {
        // A cell that is not gas only carries its gas over (most cells of the active blocks are
        // water). A gas cell loads its six neighbours' types and gas, all in flight together (a
        // missing neighbour loads this cell's and is not used).
        const float ty = cfv(D, F_TYPE, cell);
        Gas gg = read_gas(D, par, cell);
        if (ty != GAS_T) {
            write_gas(D, 1 - par, cell, gg);
            continue;
        }
        uint32_t nbr[6];
        float nty[6];
        Gas ng[6];
#pragma unroll
        for (int j = 0; j < 6; j++) nbr[j] = neighbour(g, cell, ed((uint32_t)(j >> 1), (j & 1) ? 1 : -1));
#pragma unroll
        for (int j = 0; j < 6; j++) {
            const uint32_t at = nbr[j] != NONE ? nbr[j] : cell;
            nty[j] = cfv(D, F_TYPE, at);
            ng[j] = read_gas(D, par, at);
        }
        Gas f = no_gas();
#pragma unroll
        for (uint32_t d = 0; d < 3; d++) {
            Gas lo = hll(across(D, cell, gg, d, false, nbr[2 * d], nty[2 * d], ng[2 * d]), gg, d);
            Gas hi = hll(gg, across(D, cell, gg, d, true, nbr[2 * d + 1], nty[2 * d + 1], ng[2 * d + 1]), d);
            f = {f.rho + hi.rho - lo.rho, f.m + hi.m - lo.m, f.e + hi.e - lo.e};
        }
        Gas n = floored(Gas{gg.rho - k * f.rho, gg.m - k * f.m, gg.e - k * f.e});
        write_gas(D, 1 - par, cell, n);
        V3 u = n.m / n.rho;
        float p = gas_p(n);
        float c = sqrtf(GAMMA_F * p / n.rho);
        float limit = CFL_AIR * hh / (fabsf(u.x) + fabsf(u.y) + fabsf(u.z) + 3.0f * c);
        lim = mn(lim, limit);
        if (fabsf(p - P_ATM) > 10.0f || length(u) > 0.05f) D.block_active[cell >> 6] = 1u;
    }
    for (int o = 16; o > 0; o >>= 1) lim = fminf(lim, __shfl_down_sync(0xffffffffu, lim, o));
    // The reference lowers air_dt once per workgroup, so only when there are cells.
    if ((threadIdx.x & 31) == 0 && n_cells_ > 0) atomicMin((unsigned int*)&st->s.air_dt, __float_as_uint(lim));
}
// A one-scene step's at four CTAs an SM (64 registers, a few spilled): alone it is slower than at
// three (35.5 against 34.0 us a step at 1M particles), but beside G2P and the rubber substeps the
// step's graph is faster (0.493 against 0.495 ms).
__global__ void __launch_bounds__(256, 4) k_air_substep(Dev D, int par) { air_substep_body(D, HwCta{}, par); }

// The air's substep over many scenes: substep i, for the scenes whose step has that many.
__global__ void __launch_bounds__(256, 3) k_air_substep_m(Multi M, uint32_t i, int par) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    if (i >= sD.U->mem[2]) return;
    air_substep_body(sD, c, par);
}

}  // namespace ntr
