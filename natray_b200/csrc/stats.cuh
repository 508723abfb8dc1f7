// Debug and energy statistics of the simulation (include/natray.h, ntr_sim_stats): what
// `Sim::debug_stats` (src/sim.rs:691-863) prints, computed on the device. The reference reads
// every buffer back and loops over it on the CPU; here four reduction kernels run on the
// simulation's stream (particles; cells of the step's blocks; membrane vertices; triangles)
// and only their totals come back (a few hundred bytes, plus the three most tense triangles of
// each CTA of the triangle pass). Sums are in FP64 (the reference's means and fill mean are
// sequential FP32 sums); counts, minima and maxima are exact. Minima and maxima of floats go
// through atomics on an order-preserving integer image of the float.
//
// Included at the end of sim.cu (it uses the Sim internals there).
#pragma once

namespace ntr {

__device__ __forceinline__ uint32_t fkey(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float fkey_inv(uint32_t k) {
    const uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    memcpy(&f, &b, 4);
    return f;
}

// Device accumulators of one ntr_sim_stats call.
struct StatsAcc {
    uint32_t water, full_cells, free_verts, on_water, torn, air_cells, vapour, pad;
    uint32_t lo[3], hi[3], mlo[3], mhi[3];  // ordered keys
    uint32_t fill_min, plo, phi, umax, rubber_vmax, pad2;
    unsigned long long fastest;  // speed key << 32 | ~particle index: the first of the fastest wins
    double sum_x[3], sum_v[3], ke, fill_sum, inside;
};

// One of a triangle pass CTA's three most tense triangles.
struct TensionCand {
    double tension;
    uint32_t tri;
    float l1, l2;
};

__device__ __forceinline__ float warp_min_f(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max_f(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ uint32_t warp_sum_u(uint32_t v) { return __reduce_add_sync(0xffffffffu, v); }

// Live water particles (vel.w > 0.5): count, box, sums of position and velocity, kinetic
// energy per unit mass (0.5 |v|^2 with |v|^2 in f32, as the reference), the fastest, and each
// particle's own cell counted in the step's cells (src/sim.rs:692-714).
__global__ void __launch_bounds__(256) k_stats_particles(Dev D, StatsAcc* A, uint32_t* cell_count) {
    const Grid g = grid_of(D, cur_of(D.st));
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < D.Np;
    const float4 p = in ? D.pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 v = in ? D.vel[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const bool live = in && v.w > 0.5f;
    const V3 x = xyz(p), u = xyz(v);
    const float lsq = dot(u, u);
    const float speed = sqrtf(lsq);
    if (live) {
        const I3 c = own_cell(g, x);
        const uint32_t b = block_at(g, shr2(c));
        if (b != NONE) {
            const I3 l = c - shr2(c) * 4;
            atomicAdd(cell_count + (size_t)b * 64u + (uint32_t)(l.x * 16 + l.y * 4 + l.z), 1u);
        }
    }
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = warp_sum_u(live ? 1u : 0u);
    if (n == 0) return;
    unsigned long long fast = live ? ((unsigned long long)fkey(speed) << 32) | (unsigned long long)(~i) : 0ull;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long q = __shfl_xor_sync(0xffffffffu, fast, o);
        fast = q > fast ? q : fast;
    }
    if (lane == 0) atomicMax(&A->fastest, fast);
    const float big = 3.4028235e38f;
    const float lox = warp_min_f(live ? x.x : big), loy = warp_min_f(live ? x.y : big), loz = warp_min_f(live ? x.z : big);
    const float hix = warp_max_f(live ? x.x : -big), hiy = warp_max_f(live ? x.y : -big), hiz = warp_max_f(live ? x.z : -big);
    const double sx = warp_sum_d(live ? (double)x.x : 0.0), sy = warp_sum_d(live ? (double)x.y : 0.0), sz = warp_sum_d(live ? (double)x.z : 0.0);
    const double vx = warp_sum_d(live ? (double)u.x : 0.0), vy = warp_sum_d(live ? (double)u.y : 0.0), vz = warp_sum_d(live ? (double)u.z : 0.0);
    const double ke = warp_sum_d(live ? 0.5 * (double)lsq : 0.0);
    if (lane == 0) {
        atomicAdd(&A->water, n);
        atomicMin(&A->lo[0], fkey(lox)), atomicMin(&A->lo[1], fkey(loy)), atomicMin(&A->lo[2], fkey(loz));
        atomicMax(&A->hi[0], fkey(hix)), atomicMax(&A->hi[1], fkey(hiy)), atomicMax(&A->hi[2], fkey(hiz));
        atomicAdd(&A->sum_x[0], sx), atomicAdd(&A->sum_x[1], sy), atomicAdd(&A->sum_x[2], sz);
        atomicAdd(&A->sum_v[0], vx), atomicAdd(&A->sum_v[1], vy), atomicAdd(&A->sum_v[2], vz);
        atomicAdd(&A->ke, ke);
    }
}

// The step's cells: those at least half as full as bulk water (4 particles), and the air of
// the cells typed air: count, vapour (gauge below -90 kPa), gauge range, fastest air
// (src/sim.rs:717-718, 795-813).
__global__ void __launch_bounds__(256) k_stats_cells(Dev D, StatsAcc* A, const uint32_t* cell_count) {
    const uint32_t nb = min(D.st->s.n_blocks, D.cap_blocks);
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = c < nb * 64u;
    const bool full = in && cell_count[c] >= 4u;
    const float type = in ? D.cf[(size_t)F_TYPE * D.cap_cells + c] : 1.0f;
    const bool air = in && type == 0.0f;
    float pg = 0.0f, um = 0.0f;
    if (air) {
        const float* a = D.air[0];
        const size_t cc = D.cap_cells;
        const float rho = a[c];
        const V3 m{a[cc + c], a[2 * cc + c], a[3 * cc + c]};
        const float e = a[4 * cc + c];
        pg = 0.4f * (e - 0.5f * dot(m, m) / rho) - 101325.0f;
        um = length(m) / rho;
    }
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nf = warp_sum_u(full ? 1u : 0u), na = warp_sum_u(air ? 1u : 0u), nv = warp_sum_u(air && pg < -90e3f ? 1u : 0u);
    if (na) {
        const float big = 3.4028235e38f;
        const float lo = warp_min_f(air ? pg : big), hi = warp_max_f(air ? pg : -big), umax = warp_max_f(air ? um : -big);
        if (lane == 0) {
            atomicAdd(&A->air_cells, na), atomicAdd(&A->vapour, nv);
            atomicMin(&A->plo, fkey(lo)), atomicMax(&A->phi, fkey(hi)), atomicMax(&A->umax, fkey(umax));
        }
    }
    if (nf && lane == 0) atomicAdd(&A->full_cells, nf);
}

// Membrane vertices: box of all; of the free ones (mass > 0) the count, those on water (fill
// >= 0.05), the fill's minimum and sum; the fastest (src/sim.rs:752-767).
__global__ void __launch_bounds__(256) k_stats_verts(Dev D, StatsAcc* A) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < D.Nv;
    const V3 x = in ? xyz(D.mem_x[0][i]) : v3(0.f, 0.f, 0.f);
    const bool fr = in && D.mem_mass[i] > 0.0f;
    const float fill = in ? D.mem_water[i].w : 0.0f;
    const float sp = in ? length(xyz(D.mem_v[0][i])) : 0.0f;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = warp_sum_u(in ? 1u : 0u);
    if (n == 0) return;
    const float big = 3.4028235e38f;
    const float lox = warp_min_f(in ? x.x : big), loy = warp_min_f(in ? x.y : big), loz = warp_min_f(in ? x.z : big);
    const float hix = warp_max_f(in ? x.x : -big), hiy = warp_max_f(in ? x.y : -big), hiz = warp_max_f(in ? x.z : -big);
    const uint32_t nfree = warp_sum_u(fr ? 1u : 0u), non = warp_sum_u(fr && fill >= 0.05f ? 1u : 0u);
    const float fmin = warp_min_f(fr ? fill : big);
    const double fsum = warp_sum_d(fr ? (double)fill : 0.0);
    const float vmax = warp_max_f(in ? sp : 0.0f);
    if (lane == 0) {
        atomicMin(&A->mlo[0], fkey(lox)), atomicMin(&A->mlo[1], fkey(loy)), atomicMin(&A->mlo[2], fkey(loz));
        atomicMax(&A->mhi[0], fkey(hix)), atomicMax(&A->mhi[1], fkey(hiy)), atomicMax(&A->mhi[2], fkey(hiz));
        atomicAdd(&A->free_verts, nfree), atomicAdd(&A->on_water, non);
        if (nfree) atomicMin(&A->fill_min, fkey(fmin)), atomicAdd(&A->fill_sum, fsum);
        atomicMax(&A->rubber_vmax, fkey(vmax));
    }
}

// Ogden stress sigma(a, b) = sum_i mu_i (a^alpha_i - b^alpha_i), and the plane-stress principal
// stress of stretches (l1, l2) with the wrinkling branch (src/balloon.rs:51-63), in f64.
__device__ __forceinline__ double ogden_sigma(const double mu[3], double a, double b) {
    const double al[3] = {1.3, 5.0, -2.0};
    double s = 0.0;
    for (int i = 0; i < 3; i++) s += mu[i] * (pow(a, al[i]) - pow(b, al[i]));
    return s;
}
__device__ __forceinline__ double ogden_stress1(const double mu[3], double l1, double l2) {
    const double major = fmax(l1, l2), minor = fmin(l1, l2);
    if (major <= 1.0) return 0.0;
    const double natural = pow(major, -0.5);
    if (minor < natural) return l1 >= l2 ? ogden_sigma(mu, major, natural) : 0.0;
    return ogden_sigma(mu, l1, 1.0 / (l1 * l2));
}

// Triangles: the enclosed volume (sum of a . (b x c) / 6 in f64), the torn ones, and each CTA's
// three most tense intact ones (tension = first principal stress x thickness / (l1 l2), from
// the stretches of C = F^T F, src/sim.rs:746-785).
__global__ void __launch_bounds__(256) k_stats_tris(Dev D, StatsAcc* A, TensionCand* cand) {
    __shared__ double s_t[8];
    __shared__ uint32_t s_i[8];
    __shared__ uint32_t s_pick;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < D.Nt;
    double vol = 0.0, ten = -1.0;
    float l1f = 0.f, l2f = 0.f;
    bool torn = false;
    if (in) {
        const Tri t = D.tris[i];
        const float4 pa = D.mem_x[0][t.v0], pb = D.mem_x[0][t.v1], pc = D.mem_x[0][t.v2];
        const double ax = pa.x, ay = pa.y, az = pa.z, bx = pb.x, by = pb.y, bz = pb.z, cx = pc.x, cy = pc.y, cz = pc.z;
        // b x c, then a . (b x c) (glam's cross and dot)
        const double kx = by * cz - cy * bz, ky = bz * cx - cz * bx, kz = bx * cy - cx * by;
        vol = (ax * kx + ay * ky + az * kz) / 6.0;
        torn = D.alive[i] == 0u;
        if (!torn) {
            const double m0 = t.dm_inv.x, m1 = t.dm_inv.y, m2 = t.dm_inv.z, m3 = t.dm_inv.w;
            const double e1x = bx - ax, e1y = by - ay, e1z = bz - az, e2x = cx - ax, e2y = cy - ay, e2z = cz - az;
            const double f0x = e1x * m0 + e2x * m2, f0y = e1y * m0 + e2y * m2, f0z = e1z * m0 + e2z * m2;
            const double f1x = e1x * m1 + e2x * m3, f1y = e1y * m1 + e2y * m3, f1z = e1z * m1 + e2z * m3;
            const double c00 = f0x * f0x + f0y * f0y + f0z * f0z, c01 = f0x * f1x + f0y * f1y + f0z * f1z;
            const double c11 = f1x * f1x + f1y * f1y + f1z * f1z;
            const double mid = 0.5 * (c00 + c11);
            const double dd = c00 - c11;
            const double dev = sqrt(0.25 * (dd * dd) + c01 * c01);
            const double l1 = sqrt(mid + dev), l2 = sqrt(fmax(mid - dev, 0.0));
            const double mu[3] = {D.U->rubber[0], D.U->rubber[1], D.U->rubber[2]};
            ten = ogden_stress1(mu, l1, l2) * (double)D.U->rubber[3] / fmax(l1 * l2, 1e-9);
            l1f = (float)l1, l2f = (float)l2;
        }
    }
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const double vs = warp_sum_d(vol);
    const uint32_t nt = warp_sum_u(torn ? 1u : 0u);
    if (lane == 0) {
        atomicAdd(&A->inside, vs);
        if (nt) atomicAdd(&A->torn, nt);
    }
    // Three rounds of the CTA's argmax (ties: the lower index), each pick then left out.
    for (int r = 0; r < 3; r++) {
        double bt = ten;
        uint32_t bi = in ? i : 0xffffffffu;
        for (int o = 16; o > 0; o >>= 1) {
            const double ot = __shfl_xor_sync(0xffffffffu, bt, o);
            const uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ot > bt || (ot == bt && oi < bi)) bt = ot, bi = oi;
        }
        if (lane == 0) s_t[warp] = bt, s_i[warp] = bi;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = s_t[0];
            uint32_t k = s_i[0];
            for (int w = 1; w < 8; w++)
                if (s_t[w] > t || (s_t[w] == t && s_i[w] < k)) t = s_t[w], k = s_i[w];
            s_pick = t >= 0.0 ? k : 0xffffffffu;
            cand[blockIdx.x * 3 + r] = TensionCand{t, s_pick, 0.f, 0.f};
        }
        __syncthreads();
        if (in && s_pick == i) {
            cand[blockIdx.x * 3 + r].l1 = l1f, cand[blockIdx.x * 3 + r].l2 = l2f;
            ten = -1.0;
        }
        __syncthreads();
    }
}

}  // namespace ntr
