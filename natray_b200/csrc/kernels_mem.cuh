// Rubber substep (shaders/membrane.wgsl:40-149, 258-400) with bullet contact
// (shaders/bullet.wgsl:426-611), and the bullets' own step (bullet.wgsl:92-383).
#pragma once

#include "kernels_cells.cuh"

namespace ntr {

__device__ __forceinline__ V3 qrot(float4 q, V3 v) {
    V3 qv = xyz(q);
    V3 t = 2.0f * cross(qv, v);
    return v + q.w * t + cross(qv, t);
}
__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
    V3 v = a.w * xyz(b) + b.w * xyz(a) + cross(xyz(a), xyz(b));
    return make_float4(v.x, v.y, v.z, a.w * b.w - dot(xyz(a), xyz(b)));
}
__device__ __forceinline__ float4 normalize4(float4 q) {
    float inv = 1.0f / sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    return make_float4(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
}

struct Sheet {
    float sx, sy, tangent;
};

// Ogden plane stress with wrinkling (membrane.wgsl:47-65).
__device__ __forceinline__ Sheet sheet(const ntr_gpu_params* U, float major, float minor) {
    if (major <= 1.0f) return {0.0f, 0.0f, 0.0f};
    const V3 mu = {U->rubber[0], U->rubber[1], U->rubber[2]};
    const V3 AL = {1.3f, 5.0f, -2.0f};
    float la = nt_log(major);
    V3 e1 = AL * la;
    V3 pa = {nt_exp(e1.x), nt_exp(e1.y), nt_exp(e1.z)};
    float tan_scale = 1.0f / (major * major);
    if (minor * minor * major < 1.0f) {
        V3 e2 = ((-0.5f) * AL) * la;
        V3 pn = {nt_exp(e2.x), nt_exp(e2.y), nt_exp(e2.z)};
        return {dot(mu, pa - pn), 0.0f, dot(mu * AL, pa + 0.5f * pn) * tan_scale};
    }
    float lb = nt_log(minor);
    V3 e3 = AL * lb;
    V3 pb = {nt_exp(e3.x), nt_exp(e3.y), nt_exp(e3.z)};
    V3 e4 = (-AL) * (la + lb);
    V3 p3 = {nt_exp(e4.x), nt_exp(e4.y), nt_exp(e4.z)};
    return {dot(mu, pa - p3), dot(mu, pb - p3), dot(mu * AL, pa + p3) * tan_scale};
}

struct VertexForce {
    V3 f, n;
    float area, stiff, tension, reach, thick;
};

// The rubber's triangles, once per substep (membrane.wgsl:67-149, the part of vertex_force that
// does not depend on which of its vertices asks): the stretch, the Ogden stresses, and what each
// of its three vertices folds into its sums. One thread per triangle, so the stresses are
// computed once instead of once per vertex. Per triangle five float4 in `tri_rec`:
//   {-(h1 + h2), stiffness at v0}, {h1, at v1}, {h2, at v2}, {e1 x e2, |e1 x e2| / 6},
//   {rest / 3, tension, reach, kind}
// with the stiffness at a corner vol * (gx^2 + gy^2) * (tangent + sx), (gx, gy) the corner's
// shape gradient, and kind 0: dead at the start of the substep (not counted), 1: tore now
// (counts for the reach only), 2: counted. A vertex adds its corner's record, so it reads two
// records of each of its triangles at once, with no dependent lookups (the corner comes from
// `vtri_c`); adding -(h1 + h2) is the same as subtracting h1 + h2.
//
// `alive` holds the state at the start of the substep until this kernel writes the tears, and
// the vertices read the kind, so every vertex of a triangle sees the same thing. The reference
// writes a tear into `alive` while the triangle's other vertices may still be reading it, and
// whether they count it then depends on the threads' timing.
template <class CT>
__device__ __forceinline__ void mem_tri_body(const Dev& D, const CT& C, int par) {
    const ntr_gpu_params* U = D.U;
    const float4* X = D.mem_x[par];
    const float thick0 = U->rubber[3];
    for (uint32_t t = C.x() * blockDim.x + threadIdx.x; t < D.Nt; t += C.nx() * blockDim.x) {
        float4* rec = D.tri_rec + 5 * (size_t)t;
        if (D.alive[t] == 0u) {
            rec[4] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(0u));
            continue;
        }
        const Tri tri = D.tris[t];
        V3 x0 = xyz(X[tri.v0]);
        V3 e1 = xyz(X[tri.v1]) - x0;
        V3 e2 = xyz(X[tri.v2]) - x0;
        const float mxx = tri.dm_inv.x, myy = tri.dm_inv.y, mzz = tri.dm_inv.z, mww = tri.dm_inv.w;
        const float reach = mx(length(e1), mx(length(e2), length(e2 - e1)));
        V3 f0 = e1 * mxx + e2 * mzz;
        V3 f1 = e1 * myy + e2 * mww;
        float c00 = dot(f0, f0), c01 = dot(f0, f1), c11 = dot(f1, f1);
        float mid = 0.5f * (c00 + c11);
        float dev = sqrtf(0.25f * (c00 - c11) * (c00 - c11) + c01 * c01);
        float lx = sqrtf(mid + dev), ly = sqrtf(mx(mid - dev, 1e-12f));
        if (lx >= U->rubber2[1]) {
            D.alive[t] = 0u;
            rec[4] = make_float4(0.0f, 0.0f, reach, __uint_as_float(1u));
            continue;
        }
        Sheet sh = sheet(U, lx, ly);
        float ex = 1.0f, ey = 0.0f;
        if (dev > 1e-6f * mid) {
            float qx, qy;
            if (c00 >= c11)
                qx = mid + dev - c11, qy = c01;
            else
                qx = c01, qy = mid + dev - c00;
            float inv = 1.0f / sqrtf(qx * qx + qy * qy);
            ex = qx * inv, ey = qy * inv;
        }
        float sx = sh.sx / (lx * lx), sy = sh.sy / (ly * ly);
        float ds = sx - sy;
        float s00 = sy + ds * ex * ex;
        float s01 = ds * ex * ey;
        float s11 = sy + ds * ey * ey;
        V3 p0 = f0 * s00 + f1 * s01;
        V3 p1 = f0 * s01 + f1 * s11;
        float vol = tri.rest_area * thick0;
        V3 h1 = (-vol) * (p0 * mxx + p1 * myy);
        V3 h2 = (-vol) * (p0 * mzz + p1 * mww);
        V3 cr = cross(e1, e2);
        const float tan_sx = sh.tangent + sx;
        auto stiff = [&](float gx, float gy) { return vol * (gx * gx + gy * gy) * tan_sx; };
        rec[0] = f4(-(h1 + h2), stiff(-(mxx + mzz), -(myy + mww)));
        rec[1] = f4(h1, stiff(mxx, myy));
        rec[2] = f4(h2, stiff(mzz, mww));
        rec[3] = f4(cr, length(cr) / 6.0f);
        rec[4] = make_float4(tri.rest_area / 3.0f, sh.sx * thick0 / (lx * ly), reach, __uint_as_float(2u));
    }
}
__global__ void k_mem_tri(Dev D, int par) { mem_tri_body(D, HwCta{}, par); }

// vertex_force (membrane.wgsl:67-149): the vertex's triangles' records, folded in its order.
// Eight triangles at a time: their indices and corners, then their records, each group of
// loads issued together; the sums then run in the vertex's order.
constexpr uint32_t VF_BATCH = 8;

__device__ VertexForce vertex_force(const Dev& D, uint32_t i) {
    const float thick0 = D.U->rubber[3];
    VertexForce o = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, 0.0f, 0.0f, 0.0f, 0.0f, thick0};
    float rest = 0.0f;
    const uint32_t k0 = D.vtri_off[i], k1 = D.vtri_off[i + 1];
    for (uint32_t kb = k0; kb < k1; kb += VF_BATCH) {
        uint32_t t[VF_BATCH], c[VF_BATCH];
#pragma unroll
        for (uint32_t j = 0; j < VF_BATCH; j++) {
            const bool in = kb + j < k1;
            t[j] = in ? D.vtri[kb + j] : 0u;
            c[j] = in ? (uint32_t)D.vtri_c[kb + j] : 0u;
        }
        float4 own[VF_BATCH], nrm[VF_BATCH], info[VF_BATCH];
#pragma unroll
        for (uint32_t j = 0; j < VF_BATCH; j++) {
            own[j] = nrm[j] = info[j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (kb + j < k1) {
                const float4* rec = D.tri_rec + 5 * (size_t)t[j];
                own[j] = rec[c[j]];
                nrm[j] = rec[3];
                info[j] = rec[4];
            }
        }
#pragma unroll
        for (uint32_t j = 0; j < VF_BATCH; j++) {
            if (kb + j >= k1) break;
            const uint32_t kind = __float_as_uint(info[j].w);
            if (kind == 0u) continue;
            o.reach = mx(o.reach, info[j].z);
            if (kind == 1u) continue;
            o.f = o.f + xyz(own[j]);
            o.n = o.n + xyz(nrm[j]);
            o.area += nrm[j].w;
            rest += info[j].x;
            o.stiff += own[j].w;
            o.tension = mx(o.tension, info[j].y);
        }
    }
    if (o.area > 0.0f) o.thick = thick0 * rest / o.area;
    return o;
}

struct Near {
    float ax, ay, nx, ny, depth;
};

// The nearest point of bullet `bi`'s outline to q = (z, r) of its body frame
// (bullet.wgsl:438-472). `ol` is the bullet's outline (in shared memory).
__device__ Near nearest_surface(const float2* __restrict__ ol, float qx, float qy) {
    float2 first = ol[0], last = ol[NTR_OUTLINE - 1];
    Near o = {qx, qy, 0.0f, 0.0f, 0.0f};
    float best = BIG_F;
    for (uint32_t j = 0; j <= NTR_OUTLINE; j++) {
        float2 p0 = make_float2(first.x, 0.0f), p1 = make_float2(last.x, 0.0f);
        if (j > 0) p0 = ol[j - 1];
        if (j < NTR_OUTLINE) p1 = ol[j];
        float ex = p1.x - p0.x, ey = p1.y - p0.y;
        float len2 = ex * ex + ey * ey;
        if (len2 <= 0.0f) continue;
        float tt = clampf_(((qx - p0.x) * ex + (qy - p0.y) * ey) / len2, 0.0f, 1.0f);
        float onx = p0.x + ex * tt, ony = p0.y + ey * tt;
        float dqx = qx - onx, dqy = qy - ony;
        float d = sqrtf(dqx * dqx + dqy * dqy);
        if (d < best) {
            best = d;
            o.ax = onx, o.ay = ony;
            float nnx = -ey, nny = ex;
            float inv = 1.0f / sqrtf(nnx * nnx + nny * nny);
            o.nx = nnx * inv, o.ny = nny * inv;
        }
    }
    bool inside = false;
    if (qx > first.x && qx < last.x) {
        uint32_t k = 1;
        while (k < NTR_OUTLINE - 1 && ol[k].x < qx) k++;
        float2 a = ol[k - 1], c = ol[k];
        float f = (qx - a.x) / mx(c.x - a.x, 1e-12f);
        inside = qy < a.y * (1.0f - f) + c.y * f;
    }
    o.depth = inside ? best : -best;
    if (!inside && best > 0.0f) o.nx = (qx - o.ax) / best, o.ny = (qy - o.ay) / best;
    return o;
}

// The response to the best sample (bullet.wgsl:426-611): the rubber pushed out of the bullet and
// slowed along it, the impulses and, for a held wet vertex, the wetted-side sums into the
// bullet's fixed-point sums.
__device__ __forceinline__ void contact_response(const Dev& D, uint32_t bi, V3& x, V3& v, float m, V3 load, const VertexForce& vf, bool wet, bool& held,
                                                 float sub, V3 xb, float best, V3 on_b, V3 gap, V3 nrm, V3 rel, float share) {
    float vn = dot(rel, nrm);
    V3 rel_t = rel - vn * nrm;
    float slide = length(rel_t);
    float dvn = 0.0f, jn = 0.0f;
    V3 j = {0.0f, 0.0f, 0.0f};
    bool holds = false;
    if (!wet) {
        dvn = mx(-vn, 0.0f);
        jn = m * dvn;
        j = -m * share * dvn * nrm;
    } else {
        float ln = dot(load, nrm);
        if (ln < 0.0f) {
            dvn = -vn;
            jn = -ln * sub;
            j = mn(share, 1.0f) * ln * sub * nrm;
            holds = true;
            held = true;
        } else if (best > 0.0f) {
            dvn = mx(-vn, 0.0f);
        } else {
            return;
        }
    }
    float stop = (slide > 1e-9f && m > 0.0f) ? mn(1.0f, MU_JACKET * jn / (m * slide)) : 0.0f;
    V3 dvt = -share * stop * rel_t;
    x = x + (share * gap + sub * dvt);
    v = v + (share * dvn * nrm + dvt);
    j = j - m * dvt;
    float nl = length(vf.n);
    int32_t* hit = D.bullet_hit + bi * NTR_HIT_FIELDS;
    if (holds && nl > 0.0f) {
        float a = vf.area * 1e6f;
        V3 sx = (x - xb) * 1e3f * a;
        for (int c = 0; c < 3; c++) {
            atomicAdd(hit + 6 + c, to_fp(vf.n[c] / nl * a, FP_A));
            atomicAdd(hit + 9 + c, to_fp(sx[c], FP_X));
        }
        atomicAdd(hit + 12, to_fp(a, FP_A));
    }
    V3 jl = cross(on_b, j);
    for (int c = 0; c < 3; c++) {
        atomicAdd(hit + c, to_fp(j[c], FP_J));
        atomicAdd(hit + 3 + c, to_fp(jl[c], FP_L));
    }
}

// A triangle of vertex i's contact search (or, for k == k1, the vertex alone): its corners as
// they will be after the substep, their velocities, which corner i is, and its subdivision.
struct ContactTri {
    V3 p[3], pv[3];
    uint32_t own, n;
    bool ok;
};

__device__ __forceinline__ ContactTri contact_tri(const Dev& D, int par, uint32_t i, uint32_t k, uint32_t k1, V3 x, V3 v, float sub, float hull) {
    const float4* MX = D.mem_x[par];
    const float4* MV = D.mem_v[par];
    ContactTri t;
    for (int c = 0; c < 3; c++) t.p[c] = x, t.pv[c] = v;
    t.own = 0, t.n = 1, t.ok = true;
    if (k < k1) {
        const uint32_t tn = D.vtri[k];
        if (D.alive[tn] == 0u) {  // dead, or tore in this substep (k_mem_tri)
            t.ok = false;
            return t;
        }
        const Tri tri = D.tris[tn];
        const uint32_t ids[3] = {tri.v0, tri.v1, tri.v2};
        for (uint32_t c = 0; c < 3; c++) {
            if (ids[c] == i) {
                t.own = c;
            } else {
                t.pv[c] = xyz(MV[ids[c]]);
                t.p[c] = xyz(MX[ids[c]]) + sub * t.pv[c];
            }
        }
        const float longest = mx(distance(t.p[0], t.p[1]), mx(distance(t.p[1], t.p[2]), distance(t.p[2], t.p[0])));
        t.n = f2u(clampf_(ceilf(longest / hull), 1.0f, 8.0f));
    }
    return t;
}

// Sample m of a triangle subdivided n times: barycentric (a, c, n - a - c) / n in the order
// a = 0..n, c = 0..n - a.
__device__ __forceinline__ void contact_sample_ac(uint32_t m, uint32_t n, uint32_t& a, uint32_t& c) {
    a = 0;
    while (m > n - a) m -= n - a + 1, a++;
    c = m;
}

// What the search keeps of its best sample.
struct ContactHit {
    V3 on_b, gap, nrm, rel;
    float share, depth;
};

// One sample against a bullet, `ol` its outline (the contact search of bullet.wgsl:426-611):
// false if it does not count (no weight on this vertex, or beyond the bullet's reach). With
// `hit`, also what the response needs.
__device__ __forceinline__ bool contact_sample(const float2* ol, const ContactTri& t, uint32_t a, uint32_t c, const DBullet& b, V3 xb,
                                               float4 back, V3 w, float band, float& depth, ContactHit* hit) {
    const uint32_t n = t.n;
    V3 bary = v3((float)a, (float)c, (float)(n - a - c)) / (float)n;
    float wi = bary[t.own];
    if (wi <= 0.0f) return false;
    V3 s = bary.x * t.p[0] + bary.y * t.p[1] + bary.z * t.p[2];
    V3 r = s - xb;
    if (length(r) >= b.shape.z + band) return false;
    V3 q = qrot(back, r);
    float rho = sqrtf(q.x * q.x + q.y * q.y);
    Near nr = nearest_surface(ol, q.z, rho);
    depth = nr.depth;
    if (hit) {
        float rx = 1.0f, ry = 0.0f;
        if (rho > 1e-9f) rx = q.x / rho, ry = q.y / rho;
        hit->depth = nr.depth;
        hit->on_b = qrot(b.q, v3(rx * nr.ay, ry * nr.ay, nr.ax));
        hit->gap = hit->on_b - r;
        hit->nrm = qrot(b.q, v3(rx * nr.ny, ry * nr.ny, nr.nx));
        hit->share = wi / dot(bary, bary);
        hit->rel = bary.x * t.pv[0] + bary.y * t.pv[1] + bary.z * t.pv[2] - xyz(b.v) - cross(w, hit->on_b);
    }
    return true;
}

// Lane `src`'s contact search against a bullet (`ol` its outline), by the whole warp: the
// samples of its vertex's triangles (and of the vertex alone) shared out over the lanes, each
// lane keeping the first of its samples of greatest depth, then the warp's: the greatest depth,
// the earliest in the reference's order among equals. For finite depths that is the sample the
// reference's sequential search ends on (it takes a sample only when deeper than the best so
// far, from -band): found when its depth is above -band. Returns the sample's triangle slot and
// index. All 32 lanes call it.
__device__ bool contact_search_warp(const Dev& D, int par, int src, uint32_t i_l, V3 x_l, V3 v_l, float band_l, float sub, const DBullet& b,
                                    V3 xb, float4 back, V3 w, const float2* ol, uint32_t& k_best, uint32_t& m_best) {
    const uint32_t full = 0xffffffffu, lane = threadIdx.x & 31u;
    const uint32_t i = __shfl_sync(full, i_l, src);
    const V3 x = {__shfl_sync(full, x_l.x, src), __shfl_sync(full, x_l.y, src), __shfl_sync(full, x_l.z, src)};
    const V3 v = {__shfl_sync(full, v_l.x, src), __shfl_sync(full, v_l.y, src), __shfl_sync(full, v_l.z, src)};
    const float band = __shfl_sync(full, band_l, src);
    const uint32_t k0 = D.vtri_off[i], k1 = D.vtri_off[i + 1];
    bool have = false;
    float bd = 0.0f;
    uint32_t bo = 0u;  // (k - k0) * 64 + sample: the reference's order
    // The triangles (and the vertex alone, last), 32 at a time: lane j loads the j-th, so their
    // loads go out together. Their samples, numbered triangle by triangle in the reference's
    // order, are then shared out over the lanes: sample p of the round goes to lane p % 32, which
    // takes its triangle's corners from the lane that loaded them.
    for (uint32_t kb = k0; kb <= k1; kb += 32u) {
        const uint32_t kl = kb + lane;
        const ContactTri mine = kl <= k1 ? contact_tri(D, par, i, kl, k1, x, v, sub, b.shape.w) : ContactTri{};
        const uint32_t nk = min(32u, k1 + 1u - kb);
        // Where each triangle's samples start; a dead triangle has none.
        const uint32_t my_ns = (kl <= k1 && mine.ok) ? (mine.n + 1u) * (mine.n + 2u) / 2u : 0u;
        uint32_t start = my_ns;  // inclusive scan, then exclusive
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(full, start, o);
            if ((int)lane >= o) start += y;
        }
        const uint32_t total = __shfl_sync(full, start, nk - 1u);
        start -= my_ns;
        for (uint32_t p0 = 0; p0 < total; p0 += 32u) {
            const uint32_t p = p0 + lane;
            // The triangle of sample p: the last with start <= p (lanes past the end take 0).
            uint32_t j = 0;
            for (uint32_t q = 1; q < nk; q++)
                if (__shfl_sync(full, start, q) <= p) j = q;
            ContactTri t;
            for (int c = 0; c < 3; c++) {
                t.p[c] = {__shfl_sync(full, mine.p[c].x, j), __shfl_sync(full, mine.p[c].y, j), __shfl_sync(full, mine.p[c].z, j)};
                t.pv[c] = {__shfl_sync(full, mine.pv[c].x, j), __shfl_sync(full, mine.pv[c].y, j), __shfl_sync(full, mine.pv[c].z, j)};
            }
            t.own = __shfl_sync(full, mine.own, j);
            t.n = __shfl_sync(full, mine.n, j);
            t.ok = true;
            const uint32_t m = p - __shfl_sync(full, start, j);
            if (p >= total) continue;
            uint32_t a, c;
            contact_sample_ac(m, t.n, a, c);
            float depth;
            if (contact_sample(ol, t, a, c, b, xb, back, w, band, depth, nullptr) && (!have || depth > bd)) {
                have = true;
                bd = depth;
                bo = (kb + j - k0) * 64u + m;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const bool oh = __shfl_xor_sync(full, have, o);
        const float od = __shfl_xor_sync(full, bd, o);
        const uint32_t oo = __shfl_xor_sync(full, bo, o);
        if (oh && (!have || od > bd || (od == bd && oo < bo))) have = true, bd = od, bo = oo;
    }
    if (!have || !(bd > -band)) return false;
    k_best = k0 + bo / 64u;
    m_best = bo % 64u;
    return true;
}

// Contact of the rubber with the bullets (bullet.wgsl:426-611), for the lanes with `act`; every
// lane of the warp calls it. Per bullet in turn: the lanes near it, one after the other, have
// their search run by the whole warp (contact_search_warp), then take the response themselves.
__device__ float rubber_contact(const Dev& D, const float2* outlines, int par, uint32_t i, bool act, V3& x, V3& v, float m, V3 load,
                                const VertexForce& vf, bool wet, bool& held, float t, float sub, float now, float dt) {
    const uint32_t full = 0xffffffffu, lane = threadIdx.x & 31u;
    float limit = BIG_F;
    const float band = held ? 0.5f * vf.thick : 0.0f;
    if (act) held = false;
    const uint32_t nbu = D.U->mem[3];
    for (uint32_t bi = 0; bi < nbu; bi++) {
        const DBullet b = D.bullets[bi];
        if (b.info.z != 1u) continue;
        const float2* ol = outlines + bi * NTR_OUTLINE;
        V3 xb = xyz(b.x) - xyz(b.v) * (now - t);
        float closing = length(xyz(b.v) - v);
        const bool near = act && !(length(x - xb) > b.shape.z + vf.reach + 2.0f * closing * dt);
        if (near) limit = mn(limit, 0.25f * b.shape.w / mx(closing, 1e-6f));
        float4 back = make_float4(-b.q.x, -b.q.y, -b.q.z, b.q.w);
        V3 w = qrot(b.q, qrot(back, xyz(b.l)) / v3(b.shape.y, b.shape.y, b.shape.x));
        for (uint32_t todo = __ballot_sync(full, near); todo; todo &= todo - 1u) {
            const int src = __ffs(todo) - 1;
            uint32_t kb = 0, mb = 0;
            const bool found = contact_search_warp(D, par, src, i, x, v, band, sub, b, xb, back, w, ol, kb, mb);
            if ((int)lane != src || !found) continue;
            // The best sample again, with what the response needs.
            const uint32_t k1 = D.vtri_off[i + 1];
            const ContactTri tb = contact_tri(D, par, i, kb, k1, x, v, sub, b.shape.w);
            uint32_t a, c;
            contact_sample_ac(mb, tb.n, a, c);
            ContactHit hit;
            float depth_again;
            contact_sample(ol, tb, a, c, b, xb, back, w, band, depth_again, &hit);
            const float best = hit.depth;
            const V3 on_b = hit.on_b, gap = hit.gap, nrm = hit.nrm, rel = hit.rel;
            const float share = hit.share;
            contact_response(D, bi, x, v, m, load, vf, wet, held, sub, xb, best, on_b, gap, nrm, rel, share);
        }
    }
    return limit;
}

// The vertex of a thread of k_mem_substep: groups of 4 consecutive vertices, the 8 groups of a
// warp an eighth of the launch's vertices apart (a bijection of the launch's threads). The
// vertices near a bullet lie together in the mesh's spatial order: so their contact searches,
// the substep's only heavy work, fall to many warps (and SMs) instead of a few, and each warp
// shares its few among its lanes.
__device__ __forceinline__ uint32_t substep_vertex(uint32_t block, uint32_t thread, uint32_t n_blocks) {
    const uint32_t t = block * blockDim.x + thread;
    const uint32_t span = n_blocks * blockDim.x / 32u;  // groups in an eighth
    const uint32_t gi = t >> 2;
    return (((gi & 7u) * span + (gi >> 3)) << 2) | (t & 3u);
}

// One explicit rubber substep (membrane.wgsl:283-400). `k` is which substep of the step this
// is, `par` which pair of buffers it reads.
template <class CT>
__device__ __forceinline__ void mem_substep_body(const Dev& D, const CT& C, uint32_t k, int par) {
    DevState* st = D.st;
    const uint32_t i = substep_vertex(C.x(), threadIdx.x, C.nx());
    float lim_x = BIG_F, lim_y = BIG_F;
    const ntr_gpu_params* U = D.U;
    const float dt = dt_of(st), now = now_of(st);
    const float sub = dt / (float)max(U->mem[1], 1u);
    const float t_sub = now - dt + (float)(k + 1u) * sub;
    // What the contact with the bullets needs of this vertex; `act` when it takes part.
    bool act = false, c_held = false, c_ow = false;
    V3 c_x = {0.0f, 0.0f, 0.0f}, c_v = c_x, c_f = c_x;
    float c_m = 0.0f, c_push = 0.0f, c_w = 0.0f;
    VertexForce c_vf = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (i < D.Nv) {
        const Grid g = grid_of(D, cur_of(st));
        const float m = D.mem_mass[i];
        const float4 x4 = D.mem_x[par][i];
        float4* XO = D.mem_x[1 - par];
        float4* VO = D.mem_v[1 - par];
        if (m == 0.0f) {
            XO[i] = x4;
            VO[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else {
            const float hh = g.h;
            const VertexForce vf = vertex_force(D, i);
            lim_x = sqrtf(m / mx(vf.stiff, 1e-30f));
            if (vf.tension > 0.0f) lim_y = sqrtf(U->fluid[0] * hh * hh * hh / (4.0f * PI_F * vf.tension));
            V3 f = vf.f + m * v3(U->gravity[0], U->gravity[1], U->gravity[2]);
            const float4 v4 = D.mem_v[par][i];
            V3 v = xyz(v4);
            float nl = length(vf.n);
            const size_t first = (size_t)i * NTR_LAYER_MODES;
            bool held = v4.w > 0.0f;
            const float4 mw = D.mem_water[i];
            const bool ow = mw.w >= CONTACT_F;
            float push = (ow && nl > 0.0f) ? -dot(f, vf.n / mx(nl, 1e-30f)) : 0.0f;
            D.mem_push[i] = make_float2(held ? 0.0f : push, vf.area);
            if (sub <= 0.0f) {
                XO[i] = x4;
                VO[i] = v4;
            } else {
                if (ow && nl > 0.0f) {
                    V3 n = vf.n / nl;
                    V3 vw = xyz(mw);
                    V3 rel = v - vw;
                    V3 rel_t = rel - dot(rel, n) * n;
                    V3 ft = f - dot(f, n) * n;
                    float kk = sqrtf(U->fluid[0] * MU_WATER) * vf.area;
                    const V3 TAU0 = {2.0e-6f, 3.170e-5f, 5.024e-4f}, TAU1 = {7.962e-3f, 1.262e-1f, 2.0f};
                    const V3 LW0 = {573.42f, 158.41f, 38.750f}, LW1 = {10.049f, 2.2387f, 0.9494f};
                    V3 x0 = v3(-sub, -sub, -sub) / TAU0, x1 = v3(-sub, -sub, -sub) / TAU1;
                    V3 e0 = {nt_exp(x0.x), nt_exp(x0.y), nt_exp(x0.z)}, e1 = {nt_exp(x1.x), nt_exp(x1.y), nt_exp(x1.z)};
                    V3 g0 = (v3(1.0f, 1.0f, 1.0f) - e0) * TAU0 / v3(sub, sub, sub);
                    V3 g1 = (v3(1.0f, 1.0f, 1.0f) - e1) * TAU1 / v3(sub, sub, sub);
                    float lhs = m / sub + kk * (dot(LW0, g0) + dot(LW1, g1));
                    V3 rhs = m / sub * rel_t + ft;
                    V3 z[6];
                    for (int jj = 0; jj < 6; jj++) {
                        z[jj] = xyz(D.mem_layer[first + jj]);
                        z[jj] = z[jj] - dot(z[jj], n) * n;
                    }
                    for (int bb = 0; bb < 3; bb++) rhs = rhs - kk * LW0[bb] * (e0[bb] * z[bb] - g0[bb] * rel_t);
                    for (int bb = 0; bb < 3; bb++) rhs = rhs - kk * LW1[bb] * (e1[bb] * z[3 + bb] - g1[bb] * rel_t);
                    V3 rel_new = rhs / lhs;
                    for (int bb = 0; bb < 3; bb++) D.mem_layer[first + bb] = f4(e0[bb] * z[bb] + g0[bb] * (rel_new - rel_t), 0.0f);
                    for (int bb = 0; bb < 3; bb++) D.mem_layer[first + 3 + bb] = f4(e1[bb] * z[3 + bb] + g1[bb] * (rel_new - rel_t), 0.0f);
                    v = vw + rel_new;
                    if (held) v = v + dot(rel, n) * n;
                } else if (ow) {
                    v = xyz(mw);
                } else {
                    for (int jj = 0; jj < 6; jj++) D.mem_layer[first + jj] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    V3 fa = {0.0f, 0.0f, 0.0f};
                    if (nl > 0.0f) {
                        V3 n = vf.n / nl;
                        fa = (gas_pressure_at(D, g, par, xyz(x4) - hh * n) - gas_pressure_at(D, g, par, xyz(x4) + hh * n)) * vf.area * n;
                    }
                    v = v + sub * (f + fa) / m;
                }
                act = true;
                c_x = xyz(x4) + sub * v;
                c_v = v, c_f = f, c_m = m, c_vf = vf, c_ow = ow, c_push = push, c_w = x4.w;
                c_held = held && ow;
            }
        }
    }
    // The contact with the bullets, with every lane of the warp (rubber_contact shares a
    // vertex's search among them), then the rest of the vertex's substep.
    // The bullets' outlines, which every contact sample walks, in shared memory.
    __shared__ float2 s_outline[NTR_MAX_SHOTS * NTR_OUTLINE];
    for (uint32_t j = threadIdx.x; j < U->mem[3] * NTR_OUTLINE && j < NTR_MAX_SHOTS * NTR_OUTLINE; j += blockDim.x) s_outline[j] = D.outlines[j];
    __syncthreads();
    const float lim_c = rubber_contact(D, s_outline, par, i, act, c_x, c_v, c_m, c_f, c_vf, c_ow, c_held, t_sub, sub, now, dt);
    if (act) {
        lim_x = mn(lim_x, lim_c);
        D.mem_push[i].x = c_held ? 0.0f : c_push;
        V3 xx = c_x, v = c_v;
        if (xx.y < 0.0f) {
            float jj = mx(-v.y, 0.0f);
            xx.y = 0.0f;
            v.y = mx(v.y, 0.0f);
            float s = sqrtf(v.x * v.x + v.z * v.z);
            float keep = s > 1e-9f ? mx(0.0f, 1.0f - U->rubber2[0] * jj / s) : 0.0f;
            v = v3(v.x * keep, v.y, v.z * keep);
        }
        D.mem_x[1 - par][i] = make_float4(xx.x, xx.y, xx.z, c_w);
        D.mem_v[1 - par][i] = make_float4(v.x, v.y, v.z, c_held ? 1.0f : 0.0f);
    }
    // The longest stable substep and the capillary step, lowered with atomicMin on the bits.
    for (int o = 16; o > 0; o >>= 1) {
        lim_x = fminf(lim_x, __shfl_down_sync(0xffffffffu, lim_x, o));
        lim_y = fminf(lim_y, __shfl_down_sync(0xffffffffu, lim_y, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin((unsigned int*)&st->s.mem_dt, __float_as_uint(lim_x));
        atomicMin((unsigned int*)&st->s.cap_dt, __float_as_uint(lim_y));
    }
}
// A one-scene step's: CTAs of 128 threads (the 1M scene's 40,962 vertices in 321 CTAs instead of
// 161 of 256, spread more evenly over the 148 SMs: 67.1 -> 64.8 us a step; 64 threads: the same).
constexpr uint32_t MEM_SUB_T = 128;
__global__ void __launch_bounds__(MEM_SUB_T) k_mem_substep(Dev D, uint32_t k, int par) { mem_substep_body(D, HwCta{}, k, par); }

// ---- the bullets' step, bullet.wgsl:101-383 ---------------------------------------------------
__device__ __forceinline__ float cp_patch(float s) {
    if (s < 0.0f) return CP_WAKE * s * s;
    float beta = nt_asin(mn(s, 1.0f));
    if (beta < PI_F / 12.0f) return 2.13f * s * s;
    float x = beta / PI_F - 0.25f;
    return 0.5f + 1.81f * x - 2.0f * x * x;
}

__device__ __forceinline__ float section_r2(const DSection& s, float t) { return s.c.x + s.b.w * mx(t - s.a.w, 0.0f); }

// sample_pressure by a warp.
__device__ __forceinline__ float2 warp_sample_pressure(const Dev& D, const Grid& g, V3 x, bool gas_only, int lane) {
    I3 base = vi(vfloor(x - 0.5f));
    V3 fx = x - vf(base);
    V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    const int a = lane / 9, b = (lane / 3) % 3, c = lane % 3;
    bool present = false;
    float wp = 0.0f, w = 0.0f;
    if (lane < 27) {
        const uint32_t cell = cell_at(g, base + I3{a, b, c});
        if (cell != NONE) {
            const float ty = cfv(D, F_TYPE, cell);
            if (!(ty == SOLID_T || (gas_only && ty == WATER_T))) {
                present = true;
                w = wsel(wx, a) * wsel(wy, b) * wsel(wz, c);
                wp = w * cfv(D, F_P, cell);
            }
        }
    }
    return fold27(present, wp, w);
}

// The five samples of a bullet patch at X (grid units) by a warp: the water velocity of the
// three face lattices (warp_sample_grid with F_U + d, a_wt(d)), the fill (F_TYPE, A_WC at
// X - 0.5) and the gas pressure (warp_sample_pressure at X - 0.5, gas only, the fill's stencil).
// Each lane's four cell lookups and then all their loads go out together, instead of one
// sample's dependent chain after another's; the folds are the same, in the same order.
__device__ __forceinline__ void warp_patch_samples(const Dev& D, const Grid& g, V3 X, int lane, float2 (&s)[4], float2& gs) {
    const int a = lane / 9, b = (lane / 3) % 3, c = lane % 3;
    V3 wx[4], wy[4], wz[4];
    uint32_t cell[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const V3 x = k < 3 ? X - lattice_offset((uint32_t)k) : X - 0.5f;
        const I3 base = vi(vfloor(x - 0.5f));
        const V3 fx = x - vf(base);
        wx[k] = axis_weights(fx.x), wy[k] = axis_weights(fx.y), wz[k] = axis_weights(fx.z);
        cell[k] = lane < 27 ? cell_at(g, base + I3{a, b, c}) : NONE;
    }
    int32_t wv[4];
    float uv[4], pv = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const bool in = cell[k] != NONE;
        wv[k] = in ? accv(D, k < 3 ? a_wt((uint32_t)k) : (uint32_t)A_WC, cell[k]) : 0;
        uv[k] = in ? cfv(D, k < 3 ? F_U + (uint32_t)k : (uint32_t)F_TYPE, cell[k]) : 0.0f;
    }
    if (cell[3] != NONE) pv = cfv(D, F_P, cell[3]);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float w = 0.0f, wu = 0.0f;
        if (cell[k] != NONE) {
            w = wsel(wx[k], a) * wsel(wy[k], b) * wsel(wz[k], c) * from_fp(wv[k], FP_W);
            wu = w * uv[k];
        }
        s[k] = fold27(cell[k] != NONE, wu, w);
    }
    // The pressure sample: cells that are not solid and not water (uv[3] is the cell's type).
    const bool pp = cell[3] != NONE && !(uv[3] == SOLID_T || uv[3] == WATER_T);
    float w = 0.0f, wp = 0.0f;
    if (pp) {
        w = wsel(wx[3], a) * wsel(wy[3], b) * wsel(wz[3], c);
        wp = w * pv;
    }
    gs = fold27(pp, wp, w);
}

// push_water by a warp (integer sums: the lanes add their cells' shares in any order).
__device__ __forceinline__ void warp_push_water(const Dev& D, const Grid& g, V3 x, uint32_t d, float j, float sw, int lane) {
    if (sw <= 1e-6f || j == 0.0f) return;
    V3 lx = x - lattice_offset(d);
    I3 base = vi(vfloor(lx - 0.5f));
    V3 fx = lx - vf(base);
    V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    float hs = D.U->fluid[3];
    float k = j / (D.U->fluid[0] * hs * hs * hs * sw);
    if (lane >= 27) return;
    const int a = lane / 9, b = (lane / 3) % 3, c = lane % 3;
    const uint32_t cell = cell_at(g, base + I3{a, b, c});
    if (cell == NONE || accv(D, a_wt(d), cell) <= 0) return;
    atomicAdd(accp(D, A_BU + d, cell), to_fp(k * wsel(wx, a) * wsel(wy, b) * wsel(wz, c), FP_M));
}

// in_cavity by a warp: lane k tests section k.
__device__ __forceinline__ bool warp_in_cavity(const Dev& D, float hh, uint32_t bi, V3 p, float t, int lane) {
    static_assert(NTR_N_SEC == 32, "one lane per section");
    const float hand2 = R_HAND * R_HAND * hh * hh;
    const DSection s = D.sections[bi * NTR_N_SEC + lane];
    bool in = false;
    if (!(s.b.w <= 0.0f || section_r2(s, t) >= hand2)) {
        V3 ab = xyz(s.b) - xyz(s.a);
        float f = dot(p - xyz(s.a), ab) / mx(dot(ab, ab), 1e-20f);
        if (!(f < 0.0f || f > 1.0f)) {
            V3 dd = p - (xyz(s.a) + f * ab);
            in = dot(dd, dd) < section_r2(s, t);
        }
    }
    return __any_sync(0xffffffffu, in);
}

// The bullets' step (bullet.wgsl:186-383) in three launches:
//   k_bullet_prep, a warp per bullet: whether it flies this step, the water pressure ahead of
//     it, the membrane's contact sums (taken and cleared), into `bullet_prep`;
//   k_bullet_patch, a warp per surface patch: the patch's loads and its push on the water, into
//     `bullet_patch`;
//   k_bullet_finish, a CTA per bullet: the patches summed in the reference's order (lane l of
//     256 takes patches l, l + 256, l + 512 in turn, then a 256-wide tree), the rigid body, the
//     cavity sections.
template <class CT>
__device__ __forceinline__ void bullet_prep_body(const Dev& D, const CT& C) {
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t bi = C.x();
    // A scene without bullets still launches one CTA; it has nothing to do (and the patch and
    // finish kernels skip a bullet whose prep flag is not set).
    if (bi >= D.U->mem[3]) {
        if (threadIdx.x == 0) D.bullet_prep[bi * 4].x = 0.0f;
        return;
    }
    const int lane = (int)threadIdx.x;
    const Grid g = grid_of(D, cur_of(st));
    const DBullet b = D.bullets[bi];
    const float hh = g.h;
    int32_t* hit = D.bullet_hit + bi * NTR_HIT_FIELDS;
    uint32_t state = b.info.z;
    if (state == 0u && st->s.t_ns - st->s.dt_ns >= b.info.x) state = 1u;
    // The wetted-side sums always, the impulses only when the bullet flies this step.
    int32_t hv = 0;
    if (lane < NTR_HIT_FIELDS) hv = ((uint32_t)lane >= 6u || state == 1u) ? atomicExch(hit + lane, 0) : 0;
    int32_t h[NTR_HIT_FIELDS];
#pragma unroll
    for (int c = 0; c < NTR_HIT_FIELDS; c++) h[c] = __shfl_sync(0xffffffffu, hv, c);
    V3 ahead = xyz(b.x) + normalize(xyz(b.v) + 1e-9f) * (b.shape.z + 3.0f * hh);
    const V3 xa = (ahead - g.org) / hh - 0.5f;
    const float2 s = warp_sample_pressure(D, g, xa, false, lane);
    if (lane != 0) return;
    const float pf = s.y > 1e-6f ? s.x / s.y : 0.0f;
    V3 sn, sx;
    for (int c = 0; c < 3; c++) {
        sn[c] = from_fp(h[6 + c], FP_A);
        sx[c] = from_fp(h[9 + c], FP_X);
    }
    float sa = from_fp(h[12], FP_A);
    float4 side = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (sa > 0.0f && length(sn) > 0.0f) {
        V3 n = normalize(sn);
        side = make_float4(n.x, n.y, n.z, dot(sx, n) / sa * 1e-3f);
    }
    float4* o = D.bullet_prep + bi * 4;
    o[0] = make_float4(__uint_as_float(state), pf, 0.0f, 0.0f);
    o[1] = side;
    o[2] = make_float4(__int_as_float(h[0]), __int_as_float(h[1]), __int_as_float(h[2]), __int_as_float(h[3]));
    o[3] = make_float4(__int_as_float(h[4]), __int_as_float(h[5]), 0.0f, 0.0f);
    if (state != 1u) {
        D.bullets[bi].info.z = state;
        D.pose_log[(bi * NTR_LOG_CAP + st->s.step % NTR_LOG_CAP) * 3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}
__global__ void k_bullet_prep(Dev D) { bullet_prep_body(D, HwCta{}); }
__global__ void k_bullet_prep_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    bullet_prep_body(sD, c);
}

constexpr int BULLET_PW = 8;  // patch warps per CTA

template <class CT>
__device__ __forceinline__ void bullet_patch_body(const Dev& D, const CT& C) {
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t bi = C.y();
    const float4 pr = D.bullet_prep[bi * 4];
    if (__float_as_uint(pr.x) != 1u) return;
    const DBullet b = D.bullets[bi];
    const uint32_t k = C.x() * BULLET_PW + (threadIdx.x >> 5);
    if (k >= b.info.y) return;
    const int lane = (int)(threadIdx.x & 31u);
    const Grid g = grid_of(D, cur_of(st));
    const ntr_gpu_params* U = D.U;
    const float step = dt_of(st), t_end = now_of(st), hh = g.h;
    const float pf = pr.y;
    const float4 side = D.bullet_prep[bi * 4 + 1];
    V3 lb = qrot(make_float4(-b.q.x, -b.q.y, -b.q.z, b.q.w), xyz(b.l));
    V3 w = qrot(b.q, lb / v3(b.shape.y, b.shape.y, b.shape.x));
    const float rho = U->fluid[0];
    const V3 vhat = normalize(xyz(b.v) + 1e-9f);
    // The patch's force, torque, push on the water, and share of the wetted face.
    V3 fp = {0.0f, 0.0f, 0.0f}, tqp = {0.0f, 0.0f, 0.0f}, cenp = {0.0f, 0.0f, 0.0f};
    float cavxp = 0.0f, cavyp = 0.0f, cenwp = BIG_F;
    bool has_cav = false;
    const float4 pp = D.patches[(bi * NTR_MAX_PATCHES + k) * 2], pn = D.patches[(bi * NTR_MAX_PATCHES + k) * 2 + 1];
    V3 r = qrot(b.q, xyz(pp));
    V3 p = xyz(b.x) + r;
    V3 n = qrot(b.q, xyz(pn));
    float area = pp.w;
    V3 X = (p - g.org) / hh;
    float2 sm[4], gs;
    warp_patch_samples(D, g, X, lane, sm, gs);
    const float2 s0 = sm[0], s1 = sm[1], s2 = sm[2];
    V3 uw = {s0.y > 1e-6f ? s0.x / s0.y : 0.0f, s1.y > 1e-6f ? s1.x / s1.y : 0.0f, s2.y > 1e-6f ? s2.x / s2.y : 0.0f};
    V3 sw = {s0.y, s1.y, s2.y};
    float fill = clampf_(sm[3].y / 8.0f, 0.0f, 1.0f);
    if (warp_in_cavity(D, hh, bi, p, t_end - step, lane) || dot(r, xyz(side)) > side.w) fill = 0.0f;
    float p_gas = gs.y > 1e-6f ? gs.x / gs.y : 0.0f;
    V3 vp = xyz(b.v) + cross(w, r);
    V3 rel = vp - uw;
    float spd = length(rel);
    float wn = dot(rel, n);
    float q = 0.5f * rho * spd * spd;
    float p_water = mx(P_VAPOUR - P_ATM, pf + q * cp_patch(wn / mx(spd, 1e-9f)));
    V3 fw = -fill * p_water * area * n;
    V3 rt = rel - wn * n;
    float rtl = length(rt);
    if (rtl > 1e-9f) fw = fw - fill * CF_SKIN * 0.5f * rho * rtl * rt * area;
    fp = fw - (1.0f - fill) * mx(p_gas, P_VAPOUR - P_ATM) * area * n;
    tqp = cross(r, fp);
    warp_push_water(D, g, X, 0, -fw.x * step, sw.x, lane);
    warp_push_water(D, g, X, 1, -fw.y * step, sw.y, lane);
    warp_push_water(D, g, X, 2, -fw.z * step, sw.z, lane);
    if (wn > 0.0f && fill > 0.0f) {
        float face = fill * area * mx(dot(n, vhat), 0.0f);
        has_cav = true;
        cavxp = -dot(fw, vhat);
        cavyp = face;
        cenp = p * face;
        cenwp = dot(r, vhat);
    }
    if (lane == 0) {
        float4* o = D.bullet_patch + (bi * NTR_MAX_PATCHES + k) * 4;
        o[0] = f4(fp, cavxp);
        o[1] = f4(tqp, cavyp);
        o[2] = f4(cenp, cenwp);
        o[3] = make_float4(has_cav ? 1.0f : 0.0f, 0.0f, 0.0f, 0.0f);
    }
}
__global__ void __launch_bounds__(BULLET_PW * 32) k_bullet_patch(Dev D) { bullet_patch_body(D, HwCta{}); }
__global__ void __launch_bounds__(BULLET_PW * 32) k_bullet_patch_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    bullet_patch_body(sD, c);
}

template <class CT>
__device__ __forceinline__ void bullet_finish_body(const Dev& D, const CT& C) {
    DevState* st = D.st;
    if (st->s.dt_ns == 0) return;
    const uint32_t bi = C.x();
    if (__float_as_uint(D.bullet_prep[bi * 4].x) != 1u) return;
    const Grid g = grid_of(D, cur_of(st));
    const ntr_gpu_params* U = D.U;
    const uint32_t li = threadIdx.x;
    const DBullet b = D.bullets[bi];
    const float step = dt_of(st), t_end = now_of(st), hh = g.h;
    const float rho = U->fluid[0];
    const V3 vhat = normalize(xyz(b.v) + 1e-9f);
    __shared__ float4 red_f[256], red_t[256], red_c[256];
    const uint32_t n_patch = b.info.y;
    // Lane l's running sums over patches l, l + 256, l + 512, in that order.
    V3 f = {0.0f, 0.0f, 0.0f}, tq = {0.0f, 0.0f, 0.0f};
    float cavx = 0.0f, cavy = 0.0f;
    float4 cen = make_float4(0.0f, 0.0f, 0.0f, BIG_F);
    for (uint32_t round = 0; round < 3; round++) {
        const uint32_t k = li + round * 256u;
        if (k < n_patch) {
            const float4* rec = D.bullet_patch + (bi * NTR_MAX_PATCHES + k) * 4;
            const float4 a = rec[0], t4 = rec[1], c4 = rec[2];
            f = f + xyz(a);
            tq = tq + xyz(t4);
            if (rec[3].x != 0.0f) {
                cavx = cavx + a.w;
                cavy = cavy + t4.w;
                V3 cx = v3(cen.x, cen.y, cen.z) + xyz(c4);
                cen = make_float4(cx.x, cx.y, cx.z, mn(cen.w, c4.w));
            }
        }
    }
    red_f[li] = make_float4(f.x, f.y, f.z, cavx);
    red_t[li] = make_float4(tq.x, tq.y, tq.z, cavy);
    red_c[li] = cen;
    __syncthreads();
    for (uint32_t off = 128; off > 0; off >>= 1) {
        if (li < off) {
            float4 a = red_f[li], o = red_f[li + off];
            red_f[li] = make_float4(a.x + o.x, a.y + o.y, a.z + o.z, a.w + o.w);
            a = red_t[li], o = red_t[li + off];
            red_t[li] = make_float4(a.x + o.x, a.y + o.y, a.z + o.z, a.w + o.w);
            a = red_c[li], o = red_c[li + off];
            red_c[li] = make_float4(a.x + o.x, a.y + o.y, a.z + o.z, mn(a.w, o.w));
        }
        __syncthreads();
    }
    int32_t s_hit[6];
    {
        const float4 h0 = D.bullet_prep[bi * 4 + 2], h1 = D.bullet_prep[bi * 4 + 3];
        s_hit[0] = __float_as_int(h0.x), s_hit[1] = __float_as_int(h0.y), s_hit[2] = __float_as_int(h0.z);
        s_hit[3] = __float_as_int(h0.w), s_hit[4] = __float_as_int(h1.x), s_hit[5] = __float_as_int(h1.y);
    }
    const float hand2 = R_HAND * R_HAND * hh * hh;
    // The new velocity and position (every thread; the 27 blocks around it are looked up in
    // parallel), then the rest by one thread.
    V3 hitv, hit_l;
    for (int c = 0; c < 3; c++) {
        hitv[c] = from_fp(s_hit[c], FP_J);
        hit_l[c] = from_fp(s_hit[3 + c], FP_L);
    }
    const float4 rf = red_f[0], rt4 = red_t[0], rc = red_c[0];
    V3 force = xyz(rf) + b.x.w * v3(U->gravity[0], U->gravity[1], U->gravity[2]);
    V3 v = xyz(b.v) + (force * step + hitv) / b.x.w;
    V3 x = xyz(b.x) + v * step;
    bool near_k = false;
    if (li < 27u) {
        const I3 c = shr2(own_cell(g, x));
        const I3 nb = c + I3{(int32_t)(li / 9u), (int32_t)((li / 3u) % 3u), (int32_t)(li % 3u)} - I3{1, 1, 1};
        near_k = block_at(g, nb) != NONE;
    }
    const bool nearb = __syncthreads_or(near_k) != 0;
    if (li == 0) {
        float drag = rf.w, face = rt4.w;
        V3 l = xyz(b.l) + xyz(rt4) * step + hit_l;
        V3 axis0 = qrot(b.q, v3(0.0f, 0.0f, 1.0f));
        float spin_extra = dot(l, axis0) * (1.0f / b.shape.x - 1.0f / b.shape.y) * step;
        float cone = length(l) / b.shape.y * step;
        float4 q = qmul(b.q, make_float4(0.0f, 0.0f, nt_sin(0.5f * spin_extra), nt_cos(0.5f * spin_extra)));
        if (cone > 1e-12f) {
            V3 ln = normalize(l) * nt_sin(0.5f * cone);
            q = qmul(make_float4(ln.x, ln.y, ln.z, nt_cos(0.5f * cone)), q);
        }
        q = normalize4(q);
        float roll = b.v.w + dot(l, axis0) / b.shape.x * step;
        uint4 info = b.info;
        info.z = 1u;
        V3 hi = g.org + v3((float)g.dims[0], (float)g.dims[1], (float)g.dims[2]) * hh;
        if (x.x < g.org.x || x.y < g.org.y || x.z < g.org.z || x.x > hi.x || x.y > hi.y || x.z > hi.z) info.z = 2u;
        float pace = nearb ? length(v) : length(v) * U->fluid[1] / 4.0f;
        if (drag > 0.0f && face > 0.0f) {
            V3 mid = xyz(rc) / face;
            V3 a = mid + vhat * (rc.w - dot(mid - xyz(b.x), vhat));
            DSection s;
            s.a = f4(a, t_end - 0.5f * step);
            s.b = f4(a + v * step, 2.0f * sqrtf(drag / (PI_F * rho * LOGVINOVICH_K)));
            s.c = make_float4(face / PI_F, 0.0f, 0.0f, 0.0f);
            D.sections[bi * NTR_N_SEC + info.w % NTR_N_SEC] = s;
            info.w += 1u;
        }
        DBullet& o = D.bullets[bi];
        o.x = f4(x, b.x.w);
        o.v = f4(v, roll);
        o.q = q;
        o.l = f4(l, pace);
        o.info = info;
        float4* e = D.pose_log + (bi * NTR_LOG_CAP + st->s.step % NTR_LOG_CAP) * 3;
        e[0] = f4(x, __uint_as_float(st->s.t_ns));
        e[1] = q;
        e[2] = f4(v, roll);
    }
    __syncthreads();
    // The reach of the open sections around the new position: a lane per section (with the one
    // opened above), then the largest. A maximum of lengths (none negative; a NaN one is passed
    // over, as by the reference's running maximum) does not depend on the order.
    if (li < 32u) {
        static_assert(NTR_N_SEC == 32, "one lane per section");
        const DSection s = D.sections[bi * NTR_N_SEC + li];
        float r = 0.0f;
        if (!(s.b.w <= 0.0f || section_r2(s, t_end) >= hand2)) r = mx(length(xyz(s.a) - x), length(xyz(s.b) - x));
        if (!(r >= 0.0f)) r = 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r = mx(r, __shfl_xor_sync(0xffffffffu, r, o));
        if (li == 0) D.bullets[bi].reach = f4(x, r > 0.0f ? r + R_HAND * hh : 0.0f);
    }
    // A cavity section still narrower than the hand-over radius is a volume source: the rate at
    // which its cylinder opens goes into A_SRC of the 27 cells around its middle, with the
    // B-spline weights of a particle there, and the pressure solve makes room for it.
    if (li < NTR_N_SEC) {
        const DSection s = D.sections[bi * NTR_N_SEC + li];
        float r2 = section_r2(s, t_end);
        if (s.b.w > 0.0f && r2 < hand2) {
            float qv = PI_F * s.b.w * length(xyz(s.b) - xyz(s.a));
            V3 xx = (0.5f * (xyz(s.a) + xyz(s.b)) - g.org) / hh - 0.5f;
            I3 base = vi(vfloor(xx - 0.5f));
            V3 fx = xx - vf(base);
            V3 wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
            const CellsNear n = near_of(g, base);
            for (int a = 0; a < 3; a++)
                for (int bb = 0; bb < 3; bb++)
                    for (int cc = 0; cc < 3; cc++) {
                        uint32_t cell = near_cell(g, n, base + I3{a, bb, cc});
                        if (cell == NONE) continue;
                        atomicAdd(accp(D, A_SRC, cell), to_fp(qv * wx[a] * wy[bb] * wz[cc], FP_Q));
                    }
        }
    }
}
__global__ void __launch_bounds__(256) k_bullet_finish(Dev D) { bullet_finish_body(D, HwCta{}); }
__global__ void __launch_bounds__(256) k_bullet_finish_m(Multi M) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    bullet_finish_body(sD, c);
}

// The rubber's substep kernels over many scenes: substep i of the step, for the scenes whose
// step has that many rubber substeps (each scene's count is its own).
__global__ void k_mem_tri_m(Multi M, uint32_t i, int par) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    if (i >= sD.U->mem[1]) return;
    mem_tri_body(sD, c, par);
}
__global__ void __launch_bounds__(256) k_mem_substep_m(Multi M, uint32_t k, int par) {
    __shared__ Dev sD;
    __shared__ Cta c;
    multi_cta(M, sD, c);
    if (sD.st->parked) return;
    if (k >= sD.U->mem[1]) return;
    mem_substep_body(sD, c, k, par);
}

}  // namespace ntr
