// Device-side types and helpers of the B200 step: the device state, the pointer table every
// kernel gets, vector arithmetic in the association the reference's WGSL writes it
// (shaders/sim_defs.wgsl, common.wgsl), and the sparse-grid lookups.
//
// The sparse grid differs from the reference in how blocks are found. The reference keeps a
// pointer per 4^3 block of the whole domain and hands out indices with atomicAdd
// (fluid.wgsl:109-125). Here each step sets one bit per claimed block in a bitmask over the
// domain; a scan of the bitmask's popcounts numbers the blocks in ascending slot order, and a
// block's index is the prefix of its word plus the set bits below it in the word. That order
// is canonical (deterministic), and nothing per slot has to be cleared between steps but the
// bitmask itself (one bit per block).
#pragma once

#include <cstdint>

#include "natray.h"

namespace ntr {

constexpr uint32_t NONE = 0xffffffffu;
constexpr uint32_t TILE = 343;
constexpr uint32_t FLT_MAX_BITS = 0x7f7fffffu;

enum { A_WC = 6, A_PC = 7, A_N = 8, A_MF = 9, A_MA = 10, A_BU = 11, A_SRC = 14, A_MW = 15, A_MV = 16 };
enum { F_U = 0, F_P = 3, F_R = 4, F_Z = 5, F_D = 6, F_Q = 8, F_DIAG = 9, F_TYPE = 10 };
enum { F_EXT = 4, F_EXT_SET = 7 };

#define GAS_T 0.0f
#define WATER_T 1.0f
#define SOLID_T 2.0f
#define COVERED_T 3.0f
#define RUBBER_T 4.0f

// Fixed-point scales (sim_defs.wgsl:127-136, bullet.wgsl:76-80).
#define FP_W 16777216.0f
#define FP_M 65536.0f
#define FP_P 65536.0f
#define FP_F 4194304.0f
#define FP_A 65536.0f
#define FP_Q 16777216.0f
#define FP_J 1073741824.0f
#define FP_L 68719476736.0f
#define FP_X 4096.0f

#define RHO_AIR 1.2f
#define MU_AIR 1.8e-5f
#define SIGMA_W 0.072f
#define PI_F 3.14159265358979f
#define GAMMA_F 1.4f
#define P_ATM 101325.0f
#define P_VAPOUR 2339.0f
#define RHO_ATM 1.204f
#define RHO_VAPOUR 0.0278f
#define CFL_AIR 0.9f
#define CONTACT_F 0.05f
#define MU_WATER 1.0e-3f
#define MU_JACKET 0.8f
#define LOGVINOVICH_K 2.0f
#define R_HAND 1.5f
#define CP_WAKE (-0.4f)
#define CF_SKIN 0.003f
#define EVAPORATION 1.3e-10f
#define WE_CRIT 12.0f
#define BIG_F 3.0e38f

struct Tri {
    uint32_t v0, v1, v2;
    float rest_area;
    float4 dm_inv;
};
static_assert(sizeof(Tri) == 32, "Tri");

struct DBullet {
    float4 x, v, q, l, shape, reach;
    uint4 info;
};
static_assert(sizeof(DBullet) == 112, "Bullet");

struct DSection {
    float4 a, b, c;
};

// The device's copy of the step state. `s` is word for word the reference's State; the
// solver scalars are also kept in double.
struct DevState {
    ntr_state s;
    double rz, alpha, beta, b_norm, r_norm;
    uint32_t solver_on;
    uint32_t ticket[4];  // arrival counters of the last-block reductions
    uint32_t nbrk;       // break-ups of this step
    uint32_t err;        // bit 0: a bounded grid barrier gave up
    uint32_t bar_count;  // grid barrier of the persistent solver: arrivals (reset per launch)
    uint32_t iters_prev;  // the last solve's iterations, kept for a joint solve's split (k_solve_reset_m)
    // The next block P2G (0) and G2P (1) hand out in a one-scene launch, zeroed by k_begin_step.
    uint32_t next_block[2];
    uint32_t pad;
    // The step's work, for its algorithmic bytes: this step's water and free-gas cells (counted
    // by k_project), and totals since ntr_sim_work last cleared them (added by the step's last
    // kernel): NTR_WORK_STEPS .. NTR_WORK_SPRAY of include/natray.h.
    uint32_t n_water, n_gas;
    unsigned long long work[6];
    // Steps this scene may still take in the current batch call (0xFFFFFFFF: no limit); a
    // batch of scenes stepped together gives each its own count (k_begin_step). A scene whose
    // budget has run out is parked for the rest of the call: its begin_step keeps the last
    // step length aside and sets none, and its kernels in the batch's launches skip it, so its
    // state stays as its last step left it (the host puts the step length back).
    uint32_t step_budget, parked, parked_dt;
};

// Every pointer and size a kernel may need. Passed by value.
struct Dev {
    const ntr_gpu_params* U;
    DevState* st;
    float4 *pos, *vel, *c0, *c1, *c2;
    uint32_t Np, Nv, Nt, cap_blocks, cap_cells, nwords, spray_cap, wet_res;
    uint32_t n_tiles, radix_passes, scan_ctas, fp64_dots;
    // The solver's grid barriers: polls before a wait gives up, and a CTA that skips its first
    // arrival (NONE: none) so that the others' waits run out (ntr_sim_test_barrier).
    uint32_t bar_spins, bar_skip;
    uint32_t* mask[2];
    uint32_t* prefix[2];
    uint32_t* block_list[2];
    uint32_t* cta_sum;
    uint32_t *pslot, *key, *key_alt, *val_alt, *key_sorted, *sorted, *hist;
    uint32_t* hist2;  // the sort's second histogram (pass 1's, counted by pass 0's scatter)
    uint32_t *block_start, *block_nb, *block_active;
    int32_t* acc;
    float* cf;
    float* air[2];
    double* xsum;   // the solver's running sums: 2 parities x 256 residues x 3 quantities
    double* spart;  // the solver's per-block partial sums when a CTA has many blocks: 3 x cap_blocks
    float4* mem_x[2];
    float4* mem_v[2];
    float4 *mem_water, *mem_layer;
    float2* mem_push;
    float* mem_mass;
    const Tri* tris;
    uint32_t *alive, *vtri_off, *vtri;
    uint8_t* vtri_c;  // per entry of vtri: which corner (0-2) of the triangle the vertex is
    float4* tri_rec;  // per triangle: what its vertices fold into their force sums, 4 float4
    DBullet* bullets;
    const float4* patches;
    const float2* outlines;
    DSection* sections;
    int32_t* bullet_hit;
    float4* bullet_prep;   // per bullet 4 float4: state and pressure ahead, wetted side, impulses
    float4* bullet_patch;  // per bullet and patch 4 float4: force, torque, cavity share
    float4* pose_log;
    float4* spray;  // 3 float4 per slot: pos + r, vel + weight, air
    float4* landed;
    uint32_t* touch;
    float4 *brk_x, *brk_v;
    uint32_t *brk_count, *brk_off;
    int32_t* tiles;     // per block: the P2G tile, 8 fields x 343 i32
    uint32_t* tile_ok;  // per block: 1 when its tile holds this step's sums
    uint32_t* coltot;   // radix sort: per digit, the elements with that digit
    uint32_t* wnb;      // solver: per cell, its 6 neighbours that are water (or NONE), 8 words
};

// Where a CTA is in its scene's grid: x() and nx() as blockIdx.x and gridDim.x of a launch for
// one scene, y() as blockIdx.y. Every step kernel's body takes its place from one of these, so
// that the same body runs in a launch for one scene (HwCta: the hardware's indices, read where
// used) and in one launch for many scenes (Cta: a batch, where each scene owns a contiguous
// range of the launch's CTAs).
// A CTA of a one-scene launch. `dynamic`: the per-block kernels may hand their blocks out from
// a counter (a many-scene launch's CTAs are tied to their scenes' blocks).
struct HwCta {
    static constexpr bool dynamic = true;
    __device__ __forceinline__ uint32_t x() const { return blockIdx.x; }
    __device__ __forceinline__ uint32_t nx() const { return gridDim.x; }
    __device__ __forceinline__ uint32_t y() const { return blockIdx.y; }
};
struct Cta {
    static constexpr bool dynamic = false;
    uint32_t x_, nx_, y_;
    __device__ __forceinline__ uint32_t x() const { return x_; }
    __device__ __forceinline__ uint32_t nx() const { return nx_; }
    __device__ __forceinline__ uint32_t y() const { return y_; }
};

// A launch over many scenes: scene s owns CTAs first[s] .. first[s + 1] - 1 of the launch (its
// grid for this kernel, possibly none), with the pointer table jobs[s].
struct Multi {
    const Dev* jobs;
    const uint32_t* first;  // n + 1 entries
    uint32_t n;
};

// The CTA's scene in a launch over many scenes: its pointer table and its place in the
// scene's grid, written to shared memory (`sD`, `sC`) so that they cost no registers. Every
// thread of the CTA calls it (it has a barrier).
__device__ __forceinline__ void multi_cta(const Multi& M, Dev& sD, Cta& sC) {
    const uint32_t b = blockIdx.x;
    uint32_t lo = 0, hi = M.n;  // the last scene whose first CTA is at or before b
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(M.first + mid) <= b) lo = mid;
        else hi = mid;
    }
    const uint32_t* src = reinterpret_cast<const uint32_t*>(M.jobs + lo);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sD);
    static_assert(sizeof(Dev) % 4 == 0, "the pointer table copies in words");
    for (uint32_t k = threadIdx.x; k < sizeof(Dev) / 4; k += blockDim.x) dst[k] = __ldg(src + k);
    if (threadIdx.x == 0) {
        const uint32_t f = __ldg(M.first + lo);
        sC = Cta{b - f, __ldg(M.first + lo + 1) - f, blockIdx.y};
    }
    __syncthreads();
}

// Packed FP32 multiply and add (two lanes of one 64-bit register pair, sm_100). Written in PTX
// with an explicit round-to-nearest modifier so that no multiply and add pair is ever fused into a
// packed FMA: each lane rounds exactly as the scalar __fmul_rn and __fadd_rn would.
__device__ __forceinline__ float2 mul2_rn(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// ---- vectors (association as written in the WGSL) ------------------------------------------
struct V3 {
    float x, y, z;
    __device__ float& operator[](int i) { return i == 0 ? x : i == 1 ? y : z; }
    __device__ float operator[](int i) const { return i == 0 ? x : i == 1 ? y : z; }
};
__device__ __forceinline__ V3 v3(float a, float b, float c) { return {a, b, c}; }
__device__ __forceinline__ V3 xyz(float4 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 operator+(V3 a, float s) { return {a.x + s, a.y + s, a.z + s}; }
__device__ __forceinline__ V3 operator-(V3 a, float s) { return {a.x - s, a.y - s, a.z - s}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V3 normalize(V3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
__device__ __forceinline__ float distance(V3 a, V3 b) { return length(a - b); }
__device__ __forceinline__ V3 vfloor(V3 a) { return {floorf(a.x), floorf(a.y), floorf(a.z)}; }
// min / max with the operand order of the CPU restatement (`b < a ? b : a`).
__device__ __forceinline__ float mn(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float mx(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float clampf_(float x, float lo, float hi) { return mn(mx(x, lo), hi); }

struct I3 {
    int32_t x, y, z;
};
__device__ __forceinline__ I3 operator+(I3 a, I3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ I3 operator-(I3 a, I3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ I3 operator*(I3 a, int32_t s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ I3 shr2(I3 a) { return {a.x >> 2, a.y >> 2, a.z >> 2}; }
__device__ __forceinline__ I3 vi(V3 a) { return {__float2int_rz(a.x), __float2int_rz(a.y), __float2int_rz(a.z)}; }
__device__ __forceinline__ V3 vf(I3 a) { return {(float)a.x, (float)a.y, (float)a.z}; }
__device__ __forceinline__ uint32_t f2u(float x) { return __float2uint_rz(x); }

// to_fp rounds half to even (sim_defs.wgsl:217-219): rint(clamp(x * scale, -2e9, 2e9)).
__device__ __forceinline__ int32_t to_fp(float x, float scale) { return __float2int_rn(clampf_(x * scale, -2e9f, 2e9f)); }
// The same rounding by addition, for the transfer kernels, which convert hundreds of values per
// particle (more than the conversion unit keeps up with): for |y| < 2^22, y + 1.5 * 2^23 lies
// in [2^23, 2^24], where floats are the integers, so the addition rounds y to the nearest
// integer, ties to even (1.5 * 2^23 is even), and the integer is the difference of the bit
// patterns. fp_round_pos does the same for 0 <= y < 2^23 with 2^23. The caller shows the range.
__device__ __forceinline__ int32_t fp_round(float y) { return __float_as_int(__fadd_rn(y, 12582912.0f)) - 0x4B400000; }
__device__ __forceinline__ int32_t fp_round_pos(float y) { return __float_as_int(__fadd_rn(y, 8388608.0f)) - 0x4B000000; }
__device__ __forceinline__ float from_fp(int32_t x, float scale) { return (float)x / scale; }

__device__ __forceinline__ V3 axis_weights(float fx) {
    return {0.5f * (1.5f - fx) * (1.5f - fx), 0.75f - (fx - 1.0f) * (fx - 1.0f), 0.5f * (fx - 0.5f) * (fx - 0.5f)};
}

// ---- float transcendentals ---------------------------------------------------------------------
// exp, log, sin, cos, asin and pow of the step, written from the mathematics so that a CPU
// evaluation of the same algorithms agrees with the device to the bit:
//   exp       Cody-Waite reduction x = k ln2 + r, |r| <= ln2/2 (ln2 as a 16-bit head plus a
//             tail), Taylor polynomial of e^r to r^7 in Horner form, times 2^k by exact
//             power-of-two multiplications.
//   log       x = m 2^e, m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh s, s = (m - 1)/(m + 1), odd
//             power series to s^11; ln x = e ln2_head + (ln m + e ln2_tail).
//   sin, cos  x = k pi/2 + r (pi/2 in three parts), Taylor polynomials to r^9 and r^10, the
//             quadrant from k mod 4.
//   asin      Maclaurin series to x^27 on |x| <= 1/2, pi/2 - 2 asin(sqrt((1 - x)/2)) above.
//   pow       exp(y ln x) for x > 0.
// Built with -fmad=false, each line is the rounded IEEE operation written.
__device__ __forceinline__ float nt_scale2(float p, int k) {
    if (k > 127) {
        p = p * 0x1p64f;
        k -= 64;
    }
    if (k < -125) {
        p = p * 0x1p-100f;
        k += 100;
    }
    return p * __uint_as_float((uint32_t)(k + 127) << 23);
}
__device__ __forceinline__ float nt_exp(float x) {
    if (x != x) return x;
    if (x > 88.72284f) return __uint_as_float(0x7f800000u);
    if (x < -103.972084f) return 0.0f;
    float k = rintf(x * 1.442695f);
    float r = __fmaf_rn(-k, 1.4286068e-06f, x - k * 0.693145751953125f);  // k * 0.693145751953125 is exact
    float p = 0.0001984127f;
    p = __fmaf_rn(p, r, 0.0013888889f);
    p = __fmaf_rn(p, r, 0.008333334f);
    p = __fmaf_rn(p, r, 0.041666668f);
    p = __fmaf_rn(p, r, 0.16666667f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    return nt_scale2(p, (int)k);
}
__device__ __forceinline__ float nt_log(float x) {
    if (x != x) return x;
    if (x < 0.0f) return __uint_as_float(0x7fc00000u);
    if (x == 0.0f) return __uint_as_float(0xff800000u);
    if (x == __uint_as_float(0x7f800000u)) return x;
    int e = 0;
    uint32_t u = __float_as_uint(x);
    if ((u >> 23) == 0) {
        x = x * 0x1p25f;
        u = __float_as_uint(x);
        e = -25;
    }
    e += (int)((u >> 23) & 0xffu) - 126;
    float m = __uint_as_float((u & 0x007fffffu) | 0x3f000000u);
    if (m < 0.70710677f) {
        m = m * 2.0f;
        e -= 1;
    }
    float s = (m - 1.0f) / (m + 1.0f);
    float z = s * s;
    float p = 0.09090909f;
    p = __fmaf_rn(p, z, 0.11111111f);
    p = __fmaf_rn(p, z, 0.14285715f);
    p = __fmaf_rn(p, z, 0.2f);
    p = __fmaf_rn(p, z, 0.33333334f);
    p = __fmaf_rn(p, z, 1.0f);
    float lm = 2.0f * s * p;
    float fe = (float)e;
    return fe * 0.693145751953125f + (lm + fe * 1.4286068e-06f);
}
__device__ __forceinline__ void nt_sincos(float x, float* so, float* co) {
    float k = rintf(x * 0.63661975f);
    float r = ((x - k * 1.5703125f) - k * 0.0004838268f) - k * 2.563283e-12f;
    float z = r * r;
    float ps = 2.7557319e-06f;
    ps = __fmaf_rn(ps, z, -0.0001984127f);
    ps = __fmaf_rn(ps, z, 0.008333334f);
    ps = __fmaf_rn(ps, z, -0.16666667f);
    float sr = __fmaf_rn(r * z, ps, r);
    float pc = -2.755732e-07f;
    pc = __fmaf_rn(pc, z, 2.4801588e-05f);
    pc = __fmaf_rn(pc, z, -0.0013888889f);
    pc = __fmaf_rn(pc, z, 0.041666668f);
    pc = __fmaf_rn(pc, z, -0.5f);
    float cr = __fmaf_rn(z, pc, 1.0f);
    int q = ((int)k) & 3;
    *so = q == 0 ? sr : q == 1 ? cr : q == 2 ? -sr : -cr;
    *co = q == 0 ? cr : q == 1 ? -sr : q == 2 ? -cr : sr;
}
__device__ __forceinline__ float nt_sin(float x) {
    float s, c;
    nt_sincos(x, &s, &c);
    return s;
}
__device__ __forceinline__ float nt_cos(float x) {
    float s, c;
    nt_sincos(x, &s, &c);
    return c;
}
__device__ __forceinline__ float nt_asin_series(float t) {
    float z = t * t;
    float p = 0.0057400377f;
    p = __fmaf_rn(p, z, 0.0064472104f);
    p = __fmaf_rn(p, z, 0.007312526f);
    p = __fmaf_rn(p, z, 0.008390335f);
    p = __fmaf_rn(p, z, 0.009761609f);
    p = __fmaf_rn(p, z, 0.011551801f);
    p = __fmaf_rn(p, z, 0.013964844f);
    p = __fmaf_rn(p, z, 0.017352764f);
    p = __fmaf_rn(p, z, 0.022372158f);
    p = __fmaf_rn(p, z, 0.030381944f);
    p = __fmaf_rn(p, z, 0.04464286f);
    p = __fmaf_rn(p, z, 0.075f);
    p = __fmaf_rn(p, z, 0.16666667f);
    return __fmaf_rn(t * z, p, t);
}
__device__ __forceinline__ float nt_asin(float x) {
    float a = fabsf(x);
    if (!(a <= 1.0f)) return __uint_as_float(0x7fc00000u);
    float r = a <= 0.5f ? nt_asin_series(a) : 1.5707964f - 2.0f * nt_asin_series(sqrtf((1.0f - a) * 0.5f));
    return x < 0.0f ? -r : r;
}
__device__ __forceinline__ float nt_pow(float x, float y) {
    if (x > 0.0f) return nt_exp(y * nt_log(x));
    if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : __uint_as_float(0x7f800000u));
    return __uint_as_float(0x7fc00000u);
}

__device__ __forceinline__ uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
__device__ __forceinline__ uint32_t hash3(uint32_t a, uint32_t b, uint32_t c) { return pcg(a ^ pcg(b ^ pcg(c))); }
__device__ __forceinline__ float rnd(uint32_t& seed) {
    seed = pcg(seed);
    return (float)(seed >> 8u) * (1.0f / 16777216.0f);
}
__device__ __forceinline__ float rnd_gauss(uint32_t& seed) {
    float u1 = mx(rnd(seed), 1e-7f);
    float u2 = rnd(seed);
    return sqrtf(-2.0f * nt_log(u1)) * nt_cos(2.0f * PI_F * u2);
}

// ---- the grid ------------------------------------------------------------------------------
struct Grid {
    float h;
    V3 org;
    uint32_t dims[3], bd[3];
    uint32_t cap_blocks, cap_cells;
    const uint32_t* mask;
    const uint32_t* prefix;
    const uint32_t* list;
    const uint32_t* nb;
};

__device__ __forceinline__ Grid grid_of(const Dev& D, int cur) {
    Grid g;
    const ntr_gpu_params* U = D.U;
    g.h = U->origin[3];
    g.org = {U->origin[0], U->origin[1], U->origin[2]};
    g.dims[0] = U->dims[0], g.dims[1] = U->dims[1], g.dims[2] = U->dims[2];
    g.bd[0] = U->bdims[0], g.bd[1] = U->bdims[1], g.bd[2] = U->bdims[2];
    g.cap_blocks = D.cap_blocks;
    g.cap_cells = D.cap_cells;
    g.mask = D.mask[cur];
    g.prefix = D.prefix[cur];
    g.list = D.block_list[cur];
    g.nb = D.block_nb;
    return g;
}

__device__ __forceinline__ uint32_t block_slot(const Grid& g, I3 b) {
    return ((uint32_t)b.x * g.bd[1] + (uint32_t)b.y) * g.bd[2] + (uint32_t)b.z;
}
__device__ __forceinline__ I3 slot_coord(const Grid& g, uint32_t s) {
    return {(int32_t)(s / (g.bd[2] * g.bd[1])), (int32_t)((s / g.bd[2]) % g.bd[1]), (int32_t)(s % g.bd[2])};
}
__device__ __forceinline__ bool in_bd(const Grid& g, I3 b) {
    return b.x >= 0 && b.y >= 0 && b.z >= 0 && (uint32_t)b.x < g.bd[0] && (uint32_t)b.y < g.bd[1] && (uint32_t)b.z < g.bd[2];
}
// Index of the block at `slot` among this step's blocks, or NONE.
__device__ __forceinline__ uint32_t lookup(const uint32_t* mask, const uint32_t* prefix, uint32_t slot, uint32_t cap) {
    uint32_t m = __ldg(mask + (slot >> 5));
    uint32_t bit = slot & 31u;
    if (!((m >> bit) & 1u)) return NONE;
    uint32_t idx = __ldg(prefix + (slot >> 5)) + __popc(m & ((1u << bit) - 1u));
    return idx < cap ? idx : NONE;
}
__device__ __forceinline__ uint32_t block_at(const Grid& g, I3 b) {
    if (!in_bd(g, b)) return NONE;
    return lookup(g.mask, g.prefix, block_slot(g, b), g.cap_blocks);
}
__device__ __forceinline__ I3 local_coord(uint32_t i) {
    uint32_t l = i % 64u;
    return {(int32_t)(l / 16u), (int32_t)((l / 4u) % 4u), (int32_t)(l % 4u)};
}
__device__ __forceinline__ I3 cell_coord(const Grid& g, uint32_t i) { return slot_coord(g, g.list[i / 64u]) * 4 + local_coord(i); }
__device__ __forceinline__ uint32_t neighbour(const Grid& g, uint32_t cell, I3 off) {
    I3 q = local_coord(cell) + off;
    I3 n = {(q.x >= 4) - (q.x < 0), (q.y >= 4) - (q.y < 0), (q.z >= 4) - (q.z < 0)};
    uint32_t b = g.nb[(cell / 64u) * 27u + (uint32_t)((n.x + 1) * 9 + (n.y + 1) * 3 + n.z + 1)];
    if (b == NONE) return NONE;
    I3 l = q - n * 4;
    return b * 64u + (uint32_t)l.x * 16u + (uint32_t)l.y * 4u + (uint32_t)l.z;
}
__device__ __forceinline__ uint32_t cell_at(const Grid& g, I3 c) {
    if (c.x < 0 || c.y < 0 || c.z < 0 || (uint32_t)c.x >= g.dims[0] || (uint32_t)c.y >= g.dims[1] || (uint32_t)c.z >= g.dims[2]) return NONE;
    uint32_t b = lookup(g.mask, g.prefix, block_slot(g, shr2(c)), g.cap_blocks);
    if (b == NONE) return NONE;
    return b * 64u + (uint32_t)(c.x & 3) * 16u + (uint32_t)(c.y & 3) * 4u + (uint32_t)(c.z & 3);
}
// The cells of a 3^3 stencil with corner `base`: the up to 2 x 2 x 2 blocks that hold the cells
// base .. base + 2 (per axis) are looked up once, all eight at the same time, instead of a
// dependent lookup per cell. near_cell gives what cell_at gives, for cells of the stencil.
struct CellsNear {
    I3 b0;
    uint32_t blk[8];  // blocks b0 + (x, y, z), x, y, z in {0, 1}, at x + 2 y + 4 z
};
__device__ __forceinline__ CellsNear near_of(const Grid& g, I3 base) {
    CellsNear n;
    n.b0 = shr2(base);
#pragma unroll
    for (int k = 0; k < 8; k++) n.blk[k] = block_at(g, n.b0 + I3{k & 1, (k >> 1) & 1, k >> 2});
    return n;
}
// `c` is a cell of the stencil: base + (0..2, 0..2, 0..2), so its block is b0 or the next one
// along each axis.
__device__ __forceinline__ uint32_t near_cell(const Grid& g, const CellsNear& n, I3 c) {
    if (c.x < 0 || c.y < 0 || c.z < 0 || (uint32_t)c.x >= g.dims[0] || (uint32_t)c.y >= g.dims[1] || (uint32_t)c.z >= g.dims[2]) return NONE;
    const I3 d = shr2(c) - n.b0;
    const uint32_t x0 = d.x ? n.blk[1] : n.blk[0], x1 = d.x ? n.blk[3] : n.blk[2];
    const uint32_t x2 = d.x ? n.blk[5] : n.blk[4], x3 = d.x ? n.blk[7] : n.blk[6];
    const uint32_t y0 = d.y ? x1 : x0, y1 = d.y ? x3 : x2;
    const uint32_t b = d.z ? y1 : y0;
    if (b == NONE) return NONE;
    return b * 64u + (uint32_t)(c.x & 3) * 16u + (uint32_t)(c.y & 3) * 4u + (uint32_t)(c.z & 3);
}
// The 27 cells of the stencil base + (0..2, 0..2, 0..2), with the work of near_cell shared:
// per axis each coordinate's block step from base's block, offset in the block and whether it
// lies in the domain; per (a, b) the two blocks the z step chooses from. cell(a, b, c) is
// near_cell(g, near_of(g, base), base + (a, b, c)).
struct Stencil27 {
    uint32_t blk[9][2];  // per a * 3 + b: the block for z step 0 and 1
    uint32_t off[9];     // per a * 3 + b: the cells' x and y offsets in the block
    uint32_t lz[3];
    bool ok[9], okz[3], zs[3];
    __device__ __forceinline__ uint32_t cell(int a, int b, int c) const {
        const int ab = a * 3 + b;
        const uint32_t bk = zs[c] ? blk[ab][1] : blk[ab][0];
        return (ok[ab] && okz[c] && bk != NONE) ? bk * 64u + off[ab] + lz[c] : NONE;
    }
};
__device__ __forceinline__ Stencil27 stencil_of(const Grid& g, const CellsNear& n, I3 base) {
    Stencil27 s;
    bool sx[3], sy[3], okx[3], oky[3];
    uint32_t lx[3], ly[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const int cx = base.x + a, cy = base.y + a, cz = base.z + a;
        okx[a] = cx >= 0 && (uint32_t)cx < g.dims[0];
        oky[a] = cy >= 0 && (uint32_t)cy < g.dims[1];
        s.okz[a] = cz >= 0 && (uint32_t)cz < g.dims[2];
        sx[a] = (cx >> 2) != n.b0.x, sy[a] = (cy >> 2) != n.b0.y, s.zs[a] = (cz >> 2) != n.b0.z;
        lx[a] = (uint32_t)(cx & 3), ly[a] = (uint32_t)(cy & 3), s.lz[a] = (uint32_t)(cz & 3);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        // blocks b0 + (sx, y, z) for (y, z) = (0,0), (1,0), (0,1), (1,1)
        const uint32_t x0 = sx[a] ? n.blk[1] : n.blk[0], x1 = sx[a] ? n.blk[3] : n.blk[2];
        const uint32_t x2 = sx[a] ? n.blk[5] : n.blk[4], x3 = sx[a] ? n.blk[7] : n.blk[6];
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const int ab = a * 3 + b;
            s.blk[ab][0] = sy[b] ? x1 : x0;
            s.blk[ab][1] = sy[b] ? x3 : x2;
            s.off[ab] = lx[a] * 16u + ly[b] * 4u;
            s.ok[ab] = okx[a] && oky[b];
        }
    }
    return s;
}
__device__ __forceinline__ I3 own_cell(const Grid& g, V3 p) { return vi(vfloor((p - g.org) / g.h)); }
__device__ __forceinline__ V3 lattice_offset(uint32_t d) {
    V3 o = {0.5f, 0.5f, 0.5f};
    if (d == 0) o.x = 0.0f;
    if (d == 1) o.y = 0.0f;
    if (d == 2) o.z = 0.0f;
    return o;
}
__device__ __forceinline__ uint32_t a_mom(uint32_t d) { return 2 * d; }
__device__ __forceinline__ uint32_t a_wt(uint32_t d) { return 2 * d + 1; }

__device__ __forceinline__ int cur_of(const DevState* st) { return (int)(st->s.step & 1u); }

}  // namespace ntr
