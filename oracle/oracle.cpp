// ORACLE - test infrastructure only. A CPU restatement of natray's simulation step, the
// checker the CUDA path is compared with and the timed CPU baseline. Nothing in the product
// (natray_b200/) may include, link or call this file; only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg use it.
//
// It follows the reference's WGSL kernels statement by statement, in the order src/sim.rs
// encodes them (src/sim.rs:390-426, 553-566):
//   shaders/sim_defs.wgsl  addressing, fixed point (to_fp rounds half to even), cell types
//   shaders/common.wgsl    pcg / hash3 / rnd / rnd_gauss
//   shaders/fluid.wgsl     begin_step .. g2p
//   shaders/membrane.wgsl  mark_rubber, mem_splat, mem_sample, mem_substep
//   shaders/air.wgsl       air_carry, air_fill, air_substep, keep_blocks
//   shaders/bullet.wgsl    bullet_step, bullet_apply, carve, rubber_contact
// and the host half of Sim::run (src/sim.rs:585-648).
//
// The reference is nondeterministic where it hands out places with atomicAdd: block indices
// (fluid.wgsl:117), particle ranks in a block (fluid.wgsl:148) and spray slots
// (fluid.wgsl:726). This restatement uses the canonical order instead: blocks by ascending
// slot, particles of a block by ascending index, spray slots in the order g2p visits the
// particles (block by block, sorted order within a block). Everything else is what the WGSL
// computes, with the same association of every floating-point expression (built with
// -ffp-contract=off), so integer results (block sets, sort order, fixed-point transfer sums)
// can be compared bit for bit.
//
// Templated on the real type: float is the FP32 oracle, double the FP64 precision oracle.
// Inner products of the solver are accumulated either in the reference's FP32 tree
// (fluid.wgsl:414-439) or in FP64 with the same tree shape.
//
// Parity of the step kernels is pinned by the oracle's own known-answer tests (tests/), and by
// the reference's scene invariants; the reference has no golden vectors for the step itself.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "natray.h"

namespace oracle {

static const uint32_t NONE = 0xffffffffu;

// ---- vectors ------------------------------------------------------------------------------
template <class R>
struct V2 {
    R x, y;
};
template <class R>
struct V3 {
    R x, y, z;
    R& operator[](int i) { return i == 0 ? x : i == 1 ? y : z; }
    R operator[](int i) const { return i == 0 ? x : i == 1 ? y : z; }
};
template <class R>
struct V4 {
    R x, y, z, w;
    V3<R> xyz() const { return {x, y, z}; }
};
template <class R> static inline V3<R> v3(R a, R b, R c) { return {a, b, c}; }
template <class R> static inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> static inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> static inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> static inline V3<R> operator*(V3<R> a, V3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> static inline V3<R> operator/(V3<R> a, V3<R> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class R> static inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> static inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> static inline V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> static inline V3<R> operator+(V3<R> a, R s) { return {a.x + s, a.y + s, a.z + s}; }
template <class R> static inline V3<R> operator-(V3<R> a, R s) { return {a.x - s, a.y - s, a.z - s}; }
template <class R> static inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> static inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> static inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> static inline V3<R> normalize(V3<R> a) { return a * (R(1) / std::sqrt(dot(a, a))); }
template <class R> static inline R distance(V3<R> a, V3<R> b) { return length(a - b); }
template <class R> static inline V3<R> vfloor(V3<R> a) { return {std::floor(a.x), std::floor(a.y), std::floor(a.z)}; }
template <class R> static inline R mn(R a, R b) { return b < a ? b : a; }
template <class R> static inline R mx(R a, R b) { return a < b ? b : a; }
template <class R> static inline R clampr(R x, R lo, R hi) { return mn(mx(x, lo), hi); }

struct I3 {
    int32_t x, y, z;
};
static inline I3 operator+(I3 a, I3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline I3 operator-(I3 a, I3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline I3 operator*(I3 a, int32_t s) { return {a.x * s, a.y * s, a.z * s}; }
static inline I3 shr2(I3 a) { return {a.x >> 2, a.y >> 2, a.z >> 2}; }

// Float to i32 as WGSL/CUDA convert: truncate, saturate, NaN to 0.
template <class R>
static inline int32_t f2i(R x) {
    if (!(x == x)) return 0;
    if (x >= R(2147483647.0)) return 2147483647;
    if (x <= R(-2147483648.0)) return (int32_t)0x80000000;
    return (int32_t)x;
}
template <class R>
static inline uint32_t f2u(R x) {
    if (!(x > R(0))) return 0;
    if (x >= R(4294967295.0)) return 0xffffffffu;
    return (uint32_t)x;
}
template <class R>
static inline I3 vi(V3<R> a) { return {f2i(a.x), f2i(a.y), f2i(a.z)}; }
template <class R>
static inline V3<R> vf(I3 a) { return {R(a.x), R(a.y), R(a.z)}; }

// to_fp: round half to even of the clamped product (sim_defs.wgsl:217-219).
template <class R>
static inline int32_t to_fp(R x, R scale) {
    R y = clampr(x * scale, R(-2e9), R(2e9));
    return (int32_t)std::nearbyint(y);
}
template <class R>
static inline R from_fp(int32_t x, R scale) { return R(x) / scale; }

static inline uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
static inline uint32_t hash3(uint32_t a, uint32_t b, uint32_t c) { return pcg(a ^ pcg(b ^ pcg(c))); }

static inline uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
static inline float bitsf(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// ---- float transcendentals ---------------------------------------------------------------------
// The float build evaluates exp, log, sin, cos, asin and pow with these rather than the C
// library, so that a GPU build that writes the same algorithms agrees with it to the bit (the
// reference's own WGSL leaves their precision to the platform). Methods, all from the
// mathematics:
//   exp       Cody-Waite reduction x = k ln2 + r, |r| <= ln2/2, ln2 split into a head with 16
//             significant bits and a tail; Taylor polynomial of e^r to r^7 (Horner); times 2^k
//             by exact power-of-two multiplications.
//   log       x = m 2^e with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s), s = (m - 1)/(m + 1),
//             odd power series of atanh to s^11; ln x = e ln2_head + (ln m + e ln2_tail).
//   sin, cos  x = k pi/2 + r with pi/2 in three parts, Taylor polynomials to r^9 and r^10,
//             quadrant from k mod 4.
//   asin      Maclaurin series to x^27 on |x| <= 1/2, asin x = pi/2 - 2 asin(sqrt((1 - x)/2))
//             above.
//   pow       exp(y ln x) for x > 0.
// The double build (the FP64 oracle) uses the C library.
namespace nm {
static inline float scale2(float p, int k) {
    if (k > 127) {
        p = p * 0x1p64f;
        k -= 64;
    }
    if (k < -125) {
        p = p * 0x1p-100f;
        k += 100;
    }
    return p * bitsf((uint32_t)(k + 127) << 23);
}
static inline float exp_(float x) {
    if (x != x) return x;
    if (x > 88.72284f) return INFINITY;
    if (x < -103.972084f) return 0.0f;
    float k = std::nearbyint(x * 1.442695f);
    float r = std::fmaf(-k, 1.4286068e-06f, x - k * 0.693145751953125f);  // k * 0.693145751953125 is exact
    float p = 0.0001984127f;
    p = std::fmaf(p, r, 0.0013888889f);
    p = std::fmaf(p, r, 0.008333334f);
    p = std::fmaf(p, r, 0.041666668f);
    p = std::fmaf(p, r, 0.16666667f);
    p = std::fmaf(p, r, 0.5f);
    p = std::fmaf(p, r, 1.0f);
    p = std::fmaf(p, r, 1.0f);
    return scale2(p, (int)k);
}
static inline float log_(float x) {
    if (x != x) return x;
    if (x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (x == INFINITY) return x;
    int e = 0;
    uint32_t u = fbits(x);
    if ((u >> 23) == 0) {
        x = x * 0x1p25f;
        u = fbits(x);
        e = -25;
    }
    e += (int)((u >> 23) & 0xffu) - 126;
    float m = bitsf((u & 0x007fffffu) | 0x3f000000u);
    if (m < 0.70710677f) {
        m = m * 2.0f;
        e -= 1;
    }
    float s = (m - 1.0f) / (m + 1.0f);
    float z = s * s;
    float p = 0.09090909f;
    p = std::fmaf(p, z, 0.11111111f);
    p = std::fmaf(p, z, 0.14285715f);
    p = std::fmaf(p, z, 0.2f);
    p = std::fmaf(p, z, 0.33333334f);
    p = std::fmaf(p, z, 1.0f);
    float lm = 2.0f * s * p;
    float fe = (float)e;
    return fe * 0.693145751953125f + (lm + fe * 1.4286068e-06f);
}
static inline void sincos_(float x, float* so, float* co) {
    float k = std::nearbyint(x * 0.63661975f);
    float r = ((x - k * 1.5703125f) - k * 0.0004838268f) - k * 2.563283e-12f;
    float z = r * r;
    float ps = 2.7557319e-06f;
    ps = std::fmaf(ps, z, -0.0001984127f);
    ps = std::fmaf(ps, z, 0.008333334f);
    ps = std::fmaf(ps, z, -0.16666667f);
    float sr = std::fmaf(r * z, ps, r);
    float pc = -2.755732e-07f;
    pc = std::fmaf(pc, z, 2.4801588e-05f);
    pc = std::fmaf(pc, z, -0.0013888889f);
    pc = std::fmaf(pc, z, 0.041666668f);
    pc = std::fmaf(pc, z, -0.5f);
    float cr = std::fmaf(z, pc, 1.0f);
    int q = ((int)k) & 3;
    float s = q == 0 ? sr : q == 1 ? cr : q == 2 ? -sr : -cr;
    float c = q == 0 ? cr : q == 1 ? -sr : q == 2 ? -cr : sr;
    *so = s;
    *co = c;
}
static inline float sin_(float x) {
    float s, c;
    sincos_(x, &s, &c);
    return s;
}
static inline float cos_(float x) {
    float s, c;
    sincos_(x, &s, &c);
    return c;
}
static inline float asin_series(float t) {
    const float C[13] = {0.16666667f, 0.075f, 0.04464286f, 0.030381944f, 0.022372158f, 0.017352764f, 0.013964844f,
                         0.011551801f, 0.009761609f, 0.008390335f, 0.007312526f, 0.0064472104f, 0.0057400377f};
    float z = t * t;
    float p = C[12];
    for (int i = 11; i >= 0; i--) p = std::fmaf(p, z, C[i]);
    return std::fmaf(t * z, p, t);
}
static inline float asin_(float x) {
    float a = std::fabs(x);
    if (!(a <= 1.0f)) return NAN;
    float r = a <= 0.5f ? asin_series(a) : 1.5707964f - 2.0f * asin_series(std::sqrt((1.0f - a) * 0.5f));
    return x < 0.0f ? -r : r;
}
static inline float pow_(float x, float y) {
    if (x > 0.0f) return exp_(y * log_(x));
    if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
    return NAN;
}
}  // namespace nm

static inline float mexp(float x) { return nm::exp_(x); }
static inline float mlog(float x) { return nm::log_(x); }
static inline float msin(float x) { return nm::sin_(x); }
static inline float mcos(float x) { return nm::cos_(x); }
static inline float masin(float x) { return nm::asin_(x); }
static inline float mpow(float x, float y) { return nm::pow_(x, y); }
static inline double mexp(double x) { return (std::exp)(x); }
static inline double mlog(double x) { return (std::log)(x); }
static inline double msin(double x) { return (std::sin)(x); }
static inline double mcos(double x) { return (std::cos)(x); }
static inline double masin(double x) { return (std::asin)(x); }
static inline double mpow(double x, double y) { return (std::pow)(x, y); }

// ---- constants (sim_defs.wgsl, fluid.wgsl, membrane.wgsl, air.wgsl, bullet.wgsl) ----------
enum { A_WC = 6, A_PC = 7, A_N = 8, A_MF = 9, A_MA = 10, A_BU = 11, A_SRC = 14, A_MW = 15, A_MV = 16, ACC_FIELDS = 19 };
enum { F_U = 0, F_P = 3, F_R = 4, F_Z = 5, F_D = 6, F_Q = 8, F_DIAG = 9, F_TYPE = 10, CELL_FIELDS = 11 };
enum { F_EXT = 4, F_EXT_SET = 7 };
static inline uint32_t a_mom(uint32_t d) { return 2 * d; }
static inline uint32_t a_wt(uint32_t d) { return 2 * d + 1; }
static const uint32_t TILE = 343;
static const uint32_t MAX_PATCHES = 576, N_SEC = 32, LOG_CAP = 256, OUTLINE = 33, HIT_FIELDS = 13;

template <class R>
struct K {
    static constexpr R GAS = R(0), WATER = R(1), SOLID = R(2), COVERED = R(3), RUBBER = R(4);
    static R FP_W() { return R(16777216.0); }
    static R FP_M() { return R(65536.0); }
    static R FP_P() { return R(65536.0); }
    static R FP_F() { return R(4194304.0); }
    static R FP_A() { return R(65536.0); }
    static R FP_Q() { return R(16777216.0); }
    static R FP_J() { return R(1073741824.0); }
    static R FP_L() { return R(68719476736.0); }
    static R FP_X() { return R(4096.0); }
    static R RHO_AIR() { return R(1.2); }
    static R MU_AIR() { return R(1.8e-5); }
    static R SIGMA_W() { return R(0.072); }
    static R PI() { return R(3.14159265358979); }
    static R GAMMA() { return R(1.4); }
    static R P_ATM() { return R(101325.0); }
    static R P_VAPOUR() { return R(2339.0); }
    static R RHO_ATM() { return R(1.204); }
    static R RHO_VAPOUR() { return R(0.0278); }
    static R P_FLOOR() { return P_VAPOUR() - P_ATM(); }
    static R CFL_AIR() { return R(0.9); }
    static R CONTACT() { return R(0.05); }
    static R MU_WATER() { return R(1.0e-3); }
    static R MU_JACKET() { return R(0.8); }
    static R LOGVINOVICH_K() { return R(2.0); }
    static R R_HAND() { return R(1.5); }
    static R CP_WAKE() { return R(-0.4); }
    static R CF_SKIN() { return R(0.003); }
    static R EVAPORATION() { return R(1.3e-10); }
    static R WE_CRIT() { return R(12.0); }
    static R BIG() { return R(3.0e38); }
};

template <class R>
struct Particle {
    V4<R> pos, vel, c0, c1, c2;
};
template <class R>
struct Gas {
    R rho;
    V3<R> m;
    R e;
};
template <class R>
struct Bullet {
    V4<R> x, v, q, l, shape, reach;
    uint32_t info[4];
};
template <class R>
struct Section {
    V4<R> a, b, c;
};
template <class R>
struct Spray {
    V4<R> pos, vel, air;
};
struct Tri {
    uint32_t v0, v1, v2;
    float rest_area;
    float dm_inv[4];
};

template <class R>
static inline V3<R> axis_weights(R fx) {
    return {R(0.5) * (R(1.5) - fx) * (R(1.5) - fx), R(0.75) - (fx - R(1.0)) * (fx - R(1.0)), R(0.5) * (fx - R(0.5)) * (fx - R(0.5))};
}

// ---- the simulation --------------------------------------------------------------------------
template <class R>
struct Sim {
    using Kc = K<R>;
    ntr_world_header hdr{};
    ntr_gpu_params U{};
    bool fp64_dots = true;

    // State (sim_defs.wgsl:24-58). Solver scalars are kept in double; in the FP32 mode they
    // hold exactly what the FP32 reference computes.
    struct St {
        uint32_t t_ns = 0, dt_ns = 0, step = 0, n_blocks = 0, n_blocks_prev = 0, overflow = 0, solve_iters = 0;
        uint32_t free_dt_ns = 0, iters_max = 0, unconverged = 0, spray_count = 0, mem_ticket = 0;
        R max_speed = 0, mem_dt = 0, cap_dt = 0, mem_dt_seen = 0, dt_flow = 0, air_dt = 0, air_dt_seen = 0;
        double rz = 0, alpha = 0, b_norm = 0, r_norm = 0, beta = 0;
        bool solver_on = false;
    } st;

    uint32_t Np = 0, Nv = 0, Nt = 0, cap_blocks = 0, cap_cells = 0, spray_cap = 0, wet_res = 0, n_shots = 0;
    uint32_t bd[3] = {0, 0, 0};
    std::vector<Particle<R>> P;
    // Sparse grid.
    std::vector<uint32_t> block_ptr, prev_ptr;
    std::vector<uint32_t> block_list, block_list_prev, block_nb, block_start, sorted, block_active;
    std::vector<uint32_t> slot_count;  // per block of this step
    std::vector<uint32_t> acc;         // i32 sums, wrapping, field-major
    std::vector<R> cf;
    std::vector<R> air[2];
    // Membrane.
    std::vector<V4<R>> mem_x[2], mem_v[2], mem_water, mem_layer;
    std::vector<V2<R>> mem_push;
    std::vector<R> mem_mass;
    std::vector<Tri> tris;
    std::vector<uint32_t> alive, vtri_off, vtri;
    std::vector<uint8_t> torn;  // triangles torn during the current rubber substep
    // Bullets.
    Bullet<R> bullets[4];
    std::vector<V4<R>> patches;  // p, n pairs
    std::vector<V2<R>> outline;
    std::vector<Section<R>> sections;
    int32_t bullet_hit[4 * 13];
    std::vector<V4<R>> pose_log;  // x, q, v per entry
    // Spray and ground.
    std::vector<Spray<R>> spray;
    std::vector<V4<R>> landed;
    std::vector<uint32_t> touch;

    // ---- helpers (sim_defs.wgsl:159-240) -------------------------------------------------
    R h() const { return R(U.origin[3]); }
    V3<R> origin() const { return {R(U.origin[0]), R(U.origin[1]), R(U.origin[2])}; }
    R dt() const { return R(st.dt_ns) * R(1e-9); }
    R now() const { return R(st.t_ns) * R(1e-9); }
    uint32_t block_slot(I3 b) const { return ((uint32_t)b.x * bd[1] + (uint32_t)b.y) * bd[2] + (uint32_t)b.z; }
    I3 slot_coord(uint32_t s) const { return {(int32_t)(s / (bd[2] * bd[1])), (int32_t)((s / bd[2]) % bd[1]), (int32_t)(s % bd[2])}; }
    static I3 local_coord(uint32_t i) {
        uint32_t l = i % 64u;
        return {(int32_t)(l / 16u), (int32_t)((l / 4u) % 4u), (int32_t)(l % 4u)};
    }
    I3 cell_coord(uint32_t i) const {
        I3 b = slot_coord(block_list[i / 64u]);
        return b * 4 + local_coord(i);
    }
    uint32_t neighbour(uint32_t cell, I3 off) const {
        I3 q = local_coord(cell) + off;
        I3 nb = {(q.x >= 4) - (q.x < 0), (q.y >= 4) - (q.y < 0), (q.z >= 4) - (q.z < 0)};
        uint32_t b = block_nb[(cell / 64u) * 27u + (uint32_t)((nb.x + 1) * 9 + (nb.y + 1) * 3 + nb.z + 1)];
        if (b == NONE) return NONE;
        I3 l = q - nb * 4;
        return b * 64u + (uint32_t)l.x * 16u + (uint32_t)l.y * 4u + (uint32_t)l.z;
    }
    size_t ai(uint32_t f, uint32_t cell) const { return (size_t)f * cap_cells + cell; }
    int32_t accv(uint32_t f, uint32_t cell) const { return (int32_t)acc[ai(f, cell)]; }
    void acc_add(uint32_t f, uint32_t cell, int32_t v) {
        uint32_t* p = &acc[ai(f, cell)];
#pragma omp atomic
        *p += (uint32_t)v;
    }
    R& cfr(uint32_t f, uint32_t cell) { return cf[ai(f, cell)]; }
    R cfv(uint32_t f, uint32_t cell) const { return cf[ai(f, cell)]; }
    R cell_type(uint32_t cell) const { return cell == NONE ? Kc::GAS : cf[ai(F_TYPE, cell)]; }
    static V3<R> lattice_offset(uint32_t d) {
        V3<R> o = {R(0.5), R(0.5), R(0.5)};
        if (d < 3) o[d] = R(0);
        return o;
    }
    I3 own_cell(V3<R> p) const { return vi(vfloor((p - origin()) / h())); }
    bool in_domain_block(I3 b) const {
        return b.x >= 0 && b.y >= 0 && b.z >= 0 && (uint32_t)b.x < bd[0] && (uint32_t)b.y < bd[1] && (uint32_t)b.z < bd[2];
    }
    uint32_t cell_at(I3 c) const {
        if (c.x < 0 || c.y < 0 || c.z < 0 || (uint32_t)c.x >= U.dims[0] || (uint32_t)c.y >= U.dims[1] || (uint32_t)c.z >= U.dims[2]) return NONE;
        uint32_t b = block_ptr[block_slot(shr2(c))];
        if (b == NONE) return NONE;
        I3 l = {c.x & 3, c.y & 3, c.z & 3};
        return b * 64u + (uint32_t)l.x * 16u + (uint32_t)l.y * 4u + (uint32_t)l.z;
    }
    void ground_touch(V3<R> p) {
        R hw = R(U.wet[0]);
        uint32_t res = U.limits[0];
        R ux = (p.x + hw) / (R(2) * hw), uz = (p.z + hw) / (R(2) * hw);
        if (ux < R(0) || uz < R(0) || ux >= R(1) || uz >= R(1)) return;
        uint32_t cx = f2u(ux * R(res)), cz = f2u(uz * R(res));
        uint32_t t = fbits((float)now());
        uint32_t* q = &touch[(size_t)cz * res + cx];
        // atomicMin on the bits of a non-negative time.
#pragma omp critical(touch)
        {
            if (t < *q) *q = t;
        }
    }
    static R rnd(uint32_t& seed) {
        seed = pcg(seed);
        return R(seed >> 8u) * (R(1) / R(16777216.0));
    }
    static R rnd_gauss(uint32_t& seed) {
        R u1 = mx(rnd(seed), R(1e-7));
        R u2 = rnd(seed);
        return std::sqrt(R(-2) * mlog(u1)) * mcos(R(2) * Kc::PI() * u2);
    }
    uint32_t n_blocks() const { return std::min(st.n_blocks, U.bdims[3]); }

    // ---- load / save ---------------------------------------------------------------------
    bool load(const void* blob, size_t len, std::string& err);
    std::vector<uint8_t> save() const;

    // ---- kernels ---------------------------------------------------------------------------
    void begin_step();
    void clear_blocks();
    void claim(I3 b, std::vector<uint8_t>& claimed, std::vector<uint32_t>& list);
    void activate_blocks();  // keep_blocks, mark_blocks, mark_rubber, blocks_ready, scan, sort
    void p2g();
    void air_carry();
    void mem_splat();
    void grid_prep();
    void air_fill();
    void bullet_step();
    void bullet_apply();
    void solve();
    void project();
    void extend();
    void mem_sample();
    void mem_substep(uint32_t k, int par);
    void air_substep(int par);
    void spray_update();
    void g2p();
    void run_step();
    void measure_rubber();
    void run_batch(uint32_t n, uint32_t stop);

    // pieces
    R face_u(uint32_t cell, uint32_t lo, uint32_t d) const {
        if (cell == NONE) return R(0);
        return bounded(cfv(F_U + d, cell), cfv(F_TYPE, cell), cell_type(lo));
    }
    static R bounded(R u, R hi, R lo) {
        if (lo == Kc::SOLID && hi == Kc::SOLID) return R(0);
        if (lo == Kc::SOLID) return mx(u, R(0));
        if (hi == Kc::SOLID) return mn(u, R(0));
        return u;
    }
    R pressure_of(uint32_t cell) const {
        if (cell == NONE) return R(0);
        R p = cfv(F_P, cell);
        return cfv(F_TYPE, cell) == Kc::WATER ? mx(p, Kc::P_FLOOR()) : p;
    }
    bool on_water(uint32_t i) const { return mem_mass[i] > R(0) && mem_water[i].w >= Kc::CONTACT(); }
    V2<R> sample_grid(V3<R> x, uint32_t fu, uint32_t fw) const;
    V2<R> sample_pressure(V3<R> x, bool gas_only) const;
    Gas<R> read_gas(int buf, uint32_t cell) const {
        const auto& a = air[buf];
        return {a[ai(0, cell)], {a[ai(1, cell)], a[ai(2, cell)], a[ai(3, cell)]}, a[ai(4, cell)]};
    }
    void write_gas(int buf, uint32_t cell, const Gas<R>& g) {
        auto& a = air[buf];
        a[ai(0, cell)] = g.rho;
        a[ai(1, cell)] = g.m.x;
        a[ai(2, cell)] = g.m.y;
        a[ai(3, cell)] = g.m.z;
        a[ai(4, cell)] = g.e;
    }
    static Gas<R> gas_at_rest(R rho, R p) { return {rho, {R(0), R(0), R(0)}, p / (Kc::GAMMA() - R(1))}; }
    static Gas<R> ambient() { return gas_at_rest(Kc::RHO_ATM(), Kc::P_ATM()); }
    static Gas<R> no_gas() { return {R(0), {R(0), R(0), R(0)}, R(0)}; }
    static R gas_p(const Gas<R>& g) { return (Kc::GAMMA() - R(1)) * (g.e - R(0.5) * dot(g.m, g.m) / g.rho); }
    static Gas<R> floored(Gas<R> o) {
        o.rho = mx(o.rho, Kc::RHO_VAPOUR());
        o.e = mx(o.e, Kc::P_VAPOUR() / (Kc::GAMMA() - R(1)) + R(0.5) * dot(o.m, o.m) / o.rho);
        return o;
    }
    bool free_gas(uint32_t cell) const { return cell == NONE || cfv(F_TYPE, cell) == Kc::GAS; }
    Gas<R> hll(const Gas<R>& l, const Gas<R>& r, uint32_t d) const;
    Gas<R> across(int buf, uint32_t cell, const Gas<R>& own, uint32_t d, bool hi) const;
    R gas_pressure_at(int buf, V3<R> x) const;
    struct VertexForce {
        V3<R> f, n;
        R area, stiff, tension, reach, thick;
        uint64_t torn;  // bit j: the vertex's j-th triangle tore in this substep
    };
    struct Sheet {
        V2<R> sig;
        R tangent;
    };
    Sheet sheet(R major, R minor) const;
    VertexForce vertex_force(int par, uint32_t i);
    V2<R> substep_one(int par, uint32_t i, uint32_t k);
    R rubber_contact(int par, uint32_t i, V3<R>& x, V3<R>& v, R m, V3<R> load, const VertexForce& vf, bool wet, bool& held, R t, R sub);
    struct Near {
        V2<R> at, n;
        R depth;
    };
    Near nearest_surface(uint32_t bi, V2<R> q) const;
    bool in_cavity(uint32_t b, V3<R> p, R t) const;
    void push_water(V3<R> x, uint32_t d, R j, R sw);
    R section_r2(const Section<R>& s, R t) const { return s.c.x + s.b.w * mx(t - s.a.w, R(0)); }
    void carve(V3<R>& x, V3<R>& v, uint32_t id) const;
    struct Gathered {
        R s;
        V3<R> g;
        R w;
    };
    uint32_t tile_cell(const uint32_t* links, uint32_t t) const {
        I3 rel = {(int32_t)(t / 49u) - 1, (int32_t)((t / 7u) % 7u) - 1, (int32_t)(t % 7u) - 1};
        I3 nb = {(rel.x + 4) / 4 - 1, (rel.y + 4) / 4 - 1, (rel.z + 4) / 4 - 1};
        uint32_t b = links[(uint32_t)((nb.x + 1) * 9 + (nb.y + 1) * 3 + nb.z + 1)];
        if (b == NONE) return NONE;
        I3 l = rel - nb * 4;
        return b * 64u + (uint32_t)l.x * 16u + (uint32_t)l.y * 4u + (uint32_t)l.z;
    }
    // Canonical spray emission: g2p records (block, rank) of each break-up, emitted after.
    struct Breakup {
        V3<R> x, v;
        uint32_t id;
    };
};

// ---- load / save --------------------------------------------------------------------------
template <class R>
static inline V4<R> ld4(const float* f) { return {R(f[0]), R(f[1]), R(f[2]), R(f[3])}; }
template <class R>
static inline void st4(float* f, const V4<R>& v) {
    f[0] = (float)v.x, f[1] = (float)v.y, f[2] = (float)v.z, f[3] = (float)v.w;
}

static size_t sec_elem(const ntr_world_header& h, int s, size_t* count) {
    size_t cp = (size_t)h.n_blocks_prev * 64;
    size_t e = 0, c = 0;
    switch (s) {
        case NTR_SEC_PARTICLES: e = 80, c = h.n_particles; break;
        case NTR_SEC_MEM_X: case NTR_SEC_MEM_V: case NTR_SEC_MEM_WATER: e = 16, c = h.n_verts; break;
        case NTR_SEC_MEM_MASS: e = 4, c = h.n_verts; break;
        case NTR_SEC_MEM_LAYER: e = 96, c = h.n_verts; break;
        case NTR_SEC_MEM_PUSH: e = 8, c = h.n_verts; break;
        case NTR_SEC_TRIS: e = 32, c = h.n_tris; break;
        case NTR_SEC_ALIVE: e = 4, c = h.n_tris; break;
        case NTR_SEC_VTRI_OFF: e = 4, c = (size_t)h.n_verts + 1; break;
        case NTR_SEC_VTRI: e = 4, c = h.n_vtri; break;
        case NTR_SEC_BULLETS: e = 112, c = 4; break;
        case NTR_SEC_PATCHES: e = 32, c = 4 * MAX_PATCHES; break;
        case NTR_SEC_OUTLINES: e = 8, c = 4 * OUTLINE; break;
        case NTR_SEC_SECTIONS: e = 48, c = 4 * N_SEC; break;
        case NTR_SEC_BULLET_HIT: e = 4, c = 4 * HIT_FIELDS; break;
        case NTR_SEC_POSE_LOG: e = 48, c = 4 * LOG_CAP; break;
        case NTR_SEC_BLOCKS_PREV: case NTR_SEC_BLOCK_ACTIVE: e = 4, c = h.n_blocks_prev; break;
        case NTR_SEC_AIR: e = 4, c = 5 * cp; break;
        case NTR_SEC_SPRAY: e = 48, c = h.n_spray; break;
        case NTR_SEC_LANDED: e = 16, c = h.n_spray; break;
        case NTR_SEC_TOUCH: e = 4, c = (size_t)h.wet_res * h.wet_res; break;
    }
    *count = c;
    return e;
}

template <class R>
bool Sim<R>::load(const void* blob, size_t len, std::string& err) {
    if (len < sizeof(ntr_world_header)) {
        err = "short blob";
        return false;
    }
    std::memcpy(&hdr, blob, sizeof hdr);
    if (hdr.magic != NTR_WORLD_MAGIC || hdr.version != NTR_WORLD_VERSION) {
        err = "bad magic";
        return false;
    }
    const uint8_t* b = (const uint8_t*)blob;
    for (int s = 0; s < NTR_SEC_COUNT; s++) {
        size_t c, e = sec_elem(hdr, s, &c);
        if (hdr.bytes[s] != e * c || hdr.offset[s] + hdr.bytes[s] > len) {
            err = "bad section " + std::to_string(s);
            return false;
        }
    }
    auto sec = [&](int s) { return (const float*)(b + hdr.offset[s]); };
    auto secu = [&](int s) { return (const uint32_t*)(b + hdr.offset[s]); };
    U = hdr.params;
    Np = hdr.n_particles, Nv = hdr.n_verts, Nt = hdr.n_tris;
    cap_blocks = hdr.block_cap, cap_cells = cap_blocks * 64, spray_cap = hdr.spray_cap, wet_res = hdr.wet_res;
    n_shots = hdr.n_shots;
    bd[0] = U.bdims[0], bd[1] = U.bdims[1], bd[2] = U.bdims[2];
    const ntr_state& s0 = hdr.state;
    st.t_ns = s0.t_ns, st.dt_ns = s0.dt_ns, st.step = s0.step, st.n_blocks = s0.n_blocks;
    st.n_blocks_prev = s0.n_blocks_prev, st.overflow = s0.overflow, st.solve_iters = s0.solve_iters;
    st.free_dt_ns = s0.free_dt_ns, st.iters_max = s0.iters_max, st.unconverged = s0.unconverged;
    st.spray_count = s0.spray_count, st.mem_ticket = s0.mem_ticket;
    st.max_speed = R(s0.max_speed), st.mem_dt = R(s0.mem_dt), st.cap_dt = R(s0.cap_dt);
    st.mem_dt_seen = R(s0.mem_dt_seen), st.dt_flow = R(s0.dt_flow), st.air_dt = R(s0.air_dt), st.air_dt_seen = R(s0.air_dt_seen);
    st.rz = s0.rz, st.alpha = s0.alpha, st.b_norm = s0.b_norm, st.r_norm = s0.r_norm, st.beta = s0.beta;

    P.resize(Np);
    const float* pp = sec(NTR_SEC_PARTICLES);
    for (uint32_t i = 0; i < Np; i++) {
        const float* a = pp + (size_t)i * 20;
        P[i] = {ld4<R>(a), ld4<R>(a + 4), ld4<R>(a + 8), ld4<R>(a + 12), ld4<R>(a + 16)};
    }
    for (int k = 0; k < 2; k++) {
        mem_x[k].resize(Nv);
        mem_v[k].resize(Nv);
    }
    mem_water.resize(Nv);
    mem_layer.resize((size_t)Nv * 6);
    mem_push.resize(Nv);
    mem_mass.resize(Nv);
    for (uint32_t i = 0; i < Nv; i++) {
        mem_x[0][i] = ld4<R>(sec(NTR_SEC_MEM_X) + 4 * i);
        mem_v[0][i] = ld4<R>(sec(NTR_SEC_MEM_V) + 4 * i);
        mem_x[1][i] = mem_x[0][i];
        mem_v[1][i] = mem_v[0][i];
        mem_water[i] = ld4<R>(sec(NTR_SEC_MEM_WATER) + 4 * i);
        mem_mass[i] = R(sec(NTR_SEC_MEM_MASS)[i]);
        mem_push[i] = {R(sec(NTR_SEC_MEM_PUSH)[2 * i]), R(sec(NTR_SEC_MEM_PUSH)[2 * i + 1])};
        for (int j = 0; j < 6; j++) mem_layer[(size_t)i * 6 + j] = ld4<R>(sec(NTR_SEC_MEM_LAYER) + 24 * (size_t)i + 4 * j);
    }
    tris.resize(Nt);
    std::memcpy(tris.data(), b + hdr.offset[NTR_SEC_TRIS], (size_t)Nt * 32);
    alive.assign(secu(NTR_SEC_ALIVE), secu(NTR_SEC_ALIVE) + Nt);
    torn.assign(Nt, 0u);
    vtri_off.assign(secu(NTR_SEC_VTRI_OFF), secu(NTR_SEC_VTRI_OFF) + Nv + 1);
    vtri.assign(secu(NTR_SEC_VTRI), secu(NTR_SEC_VTRI) + hdr.n_vtri);
    const float* bf = sec(NTR_SEC_BULLETS);
    for (int k = 0; k < 4; k++) {
        const float* q = bf + 28 * k;
        bullets[k].x = ld4<R>(q), bullets[k].v = ld4<R>(q + 4), bullets[k].q = ld4<R>(q + 8);
        bullets[k].l = ld4<R>(q + 12), bullets[k].shape = ld4<R>(q + 16), bullets[k].reach = ld4<R>(q + 20);
        std::memcpy(bullets[k].info, q + 24, 16);
    }
    patches.resize(4 * MAX_PATCHES * 2);
    for (size_t i = 0; i < patches.size(); i++) patches[i] = ld4<R>(sec(NTR_SEC_PATCHES) + 4 * i);
    outline.resize(4 * OUTLINE);
    for (size_t i = 0; i < outline.size(); i++) outline[i] = {R(sec(NTR_SEC_OUTLINES)[2 * i]), R(sec(NTR_SEC_OUTLINES)[2 * i + 1])};
    sections.resize(4 * N_SEC);
    for (size_t i = 0; i < sections.size(); i++) {
        const float* q = sec(NTR_SEC_SECTIONS) + 12 * i;
        sections[i] = {ld4<R>(q), ld4<R>(q + 4), ld4<R>(q + 8)};
    }
    std::memcpy(bullet_hit, b + hdr.offset[NTR_SEC_BULLET_HIT], sizeof bullet_hit);
    pose_log.resize(4 * LOG_CAP * 3);
    for (size_t i = 0; i < pose_log.size(); i++) pose_log[i] = ld4<R>(sec(NTR_SEC_POSE_LOG) + 4 * i);

    size_t slots = (size_t)bd[0] * bd[1] * bd[2];
    block_ptr.assign(slots, NONE);
    prev_ptr.assign(slots, NONE);
    acc.assign((size_t)ACC_FIELDS * cap_cells, 0u);
    cf.assign((size_t)CELL_FIELDS * cap_cells, R(0));
    air[0].assign((size_t)5 * cap_cells, R(0));
    air[1].assign((size_t)5 * cap_cells, R(0));
    block_list.assign(cap_blocks, 0);
    block_list_prev.assign(cap_blocks, 0);
    block_active.assign(cap_blocks, 0);
    block_nb.assign((size_t)cap_blocks * 27, NONE);
    block_start.assign((size_t)cap_blocks + 1, 0);
    slot_count.assign(cap_blocks, 0);
    sorted.assign(Np, 0);
    // The last step's blocks are this state's "current" ones; begin_step moves them to prev.
    uint32_t nbp = hdr.n_blocks_prev;
    st.n_blocks = nbp;
    const uint32_t* bp = secu(NTR_SEC_BLOCKS_PREV);
    const uint32_t* ba = secu(NTR_SEC_BLOCK_ACTIVE);
    const float* af = sec(NTR_SEC_AIR);
    for (uint32_t i = 0; i < nbp; i++) {
        block_list[i] = bp[i];
        block_ptr[bp[i]] = i;
        block_active[i] = ba[i];
    }
    for (uint32_t f = 0; f < 5; f++)
        for (size_t c = 0; c < (size_t)nbp * 64; c++) air[0][ai(f, (uint32_t)c)] = R(af[f * (size_t)nbp * 64 + c]);
    spray.assign(spray_cap, Spray<R>{});
    landed.assign(spray_cap, V4<R>{});
    for (uint32_t i = 0; i < hdr.n_spray; i++) {
        const float* q = sec(NTR_SEC_SPRAY) + 12 * (size_t)i;
        spray[i] = {ld4<R>(q), ld4<R>(q + 4), ld4<R>(q + 8)};
        landed[i] = ld4<R>(sec(NTR_SEC_LANDED) + 4 * (size_t)i);
    }
    touch.assign(secu(NTR_SEC_TOUCH), secu(NTR_SEC_TOUCH) + (size_t)wet_res * wet_res);
    return true;
}

template <class R>
std::vector<uint8_t> Sim<R>::save() const {
    ntr_world_header h = hdr;
    h.params = U;
    ntr_state& s = h.state;
    s.t_ns = st.t_ns, s.dt_ns = st.dt_ns, s.step = st.step, s.n_blocks = st.n_blocks;
    s.max_speed = (float)st.max_speed, s.n_blocks_prev = st.n_blocks_prev, s.overflow = st.overflow;
    s.solve_iters = st.solve_iters, s.rz = (float)st.rz, s.alpha = (float)st.alpha, s.b_norm = (float)st.b_norm;
    s.r_norm = (float)st.r_norm, s.free_dt_ns = st.free_dt_ns, s.iters_max = st.iters_max, s.unconverged = st.unconverged;
    s.beta = (float)st.beta, s.spray_count = st.spray_count, s.mem_dt = (float)st.mem_dt, s.cap_dt = (float)st.cap_dt;
    s.mem_dt_seen = (float)st.mem_dt_seen, s.dt_flow = (float)st.dt_flow, s.air_dt = (float)st.air_dt;
    s.air_dt_seen = (float)st.air_dt_seen, s.mem_ticket = st.mem_ticket;
    uint32_t nb = n_blocks();
    h.n_blocks_prev = nb;
    h.n_spray = std::min(st.spray_count, spray_cap);
    size_t off = (sizeof(ntr_world_header) + 255) & ~size_t(255);
    for (int k = 0; k < NTR_SEC_COUNT; k++) {
        size_t c, e = sec_elem(h, k, &c);
        h.offset[k] = off;
        h.bytes[k] = e * c;
        off += (e * c + 255) & ~size_t(255);
    }
    std::vector<uint8_t> out(off, 0);
    auto fp = [&](int k) { return (float*)(out.data() + h.offset[k]); };
    auto up = [&](int k) { return (uint32_t*)(out.data() + h.offset[k]); };
    for (uint32_t i = 0; i < Np; i++) {
        float* a = fp(NTR_SEC_PARTICLES) + (size_t)i * 20;
        st4(a, P[i].pos), st4(a + 4, P[i].vel), st4(a + 8, P[i].c0), st4(a + 12, P[i].c1), st4(a + 16, P[i].c2);
    }
    for (uint32_t i = 0; i < Nv; i++) {
        st4(fp(NTR_SEC_MEM_X) + 4 * i, mem_x[0][i]);
        st4(fp(NTR_SEC_MEM_V) + 4 * i, mem_v[0][i]);
        st4(fp(NTR_SEC_MEM_WATER) + 4 * i, mem_water[i]);
        fp(NTR_SEC_MEM_MASS)[i] = (float)mem_mass[i];
        fp(NTR_SEC_MEM_PUSH)[2 * i] = (float)mem_push[i].x;
        fp(NTR_SEC_MEM_PUSH)[2 * i + 1] = (float)mem_push[i].y;
        for (int j = 0; j < 6; j++) st4(fp(NTR_SEC_MEM_LAYER) + 24 * (size_t)i + 4 * j, mem_layer[(size_t)i * 6 + j]);
    }
    std::memcpy(out.data() + h.offset[NTR_SEC_TRIS], tris.data(), (size_t)Nt * 32);
    std::memcpy(up(NTR_SEC_ALIVE), alive.data(), (size_t)Nt * 4);
    std::memcpy(up(NTR_SEC_VTRI_OFF), vtri_off.data(), ((size_t)Nv + 1) * 4);
    std::memcpy(up(NTR_SEC_VTRI), vtri.data(), vtri.size() * 4);
    for (int k = 0; k < 4; k++) {
        float* q = fp(NTR_SEC_BULLETS) + 28 * k;
        st4(q, bullets[k].x), st4(q + 4, bullets[k].v), st4(q + 8, bullets[k].q), st4(q + 12, bullets[k].l);
        st4(q + 16, bullets[k].shape), st4(q + 20, bullets[k].reach);
        std::memcpy(q + 24, bullets[k].info, 16);
    }
    for (size_t i = 0; i < patches.size(); i++) st4(fp(NTR_SEC_PATCHES) + 4 * i, patches[i]);
    for (size_t i = 0; i < outline.size(); i++) {
        fp(NTR_SEC_OUTLINES)[2 * i] = (float)outline[i].x;
        fp(NTR_SEC_OUTLINES)[2 * i + 1] = (float)outline[i].y;
    }
    for (size_t i = 0; i < sections.size(); i++) {
        float* q = fp(NTR_SEC_SECTIONS) + 12 * i;
        st4(q, sections[i].a), st4(q + 4, sections[i].b), st4(q + 8, sections[i].c);
    }
    std::memcpy(out.data() + h.offset[NTR_SEC_BULLET_HIT], bullet_hit, sizeof bullet_hit);
    for (size_t i = 0; i < pose_log.size(); i++) st4(fp(NTR_SEC_POSE_LOG) + 4 * i, pose_log[i]);
    for (uint32_t i = 0; i < nb; i++) {
        up(NTR_SEC_BLOCKS_PREV)[i] = block_list[i];
        up(NTR_SEC_BLOCK_ACTIVE)[i] = block_active[i];
    }
    for (uint32_t f = 0; f < 5; f++)
        for (size_t c = 0; c < (size_t)nb * 64; c++) fp(NTR_SEC_AIR)[f * (size_t)nb * 64 + c] = (float)air[0][ai(f, (uint32_t)c)];
    for (uint32_t i = 0; i < h.n_spray; i++) {
        float* q = fp(NTR_SEC_SPRAY) + 12 * (size_t)i;
        st4(q, spray[i].pos), st4(q + 4, spray[i].vel), st4(q + 8, spray[i].air);
        st4(fp(NTR_SEC_LANDED) + 4 * (size_t)i, landed[i]);
    }
    std::memcpy(up(NTR_SEC_TOUCH), touch.data(), touch.size() * 4);
    std::memcpy(out.data(), &h, sizeof h);
    return out;
}

// ---- begin_step, fluid.wgsl:33-89 -----------------------------------------------------------
template <class R>
void Sim<R>::begin_step() {
    R vmax = st.max_speed;
    uint32_t arrive = U.limits[3];
    for (uint32_t k = 0; k < U.mem[3]; k++) {
        const Bullet<R>& b = bullets[k];
        if (b.info[2] == 1u) {
            vmax = mx(vmax, b.l.w);
        } else if (b.info[2] == 0u) {
            if (b.info[0] > st.t_ns)
                arrive = std::min(arrive, b.info[0]);
            else
                vmax = mx(vmax, length(b.v.xyz()));
        }
    }
    R mem_dt = st.mem_dt, air_dt = st.air_dt;
    R dt_s = mn(R(U.fluid[2]), st.cap_dt);
    if (vmax > R(0)) dt_s = mn(dt_s, R(U.fluid[1]) * h() / vmax);
    st.dt_flow = dt_s;
    st.mem_dt_seen = mem_dt;
    st.air_dt_seen = air_dt;
    dt_s = mn(dt_s, mn(R(U.mem[1]) * mem_dt, R(U.mem[2]) * air_dt));
    if (st.free_dt_ns > 0u) dt_s = mn(dt_s, R(1.25) * R(st.free_dt_ns) * R(1e-9));
    uint32_t free_ns = std::max(f2u(dt_s * R(1e9)), 20u);
    uint32_t stop = U.limits[3];
    bool live = st.t_ns < stop;
    uint32_t dt_ns = 0;
    if (live) {
        dt_ns = std::min(free_ns, std::min(stop, arrive) - st.t_ns);
        st.free_dt_ns = free_ns;
        st.t_ns += dt_ns;
        st.step += 1;
        st.max_speed = R(0);
        st.mem_dt = R(3.4028234663852886e38);
        st.cap_dt = R(3.4028234663852886e38);
        st.air_dt = R(3.4028234663852886e38);
        st.mem_ticket = 0;
        st.n_blocks_prev = n_blocks();
        st.n_blocks = 0;
    }
    st.dt_ns = dt_ns;
}

// ---- block activation, fluid.wgsl:93-196, membrane.wgsl:164-180, air.wgsl:271-277 ---------
template <class R>
void Sim<R>::clear_blocks() {
    uint32_t n = st.n_blocks_prev;
    for (uint32_t b = 0; b < n; b++) {
        uint32_t s = block_list[b];
        block_ptr[s] = NONE;
        block_list_prev[b] = s;
        prev_ptr[s] = b;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n * 64; i++)
        for (uint32_t f = 0; f < ACC_FIELDS; f++) acc[ai(f, (uint32_t)i)] = 0;
}

template <class R>
void Sim<R>::claim(I3 b, std::vector<uint8_t>& claimed, std::vector<uint32_t>& list) {
    uint32_t s = block_slot(b);
    if (!claimed[s]) {
        claimed[s] = 1;
        list.push_back(s);
    }
}

template <class R>
void Sim<R>::activate_blocks() {
    // Claims: the union of every particle's transfer stencil (cells floor(x) - 1 .. + 2), the
    // blocks around rubber off the water (cells - 2 .. + 3), and the blocks whose air was active.
    size_t slots = (size_t)bd[0] * bd[1] * bd[2];
    std::vector<uint8_t> claimed(slots, 0);
    std::vector<uint32_t> list;
    I3 bmax = {(int32_t)bd[0] - 1, (int32_t)bd[1] - 1, (int32_t)bd[2] - 1};
    auto clampi = [](int32_t v, int32_t lo, int32_t hi) { return std::min(std::max(v, lo), hi); };
    auto claim_range = [&](I3 lo_c, I3 hi_c) {
        I3 lo = shr2(lo_c), hi = shr2(hi_c);
        lo = {clampi(lo.x, 0, bmax.x), clampi(lo.y, 0, bmax.y), clampi(lo.z, 0, bmax.z)};
        hi = {clampi(hi.x, 0, bmax.x), clampi(hi.y, 0, bmax.y), clampi(hi.z, 0, bmax.z)};
        for (int32_t x = lo.x; x <= hi.x; x++)
            for (int32_t y = lo.y; y <= hi.y; y++)
                for (int32_t z = lo.z; z <= hi.z; z++) claim({x, y, z}, claimed, list);
    };
    if (st.dt_ns > 0) {
        // keep_blocks
        for (uint32_t i = 0; i < st.n_blocks_prev; i++)
            if (block_active[i] != 0) claim(slot_coord(block_list_prev[i]), claimed, list);
        // mark_blocks
        for (uint32_t i = 0; i < Np; i++) {
            if (P[i].vel.w < R(0.5)) continue;
            I3 c = own_cell(P[i].pos.xyz());
            claim_range(c - I3{1, 1, 1}, c + I3{2, 2, 2});
        }
        // mark_rubber
        for (uint32_t i = 0; i < Nv; i++) {
            if (mem_push[i].y <= R(0) || on_water(i)) continue;
            I3 c = own_cell(mem_x[0][i].xyz());
            claim_range(c - I3{2, 2, 2}, c + I3{3, 3, 3});
        }
    }
    std::sort(list.begin(), list.end());
    uint32_t n = (uint32_t)list.size();
    st.n_blocks = n;
    if (n > U.bdims[3]) {
        st.overflow = 1;
        n = U.bdims[3];
    }
    for (uint32_t b = 0; b < n; b++) {
        block_list[b] = list[b];
        block_ptr[list[b]] = b;
    }
    // Counting sort by block, particles in index order within a block.
    std::fill(slot_count.begin(), slot_count.begin() + n, 0u);
    std::vector<uint32_t> key(Np, NONE);
    if (st.dt_ns > 0) {
        for (uint32_t i = 0; i < Np; i++) {
            if (P[i].vel.w < R(0.5)) continue;
            I3 c = own_cell(P[i].pos.xyz());
            I3 b = shr2(c);
            if (!in_domain_block(b)) continue;
            uint32_t bi = block_ptr[block_slot(b)];
            if (bi == NONE) continue;
            key[i] = bi;
            slot_count[bi]++;
        }
    }
    uint32_t run = 0;
    for (uint32_t b = 0; b < n; b++) {
        block_start[b] = run;
        run += slot_count[b];
    }
    block_start[n] = run;
    std::vector<uint32_t> fillp(block_start.begin(), block_start.begin() + n);
    for (uint32_t i = 0; i < Np; i++)
        if (key[i] != NONE) sorted[fillp[key[i]]++] = i;
}

// ---- p2g, fluid.wgsl:198-303 -------------------------------------------------------------------
template <class R>
void Sim<R>::p2g() {
    const uint32_t n = n_blocks();
    const R hh = h();
    const V3<R> org = origin();
#pragma omp parallel
    {
        std::vector<uint32_t> tile(8 * TILE);
#pragma omp for schedule(dynamic, 8)
        for (int64_t bb = 0; bb < (int64_t)n; bb++) {
            uint32_t b = (uint32_t)bb;
            I3 bc = slot_coord(block_list[b]);
            uint32_t links[27];
            for (uint32_t li = 0; li < 27; li++) {
                I3 nb = bc + I3{(int32_t)(li / 9u), (int32_t)((li / 3u) % 3u), (int32_t)(li % 3u)} - I3{1, 1, 1};
                uint32_t idx = NONE;
                if (in_domain_block(nb)) idx = block_ptr[block_slot(nb)];
                links[li] = idx;
                block_nb[(size_t)b * 27 + li] = idx;
            }
            uint32_t count = block_start[b + 1] - block_start[b];
            if (count == 0) {
                for (uint32_t li = 0; li < 64; li++) acc[ai(A_N, b * 64 + li)] = 0;
                continue;
            }
            std::fill(tile.begin(), tile.end(), 0u);
            uint32_t own[64] = {0};
            I3 corner = bc * 4 - I3{1, 1, 1};
            uint32_t first = block_start[b];
            for (uint32_t k = 0; k < count; k++) {
                const Particle<R>& p = P[sorted[first + k]];
                V3<R> x = (p.pos.xyz() - org) / hh;
                auto splat = [&](V3<R> o, uint32_t fa, R val, V3<R> grad, uint32_t fw, R scale) {
                    I3 base = vi(vfloor(x - o - R(0.5)));
                    V3<R> fx = x - o - vf<R>(base);
                    V3<R> wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
                    I3 t = base - corner;
                    uint32_t t0 = (uint32_t)t.x * 49u + (uint32_t)t.y * 7u + (uint32_t)t.z;
                    V3<R> hg = grad * hh;
                    for (uint32_t a = 0; a < 3; a++)
                        for (uint32_t bq = 0; bq < 3; bq++)
                            for (uint32_t c = 0; c < 3; c++) {
                                R weight = wx[a] * wy[bq] * wz[c];
                                uint32_t tt = t0 + a * 49u + bq * 7u + c;
                                R node = val + dot(hg, v3(R(a), R(bq), R(c)) - fx);
                                tile[fa * TILE + tt] += (uint32_t)to_fp(weight * node, scale);
                                tile[fw * TILE + tt] += (uint32_t)to_fp(weight, Kc::FP_W());
                            }
                };
                splat({R(0), R(0.5), R(0.5)}, a_mom(0), p.vel.x, p.c0.xyz(), a_wt(0), Kc::FP_M());
                splat({R(0.5), R(0), R(0.5)}, a_mom(1), p.vel.y, p.c1.xyz(), a_wt(1), Kc::FP_M());
                splat({R(0.5), R(0.5), R(0)}, a_mom(2), p.vel.z, p.c2.xyz(), a_wt(2), Kc::FP_M());
                splat({R(0.5), R(0.5), R(0.5)}, A_PC, p.c0.w * R(1e-6), {R(0), R(0), R(0)}, A_WC, Kc::FP_P());
                I3 l = own_cell(p.pos.xyz()) - bc * 4;
                own[l.x * 16 + l.y * 4 + l.z]++;
            }
            for (uint32_t t = 0; t < TILE; t++) {
                uint32_t cell = tile_cell(links, t);
                if (cell == NONE) continue;
                for (uint32_t f = 0; f < 8; f++) {
                    uint32_t v = tile[f * TILE + t];
                    if (v != 0) acc_add(f, cell, (int32_t)v);
                }
            }
            for (uint32_t li = 0; li < 64; li++) acc[ai(A_N, b * 64 + li)] = own[li];
        }
    }
}

// ---- air_carry, air.wgsl:85-99 ------------------------------------------------------------------
template <class R>
void Sim<R>::air_carry() {
    const uint32_t n = n_blocks();
#pragma omp parallel for schedule(static)
    for (int64_t bb = 0; bb < (int64_t)n; bb++) {
        uint32_t b = (uint32_t)bb;
        uint32_t s = block_list[b];
        uint32_t o = prev_ptr[s];
        bool carried = o < st.n_blocks_prev && block_list_prev[o] == s;
        for (uint32_t li = 0; li < 64; li++) {
            Gas<R> g = ambient();
            if (carried) g = read_gas(0, o * 64 + li);
            write_gas(1, b * 64 + li, g);
        }
        block_active[b] = 0;
    }
}

// ---- mem_splat, membrane.wgsl:182-217 -------------------------------------------------------------
template <class R>
void Sim<R>::mem_splat() {
    const R hh = h();
    const V3<R> org = origin();
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)Nv; ii++) {
        uint32_t i = (uint32_t)ii;
        if (mem_mass[i] == R(0)) continue;
        V2<R> pa = mem_push[i];
        if (pa.y <= R(0)) continue;
        uint32_t own = cell_at(own_cell(mem_x[0][i].xyz()));
        if (own != NONE) {
            R a = pa.y * R(1e6);
            acc_add(A_MW, own, to_fp(a, Kc::FP_A()));
            V3<R> mv = mem_v[0][i].xyz();
            for (uint32_t d = 0; d < 3; d++) acc_add(A_MV + d, own, to_fp(a * mv[d], Kc::FP_A()));
        }
        if (!on_water(i)) continue;
        V3<R> x = (mem_x[0][i].xyz() - org) / hh - R(0.5);
        I3 base = vi(vfloor(x - R(0.5)));
        V3<R> fx = x - vf<R>(base);
        V3<R> wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                for (int c = 0; c < 3; c++) {
                    uint32_t cell = cell_at(base + I3{a, b, c});
                    if (cell == NONE) continue;
                    R w = wx[a] * wy[b] * wz[c];
                    acc_add(A_MF, cell, to_fp(w * pa.x, Kc::FP_F()));
                    acc_add(A_MA, cell, to_fp(w * pa.y * R(1e6), Kc::FP_A()));
                }
    }
}

// ---- grid_prep, fluid.wgsl:305-356 -----------------------------------------------------------------
template <class R>
void Sim<R>::grid_prep() {
    const uint32_t n = n_blocks() * 64;
    const R hh = h();
    const V3<R> org = origin();
    const V3<R> knot = {R(U.knot[0]), R(U.knot[1]), R(U.knot[2])};
    const R kr = R(U.knot[3]) + R(0.5) * hh;
    const R grav[3] = {R(U.gravity[0]), R(U.gravity[1]), R(U.gravity[2])};
#pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < (int64_t)n; ci++) {
        uint32_t cell = (uint32_t)ci;
        R ty = Kc::GAS;
        I3 c = cell_coord(cell);
        bool ground = org.y + (R(c.y) + R(0.5)) * hh < R(0);
        V3<R> p = org + (vf<R>(c) + R(0.5)) * hh - knot;
        bool knot_c = p.y > R(0) && p.y < R(2) * kr && std::sqrt(p.x * p.x + p.z * p.z) < kr;
        if (ground || knot_c)
            ty = Kc::SOLID;
        else if (accv(A_N, cell) > 0)
            ty = Kc::WATER;
        cfr(F_TYPE, cell) = ty;
        for (uint32_t d = 0; d < 3; d++) {
            R w = from_fp(accv(a_wt(d), cell), Kc::FP_W());
            R u = R(0);
            if (w > R(1e-6)) u = from_fp(accv(a_mom(d), cell), Kc::FP_M()) / w + dt() * grav[d];
            cfr(F_U + d, cell) = u;
        }
        R wc = from_fp(accv(A_WC, cell), Kc::FP_W());
        R ma = from_fp(accv(A_MA, cell), Kc::FP_A());
        if (ty == Kc::GAS && accv(A_MW, cell) > 0) {
            ty = Kc::RUBBER;
            cfr(F_TYPE, cell) = ty;
        }
        R pr = R(0);
        if (ty == Kc::WATER && wc > R(1e-6)) {
            pr = from_fp(accv(A_PC, cell), Kc::FP_P()) / wc * R(1e6);
        } else if (ty != Kc::WATER && ty != Kc::SOLID && ma > R(0)) {
            ty = Kc::COVERED;
            cfr(F_TYPE, cell) = ty;
            pr = from_fp(accv(A_MF, cell), Kc::FP_F()) / ma * R(1e6);
        }
        cfr(F_P, cell) = pr;
    }
}

// ---- air_fill (reads the second air buffer, writes the first), air.wgsl:101-148 ---------------
template <class R>
void Sim<R>::air_fill() {
    const uint32_t n = n_blocks() * 64;
    static const I3 E6[6] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < (int64_t)n; ci++) {
        uint32_t cell = (uint32_t)ci;
        R ty = cfv(F_TYPE, cell);
        if (ty == Kc::WATER || ty == Kc::SOLID) {
            write_gas(0, cell, no_gas());
            continue;
        }
        Gas<R> g = read_gas(1, cell);
        if (g.rho <= R(0)) {
            Gas<R> sum = no_gas();
            R cnt = R(0);
            for (int k = 0; k < 6; k++) {
                uint32_t nb = neighbour(cell, E6[k]);
                if (nb == NONE) continue;
                Gas<R> q = read_gas(1, nb);
                if (q.rho > R(0)) {
                    sum = {sum.rho + q.rho, sum.m + q.m, sum.e + q.e};
                    cnt += R(1);
                }
            }
            if (cnt > R(0))
                g = {sum.rho / cnt, sum.m / cnt, sum.e / cnt};
            else
                g = gas_at_rest(Kc::RHO_VAPOUR(), Kc::P_VAPOUR());
        }
        write_gas(0, cell, g);
        if (ty == Kc::GAS) cfr(F_P, cell) = gas_p(g) - Kc::P_ATM();
        if (ty == Kc::RUBBER) {
            R p = Kc::BIG();
            for (int k = 0; k < 6; k++) {
                uint32_t nb = neighbour(cell, E6[k]);
                if (nb == NONE || !free_gas(nb)) continue;
                Gas<R> q = read_gas(1, nb);
                if (q.rho > R(0)) p = mn(p, gas_p(q));
            }
            cfr(F_P, cell) = (p < Kc::BIG() ? p : gas_p(g)) - Kc::P_ATM();
        }
    }
}

// ---- bullets, bullet.wgsl ------------------------------------------------------------------------
template <class R>
static inline V3<R> qrot(V4<R> q, V3<R> v) {
    V3<R> qv = q.xyz();
    V3<R> t = R(2) * cross(qv, v);
    return v + q.w * t + cross(qv, t);
}
template <class R>
static inline V4<R> qmul(V4<R> a, V4<R> b) {
    V3<R> v = a.w * b.xyz() + b.w * a.xyz() + cross(a.xyz(), b.xyz());
    return {v.x, v.y, v.z, a.w * b.w - dot(a.xyz(), b.xyz())};
}
template <class R>
static inline V4<R> normalize4(V4<R> q) {
    R inv = R(1) / std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    return {q.x * inv, q.y * inv, q.z * inv, q.w * inv};
}
template <class R>
static R cp_patch(R s) {
    if (s < R(0)) return K<R>::CP_WAKE() * s * s;
    R beta = masin(mn(s, R(1)));
    if (beta < K<R>::PI() / R(12)) return R(2.13) * s * s;
    R x = beta / K<R>::PI() - R(0.25);
    return R(0.5) + R(1.81) * x - R(2) * x * x;
}

template <class R>
V2<R> Sim<R>::sample_grid(V3<R> x, uint32_t fu, uint32_t fw) const {
    I3 base = vi(vfloor(x - R(0.5)));
    V3<R> fx = x - vf<R>(base);
    V3<R> wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    V2<R> s = {R(0), R(0)};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++) {
                uint32_t cell = cell_at(base + I3{a, b, c});
                if (cell == NONE) continue;
                R w = wx[a] * wy[b] * wz[c] * from_fp(accv(fw, cell), Kc::FP_W());
                s = {s.x + w * cfv(fu, cell), s.y + w};
            }
    return s;
}

template <class R>
V2<R> Sim<R>::sample_pressure(V3<R> x, bool gas_only) const {
    I3 base = vi(vfloor(x - R(0.5)));
    V3<R> fx = x - vf<R>(base);
    V3<R> wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    V2<R> s = {R(0), R(0)};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++) {
                uint32_t cell = cell_at(base + I3{a, b, c});
                if (cell == NONE) continue;
                R ty = cfv(F_TYPE, cell);
                if (ty == Kc::SOLID || (gas_only && ty == Kc::WATER)) continue;
                R w = wx[a] * wy[b] * wz[c];
                s = {s.x + w * cfv(F_P, cell), s.y + w};
            }
    return s;
}

template <class R>
void Sim<R>::push_water(V3<R> x, uint32_t d, R j, R sw) {
    if (sw <= R(1e-6) || j == R(0)) return;
    V3<R> lx = x - lattice_offset(d);
    I3 base = vi(vfloor(lx - R(0.5)));
    V3<R> fx = lx - vf<R>(base);
    V3<R> wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    R hs = R(U.fluid[3]);
    R k = j / (R(U.fluid[0]) * hs * hs * hs * sw);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++) {
                uint32_t cell = cell_at(base + I3{a, b, c});
                if (cell == NONE || accv(a_wt(d), cell) <= 0) continue;
                acc_add(A_BU + d, cell, to_fp(k * wx[a] * wy[b] * wz[c], Kc::FP_M()));
            }
}

template <class R>
bool Sim<R>::in_cavity(uint32_t b, V3<R> p, R t) const {
    R hand2 = Kc::R_HAND() * Kc::R_HAND() * h() * h();
    for (uint32_t k = 0; k < N_SEC; k++) {
        const Section<R>& s = sections[b * N_SEC + k];
        if (s.b.w <= R(0) || section_r2(s, t) >= hand2) continue;
        V3<R> ab = s.b.xyz() - s.a.xyz();
        R f = dot(p - s.a.xyz(), ab) / mx(dot(ab, ab), R(1e-20));
        if (f < R(0) || f > R(1)) continue;
        V3<R> d = p - (s.a.xyz() + f * ab);
        if (dot(d, d) < section_r2(s, t)) return true;
    }
    return false;
}

template <class R>
void Sim<R>::bullet_step() {
    const R step = dt(), t_end = now(), hh = h();
    const V3<R> org = origin();
    for (uint32_t bi = 0; bi < U.mem[3]; bi++) {
        Bullet<R> b = bullets[bi];
        // li == 0: state, the pressure ahead, and the side of the rubber it holds.
        uint32_t state = b.info[2];
        if (state == 0u && st.t_ns - st.dt_ns >= b.info[0]) state = 1u;
        V3<R> ahead = b.x.xyz() + normalize(b.v.xyz() + R(1e-9)) * (b.shape.z + R(3) * hh);
        V2<R> sp0 = sample_pressure((ahead - org) / hh - R(0.5), false);
        R pf = sp0.y > R(1e-6) ? sp0.x / sp0.y : R(0);
        V3<R> sn, sx;
        for (int c = 0; c < 3; c++) {
            sn[c] = from_fp(bullet_hit[bi * HIT_FIELDS + 6 + c], Kc::FP_A());
            bullet_hit[bi * HIT_FIELDS + 6 + c] = 0;
            sx[c] = from_fp(bullet_hit[bi * HIT_FIELDS + 9 + c], Kc::FP_X());
            bullet_hit[bi * HIT_FIELDS + 9 + c] = 0;
        }
        R sa = from_fp(bullet_hit[bi * HIT_FIELDS + 12], Kc::FP_A());
        bullet_hit[bi * HIT_FIELDS + 12] = 0;
        V4<R> side = {R(0), R(0), R(0), R(0)};
        if (sa > R(0) && length(sn) > R(0)) {
            V3<R> n = normalize(sn);
            side = {n.x, n.y, n.z, dot(sx, n) / sa * R(1e-3)};
        }
        if (state != 1u) {
            bullets[bi].info[2] = state;
            V4<R>& e = pose_log[(bi * LOG_CAP + st.step % LOG_CAP) * 3];
            e = {R(0), R(0), R(0), R(0)};
            continue;
        }
        V3<R> lb = qrot(V4<R>{-b.q.x, -b.q.y, -b.q.z, b.q.w}, b.l.xyz());
        V3<R> w = qrot(b.q, lb / V3<R>{b.shape.y, b.shape.y, b.shape.x});
        const R rho = R(U.fluid[0]);
        const V3<R> vhat = normalize(b.v.xyz() + R(1e-9));
        // Per thread partial sums over patches li, li + 256, li + 512, then the 256-wide tree.
        struct Red {
            V4<R> f, t, c;
        };
        std::vector<Red> red(256);
        for (uint32_t li = 0; li < 256; li++) {
            V3<R> f = {R(0), R(0), R(0)}, tq = {R(0), R(0), R(0)};
            V4<R> cav = {R(0), R(0), R(0), R(0)};
            V4<R> cen = {R(0), R(0), R(0), Kc::BIG()};
            for (uint32_t k = li; k < b.info[1]; k += 256u) {
                V4<R> pp = patches[(bi * MAX_PATCHES + k) * 2], pn = patches[(bi * MAX_PATCHES + k) * 2 + 1];
                V3<R> r = qrot(b.q, pp.xyz());
                V3<R> p = b.x.xyz() + r;
                V3<R> n = qrot(b.q, pn.xyz());
                R area = pp.w;
                V3<R> X = (p - org) / hh;
                V3<R> uw, sw;
                for (uint32_t d = 0; d < 3; d++) {
                    V2<R> s = sample_grid(X - lattice_offset(d), F_U + d, a_wt(d));
                    uw[d] = s.y > R(1e-6) ? s.x / s.y : R(0);
                    sw[d] = s.y;
                }
                R fill = clampr(sample_grid(X - R(0.5), F_TYPE, A_WC).y / R(8), R(0), R(1));
                if (in_cavity(bi, p, t_end - step) || dot(r, side.xyz()) > side.w) fill = R(0);
                V2<R> gs = sample_pressure(X - R(0.5), true);
                R p_gas = gs.y > R(1e-6) ? gs.x / gs.y : R(0);
                V3<R> vp = b.v.xyz() + cross(w, r);
                V3<R> rel = vp - uw;
                R spd = length(rel);
                R wn = dot(rel, n);
                R q = R(0.5) * rho * spd * spd;
                R p_water = mx(Kc::P_FLOOR(), pf + q * cp_patch(wn / mx(spd, R(1e-9))));
                V3<R> fw = -fill * p_water * area * n;
                V3<R> rt = rel - wn * n;
                R rtl = length(rt);
                if (rtl > R(1e-9)) fw = fw - fill * Kc::CF_SKIN() * R(0.5) * rho * rtl * rt * area;
                V3<R> fp = fw - (R(1) - fill) * mx(p_gas, Kc::P_FLOOR()) * area * n;
                f = f + fp;
                tq = tq + cross(r, fp);
                for (uint32_t d = 0; d < 3; d++) push_water(X, d, -fw[d] * step, sw[d]);
                if (wn > R(0) && fill > R(0)) {
                    R face = fill * area * mx(dot(n, vhat), R(0));
                    cav = {cav.x + -dot(fw, vhat), cav.y + face, cav.z, cav.w};
                    V3<R> cx = cen.xyz() + p * face;
                    cen = {cx.x, cx.y, cx.z, mn(cen.w, dot(r, vhat))};
                }
            }
            red[li] = {{f.x, f.y, f.z, cav.x}, {tq.x, tq.y, tq.z, cav.y}, cen};
        }
        for (uint32_t off = 128; off > 0; off >>= 1)
            for (uint32_t li = 0; li < off; li++) {
                Red& a = red[li];
                const Red& o = red[li + off];
                a.f = {a.f.x + o.f.x, a.f.y + o.f.y, a.f.z + o.f.z, a.f.w + o.f.w};
                a.t = {a.t.x + o.t.x, a.t.y + o.t.y, a.t.z + o.t.z, a.t.w + o.t.w};
                a.c = {a.c.x + o.c.x, a.c.y + o.c.y, a.c.z + o.c.z, mn(a.c.w, o.c.w)};
            }
        V3<R> hit, hit_l;
        for (int c = 0; c < 3; c++) {
            hit[c] = from_fp(bullet_hit[bi * HIT_FIELDS + c], Kc::FP_J());
            bullet_hit[bi * HIT_FIELDS + c] = 0;
            hit_l[c] = from_fp(bullet_hit[bi * HIT_FIELDS + 3 + c], Kc::FP_L());
            bullet_hit[bi * HIT_FIELDS + 3 + c] = 0;
        }
        V3<R> grav = {R(U.gravity[0]), R(U.gravity[1]), R(U.gravity[2])};
        V3<R> force = red[0].f.xyz() + b.x.w * grav;
        R drag = red[0].f.w;
        R face = red[0].t.w;
        V3<R> v = b.v.xyz() + (force * step + hit) / b.x.w;
        V3<R> x = b.x.xyz() + v * step;
        V3<R> l = b.l.xyz() + red[0].t.xyz() * step + hit_l;
        V3<R> axis0 = qrot(b.q, V3<R>{R(0), R(0), R(1)});
        R spin_extra = dot(l, axis0) * (R(1) / b.shape.x - R(1) / b.shape.y) * step;
        R cone = length(l) / b.shape.y * step;
        V4<R> q = qmul(b.q, V4<R>{R(0), R(0), msin(R(0.5) * spin_extra), mcos(R(0.5) * spin_extra)});
        if (cone > R(1e-12)) {
            V3<R> ln = normalize(l) * msin(R(0.5) * cone);
            q = qmul(V4<R>{ln.x, ln.y, ln.z, mcos(R(0.5) * cone)}, q);
        }
        q = normalize4(q);
        R roll = b.v.w + dot(l, axis0) / b.shape.x * step;
        uint32_t info[4] = {b.info[0], b.info[1], 1u, b.info[3]};
        V3<R> hi = org + v3(R(U.dims[0]), R(U.dims[1]), R(U.dims[2])) * hh;
        if (x.x < org.x || x.y < org.y || x.z < org.z || x.x > hi.x || x.y > hi.y || x.z > hi.z) info[2] = 2u;
        I3 c = shr2(own_cell(x));
        bool nearb = false;
        for (uint32_t k = 0; k < 27; k++) {
            I3 nb = c + I3{(int32_t)(k / 9u), (int32_t)((k / 3u) % 3u), (int32_t)(k % 3u)} - I3{1, 1, 1};
            if (in_domain_block(nb) && block_ptr[block_slot(nb)] != NONE) nearb = true;
        }
        R pace = nearb ? length(v) : length(v) * R(U.fluid[1]) / R(4);
        if (drag > R(0) && face > R(0)) {
            V3<R> mid = red[0].c.xyz() / face;
            V3<R> a = mid + vhat * (red[0].c.w - dot(mid - b.x.xyz(), vhat));
            Section<R> s;
            s.a = {a.x, a.y, a.z, t_end - R(0.5) * step};
            V3<R> bb = a + v * step;
            s.b = {bb.x, bb.y, bb.z, R(2) * std::sqrt(drag / (Kc::PI() * rho * Kc::LOGVINOVICH_K()))};
            s.c = {face / Kc::PI(), R(0), R(0), R(0)};
            sections[bi * N_SEC + info[3] % N_SEC] = s;
            info[3] += 1u;
        }
        R reach = R(0);
        const R hand2 = Kc::R_HAND() * Kc::R_HAND() * hh * hh;
        for (uint32_t k = 0; k < N_SEC; k++) {
            const Section<R>& s = sections[bi * N_SEC + k];
            if (s.b.w <= R(0) || section_r2(s, t_end) >= hand2) continue;
            reach = mx(reach, mx(length(s.a.xyz() - x), length(s.b.xyz() - x)));
        }
        Bullet<R>& o = bullets[bi];
        o.x = {x.x, x.y, x.z, b.x.w};
        o.v = {v.x, v.y, v.z, roll};
        o.q = q;
        o.l = {l.x, l.y, l.z, pace};
        o.reach = {x.x, x.y, x.z, reach > R(0) ? reach + Kc::R_HAND() * hh : R(0)};
        std::memcpy(o.info, info, 16);
        uint32_t tb = st.t_ns;
        float tf;
        std::memcpy(&tf, &tb, 4);
        V4<R>* e = &pose_log[(bi * LOG_CAP + st.step % LOG_CAP) * 3];
        e[0] = {x.x, x.y, x.z, R(tf)};
        e[1] = q;
        e[2] = {v.x, v.y, v.z, roll};
        // Sections thinner than the grid push the water out of the way as they open.
        for (uint32_t li = 0; li < N_SEC; li++) {
            const Section<R>& s = sections[bi * N_SEC + li];
            R r2 = section_r2(s, t_end);
            if (!(s.b.w > R(0) && r2 < hand2)) continue;
            R qv = Kc::PI() * s.b.w * length(s.b.xyz() - s.a.xyz());
            V3<R> xx = (R(0.5) * (s.a.xyz() + s.b.xyz()) - org) / hh - R(0.5);
            I3 base = vi(vfloor(xx - R(0.5)));
            V3<R> fx = xx - vf<R>(base);
            V3<R> wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
            for (int a = 0; a < 3; a++)
                for (int bb2 = 0; bb2 < 3; bb2++)
                    for (int cc = 0; cc < 3; cc++) {
                        uint32_t cell = cell_at(base + I3{a, bb2, cc});
                        if (cell == NONE) continue;
                        acc_add(A_SRC, cell, to_fp(qv * wx[a] * wy[bb2] * wz[cc], Kc::FP_Q()));
                    }
        }
    }
}

template <class R>
void Sim<R>::bullet_apply() {
    const uint32_t n = n_blocks() * 64;
#pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < (int64_t)n; ci++) {
        uint32_t cell = (uint32_t)ci;
        for (uint32_t d = 0; d < 3; d++) {
            int32_t du = accv(A_BU + d, cell);
            if (du != 0) cfr(F_U + d, cell) = cfv(F_U + d, cell) + from_fp(du, Kc::FP_M());
        }
    }
}

// ---- pressure solve, fluid.wgsl:381-578 ---------------------------------------------------------
template <class R, class A>
struct Acc4 {
    A x, y, z, w;
};

// Symmetric red-black Gauss-Seidel inside one block, two sweeps (fluid.wgsl:390-410).
template <class R>
static void precondition_block(const R* r, const R* diag, const bool* water, R* zl) {
    for (int li = 0; li < 64; li++) zl[li] = R(0);
    for (uint32_t k = 0; k < 5; k++) {
        for (int li = 0; li < 64; li++) {
            int lx = li / 16, ly = (li / 4) % 4, lz = li % 4;
            uint32_t colour = (uint32_t)(lx + ly + lz) % 2u;
            if (!(water[li] && colour == k % 2u)) continue;
            R s = r[li];
            if (lx > 0 && water[li - 16]) s += zl[li - 16];
            if (lx < 3 && water[li + 16]) s += zl[li + 16];
            if (ly > 0 && water[li - 4]) s += zl[li - 4];
            if (ly < 3 && water[li + 4]) s += zl[li + 4];
            if (lz > 0 && water[li - 1]) s += zl[li - 1];
            if (lz < 3 && water[li + 1]) s += zl[li + 1];
            zl[li] = s / diag[li];
        }
    }
}

// The 64-wide tree of block_sum (fluid.wgsl:414-422).
template <class A>
static void tree64(A* v) {
    for (int off = 32; off > 0; off >>= 1)
        for (int li = 0; li < off; li++) v[li] += v[li + off];
}
// total(): 256 strided partial sums, then the 256-wide tree (fluid.wgsl:426-439).
template <class A>
static A total256(const std::vector<A>& part, uint32_t n) {
    A red[256];
    for (uint32_t li = 0; li < 256; li++) {
        A s = A(0);
        for (uint32_t i = li; i < n; i += 256) s += part[i];
        red[li] = s;
    }
    for (int off = 128; off > 0; off >>= 1)
        for (int li = 0; li < off; li++) red[li] += red[li + off];
    return red[0];
}

template <class R>
void Sim<R>::solve() {
    const uint32_t nb = n_blocks();
    const R hh = h();
    const R grav_w = R(U.gravity[3]);
    const R rho = R(U.fluid[0]);
    const R tol = R(U.solve[0]);
    static const I3 E[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    // Partials per block: x, y, z components kept as separate arrays of the accumulator type.
    std::vector<double> px(nb), py(nb), pz(nb);
    auto run_block_sum = [&](uint32_t b, const R* vx, const R* vy, const R* vz) {
        if (fp64_dots) {
            double ax[64], ay[64], az[64];
            for (int i = 0; i < 64; i++) ax[i] = (double)vx[i], ay[i] = (double)vy[i], az[i] = (double)vz[i];
            tree64(ax), tree64(ay), tree64(az);
            px[b] = ax[0], py[b] = ay[0], pz[b] = az[0];
        } else {
            R ax[64], ay[64], az[64];
            for (int i = 0; i < 64; i++) ax[i] = vx[i], ay[i] = vy[i], az[i] = vz[i];
            tree64(ax), tree64(ay), tree64(az);
            px[b] = (double)ax[0], py[b] = (double)ay[0], pz[b] = (double)az[0];
        }
    };
    auto total = [&](const std::vector<double>& part) -> double {
        if (fp64_dots) return total256(part, nb);
        std::vector<R> pr(nb);
        for (uint32_t i = 0; i < nb; i++) pr[i] = (R)part[i];
        return (double)total256(pr, nb);
    };
    // In the FP64 mode products are formed in double from the FP32 factors.
    auto prod = [&](R a, R b, R& out_r, double& out_d) {
        out_r = a * b;
        out_d = (double)a * (double)b;
    };
    (void)prod;

    // solve_init
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t bb = 0; bb < (int64_t)nb; bb++) {
        uint32_t b = (uint32_t)bb;
        R r[64], dg[64], bv[64], zl[64];
        bool water[64];
        for (uint32_t li = 0; li < 64; li++) {
            uint32_t cell = b * 64 + li;
            water[li] = cfv(F_TYPE, cell) == Kc::WATER;
            R diag = R(1), rr = R(0), bq = R(0);
            if (water[li]) {
                R cs = grav_w * dt();
                R kc = hh * hh / (cs * cs);
                R div = R(0), off = R(0);
                diag = kc;
                bq = kc * cfv(F_P, cell);
                for (uint32_t d = 0; d < 3; d++) {
                    I3 e = E[d];
                    I3 me = {-e.x, -e.y, -e.z};
                    div += face_u(neighbour(cell, e), cell, d) - face_u(cell, neighbour(cell, me), d);
                    for (int s = -1; s <= 1; s += 2) {
                        uint32_t nbc = neighbour(cell, e * s);
                        R nt = cell_type(nbc);
                        if (nt == Kc::SOLID) continue;
                        diag += R(1);
                        if (nt == Kc::WATER)
                            off -= cfv(F_P, nbc);
                        else
                            bq += pressure_of(nbc);
                    }
                }
                div -= from_fp(accv(A_SRC, cell), Kc::FP_Q()) / (hh * hh);
                bq -= rho * hh / dt() * div;
                rr = bq - diag * cfv(F_P, cell) - off;
                cfr(F_DIAG, cell) = diag;
                cfr(F_R, cell) = rr;
            }
            r[li] = rr, dg[li] = diag, bv[li] = bq;
        }
        precondition_block(r, dg, water, zl);
        R vx[64], vy[64], vz[64];
        for (uint32_t li = 0; li < 64; li++) {
            if (water[li]) cfr(F_Z, b * 64 + li) = zl[li];
        }
        if (fp64_dots) {
            double ax[64], ay[64], az[64];
            for (int i = 0; i < 64; i++) {
                ax[i] = (double)r[i] * (double)zl[i];
                ay[i] = (double)r[i] * (double)r[i];
                az[i] = (double)bv[i] * (double)bv[i];
            }
            tree64(ax), tree64(ay), tree64(az);
            px[b] = ax[0], py[b] = ay[0], pz[b] = az[0];
        } else {
            for (int i = 0; i < 64; i++) vx[i] = r[i] * zl[i], vy[i] = r[i] * r[i], vz[i] = bv[i] * bv[i];
            run_block_sum(b, vx, vy, vz);
        }
    }
    // solve_start
    {
        double sx = total(px), sy = total(py), sz = total(pz);
        st.rz = sx;
        st.beta = 0;
        if (fp64_dots) {
            st.b_norm = std::sqrt(sz);
            st.r_norm = std::sqrt(sy);
        } else {
            st.b_norm = (double)std::sqrt((R)sz);
            st.r_norm = (double)std::sqrt((R)sy);
        }
        st.solve_iters = 0;
        auto converged = [&](double rr) {
            if (fp64_dots) return std::sqrt(rr) <= (double)tol * std::max(st.b_norm, 1.0);
            return std::sqrt((R)rr) <= tol * mx((R)st.b_norm, R(1));
        };
        st.solver_on = sx > 0.0 && !converged(sy);
        uint32_t limit = U.limits[2];
        for (uint32_t it = 0; it < limit && st.solver_on; it++) {
            uint32_t old = st.solve_iters % 2u;
            R beta = (R)st.beta;
            // solve_q
#pragma omp parallel for schedule(dynamic, 16)
            for (int64_t bb = 0; bb < (int64_t)nb; bb++) {
                uint32_t b = (uint32_t)bb;
                R v[64];
                double vd[64];
                for (uint32_t li = 0; li < 64; li++) {
                    uint32_t cell = b * 64 + li;
                    v[li] = R(0), vd[li] = 0.0;
                    if (cfv(F_TYPE, cell) != Kc::WATER) continue;
                    R dn = cfv(F_Z, cell) + beta * cfv(F_D + old, cell);
                    R q = cfv(F_DIAG, cell) * dn;
                    for (uint32_t d = 0; d < 3; d++)
                        for (int k = -1; k <= 1; k += 2) {
                            uint32_t nbc = neighbour(cell, E[d] * k);
                            if (cell_type(nbc) == Kc::WATER) q -= cfv(F_Z, nbc) + beta * cfv(F_D + old, nbc);
                        }
                    cfr(F_D + 1 - old, cell) = dn;
                    cfr(F_Q, cell) = q;
                    v[li] = dn * q;
                    vd[li] = (double)dn * (double)q;
                }
                if (fp64_dots) {
                    tree64(vd);
                    px[b] = vd[0];
                } else {
                    tree64(v);
                    px[b] = (double)v[0];
                }
            }
            // solve_alpha
            {
                double s = total(px);
                if (fp64_dots)
                    st.alpha = s > 0.0 ? st.rz / s : 0.0;
                else
                    st.alpha = s > 0.0 ? (double)((R)st.rz / (R)s) : 0.0;
            }
            // solve_update
            R a = (R)st.alpha;
#pragma omp parallel for schedule(dynamic, 16)
            for (int64_t bb = 0; bb < (int64_t)nb; bb++) {
                uint32_t b = (uint32_t)bb;
                R r[64], dg[64], zl[64];
                bool water[64];
                for (uint32_t li = 0; li < 64; li++) {
                    uint32_t cell = b * 64 + li;
                    water[li] = cfv(F_TYPE, cell) == Kc::WATER;
                    R diag = R(1), rr = R(0);
                    if (water[li]) {
                        cfr(F_P, cell) = cfv(F_P, cell) + a * cfv(F_D + 1 - old, cell);
                        rr = cfv(F_R, cell) - a * cfv(F_Q, cell);
                        cfr(F_R, cell) = rr;
                        diag = cfv(F_DIAG, cell);
                    }
                    r[li] = rr, dg[li] = diag;
                }
                precondition_block(r, dg, water, zl);
                for (uint32_t li = 0; li < 64; li++)
                    if (water[li]) cfr(F_Z, b * 64 + li) = zl[li];
                if (fp64_dots) {
                    double ax[64], ay[64];
                    for (int i = 0; i < 64; i++) ax[i] = (double)r[i] * (double)zl[i], ay[i] = (double)r[i] * (double)r[i];
                    tree64(ax), tree64(ay);
                    px[b] = ax[0], py[b] = ay[0];
                } else {
                    R ax[64], ay[64];
                    for (int i = 0; i < 64; i++) ax[i] = r[i] * zl[i], ay[i] = r[i] * r[i];
                    tree64(ax), tree64(ay);
                    px[b] = (double)ax[0], py[b] = (double)ay[0];
                }
            }
            // solve_beta
            {
                double sx2 = total(px), sy2 = total(py);
                st.solve_iters += 1;
                if (fp64_dots) {
                    st.r_norm = std::sqrt(sy2);
                    st.beta = st.rz > 0.0 ? sx2 / st.rz : 0.0;
                } else {
                    st.r_norm = (double)std::sqrt((R)sy2);
                    st.beta = st.rz > 0.0 ? (double)((R)sx2 / (R)st.rz) : 0.0;
                }
                st.rz = sx2;
                bool done = converged(sy2);
                if (done || st.solve_iters >= U.limits[2]) {
                    st.iters_max = std::max(st.iters_max, st.solve_iters);
                    st.unconverged += done ? 0u : 1u;
                    st.solver_on = false;
                }
            }
        }
    }
}

// ---- project, extend, fluid.wgsl:580-674 -------------------------------------------------------
template <class R>
void Sim<R>::project() {
    const uint32_t n = n_blocks() * 64;
    const R k = dt() / (R(U.fluid[0]) * h());
    static const I3 M[3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
#pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < (int64_t)n; ci++) {
        uint32_t cell = (uint32_t)ci;
        R ty = cfv(F_TYPE, cell);
        for (uint32_t d = 0; d < 3; d++) {
            uint32_t nb = neighbour(cell, M[d]);
            R nt = cell_type(nb);
            R u = bounded(cfv(F_U + d, cell), ty, nt);
            if (ty != Kc::SOLID && nt != Kc::SOLID && (ty == Kc::WATER || nt == Kc::WATER)) u -= k * (pressure_of(cell) - pressure_of(nb));
            cfr(F_U + d, cell) = u;
        }
    }
}

template <class R>
void Sim<R>::extend() {
    const uint32_t n = n_blocks() * 64;
    static const I3 M[3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
    static const I3 E6[6] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    auto face_set = [&](uint32_t cell, uint32_t d) {
        if (cell == NONE) return false;
        return cfv(F_TYPE, cell) == Kc::WATER || cell_type(neighbour(cell, M[d])) == Kc::WATER;
    };
#pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < (int64_t)n; ci++) {
        uint32_t cell = (uint32_t)ci;
        uint32_t done = 0;
        for (uint32_t d = 0; d < 3; d++) {
            R u = cfv(F_U + d, cell);
            if (face_set(cell, d)) {
                done |= 1u << d;
            } else {
                R sum = R(0), cnt = R(0);
                for (int k = 0; k < 6; k++) {
                    uint32_t nb = neighbour(cell, E6[k]);
                    if (face_set(nb, d)) {
                        sum += cfv(F_U + d, nb);
                        cnt += R(1);
                    }
                }
                if (cnt > R(0)) {
                    u = sum / cnt;
                    done |= 1u << d;
                }
            }
            cfr(F_EXT + d, cell) = u;
        }
        cfr(F_EXT_SET, cell) = R(done);
    }
    auto ext_set = [&](uint32_t cell, uint32_t d) {
        return cell != NONE && ((f2u(cfv(F_EXT_SET, cell)) >> d) & 1u) != 0u;
    };
#pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < (int64_t)n; ci++) {
        uint32_t cell = (uint32_t)ci;
        R ty = cfv(F_TYPE, cell);
        for (uint32_t d = 0; d < 3; d++) {
            R u = cfv(F_U + d, cell);
            if (ext_set(cell, d)) {
                u = cfv(F_EXT + d, cell);
            } else {
                R sum = R(0), cnt = R(0);
                for (int k = 0; k < 6; k++) {
                    uint32_t nb = neighbour(cell, E6[k]);
                    if (ext_set(nb, d)) {
                        sum += cfv(F_EXT + d, nb);
                        cnt += R(1);
                    }
                }
                if (cnt > R(0)) u = sum / cnt;
            }
            cfr(F_U + d, cell) = bounded(u, ty, cell_type(neighbour(cell, M[d])));
        }
    }
}

// ---- mem_sample, membrane.wgsl:219-256 ------------------------------------------------------------
template <class R>
void Sim<R>::mem_sample() {
    const R hh = h();
    const V3<R> org = origin();
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)Nv; ii++) {
        uint32_t i = (uint32_t)ii;
        if (mem_mass[i] == R(0)) continue;
        V3<R> x = (mem_x[0][i].xyz() - org) / hh;
        V3<R> v = {R(0), R(0), R(0)};
        for (uint32_t d = 0; d < 3; d++) {
            V2<R> s = sample_grid(x - lattice_offset(d), F_U + d, a_wt(d));
            v[d] = s.y > R(1e-6) ? s.x / s.y : R(0);
        }
        R fill = sample_grid(x - R(0.5), F_TYPE, A_WC).y / R(8);
        mem_water[i] = {v.x, v.y, v.z, fill};
    }
}

// ---- mem_substep, membrane.wgsl:47-400, bullet.wgsl:426-611 ------------------------------------------
template <class R>
typename Sim<R>::Sheet Sim<R>::sheet(R major, R minor) const {
    if (major <= R(1)) return {{R(0), R(0)}, R(0)};
    const V3<R> mu = {R(U.rubber[0]), R(U.rubber[1]), R(U.rubber[2])};
    const V3<R> AL = {R(1.3), R(5.0), R(-2.0)};
    R la = mlog(major);
    V3<R> e1 = AL * la;
    V3<R> pa = {mexp(e1.x), mexp(e1.y), mexp(e1.z)};
    R tan_scale = R(1) / (major * major);
    if (minor * minor * major < R(1)) {
        V3<R> e2 = (R(-0.5) * AL) * la;
        V3<R> pn = {mexp(e2.x), mexp(e2.y), mexp(e2.z)};
        return {{dot(mu, pa - pn), R(0)}, dot(mu * AL, pa + R(0.5) * pn) * tan_scale};
    }
    R lb = mlog(minor);
    V3<R> e3 = AL * lb;
    V3<R> pb = {mexp(e3.x), mexp(e3.y), mexp(e3.z)};
    V3<R> e4 = (-AL) * (la + lb);
    V3<R> p3 = {mexp(e4.x), mexp(e4.y), mexp(e4.z)};
    return {{dot(mu, pa - p3), dot(mu, pb - p3)}, dot(mu * AL, pa + p3) * tan_scale};
}

template <class R>
typename Sim<R>::VertexForce Sim<R>::vertex_force(int par, uint32_t i) {
    const auto& X = mem_x[par];
    VertexForce o = {{R(0), R(0), R(0)}, {R(0), R(0), R(0)}, R(0), R(0), R(0), R(0), R(U.rubber[3]), 0u};
    R rest = R(0);
    const R thick0 = R(U.rubber[3]);
    // `alive` holds the state at the start of the substep for the whole substep: every vertex
    // of a triangle sees it alive, evaluates the same stretch and so the same tear (the
    // reference writes the tear at once, and what the triangle's other vertices then see depends
    // on the threads' timing). Tears are committed after the substep (mem_substep).
    for (uint32_t k = vtri_off[i]; k < vtri_off[i + 1]; k++) {
        uint32_t t = vtri[k];
        if (alive[t] == 0u) continue;
        const Tri& tri = tris[t];
        V3<R> x0 = X[tri.v0].xyz();
        V3<R> e1 = X[tri.v1].xyz() - x0;
        V3<R> e2 = X[tri.v2].xyz() - x0;
        const R mxx = R(tri.dm_inv[0]), myy = R(tri.dm_inv[1]), mzz = R(tri.dm_inv[2]), mww = R(tri.dm_inv[3]);
        o.reach = mx(o.reach, mx(length(e1), mx(length(e2), length(e2 - e1))));
        V3<R> f0 = e1 * mxx + e2 * mzz;
        V3<R> f1 = e1 * myy + e2 * mww;
        R c00 = dot(f0, f0), c01 = dot(f0, f1), c11 = dot(f1, f1);
        R mid = R(0.5) * (c00 + c11);
        R dev = std::sqrt(R(0.25) * (c00 - c11) * (c00 - c11) + c01 * c01);
        V2<R> l = {std::sqrt(mid + dev), std::sqrt(mx(mid - dev, R(1e-12)))};
        if (l.x >= R(U.rubber2[1])) {
#pragma omp atomic write
            torn[t] = 1u;
            o.torn |= 1ull << (k - vtri_off[i]);
            continue;
        }
        Sheet sh = sheet(l.x, l.y);
        V2<R> sig = sh.sig;
        V2<R> e = {R(1), R(0)};
        if (dev > R(1e-6) * mid) {
            V2<R> q = c00 >= c11 ? V2<R>{mid + dev - c11, c01} : V2<R>{c01, mid + dev - c00};
            R inv = R(1) / std::sqrt(q.x * q.x + q.y * q.y);
            e = {q.x * inv, q.y * inv};
        }
        V2<R> s = {sig.x / (l.x * l.x), sig.y / (l.y * l.y)};
        R ds = s.x - s.y;
        R s00 = s.y + ds * e.x * e.x;
        R s01 = ds * e.x * e.y;
        R s11 = s.y + ds * e.y * e.y;
        V3<R> p0 = f0 * s00 + f1 * s01;
        V3<R> p1 = f0 * s01 + f1 * s11;
        R vol = R(tri.rest_area) * thick0;
        V3<R> h1 = (-vol) * (p0 * mxx + p1 * myy);
        V3<R> h2 = (-vol) * (p0 * mzz + p1 * mww);
        V2<R> grad = {mxx, myy};
        if (i == tri.v0) {
            o.f = o.f - (h1 + h2);
            grad = {-(mxx + mzz), -(myy + mww)};
        } else if (i == tri.v1) {
            o.f = o.f + h1;
        } else {
            o.f = o.f + h2;
            grad = {mzz, mww};
        }
        V3<R> cr = cross(e1, e2);
        o.n = o.n + cr;
        o.area += length(cr) / R(6);
        rest += R(tri.rest_area) / R(3);
        o.stiff += vol * (grad.x * grad.x + grad.y * grad.y) * (sh.tangent + s.x);
        o.tension = mx(o.tension, sig.x * thick0 / (l.x * l.y));
    }
    if (o.area > R(0)) o.thick = thick0 * rest / o.area;
    return o;
}

template <class R>
Gas<R> Sim<R>::hll(const Gas<R>& l, const Gas<R>& r, uint32_t d) const {
    const R G = Kc::GAMMA();
    R pl = gas_p(l), pr = gas_p(r);
    R ul = l.m[d] / l.rho, ur = r.m[d] / r.rho;
    R cl = std::sqrt(G * pl / l.rho), cr = std::sqrt(G * pr / r.rho);
    R sl = mn(ul - cl, ur - cr), sr = mx(ul + cl, ur + cr);
    auto flux = [&](const Gas<R>& g, R p, R u) {
        V3<R> m = g.m * u;
        m[d] += p;
        return Gas<R>{g.rho * u, m, (g.e + p) * u};
    };
    Gas<R> fl = flux(l, pl, ul), fr = flux(r, pr, ur);
    if (sl >= R(0)) return fl;
    if (sr <= R(0)) return fr;
    R k = R(1) / (sr - sl);
    R a = sr * k, b = -sl * k, c = sl * sr * k;
    return {a * fl.rho + b * fr.rho + c * (r.rho - l.rho), a * fl.m + b * fr.m + c * (r.m - l.m), a * fl.e + b * fr.e + c * (r.e - l.e)};
}

template <class R>
Gas<R> Sim<R>::across(int buf, uint32_t cell, const Gas<R>& own, uint32_t d, bool hi) const {
    I3 e = {0, 0, 0};
    int s = hi ? 1 : -1;
    if (d == 0) e.x = s;
    if (d == 1) e.y = s;
    if (d == 2) e.z = s;
    uint32_t nb = neighbour(cell, e);
    if (nb == NONE) return ambient();
    if (free_gas(nb)) return read_gas(buf, nb);
    R w = cfv(F_U + d, hi ? nb : cell);
    if (cfv(F_TYPE, nb) == Kc::RUBBER) w = from_fp(accv(A_MV + d, nb), Kc::FP_A()) / from_fp(accv(A_MW, nb), Kc::FP_A());
    Gas<R> g = own;
    R u = own.m[d] / own.rho;
    g.m[d] = own.rho * (R(2) * w - u);
    g.e = own.e + R(0.5) * (g.m[d] * g.m[d] - own.m[d] * own.m[d]) / own.rho;
    return g;
}

template <class R>
R Sim<R>::gas_pressure_at(int buf, V3<R> x) const {
    const V3<R> org = origin();
    const R hh = h();
    I3 base = vi(vfloor((x - org) / hh - R(1)));
    V3<R> fx = (x - org) / hh - R(0.5) - vf<R>(base);
    V3<R> wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
    V2<R> s = {R(0), R(0)};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++) {
                uint32_t cell = cell_at(base + I3{a, b, c});
                R w = wx[a] * wy[b] * wz[c];
                if (cell == NONE)
                    s = {s.x + w * Kc::P_ATM(), s.y + w};
                else if (free_gas(cell))
                    s = {s.x + w * gas_p(read_gas(buf, cell)), s.y + w};
            }
    return s.y > R(1e-6) ? s.x / s.y : Kc::P_ATM();
}

template <class R>
typename Sim<R>::Near Sim<R>::nearest_surface(uint32_t bi, V2<R> q) const {
    auto ol = [&](uint32_t k) { return outline[bi * OUTLINE + k]; };
    V2<R> first = ol(0), last = ol(OUTLINE - 1);
    Near o = {q, {R(0), R(0)}, R(0)};
    R best = Kc::BIG();
    for (uint32_t j = 0; j <= OUTLINE; j++) {
        V2<R> p0 = {first.x, R(0)}, p1 = {last.x, R(0)};
        if (j > 0) p0 = ol(j - 1);
        if (j < OUTLINE) p1 = ol(j);
        V2<R> e = {p1.x - p0.x, p1.y - p0.y};
        R len2 = e.x * e.x + e.y * e.y;
        if (len2 <= R(0)) continue;
        R tt = clampr(((q.x - p0.x) * e.x + (q.y - p0.y) * e.y) / len2, R(0), R(1));
        V2<R> on = {p0.x + e.x * tt, p0.y + e.y * tt};
        V2<R> dq = {q.x - on.x, q.y - on.y};
        R d = std::sqrt(dq.x * dq.x + dq.y * dq.y);
        if (d < best) {
            best = d;
            o.at = on;
            V2<R> nn = {-e.y, e.x};
            R inv = R(1) / std::sqrt(nn.x * nn.x + nn.y * nn.y);
            o.n = {nn.x * inv, nn.y * inv};
        }
    }
    bool inside = false;
    if (q.x > first.x && q.x < last.x) {
        uint32_t k = 1;
        while (k < OUTLINE - 1 && ol(k).x < q.x) k++;
        V2<R> a = ol(k - 1), c = ol(k);
        R f = (q.x - a.x) / mx(c.x - a.x, R(1e-12));
        inside = q.y < a.y * (R(1) - f) + c.y * f;
    }
    o.depth = inside ? best : -best;
    if (!inside && best > R(0)) o.n = {(q.x - o.at.x) / best, (q.y - o.at.y) / best};
    return o;
}

template <class R>
R Sim<R>::rubber_contact(int par, uint32_t i, V3<R>& x, V3<R>& v, R m, V3<R> load, const VertexForce& vf, bool wet, bool& held, R t, R sub) {
    const auto& MX = mem_x[par];
    const auto& MV = mem_v[par];
    R limit = Kc::BIG();
    R band = held ? R(0.5) * vf.thick : R(0);
    held = false;
    for (uint32_t bi = 0; bi < U.mem[3]; bi++) {
        const Bullet<R>& b = bullets[bi];
        if (b.info[2] != 1u) continue;
        V3<R> xb = b.x.xyz() - b.v.xyz() * (now() - t);
        R closing = length(b.v.xyz() - v);
        if (length(x - xb) > b.shape.z + vf.reach + R(2) * closing * dt()) continue;
        limit = mn(limit, R(0.25) * b.shape.w / mx(closing, R(1e-6)));
        V4<R> back = {-b.q.x, -b.q.y, -b.q.z, b.q.w};
        V3<R> w = qrot(b.q, qrot(back, b.l.xyz()) / V3<R>{b.shape.y, b.shape.y, b.shape.x});
        R best = -band;
        bool found = false;
        V3<R> gap = {R(0), R(0), R(0)}, on_b = gap, nrm = gap, rel = gap;
        R share = R(0);
        for (uint32_t k = vtri_off[i]; k <= vtri_off[i + 1]; k++) {
            V3<R> p[3] = {x, x, x};
            V3<R> pv[3] = {v, v, v};
            uint32_t own = 0, n = 1;
            if (k < vtri_off[i + 1]) {
                uint32_t tn = vtri[k];
                if (alive[tn] == 0u || ((vf.torn >> (k - vtri_off[i])) & 1u)) continue;
                const Tri& tri = tris[tn];
                uint32_t ids[3] = {tri.v0, tri.v1, tri.v2};
                for (uint32_t c = 0; c < 3; c++) {
                    if (ids[c] == i) {
                        own = c;
                    } else {
                        pv[c] = MV[ids[c]].xyz();
                        p[c] = MX[ids[c]].xyz() + sub * pv[c];
                    }
                }
                R longest = mx(distance(p[0], p[1]), mx(distance(p[1], p[2]), distance(p[2], p[0])));
                n = f2u(clampr(std::ceil(longest / b.shape.w), R(1), R(8)));
            }
            for (uint32_t a = 0; a <= n; a++) {
                for (uint32_t c = 0; c <= n - a; c++) {
                    V3<R> bary = v3(R(a), R(c), R(n - a - c)) / R(n);
                    R wi = bary[own];
                    if (wi <= R(0)) continue;
                    V3<R> s = bary.x * p[0] + bary.y * p[1] + bary.z * p[2];
                    V3<R> r = s - xb;
                    if (length(r) >= b.shape.z + band) continue;
                    V3<R> q = qrot(back, r);
                    R rho = std::sqrt(q.x * q.x + q.y * q.y);
                    Near near = nearest_surface(bi, V2<R>{q.z, rho});
                    if (near.depth <= best) continue;
                    V2<R> radial = rho > R(1e-9) ? V2<R>{q.x / rho, q.y / rho} : V2<R>{R(1), R(0)};
                    best = near.depth;
                    found = true;
                    on_b = qrot(b.q, V3<R>{radial.x * near.at.y, radial.y * near.at.y, near.at.x});
                    gap = on_b - r;
                    nrm = qrot(b.q, V3<R>{radial.x * near.n.y, radial.y * near.n.y, near.n.x});
                    share = wi / dot(bary, bary);
                    rel = bary.x * pv[0] + bary.y * pv[1] + bary.z * pv[2] - b.v.xyz() - cross(w, on_b);
                }
            }
        }
        if (!found) continue;
        R vn = dot(rel, nrm);
        V3<R> rel_t = rel - vn * nrm;
        R slide = length(rel_t);
        R dvn = R(0), jn = R(0);
        V3<R> j = {R(0), R(0), R(0)};
        bool holds = false;
        if (!wet) {
            dvn = mx(-vn, R(0));
            jn = m * dvn;
            j = -m * share * dvn * nrm;
        } else {
            R ln = dot(load, nrm);
            if (ln < R(0)) {
                dvn = -vn;
                jn = -ln * sub;
                j = mn(share, R(1)) * ln * sub * nrm;
                holds = true;
                held = true;
            } else if (best > R(0)) {
                dvn = mx(-vn, R(0));
            } else {
                continue;
            }
        }
        R stop = (slide > R(1e-9) && m > R(0)) ? mn(R(1), Kc::MU_JACKET() * jn / (m * slide)) : R(0);
        V3<R> dvt = -share * stop * rel_t;
        x = x + (share * gap + sub * dvt);
        v = v + (share * dvn * nrm + dvt);
        j = j - m * dvt;
        R nl = length(vf.n);
        if (holds && nl > R(0)) {
            R a = vf.area * R(1e6);
            V3<R> sx = (x - xb) * R(1e3) * a;
            for (int c = 0; c < 3; c++) {
#pragma omp atomic
                bullet_hit[bi * HIT_FIELDS + 6 + c] += to_fp(vf.n[c] / nl * a, Kc::FP_A());
#pragma omp atomic
                bullet_hit[bi * HIT_FIELDS + 9 + c] += to_fp(sx[c], Kc::FP_X());
            }
#pragma omp atomic
            bullet_hit[bi * HIT_FIELDS + 12] += to_fp(a, Kc::FP_A());
        }
        V3<R> jl = cross(on_b, j);
        for (int c = 0; c < 3; c++) {
#pragma omp atomic
            bullet_hit[bi * HIT_FIELDS + c] += to_fp(j[c], Kc::FP_J());
#pragma omp atomic
            bullet_hit[bi * HIT_FIELDS + 3 + c] += to_fp(jl[c], Kc::FP_L());
        }
    }
    return limit;
}

template <class R>
V2<R> Sim<R>::substep_one(int par, uint32_t i, uint32_t k) {
    const R BIG = Kc::BIG();
    R m = mem_mass[i];
    V4<R> x = mem_x[par][i];
    auto& XO = mem_x[1 - par];
    auto& VO = mem_v[1 - par];
    if (m == R(0)) {
        XO[i] = x;
        VO[i] = {R(0), R(0), R(0), R(0)};
        return {BIG, BIG};
    }
    const R hh = h();
    R sub = dt() / R(std::max(U.mem[1], 1u));
    R t_sub = now() - dt() + R(k + 1u) * sub;
    VertexForce vf = vertex_force(par, i);
    V2<R> limits = {std::sqrt(m / mx(vf.stiff, R(1e-30))), BIG};
    if (vf.tension > R(0)) limits.y = std::sqrt(R(U.fluid[0]) * hh * hh * hh / (R(4) * Kc::PI() * vf.tension));
    V3<R> grav = {R(U.gravity[0]), R(U.gravity[1]), R(U.gravity[2])};
    V3<R> f = vf.f + m * grav;
    V3<R> v = mem_v[par][i].xyz();
    R nl = length(vf.n);
    size_t first = (size_t)i * 6;
    bool held = mem_v[par][i].w > R(0);
    bool ow = on_water(i);
    R push = (ow && nl > R(0)) ? -dot(f, vf.n / mx(nl, R(1e-30))) : R(0);
    mem_push[i] = {held ? R(0) : push, vf.area};
    if (sub <= R(0)) {
        XO[i] = x;
        VO[i] = mem_v[par][i];
        return limits;
    }
    if (ow && nl > R(0)) {
        V3<R> n = vf.n / nl;
        V3<R> vw = mem_water[i].xyz();
        V3<R> rel = v - vw;
        V3<R> rel_t = rel - dot(rel, n) * n;
        V3<R> ft = f - dot(f, n) * n;
        R kk = std::sqrt(R(U.fluid[0]) * Kc::MU_WATER()) * vf.area;
        const V3<R> TAU[2] = {{R(2.0e-6), R(3.170e-5), R(5.024e-4)}, {R(7.962e-3), R(1.262e-1), R(2.0)}};
        const V3<R> LW[2] = {{R(573.42), R(158.41), R(38.750)}, {R(10.049), R(2.2387), R(0.9494)}};
        V3<R> e[2], g[2];
        for (int a = 0; a < 2; a++) {
            V3<R> ex = V3<R>{-sub, -sub, -sub} / TAU[a];
            e[a] = {mexp(ex.x), mexp(ex.y), mexp(ex.z)};
            g[a] = (V3<R>{R(1), R(1), R(1)} - e[a]) * TAU[a] / V3<R>{sub, sub, sub};
        }
        R lhs = m / sub + kk * (dot(LW[0], g[0]) + dot(LW[1], g[1]));
        V3<R> rhs = m / sub * rel_t + ft;
        V3<R> z[6];
        for (int j = 0; j < 6; j++) {
            z[j] = mem_layer[first + j].xyz();
            z[j] = z[j] - dot(z[j], n) * n;
        }
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 3; b++) rhs = rhs - kk * LW[a][b] * (e[a][b] * z[3 * a + b] - g[a][b] * rel_t);
        V3<R> rel_new = rhs / lhs;
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 3; b++) {
                V3<R> zz = e[a][b] * z[3 * a + b] + g[a][b] * (rel_new - rel_t);
                mem_layer[first + 3 * a + b] = {zz.x, zz.y, zz.z, R(0)};
            }
        v = vw + rel_new;
        if (held) v = v + dot(rel, n) * n;
    } else if (ow) {
        v = mem_water[i].xyz();
    } else {
        for (int j = 0; j < 6; j++) mem_layer[first + j] = {R(0), R(0), R(0), R(0)};
        V3<R> fa = {R(0), R(0), R(0)};
        if (nl > R(0)) {
            V3<R> n = vf.n / nl;
            fa = (gas_pressure_at(par, x.xyz() - hh * n) - gas_pressure_at(par, x.xyz() + hh * n)) * vf.area * n;
        }
        v = v + sub * (f + fa) / m;
    }
    V3<R> xx = x.xyz() + sub * v;
    bool wet = ow;
    held = held && wet;
    limits.x = mn(limits.x, rubber_contact(par, i, xx, v, m, f, vf, wet, held, t_sub, sub));
    mem_push[i].x = held ? R(0) : push;
    if (xx.y < R(0)) {
        R j = mx(-v.y, R(0));
        xx.y = R(0);
        v.y = mx(v.y, R(0));
        R s = std::sqrt(v.x * v.x + v.z * v.z);
        R keep = s > R(1e-9) ? mx(R(0), R(1) - R(U.rubber2[0]) * j / s) : R(0);
        v = {v.x * keep, v.y, v.z * keep};
    }
    XO[i] = {xx.x, xx.y, xx.z, x.w};
    VO[i] = {v.x, v.y, v.z, held ? R(1) : R(0)};
    return limits;
}

template <class R>
void Sim<R>::mem_substep(uint32_t k, int par) {
    R lo_x = Kc::BIG(), lo_y = Kc::BIG();
#pragma omp parallel for schedule(static) reduction(min : lo_x, lo_y)
    for (int64_t ii = 0; ii < (int64_t)Nv; ii++) {
        V2<R> l = substep_one(par, (uint32_t)ii, k);
        lo_x = mn(lo_x, l.x);
        lo_y = mn(lo_y, l.y);
    }
    for (uint32_t t = 0; t < Nt; t++)
        if (torn[t]) alive[t] = 0u, torn[t] = 0u;
    st.mem_dt = mn(st.mem_dt, lo_x);
    st.cap_dt = mn(st.cap_dt, lo_y);
}

template <class R>
void Sim<R>::air_substep(int par) {
    const uint32_t nb = n_blocks();
    const R hh = h();
    R lim_all = Kc::BIG();
#pragma omp parallel for schedule(static) reduction(min : lim_all)
    for (int64_t bb = 0; bb < (int64_t)nb; bb++) {
        uint32_t b = (uint32_t)bb;
        for (uint32_t li = 0; li < 64; li++) {
            uint32_t cell = b * 64 + li;
            Gas<R> g = read_gas(par, cell);
            if (!free_gas(cell)) {
                write_gas(1 - par, cell, g);
                continue;
            }
            Gas<R> f = no_gas();
            for (uint32_t d = 0; d < 3; d++) {
                Gas<R> lo = hll(across(par, cell, g, d, false), g, d);
                Gas<R> hi = hll(g, across(par, cell, g, d, true), d);
                f = {f.rho + hi.rho - lo.rho, f.m + hi.m - lo.m, f.e + hi.e - lo.e};
            }
            R k = dt() / R(std::max(U.mem[2], 1u)) / hh;
            Gas<R> n = floored(Gas<R>{g.rho - k * f.rho, g.m - k * f.m, g.e - k * f.e});
            write_gas(1 - par, cell, n);
            V3<R> u = n.m / n.rho;
            R p = gas_p(n);
            R c = std::sqrt(Kc::GAMMA() * p / n.rho);
            R limit = Kc::CFL_AIR() * hh / (std::fabs(u.x) + std::fabs(u.y) + std::fabs(u.z) + R(3) * c);
            lim_all = mn(lim_all, limit);
            if (std::fabs(p - Kc::P_ATM()) > R(10) || length(u) > R(0.05)) block_active[b] = 1u;
        }
    }
    if (nb > 0) st.air_dt = mn(st.air_dt, lim_all);
}

// ---- spray, g2p, fluid.wgsl:676-901 ------------------------------------------------------------
template <class R>
void Sim<R>::spray_update() {
    const uint32_t n = std::min(st.spray_count, spray_cap);
    const R step = dt();
    const V3<R> grav = {R(U.gravity[0]), R(U.gravity[1]), R(U.gravity[2])};
    const R rhow = R(U.fluid[0]);
    auto drag_cd = [](R re) {
        if (re < R(1e-4)) return R(24) / R(1e-4);
        return R(24) / re * (R(1) + R(0.15) * mpow(re, R(0.687))) + R(0.42) / (R(1) + R(42500) * mpow(re, R(-1.16)));
    };
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ii++) {
        Spray<R>& s = spray[ii];
        R r = s.pos.w;
        if (r <= R(0)) continue;
        R sp = length(s.vel.xyz());
        R re = R(2) * r * sp * Kc::RHO_AIR() / Kc::MU_AIR();
        R k = R(3) * Kc::RHO_AIR() * drag_cd(re) * sp / (R(8) * rhow * r);
        V3<R> v = (s.vel.xyz() + step * grav) / (R(1) + k * step);
        r = std::sqrt(mx(r * r - Kc::EVAPORATION() * step, R(0)));
        if (r < R(2.5e-6)) r = R(0);
        V3<R> pos = s.pos.xyz() + step * v;
        if (pos.y <= r) {
            landed[ii] = {pos.x, pos.z, r * mpow(s.vel.w, R(1) / R(3)), now()};
            r = R(0);
        }
        s.pos = {pos.x, pos.y, pos.z, r};
        s.vel = {v.x, v.y, v.z, s.vel.w};
    }
}

template <class R>
void Sim<R>::carve(V3<R>& x, V3<R>& v, uint32_t id) const {
    R t = now();
    R hand2 = Kc::R_HAND() * Kc::R_HAND() * h() * h();
    for (uint32_t bi = 0; bi < U.mem[3]; bi++) {
        V4<R> reach = bullets[bi].reach;
        if (reach.w <= R(0) || distance(x, reach.xyz()) > reach.w) continue;
        for (uint32_t k = 0; k < N_SEC; k++) {
            const Section<R>& s = sections[bi * N_SEC + k];
            R r2 = section_r2(s, t);
            if (s.b.w <= R(0) || r2 >= hand2) continue;
            V3<R> ab = s.b.xyz() - s.a.xyz();
            R f = dot(x - s.a.xyz(), ab) / mx(dot(ab, ab), R(1e-20));
            if (f < R(0) || f > R(1)) continue;
            V3<R> on = s.a.xyz() + f * ab;
            V3<R> d = x - on;
            if (dot(d, d) >= r2) continue;
            if (dot(d, d) < R(1e-14)) {
                uint32_t seed = hash3(id, st.step, k);
                R g0 = rnd_gauss(seed);
                R g1 = rnd_gauss(seed);
                R g2 = rnd_gauss(seed);
                d = cross(ab + R(1e-9), V3<R>{g0, g1, g2});
            }
            V3<R> dir = normalize(d);
            R r = std::sqrt(r2);
            x = on + dir * r;
            R wall = s.b.w / (R(2) * r);
            v = v + dir * mx(wall - dot(v, dir), R(0));
        }
    }
}

template <class R>
void Sim<R>::g2p() {
    const uint32_t nb = n_blocks();
    const R hh = h();
    const V3<R> org = origin();
    const R step = dt();
    const R spacing = R(U.fluid[3]);
    const R rhow = R(U.fluid[0]);
    const V3<R> lo = org + R(3.5) * hh;
    const V3<R> hi = org + (v3(R(U.dims[0]), R(U.dims[1]), R(U.dims[2])) - R(4.5)) * hh;
    const R r_thin = R(0.75) * spacing;
    const R t_thin = R(3) * std::sqrt(rhow * r_thin * r_thin * r_thin / Kc::SIGMA_W());
    const R cs = R(4) / (hh * hh);
    std::vector<std::vector<Breakup>> brk(nb);
    R fastest_all = R(0);
#pragma omp parallel
    {
        std::vector<R> tg(8 * TILE);
#pragma omp for schedule(dynamic, 8) reduction(max : fastest_all)
        for (int64_t bb = 0; bb < (int64_t)nb; bb++) {
            uint32_t b = (uint32_t)bb;
            const uint32_t* links = &block_nb[(size_t)b * 27];
            uint32_t count = block_start[b + 1] - block_start[b];
            if (count == 0) continue;
            for (uint32_t t = 0; t < TILE; t++) {
                uint32_t cell = tile_cell(links, t);
                bool water = cell != NONE && cfv(F_TYPE, cell) == Kc::WATER;
                for (uint32_t d = 0; d < 3; d++) {
                    R u = R(0), w = R(0);
                    if (cell != NONE) {
                        u = cfv(F_U + d, cell);
                        w = from_fp(accv(a_wt(d), cell), Kc::FP_W());
                    }
                    tg[a_mom(d) * TILE + t] = u;
                    tg[a_wt(d) * TILE + t] = w;
                }
                tg[A_PC * TILE + t] = water ? pressure_of(cell) : R(0);
                tg[A_WC * TILE + t] = water ? R(1) : R(0);
            }
            I3 corner = slot_coord(block_list[b]) * 4 - I3{1, 1, 1};
            uint32_t first = block_start[b];
            for (uint32_t k = 0; k < count; k++) {
                uint32_t i = sorted[first + k];
                Particle<R> p = P[i];
                V3<R> X = (p.pos.xyz() - org) / hh;
                auto gather = [&](V3<R> o, uint32_t fa, uint32_t fw) {
                    I3 base = vi(vfloor(X - o - R(0.5)));
                    V3<R> fx = X - o - vf<R>(base);
                    V3<R> wx = axis_weights(fx.x), wy = axis_weights(fx.y), wz = axis_weights(fx.z);
                    I3 tq = base - corner;
                    uint32_t t0 = (uint32_t)tq.x * 49u + (uint32_t)tq.y * 7u + (uint32_t)tq.z;
                    Gathered r = {R(0), {R(0), R(0), R(0)}, R(0)};
                    for (uint32_t a = 0; a < 3; a++)
                        for (uint32_t bq = 0; bq < 3; bq++)
                            for (uint32_t c = 0; c < 3; c++) {
                                R weight = wx[a] * wy[bq] * wz[c];
                                uint32_t t = t0 + a * 49u + bq * 7u + c;
                                R u = weight * tg[fa * TILE + t];
                                r.s += u;
                                // Fused multiply-adds, as the CUDA gather.
                                V3<R> d = v3(R(a), R(bq), R(c)) - fx;
                                r.g = {std::fma(u, d.x, r.g.x), std::fma(u, d.y, r.g.y), std::fma(u, d.z, r.g.z)};
                                r.w = std::fma(weight, tg[fw * TILE + t], r.w);
                            }
                    r.g = r.g * hh;
                    return r;
                };
                Gathered gu = gather({R(0), R(0.5), R(0.5)}, a_mom(0), a_wt(0));
                Gathered gv = gather({R(0.5), R(0), R(0.5)}, a_mom(1), a_wt(1));
                Gathered gw = gather({R(0.5), R(0.5), R(0)}, a_mom(2), a_wt(2));
                Gathered gp = gather({R(0.5), R(0.5), R(0.5)}, A_PC, A_WC);
                V3<R> v = {gu.s, gv.s, gw.s};
                R m_near = gu.w + gv.w + gw.w;
                V3<R> x = p.pos.xyz() + step * v;
                if (U.mem[3] > 0u) carve(x, v, i);
                bool escaped = x.x < lo.x || x.z < lo.z || x.x > hi.x || x.z > hi.z || x.y > hi.y;
                R fill = m_near / R(24);
                bool on_ground = x.y < R(1.5) * spacing;
                I3 oc = vi(vfloor(X)) - corner;
                uint32_t own_t = tile_cell(links, (uint32_t)oc.x * 49u + (uint32_t)oc.y * 7u + (uint32_t)oc.z);
                bool covered = own_t != NONE && accv(A_MA, own_t) > 0;
                R thin_age = (fill < R(0.45) && !on_ground && !covered) ? p.c1.w + step : R(0);
                if (escaped || (!covered && fill < R(0.2)) || thin_age > t_thin) {
                    if (on_ground)
                        ground_touch(x);
                    else
                        brk[b].push_back({x, v, i});
                    P[i].vel = {v.x, v.y, v.z, R(0)};
                    continue;
                }
                V3<R> xx = x, vv = v;
                if (xx.y < R(0.3) * spacing) {
                    xx.y = R(0.3) * spacing;
                    vv.y = mx(vv.y, R(0));
                }
                if (xx.y < R(0.7) * spacing) ground_touch(xx);
                P[i].pos = {xx.x, xx.y, xx.z, p.pos.w};
                P[i].vel = {vv.x, vv.y, vv.z, R(1)};
                V3<R> c0 = gu.g * cs, c1 = gv.g * cs, c2 = gw.g * cs;
                P[i].c0 = {c0.x, c0.y, c0.z, gp.w > R(1e-6) ? gp.s / gp.w : R(0)};
                P[i].c1 = {c1.x, c1.y, c1.z, thin_age};
                P[i].c2 = {c2.x, c2.y, c2.z, R(0)};
                fastest_all = mx(fastest_all, length(vv));
            }
        }
    }
    st.max_speed = mx(st.max_speed, fastest_all);
    // Break-ups in canonical order: block by block, sorted order within a block.
    const R hs = spacing;
    const R vol = hs * hs * hs;
    for (uint32_t b = 0; b < nb; b++) {
        for (const Breakup& e : brk[b]) {
            uint32_t firsts = st.spray_count;
            st.spray_count += 5u;
            if (firsts >= spray_cap) continue;
            uint32_t seed = hash3(st.step, e.id, 0xb4eau);
            R speed = length(e.v);
            R bd2 = Kc::WE_CRIT() * Kc::SIGMA_W() / (Kc::RHO_AIR() * mx(speed * speed, R(1e-4)));
            R d_med = mn(R(0.55) * hs, R(0.5) * bd2);
            R dd[4];
            R used = R(0);
            for (int k = 0; k < 4; k++) {
                dd[k] = clampr(d_med * mexp(R(0.5) * rnd_gauss(seed)), R(2e-5), R(1.24) * hs);
                used += R(0.5236) * dd[k] * dd[k] * dd[k];
            }
            R df = R(0.5) * d_med;
            bool fine = df < R(1e-4);
            R fit = mpow(vol / used, R(1) / R(3));
            R scale = fine ? mn(R(1), fit) : fit;
            bool stop = false;
            for (uint32_t k = 0; k < 4; k++) {
                uint32_t slot = firsts + k;
                if (slot >= spray_cap) {
                    stop = true;
                    break;
                }
                R dk = dd[k] * scale;
                R spread = std::sqrt(Kc::SIGMA_W() / (rhow * dk)) + R(0.05) * speed;
                R g0 = rnd_gauss(seed);
                R g1 = rnd_gauss(seed);
                R g2 = rnd_gauss(seed);
                V3<R> u = normalize(V3<R>{g0, g1, g2} + R(1e-6));
                R o0 = rnd(seed);
                R o1 = rnd(seed);
                R o2 = rnd(seed);
                V3<R> off = (V3<R>{o0, o1, o2} - R(0.5)) * hs;
                R rr = rnd(seed);
                V3<R> px = e.x + off;
                V3<R> pv = e.v + u * spread * rr;
                spray[slot] = {{px.x, px.y, px.z, R(0.5) * dk}, {pv.x, pv.y, pv.z, R(1)}, {R(0), R(0), R(0), now()}};
            }
            if (stop) continue;
            uint32_t slot = firsts + 4;
            if (slot >= spray_cap) continue;
            R nn = (vol - used * scale * scale * scale) / (R(0.5236) * df * df * df);
            spray[slot] = {{e.x.x, e.x.y, e.x.z, (fine && nn >= R(2)) ? R(0.5) * df : R(0)}, {e.v.x, e.v.y, e.v.z, mx(nn, R(2))}, {R(0), R(0), R(0), now()}};
        }
    }
}

// ---- one step, and the host's batch (src/sim.rs:553-648) ------------------------------------------
template <class R>
void Sim<R>::run_step() {
    begin_step();
    if (st.dt_ns == 0) return;
    clear_blocks();
    activate_blocks();
    p2g();
    air_carry();
    mem_splat();
    grid_prep();
    air_fill();
    bullet_step();
    bullet_apply();
    solve();
    project();
    extend();
    mem_sample();
    uint32_t n_mem = U.mem[1], n_air = U.mem[2];
    for (uint32_t i = 0; i < std::max(n_mem, n_air); i++) {
        if (i < n_mem) mem_substep(i, (int)(i % 2));
        if (i < n_air) air_substep((int)(i % 2));
    }
    spray_update();
    g2p();
}

static uint32_t substeps_for(float dt, float sub_dt) {
    float n = std::ceil(1.1f * dt / sub_dt);
    if (!std::isfinite(n)) return 2;
    uint32_t k = n <= 0.0f ? 0u : (n >= 4294967296.0f ? 0xffffffffu : (uint32_t)n);
    k = std::min(std::max(k, 2u), 256u);
    return (k + 1) / 2 * 2;
}

template <class R>
void Sim<R>::measure_rubber() {
    // A substep of no length (src/sim.rs:524-541).
    uint32_t save_dt = st.dt_ns;
    st.dt_ns = 0;
    mem_substep(0, 0);
    st.dt_ns = save_dt;
    float dtm = std::min((float)U.fluid[2], (float)st.cap_dt);
    hdr.substeps = substeps_for(dtm, (float)st.mem_dt);
    hdr.air_substeps = substeps_for(dtm, (float)st.air_dt);
}

template <class R>
void Sim<R>::run_batch(uint32_t n, uint32_t stop) {
    U.limits[2] = hdr.iters;
    U.limits[3] = stop;
    U.mem[1] = hdr.substeps;
    U.mem[2] = hdr.air_substeps;
    st.iters_max = 0;
    st.unconverged = 0;
    for (uint32_t k = 0; k < n; k++) run_step();
    hdr.unconverged += st.unconverged;
    uint32_t mxi = hdr.max_iters ? hdr.max_iters : 4096;
    if (st.unconverged > 0)
        hdr.iters = std::min(hdr.iters * 2, mxi);
    else if (st.iters_max > 0)
        hdr.iters = std::min(std::max(st.iters_max + st.iters_max / 4 + 2, std::min(8u, mxi)), mxi);
    hdr.substeps = substeps_for((float)st.dt_flow, (float)st.mem_dt_seen);
    hdr.air_substeps = substeps_for((float)st.dt_flow, (float)st.air_dt_seen);
}

struct Handle {
    int fp64 = 0;
    Sim<float>* f = nullptr;
    Sim<double>* d = nullptr;
    std::string err;
};

}  // namespace oracle

using namespace oracle;

extern "C" {

// Creates an oracle from a world blob. real64: FP64 arithmetic throughout. fp64_dots: solver
// inner products accumulated in FP64 (otherwise the reference's FP32 tree).
__attribute__((visibility("default"))) void* oracle_create(const void* blob, size_t len, int real64, int fp64_dots, char* err, size_t errcap) {
    Handle* h = new Handle;
    h->fp64 = real64;
    std::string e;
    bool ok;
    if (real64) {
        h->d = new Sim<double>;
        h->d->fp64_dots = fp64_dots != 0;
        ok = h->d->load(blob, len, e);
        if (ok && h->d->hdr.substeps == 0) h->d->measure_rubber();
    } else {
        h->f = new Sim<float>;
        h->f->fp64_dots = fp64_dots != 0;
        ok = h->f->load(blob, len, e);
        if (ok && h->f->hdr.substeps == 0) h->f->measure_rubber();
    }
    if (!ok) {
        if (err && errcap) snprintf(err, errcap, "%s", e.c_str());
        delete h->f;
        delete h->d;
        delete h;
        return nullptr;
    }
    return h;
}

__attribute__((visibility("default"))) void oracle_destroy(void* p) {
    Handle* h = (Handle*)p;
    if (!h) return;
    delete h->f;
    delete h->d;
    delete h;
}

// One batch of n steps stopping at stop_ns (Sim::run). Returns the steps that ran, or -1 on
// block overflow.
__attribute__((visibility("default"))) int oracle_step(void* p, uint32_t n, uint32_t stop) {
    Handle* h = (Handle*)p;
    uint32_t before, after, ovf;
    if (h->fp64) {
        before = h->d->st.step;
        h->d->run_batch(n, stop);
        after = h->d->st.step;
        ovf = h->d->st.overflow;
    } else {
        before = h->f->st.step;
        h->f->run_batch(n, stop);
        after = h->f->st.step;
        ovf = h->f->st.overflow;
    }
    if (ovf) return -1;
    return (int)(after - before);
}

// Snapshot as a world blob. Returns the size; copies when cap is large enough.
__attribute__((visibility("default"))) size_t oracle_snapshot(void* p, void* buf, size_t cap) {
    Handle* h = (Handle*)p;
    std::vector<uint8_t> v = h->fp64 ? h->d->save() : h->f->save();
    if (buf && cap >= v.size()) std::memcpy(buf, v.data(), v.size());
    return v.size();
}

// Intermediate buffers of the last step. what: 0 block list (u32), 1 sorted (u32),
// 2 block_start (u32, n+1), 3 acc (i32, 19 fields x n*64), 4 cf (f32, 11 x n*64),
// 5 block_nb (u32, 27 n), 6 air (f32, 5 x n*64). Returns the element count.
__attribute__((visibility("default"))) size_t oracle_get(void* p, int what, void* out, size_t cap_elems) {
    Handle* hd = (Handle*)p;
    auto run = [&](auto* s) -> size_t {
        uint32_t n = s->n_blocks();
        size_t cells = (size_t)n * 64;
        size_t count = 0;
        switch (what) {
            case 0: count = n; break;
            case 1: count = s->block_start[n]; break;
            case 2: count = (size_t)n + 1; break;
            case 3: count = ACC_FIELDS * cells; break;
            case 4: count = CELL_FIELDS * cells; break;
            case 5: count = (size_t)n * 27; break;
            case 6: count = 5 * cells; break;
            default: return 0;
        }
        if (!out || cap_elems < count) return count;
        uint32_t* u = (uint32_t*)out;
        float* f = (float*)out;
        switch (what) {
            case 0: std::memcpy(u, s->block_list.data(), n * 4); break;
            case 1: std::memcpy(u, s->sorted.data(), count * 4); break;
            case 2: std::memcpy(u, s->block_start.data(), count * 4); break;
            case 3:
                for (uint32_t fl = 0; fl < ACC_FIELDS; fl++) std::memcpy(u + fl * cells, s->acc.data() + (size_t)fl * s->cap_cells, cells * 4);
                break;
            case 4:
                for (uint32_t fl = 0; fl < CELL_FIELDS; fl++)
                    for (size_t c = 0; c < cells; c++) f[fl * cells + c] = (float)s->cf[(size_t)fl * s->cap_cells + c];
                break;
            case 5: std::memcpy(u, s->block_nb.data(), count * 4); break;
            case 6:
                for (uint32_t fl = 0; fl < 5; fl++)
                    for (size_t c = 0; c < cells; c++) f[fl * cells + c] = (float)s->air[0][(size_t)fl * s->cap_cells + c];
                break;
        }
        return count;
    };
    return hd->fp64 ? run(hd->d) : run(hd->f);
}

// Solver scalars of the last step as doubles: rz, alpha, beta, b_norm, r_norm, iterations.
__attribute__((visibility("default"))) void oracle_solver(void* p, double out[6]) {
    Handle* hd = (Handle*)p;
    auto run = [&](auto* s) {
        out[0] = s->st.rz, out[1] = s->st.alpha, out[2] = s->st.beta, out[3] = s->st.b_norm, out[4] = s->st.r_norm;
        out[5] = s->st.solve_iters;
    };
    hd->fp64 ? run(hd->d) : run(hd->f);
}

// The float transcendentals, for testing: fn 0 exp, 1 log, 2 sin, 3 cos, 4 asin, 5 pow(x, y).
__attribute__((visibility("default"))) void oracle_math(int fn, const float* x, const float* y, float* out, size_t n) {
    for (size_t i = 0; i < n; i++) {
        switch (fn) {
            case 0: out[i] = nm::exp_(x[i]); break;
            case 1: out[i] = nm::log_(x[i]); break;
            case 2: out[i] = nm::sin_(x[i]); break;
            case 3: out[i] = nm::cos_(x[i]); break;
            case 4: out[i] = nm::asin_(x[i]); break;
            case 5: out[i] = nm::pow_(x[i], y[i]); break;
            default: out[i] = NAN;
        }
    }
}

__attribute__((visibility("default"))) void oracle_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
    (void)n;
#endif
}

__attribute__((visibility("default"))) int oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
