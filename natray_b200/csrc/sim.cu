// The simulation on one B200: device state, the step as one CUDA graph, and the C ABI of
// include/natray.h that replaces the reference's wgpu dispatch (src/gpu.rs:60-214, src/sim.rs:
// 208-689).
//
// A step is ~30 kernels plus two per solver iteration and one or two per substep. The host
// never synchronises inside a batch: the step length, the block set, the solver's convergence
// and every dispatch size are decided on the device, as in the reference. The host captures
// one step into a CUDA graph per (solver iterations, rubber substeps, air substeps, precision)
// and launches it n times for a batch, then reads the state back once (src/sim.rs:585-648).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <condition_variable>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "capi_util.hpp"
#include "kernels_g2p.cuh"
#include "kernels_solve.cuh"
#include "kernels_grid.cuh"
#include "world.hpp"

namespace ntr {

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            return fail(NTR_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));           \
        }                                                                                          \
    } while (0)

struct GraphKey {
    uint32_t n_mem, n_air, fp64, size;
    bool operator<(const GraphKey& o) const {
        return std::tie(n_mem, n_air, fp64, size) < std::tie(o.n_mem, o.n_air, o.fp64, o.size);
    }
};

struct StepGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0;
};

// Makes `device` current for the rest of the calling scope and puts the thread's own current
// device back when the scope ends, so a call on a simulation or batch of another GPU leaves the
// caller's CUDA (or torch) context where it was.
struct DeviceScope {
    int saved = -1;
    bool ok = false;
    explicit DeviceScope(int device) {
        if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
        ok = saved == device || cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceScope() {
        int now = -1;
        if (saved >= 0 && cudaGetDevice(&now) == cudaSuccess && now != saved) cudaSetDevice(saved);
    }
};

// A one-scene step's default cap on P2G's and G2P's CTAs an SM. Each takes at most what an SM
// holds at once (P2G four, G2P six at 1M particles); five leaves G2P one CTA's registers short of
// that on every SM, where the rubber's substep and sampling CTAs run beside it instead of waiting
// for G2P's end: 0.524 -> 0.515 ms a step over the bench's 300 steps of the 1M scene (four: 0.524).
constexpr uint32_t SIM_BLOCK_CTAS = 5;

struct Sim {
    int device = 0;
    int sms = 148;
    uint32_t coop_ctas = 148;
    uint32_t p2g_occ = 1, g2p128_occ = 1, g2p256_occ = 1;  // DevFacts
    // The scene's size class for its launch grids: its block count at the last read-back with a
    // quarter to spare, rounded up to a power of two (0: not known yet, full grids).
    uint32_t size_class = 0;
    cudaError_t launch_err = cudaSuccess;
    cudaStream_t stream = nullptr;
    cudaStream_t aux = nullptr;   // the second stream of the step's forks
    cudaStream_t aux2 = nullptr;  // and the third (the air substeps)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_fork[3] = {nullptr, nullptr, nullptr}, ev_join[3] = {nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> ev_sub;  // per substep: the rubber's, the air's
    World host;  // header (params, host control) of the world; sections are not kept
    ntr_gpu_params U{};
    Dev D{};
    std::vector<void*> allocs;
    size_t device_bytes = 0;
    DevState* h_state = nullptr;  // pinned
    bool own_h_state = true;      // false: a batch slot's, kept across its scenes
    ntr_gpu_params* h_params = nullptr;  // pinned staging of the parameters a step call uploads
    std::map<GraphKey, StepGraph> graphs;
    uint64_t last_launches = 0;
    double last_ms = 0.0;
    double step_ms = 0.0;
    void* stats_mem = nullptr;  // ntr_sim_stats' scratch, allocated at its first call
    cudaEvent_t ev_out = nullptr;  // ntr_sim_pack_particles: the caller's stream waits on it
    uint32_t batch_steps = 0;  // ntr_sim_set_batch_steps: fixed steps per ntr_sim_advance batch (0: by time)
    uint32_t fp64 = 1;
    ntr_tuning tune{0u, 8u, SIM_BLOCK_CTAS, 0u};  // launch shapes (ntr_sim_set_tuning)
    bool own_streams = true;  // false: the streams, events and h_params are a batch slot's, kept across its scenes

    ~Sim() {
        DeviceScope scope(device);
        for (auto& kv : graphs) {
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
        }
        for (void* p : allocs) cudaFree(p);
        if (stats_mem) cudaFree(stats_mem);
        if (ev_out) cudaEventDestroy(ev_out);
        if (h_state && own_h_state) cudaFreeHost(h_state);
        for (cudaEvent_t e : ev_sub)
            if (e) cudaEventDestroy(e);
        if (!own_streams) return;
        if (h_params) cudaFreeHost(h_params);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (int k = 0; k < 3; k++) {
            if (ev_fork[k]) cudaEventDestroy(ev_fork[k]);
            if (ev_join[k]) cudaEventDestroy(ev_join[k]);
        }
        if (aux2) cudaStreamDestroy(aux2);
        if (aux) cudaStreamDestroy(aux);
        if (stream) cudaStreamDestroy(stream);
    }

    bool dry = false;  // allocate() only counts the bytes
    // When set, allocations are carved from this device region (a batch slot's, kept across the
    // scenes it holds) instead of made one by one: no cudaMalloc or cudaFree, which synchronise
    // the whole device, when a scene is admitted or retired.
    uint8_t* arena = nullptr;
    size_t arena_cap = 0, arena_used = 0;

    template <class T>
    ntr_status alloc(T*& p, size_t count) {
        void* q = nullptr;
        size_t bytes = (std::max<size_t>(count * sizeof(T), 16) + 255) & ~(size_t)255;
        if (dry) {
            device_bytes += bytes;
            p = nullptr;
            return NTR_OK;
        }
        if (arena) {
            if (arena_used + bytes > arena_cap) return fail(NTR_E_NOMEM, "the slot's device region is too small for the scene");
            p = (T*)(arena + arena_used);
            arena_used += bytes;
            device_bytes += bytes;
            return NTR_OK;
        }
        cudaError_t e = cudaMalloc(&q, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(NTR_E_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
        }
        allocs.push_back(q);
        device_bytes += bytes;
        p = (T*)q;
        return NTR_OK;
    }
};

static ntr_status check_device(int device) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(NTR_E_NODEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= n) return fail(NTR_E_INVALID, "device index out of range");
    return NTR_OK;
}

// What the library needs to know of a device, asked once per device (cudaGetDeviceProperties
// takes milliseconds, which a serving loop admitting scenes would pay every time).
struct DevFacts {
    int sms = 0, major = 0, minor = 0;
    uint32_t coop_ctas = 0;  // CTAs of a persistent solve that the device holds at once (at most 256)
    uint32_t coop_all = 0;   // CTAs of the solve the device holds at once, uncapped (a joint solve of many systems)
    // CTAs an SM holds at once of the one-scene P2G and G2P (of 128 and 256 threads), which hand
    // their blocks out from a counter: more than that only wait for the counter to run out.
    uint32_t p2g_occ = 1, g2p128_occ = 1, g2p256_occ = 1;
    bool known = false;
};
static ntr_status device_facts(int device, DevFacts& out) {
    static std::mutex mu;
    static DevFacts cache[64];
    if (device < 0 || device >= 64) return fail(NTR_E_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    DevFacts& f = cache[device];
    if (!f.known) {
        DeviceScope scope(device);
        if (!scope.ok) return fail(NTR_E_CUDA, "cudaSetDevice failed");
        CU(cudaDeviceGetAttribute(&f.sms, cudaDevAttrMultiProcessorCount, device));
        CU(cudaDeviceGetAttribute(&f.major, cudaDevAttrComputeCapabilityMajor, device));
        CU(cudaDeviceGetAttribute(&f.minor, cudaDevAttrComputeCapabilityMinor, device));
        if (f.major >= 10) {
            // The persistent solver's grid must be co-resident: at most what occupancy allows,
            // for the one-scene and the many-scene solve alike. CTA c owns the blocks c (mod 256)
            // (and c + G, ... with fewer CTAs): at most 256.
            int occ = 1 << 30, o = 0;
            CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_solve<true>, SOLVE_T, 0));
            occ = std::min(occ, o);
            CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_solve<false>, SOLVE_T, 0));
            occ = std::min(occ, o);
            CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_solve_batch<true>, SOLVE_T, 0));
            occ = std::min(occ, o);
            CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_solve_batch<false>, SOLVE_T, 0));
            occ = std::min(occ, o);
            f.coop_ctas = (uint32_t)std::min(256, f.sms * occ);
            f.coop_all = (uint32_t)(f.sms * occ);
            CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_p2g, P2G_T, 0));
            f.p2g_occ = (uint32_t)std::max(o, 1);
            CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_g2p<128>, 128, 0));
            f.g2p128_occ = (uint32_t)std::max(o, 1);
            CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_g2p<256>, 256, 0));
            f.g2p256_occ = (uint32_t)std::max(o, 1);
        }
        f.known = true;
    }
    out = f;
    return NTR_OK;
}

static uint32_t radix_passes_for(uint32_t cap) {
    // The key NONE sorts as 2^(8p) - 1, which no valid block index may reach.
    uint32_t p = 1;
    while (p < 4 && (uint64_t)cap >= (1ull << (8 * p))) p++;
    return p;
}

// ---- allocation and upload --------------------------------------------------------------------
static ntr_status allocate(Sim& S) {
    const ntr_world_header& h = S.host.h;
    Dev& D = S.D;
    D.Np = h.n_particles, D.Nv = h.n_verts, D.Nt = h.n_tris;
    D.cap_blocks = h.block_cap;
    D.cap_cells = h.block_cap * 64u;
    D.spray_cap = h.spray_cap;
    D.wet_res = h.wet_res;
    const size_t slots = (size_t)h.params.bdims[0] * h.params.bdims[1] * h.params.bdims[2];
    D.nwords = (uint32_t)((slots + 31) / 32);
    D.scan_ctas = (D.nwords + SCAN_T * SCAN_W - 1) / (SCAN_T * SCAN_W);
    D.n_tiles = (D.Np + RADIX_TILE - 1) / RADIX_TILE;
    if (D.n_tiles == 0) D.n_tiles = 1;
    D.radix_passes = radix_passes_for(D.cap_blocks);
    D.fp64_dots = S.fp64;
    D.bar_spins = BARRIER_SPINS;
    D.bar_skip = NONE;
    ntr_status r;
#define AL(p, n) \
    if ((r = S.alloc(p, n)) != NTR_OK) return r
    ntr_gpu_params* u;
    AL(u, 1);
    D.U = u;
    AL(D.st, 1);
    AL(D.pos, D.Np);
    AL(D.vel, D.Np);
    AL(D.c0, D.Np);
    AL(D.c1, D.Np);
    AL(D.c2, D.Np);
    for (int k = 0; k < 2; k++) {
        AL(D.mask[k], D.nwords);
        AL(D.prefix[k], D.nwords + 1);
        AL(D.block_list[k], D.cap_blocks);
    }
    AL(D.cta_sum, D.scan_ctas + 1);
    AL(D.pslot, D.Np);
    AL(D.key, D.Np);
    AL(D.key_alt, D.Np);
    AL(D.val_alt, D.Np);
    AL(D.key_sorted, D.Np);
    AL(D.sorted, D.Np);
    AL(D.hist, 256u * D.n_tiles);
    AL(D.hist2, 256u * D.n_tiles);
    AL(D.block_start, D.cap_blocks + 1);
    AL(D.block_nb, (size_t)D.cap_blocks * 27);
    AL(D.block_active, D.cap_blocks);
    AL(D.acc, (size_t)NTR_ACC_FIELDS * D.cap_cells);
    AL(D.cf, (size_t)NTR_CELL_FIELDS * D.cap_cells);
    AL(D.air[0], (size_t)NTR_AIR_FIELDS * D.cap_cells);
    AL(D.air[1], (size_t)NTR_AIR_FIELDS * D.cap_cells);
    AL(D.xsum, 2u * 256u * SOLVE_XQ);
    AL(D.spart, 3u * (size_t)D.cap_blocks);
    for (int k = 0; k < 2; k++) {
        AL(D.mem_x[k], D.Nv);
        AL(D.mem_v[k], D.Nv);
    }
    AL(D.mem_water, D.Nv);
    AL(D.mem_layer, (size_t)D.Nv * NTR_LAYER_MODES);
    AL(D.mem_push, D.Nv);
    AL(D.mem_mass, D.Nv);
    Tri* tris;
    AL(tris, D.Nt);
    D.tris = tris;
    AL(D.alive, D.Nt);
    AL(D.tri_rec, (size_t)D.Nt * 5);
    AL(D.vtri_off, D.Nv + 1);
    AL(D.vtri, h.n_vtri);
    AL(D.vtri_c, h.n_vtri);
    AL(D.bullets, NTR_MAX_SHOTS);
    float4* pat;
    AL(pat, NTR_MAX_SHOTS * NTR_MAX_PATCHES * 2);
    D.patches = pat;
    float2* ol;
    AL(ol, NTR_MAX_SHOTS * NTR_OUTLINE);
    D.outlines = ol;
    AL(D.sections, NTR_MAX_SHOTS * NTR_N_SEC);
    AL(D.bullet_hit, NTR_MAX_SHOTS * NTR_HIT_FIELDS);
    AL(D.bullet_prep, NTR_MAX_SHOTS * 4);
    AL(D.bullet_patch, NTR_MAX_SHOTS * NTR_MAX_PATCHES * 4);
    AL(D.pose_log, NTR_MAX_SHOTS * NTR_LOG_CAP * 3);
    AL(D.spray, (size_t)D.spray_cap * 3);
    AL(D.landed, D.spray_cap);
    AL(D.touch, (size_t)D.wet_res * D.wet_res);
    AL(D.brk_x, D.Np); AL(D.brk_v, D.Np);
    AL(D.brk_count, D.cap_blocks);
    AL(D.brk_off, D.cap_blocks);
    AL(D.tiles, (size_t)D.cap_blocks * 8 * TILE);
    AL(D.tile_ok, D.cap_blocks);
    AL(D.coltot, 256);
    AL(D.wnb, (size_t)D.cap_cells * 8);
#undef AL
    return NTR_OK;
}

// Writes the world's state (not its static scene) to the device.
static ntr_status upload_state(Sim& S, const World& w) {
    const ntr_world_header& h = w.h;
    Dev& D = S.D;
    // Particles: AoS of 20 floats to five float4 arrays.
    {
        std::vector<float4> a[5];
        for (auto& v : a) v.resize(D.Np);
        const float* p = w.as<float>(NTR_SEC_PARTICLES);
        for (uint32_t i = 0; i < D.Np; i++)
            for (int k = 0; k < 5; k++) a[k][i] = make_float4(p[20 * (size_t)i + 4 * k], p[20 * (size_t)i + 4 * k + 1], p[20 * (size_t)i + 4 * k + 2], p[20 * (size_t)i + 4 * k + 3]);
        float4* dst[5] = {D.pos, D.vel, D.c0, D.c1, D.c2};
        for (int k = 0; k < 5; k++) CU(cudaMemcpyAsync(dst[k], a[k].data(), (size_t)D.Np * 16, cudaMemcpyHostToDevice, S.stream));
    }
    CU(cudaMemcpyAsync(D.mem_x[0], w.sec[NTR_SEC_MEM_X].data(), (size_t)D.Nv * 16, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.mem_x[1], w.sec[NTR_SEC_MEM_X].data(), (size_t)D.Nv * 16, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.mem_v[0], w.sec[NTR_SEC_MEM_V].data(), (size_t)D.Nv * 16, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.mem_v[1], w.sec[NTR_SEC_MEM_V].data(), (size_t)D.Nv * 16, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.mem_water, w.sec[NTR_SEC_MEM_WATER].data(), (size_t)D.Nv * 16, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.mem_layer, w.sec[NTR_SEC_MEM_LAYER].data(), (size_t)D.Nv * 96, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.mem_push, w.sec[NTR_SEC_MEM_PUSH].data(), (size_t)D.Nv * 8, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.alive, w.sec[NTR_SEC_ALIVE].data(), (size_t)D.Nt * 4, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.bullets, w.sec[NTR_SEC_BULLETS].data(), w.sec[NTR_SEC_BULLETS].size(), cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.sections, w.sec[NTR_SEC_SECTIONS].data(), w.sec[NTR_SEC_SECTIONS].size(), cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.bullet_hit, w.sec[NTR_SEC_BULLET_HIT].data(), w.sec[NTR_SEC_BULLET_HIT].size(), cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.pose_log, w.sec[NTR_SEC_POSE_LOG].data(), w.sec[NTR_SEC_POSE_LOG].size(), cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemsetAsync(D.spray, 0, (size_t)D.spray_cap * 48, S.stream));
    CU(cudaMemsetAsync(D.landed, 0, (size_t)D.spray_cap * 16, S.stream));
    if (h.n_spray) {
        CU(cudaMemcpyAsync(D.spray, w.sec[NTR_SEC_SPRAY].data(), (size_t)h.n_spray * 48, cudaMemcpyHostToDevice, S.stream));
        CU(cudaMemcpyAsync(D.landed, w.sec[NTR_SEC_LANDED].data(), (size_t)h.n_spray * 16, cudaMemcpyHostToDevice, S.stream));
    }
    CU(cudaMemcpyAsync(D.touch, w.sec[NTR_SEC_TOUCH].data(), (size_t)D.wet_res * D.wet_res * 4, cudaMemcpyHostToDevice, S.stream));
    // Grid: the last step's blocks become the "current" ones of parity step & 1.
    CU(cudaMemsetAsync(D.acc, 0, (size_t)NTR_ACC_FIELDS * D.cap_cells * 4, S.stream));
    CU(cudaMemsetAsync(D.cf, 0, (size_t)NTR_CELL_FIELDS * D.cap_cells * 4, S.stream));
    CU(cudaMemsetAsync(D.air[0], 0, (size_t)NTR_AIR_FIELDS * D.cap_cells * 4, S.stream));
    CU(cudaMemsetAsync(D.air[1], 0, (size_t)NTR_AIR_FIELDS * D.cap_cells * 4, S.stream));
    CU(cudaMemsetAsync(D.block_active, 0, (size_t)D.cap_blocks * 4, S.stream));
    const int cur = (int)(h.state.step & 1u);
    const uint32_t nbp = h.n_blocks_prev;
    {
        std::vector<uint32_t> mask(D.nwords, 0u), prefix(D.nwords + 1, 0u);
        const uint32_t* bl = w.as<uint32_t>(NTR_SEC_BLOCKS_PREV);
        for (uint32_t b = 0; b < nbp; b++) {
            if (b > 0 && bl[b] <= bl[b - 1]) return fail(NTR_E_INVALID, "world blob block list is not ascending");
            if ((size_t)bl[b] >= (size_t)D.nwords * 32) return fail(NTR_E_INVALID, "world blob block slot out of range");
            mask[bl[b] >> 5] |= 1u << (bl[b] & 31u);
        }
        uint32_t run = 0;
        for (uint32_t k = 0; k < D.nwords; k++) {
            prefix[k] = run;
            run += __builtin_popcount(mask[k]);
        }
        prefix[D.nwords] = run;
        CU(cudaMemcpyAsync(D.mask[cur], mask.data(), (size_t)D.nwords * 4, cudaMemcpyHostToDevice, S.stream));
        CU(cudaMemcpyAsync(D.prefix[cur], prefix.data(), ((size_t)D.nwords + 1) * 4, cudaMemcpyHostToDevice, S.stream));
        CU(cudaMemsetAsync(D.mask[cur ^ 1], 0, (size_t)D.nwords * 4, S.stream));
        CU(cudaMemsetAsync(D.prefix[cur ^ 1], 0, ((size_t)D.nwords + 1) * 4, S.stream));
        if (nbp) {
            CU(cudaMemcpyAsync(D.block_list[cur], bl, (size_t)nbp * 4, cudaMemcpyHostToDevice, S.stream));
            CU(cudaMemcpyAsync(D.block_active, w.sec[NTR_SEC_BLOCK_ACTIVE].data(), (size_t)nbp * 4, cudaMemcpyHostToDevice, S.stream));
            const float* af = w.as<float>(NTR_SEC_AIR);
            for (uint32_t f = 0; f < NTR_AIR_FIELDS; f++)
                CU(cudaMemcpyAsync(D.air[0] + (size_t)f * D.cap_cells, af + (size_t)f * nbp * 64, (size_t)nbp * 64 * 4, cudaMemcpyHostToDevice, S.stream));
        }
    }
    DevState ds;
    std::memset(&ds, 0, sizeof ds);
    ds.step_budget = 0xFFFFFFFFu;
    ds.s = h.state;
    ds.s.n_blocks = nbp;
    ds.rz = h.state.rz, ds.alpha = h.state.alpha, ds.beta = h.state.beta, ds.b_norm = h.state.b_norm, ds.r_norm = h.state.r_norm;
    CU(cudaMemcpyAsync(D.st, &ds, sizeof ds, cudaMemcpyHostToDevice, S.stream));
    return NTR_OK;
}

static ntr_status upload_static(Sim& S, const World& w) {
    Dev& D = S.D;
    CU(cudaMemcpyAsync((void*)D.tris, w.sec[NTR_SEC_TRIS].data(), (size_t)D.Nt * 32, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.vtri_off, w.sec[NTR_SEC_VTRI_OFF].data(), ((size_t)D.Nv + 1) * 4, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync(D.vtri, w.sec[NTR_SEC_VTRI].data(), w.sec[NTR_SEC_VTRI].size(), cudaMemcpyHostToDevice, S.stream));
    {
        // Which corner of each of its triangles a vertex is: the first of v0, v1, v2 that it
        // equals (the order in which membrane.wgsl's vertex_force tests them).
        const uint32_t* off = w.as<uint32_t>(NTR_SEC_VTRI_OFF);
        const uint32_t* vt = w.as<uint32_t>(NTR_SEC_VTRI);
        const Tri* tr = w.as<Tri>(NTR_SEC_TRIS);
        const size_t n_vt = w.sec[NTR_SEC_VTRI].size() / 4;
        std::vector<uint8_t> corner(n_vt, 2);
        for (uint32_t i = 0; i < D.Nv; i++)
            for (uint32_t k = off[i]; k < off[i + 1] && k < n_vt; k++) {
                const uint32_t t = vt[k];
                if (t < D.Nt) corner[k] = tr[t].v0 == i ? 0 : tr[t].v1 == i ? 1 : 2;
            }
        if (n_vt) CU(cudaMemcpyAsync(D.vtri_c, corner.data(), n_vt, cudaMemcpyHostToDevice, S.stream));
    }
    CU(cudaMemcpyAsync(D.mem_mass, w.sec[NTR_SEC_MEM_MASS].data(), (size_t)D.Nv * 4, cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync((void*)D.patches, w.sec[NTR_SEC_PATCHES].data(), w.sec[NTR_SEC_PATCHES].size(), cudaMemcpyHostToDevice, S.stream));
    CU(cudaMemcpyAsync((void*)D.outlines, w.sec[NTR_SEC_OUTLINES].data(), w.sec[NTR_SEC_OUTLINES].size(), cudaMemcpyHostToDevice, S.stream));
    return NTR_OK;
}

// The parameters of a step call, through a pinned buffer so that the copy is an asynchronous
// DMA (the call before has read its state back, so the buffer is free).
static ntr_status push_params(Sim& S) {
    *S.h_params = S.U;
    CU(cudaMemcpyAsync((void*)S.D.U, S.h_params, sizeof(ntr_gpu_params), cudaMemcpyHostToDevice, S.stream));
    return NTR_OK;
}

static ntr_status read_state(Sim& S) {
    CU(cudaMemcpyAsync(S.h_state, S.D.st, sizeof(DevState), cudaMemcpyDeviceToHost, S.stream));
    CU(cudaStreamSynchronize(S.stream));
    return NTR_OK;
}

// The zero-length rubber substep that sizes the first step (src/sim.rs:524-541).
static ntr_status measure_rubber(Sim& S) {
    Dev& D = S.D;
    CU(cudaMemsetAsync(&D.st->s.dt_ns, 0, 4, S.stream));
    k_mem_tri<<<std::max((D.Nt + 255) / 256, 1u), 256, 0, S.stream>>>(D, 0);
    k_mem_substep<<<std::max((D.Nv + MEM_SUB_T - 1) / MEM_SUB_T, 1u), MEM_SUB_T, 0, S.stream>>>(D, 0, 0);
    CU(cudaGetLastError());
    ntr_status r = read_state(S);
    if (r != NTR_OK) return r;
    const ntr_state& s = S.h_state->s;
    float dtm = std::min(S.U.fluid[2], s.cap_dt);
    S.host.h.substeps = substeps_for(dtm, s.mem_dt);
    S.host.h.air_substeps = substeps_for(dtm, s.air_dt);
    return NTR_OK;
}

// ---- the step -----------------------------------------------------------------------------------
// Per-kernel device timing of the profiling mode, the reference's NATRAY_PROF
// (src/sim.rs:594-614, 670-689): an event after every launch of a step run outside the graph.
struct Prof {
    std::vector<cudaEvent_t> ev;
    std::vector<const char*> name;
    size_t next = 0;
    cudaError_t err = cudaSuccess;
    void mark(const char* n, cudaStream_t s) {
        if (next == ev.size()) {
            cudaEvent_t e;
            cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) {
                err = r;
                return;
            }
            ev.push_back(e);
            name.push_back(nullptr);
        }
        name[next] = n;
        cudaError_t r = cudaEventRecord(ev[next++], s);
        if (r != cudaSuccess) err = r;
    }
    ~Prof() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};
static ntr_status prof_report(Prof& prof, char* report, size_t cap, size_t* len);

// The pressure solve as one cooperative launch of `ctas` CTAs on `s`: of S alone (jobs == NULL),
// or of the `n_jobs` simulations whose pointer tables are at `jobs` on the device. Each job's
// barrier counter must be zero (the step resets it before the launch).
static uint64_t enqueue_solve(Sim& S, cudaStream_t s, const Dev* jobs, uint32_t n_jobs, bool fp64, Prof* prof, uint32_t ctas) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(SOLVE_T);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaError_t e;
    if (!jobs)
        e = fp64 ? cudaLaunchKernelEx(&cfg, k_solve<true>, S.D) : cudaLaunchKernelEx(&cfg, k_solve<false>, S.D);
    else
        e = fp64 ? cudaLaunchKernelEx(&cfg, k_solve_batch<true>, jobs, n_jobs) : cudaLaunchKernelEx(&cfg, k_solve_batch<false>, jobs, n_jobs);
    if (e != cudaSuccess) S.launch_err = e;
    if (prof) prof->mark(fp64 ? "k_solve<true>" : "k_solve<false>", s);
    return 1;
}

// Launch grids sized to the scene. The per-cell, per-block and solver kernels loop over their
// work, so any grid gives the same results, bit for bit; a scene of a few hundred blocks gets as
// many CTAs as its cells and blocks can use (a cell a thread, a block a CTA, a block a solver
// warp) instead of the GPU's worth its kernels would otherwise spend launching CTAs with nothing
// to do. The launch-shape tuning (ntr_sim_set_tuning) caps them.
struct Grids {
    uint32_t cell, p2g, g2p, solve;
    bool g2p_wide;  // G2P in CTAs of 256 threads (scenes under 300k particles), else 128
    uint32_t blk;   // CTAs of a scene's per-block kernels in a many-scene launch (a fixed stride)
};
static Grids launch_grids(const Sim& S) {
    const bool wide = S.D.Np < 300000u;
    const uint32_t per_sm = S.tune.block_ctas_per_sm;
    Grids g{(uint32_t)S.sms * S.tune.cell_ctas_per_sm, (uint32_t)S.sms * std::min(per_sm, S.p2g_occ),
            (uint32_t)S.sms * std::min(per_sm, wide ? S.g2p256_occ : S.g2p128_occ),
            S.tune.solve_ctas ? S.tune.solve_ctas : S.coop_ctas, wide, (uint32_t)S.sms * per_sm};
    const uint32_t nb = S.size_class;
    if (nb) {
        g.cell = std::max(1u, std::min(g.cell, (nb * 64u + 255u) / 256u));
        g.blk = std::max(1u, std::min(g.blk, nb));
        g.p2g = std::max(1u, std::min(g.p2g, nb));
        g.g2p = std::max(1u, std::min(g.g2p, nb));
        if (!S.tune.solve_ctas) g.solve = std::max(1u, std::min(g.solve, (nb + SOLVE_T / 32 - 1) / (SOLVE_T / 32)));
    }
    return g;
}
static uint32_t size_class_of(uint32_t n_blocks) {
    if (n_blocks == 0) return 0;
    uint32_t want = n_blocks + n_blocks / 4 + 1, c = 64;
    while (c < want && c < (1u << 30)) c <<= 1;
    return c;
}

// One step on stream `s`, with the side streams forked from and joined back into it.
static uint64_t enqueue_step(Sim& S, cudaStream_t s, uint32_t n_mem, uint32_t n_air, bool fp64, Prof* prof) {
    Dev& D = S.D;
    uint64_t n = 0;
    const Grids grids = launch_grids(S);
    const uint32_t G_cell = grids.cell;
    const uint32_t g_vert = (D.Nv + 255) / 256 ? (D.Nv + 255) / 256 : 1;
    const uint32_t g_tri = std::max((D.Nt + 127) / 128, 1u);  // k_mem_tri in CTAs of 128 (24.4 -> 22.9 us a step at 1M)
    const uint32_t n_shots = S.U.mem[3] ? S.U.mem[3] : 1;
#define L(kern, grid, block, ...)                       \
    do {                                                \
        kern<<<(grid), (block), 0, s>>>(__VA_ARGS__);   \
        n++;                                            \
        if (prof) prof->mark(#kern, s);                 \
    } while (0)
    // Independent work goes to a second stream: (in the profiling mode everything stays on one).
    cudaStream_t a = prof ? s : S.aux;
    auto fork = [&](int k) {
        if (a == s) return;
        cudaEventRecord(S.ev_fork[k], s);
        cudaStreamWaitEvent(a, S.ev_fork[k], 0);
    };
    auto join = [&](int k) {
        if (a == s) return;
        cudaEventRecord(S.ev_join[k], a);
        cudaStreamWaitEvent(s, S.ev_join[k], 0);
    };
#define LA(kern, grid, block, ...)                      \
    do {                                                \
        kern<<<(grid), (block), 0, a>>>(__VA_ARGS__);   \
        n++;                                            \
        if (prof) prof->mark(#kern, a);                 \
    } while (0)
    if (prof) prof->mark("start", s);
    L(k_begin_step, 1, 32, D);
    // The side stream clears the last step's sums while the blocks are found and the particles
    // sorted; it then splats the rubber and carries the air (which need the block set but touch
    // none of what the sort and P2G read or write).
    fork(0);
    LA(k_clear_acc, G_cell, 256, D);
    // The first rubber substep's triangle records need only the membrane as the last step left
    // it (nothing before that substep writes its positions or `alive`): made here, beside the
    // sort, instead of in the rubber's chain after the pressure solve.
    if (n_mem > 0) LA(k_mem_tri, g_tri, 128, D, 0);
    // The spray's flight reads only the spray, the step length and the spray count from before
    // this step's break-ups (k_spray_scan advances it): beside the sort too.
    LA(k_spray_update, G_cell, 256, D);
    L(k_clear_mask, std::max((D.nwords + 255) / 256, 1u), 256, D);
    L(k_mark, (uint32_t)(((uint64_t)warp_round(D.Np) + warp_round(D.cap_blocks) + warp_round(D.Nv) + 255) / 256), 256, D);
    L(k_scan_words_a, D.scan_ctas, SCAN_T, D);
    L(k_scan_words_b, D.scan_ctas, SCAN_T, D);
    if (a != s) {
        cudaEventRecord(S.ev_fork[1], s);
        cudaStreamWaitEvent(a, S.ev_fork[1], 0);
    }
    LA(k_mem_splat, g_vert, 256, D);
    LA(k_air_carry, G_cell, 256, D);
    // The sort: the keys with pass 0's histogram, then per pass the scan and the scatter; pass
    // 0's scatter counts pass 1's histogram, later passes (more than 65,535 blocks) count their own.
    L(k_keys_hist, D.n_tiles, KEYS_T, D);
    {
        const uint32_t P = D.radix_passes;
        const uint32_t* kin = D.key;
        const uint32_t* vin = nullptr;
        for (uint32_t p = 0; p < P; p++) {
            bool to_final = ((P - 1 - p) % 2) == 0;
            uint32_t* kout = to_final ? D.key_sorted : D.key_alt;
            uint32_t* vout = to_final ? D.sorted : D.val_alt;
            uint32_t* h = (p % 2 == 0) ? D.hist : D.hist2;
            if (p >= 2) L(k_radix_hist, D.n_tiles, RADIX_T, D, h, kin, 8u * p);
            L(k_radix_scan, 256, 256, D, h);
            L(k_radix_scatter, D.n_tiles, SCAT_T, D, h, kin, vin, kout, vout, 8u * p, (p == 0 && P > 1) ? D.hist2 : nullptr);
            kin = kout;
            vin = vout;
        }
    }
    L(k_block_bounds, (D.Np + 1 + 255) / 256, 256, D);
    L(k_p2g, grids.p2g, P2G_T, D);
    // The side stream (the rubber's splat, the air's carry) is long done by now; the gather of
    // the tiles and the cells' grid_prep then go in one pass.
    join(0);
    L(k_gather_prep, G_cell, 256, D);
    L(k_air_fill, G_cell, 256, D);
    L(k_bullet_prep, n_shots, 32, D);
    {
        const dim3 gp((NTR_MAX_PATCHES + BULLET_PW - 1) / BULLET_PW, n_shots);
        L(k_bullet_patch, gp, BULLET_PW * 32, D);
    }
    L(k_bullet_finish, n_shots, 256, D);
    L(k_bullet_apply, G_cell, 256, D);
    // (k_bullet_apply has set the pressure solve's grid barrier counter to zero.)
    n += enqueue_solve(S, s, nullptr, 1u, fp64, prof, grids.solve);
    L(k_project, G_cell, 256, D);
    L(k_extend_1, G_cell, 256, D);
    L(k_extend_2, G_cell, 256, D);
    // G2P shares nothing with the rubber and air substeps: they run side by side.
    // The rubber substeps on one side stream and the air substeps on another: rubber substep i
    // reads the air buffer that air substep i - 1 writes, and air substep i overwrites the one
    // rubber substep i - 1 reads, so substep i of the two runs side by side and each waits for
    // the other's substep i - 1.
    cudaStream_t a2 = prof ? s : S.aux2;
    const uint32_t n_sub = std::max(n_mem, n_air);
    if (a != s && S.ev_sub.size() < 2 * (size_t)n_sub) {
        while (S.ev_sub.size() < 2 * (size_t)n_sub) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) S.launch_err = cudaErrorMemoryAllocation;
            S.ev_sub.push_back(e);
        }
    }
    fork(1);
    if (a2 != s) {
        cudaEventRecord(S.ev_fork[2], s);
        cudaStreamWaitEvent(a2, S.ev_fork[2], 0);
    }
    LA(k_mem_sample, (uint32_t)(((uint64_t)D.Nv * 4 + 127) / 128), 128, D);
    for (uint32_t i = 0; i < n_sub; i++) {
        if (i < n_mem) {
            if (a != s && i >= 1 && i - 1 < n_air) cudaStreamWaitEvent(a, S.ev_sub[2 * (i - 1) + 1], 0);
            if (i > 0) LA(k_mem_tri, g_tri, 128, D, (int)(i % 2));
            LA(k_mem_substep, std::max((D.Nv + MEM_SUB_T - 1) / MEM_SUB_T, 1u), MEM_SUB_T, D, i, (int)(i % 2));
            if (a != s) cudaEventRecord(S.ev_sub[2 * i], a);
        }
        if (i < n_air) {
            if (a2 != s && i >= 1 && i - 1 < n_mem) cudaStreamWaitEvent(a2, S.ev_sub[2 * (i - 1)], 0);
            k_air_substep<<<G_cell, 256, 0, a2>>>(D, (int)(i % 2));
            n++;
            if (prof) prof->mark("k_air_substep", a2);
            if (a2 != s) cudaEventRecord(S.ev_sub[2 * i + 1], a2);
        }
    }
    // Past 300k particles the blocks outnumber the resident CTAs: smaller CTAs, more of them.
    if (!grids.g2p_wide)
        L(k_g2p<128>, grids.g2p, 128, D);
    else
        L(k_g2p<256>, grids.g2p, 256, D);
    // The break-ups' drops go into spray slots past the old count, which nothing on the side
    // streams touches: they follow G2P while the rubber and the air finish.
    L(k_spray_scan, 1, 1024, D);
    L(k_spray_emit, G_cell, 256, D);
    join(1);
    if (a2 != s) {
        cudaEventRecord(S.ev_join[2], a2);
        cudaStreamWaitEvent(s, S.ev_join[2], 0);
    }
#undef L
#undef LA
    return n;
}

// The step captured as a graph, cached by its shape.
static ntr_status get_graph(Sim& S, StepGraph*& out) {
    // The size class follows the block count the last read-back saw.
    if (S.h_state) S.size_class = size_class_of(std::max(S.h_state->s.n_blocks, S.h_state->s.n_blocks_prev));
    GraphKey key{S.host.h.substeps, S.host.h.air_substeps, S.fp64, S.size_class};
    auto it = S.graphs.find(key);
    if (it != S.graphs.end()) {
        out = &it->second;
        return NTR_OK;
    }
    // Bound the cache: a new shape replaces the oldest when there are many.
    if (S.graphs.size() >= 16) {
        auto victim = S.graphs.begin();
        cudaGraphExecDestroy(victim->second.exec);
        cudaGraphDestroy(victim->second.graph);
        S.graphs.erase(victim);
    }
    StepGraph g;
    S.launch_err = cudaSuccess;
    CU(cudaStreamBeginCapture(S.stream, cudaStreamCaptureModeThreadLocal));
    g.launches = enqueue_step(S, S.stream, key.n_mem, key.n_air, key.fp64 != 0, nullptr);
    cudaError_t le = cudaGetLastError();
    cudaError_t ce = cudaStreamEndCapture(S.stream, &g.graph);
    if (S.launch_err != cudaSuccess) le = S.launch_err;
    if (le != cudaSuccess) {
        if (g.graph) cudaGraphDestroy(g.graph);
        return fail(NTR_E_CUDA, std::string("kernel launch during capture: ") + cudaGetErrorString(le));
    }
    if (ce != cudaSuccess) return fail(NTR_E_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce));
    CU(cudaGraphInstantiate(&g.exec, g.graph, 0));
    auto res = S.graphs.emplace(key, g);
    out = &res.first->second;
    return NTR_OK;
}

// Sim::run (src/sim.rs:585-648).
static ntr_status run_batch(Sim& S, uint32_t n, uint32_t stop, uint32_t* taken, Prof* prof = nullptr) {
    ntr_world_header& h = S.host.h;
    S.U.limits[2] = h.iters;
    S.U.limits[3] = stop;
    S.U.mem[1] = h.substeps;
    S.U.mem[2] = h.air_substeps;
    ntr_status r = push_params(S);
    if (r != NTR_OK) return r;
    // The solver's most-iterations and out-of-iterations counters start from zero in every batch.
    CU(cudaMemsetAsync(&S.D.st->s.iters_max, 0, 8, S.stream));
    StepGraph* g = nullptr;
    if (!prof) {
        if ((r = get_graph(S, g)) != NTR_OK) return r;
    } else {
        S.size_class = size_class_of(std::max(S.h_state->s.n_blocks, S.h_state->s.n_blocks_prev));
    }
    const uint32_t before = S.h_state->s.step;
    uint64_t launches = 0;
    CU(cudaEventRecord(S.ev0, S.stream));
    if (prof) {
        S.launch_err = cudaSuccess;
        for (uint32_t k = 0; k < n; k++) launches += enqueue_step(S, S.stream, h.substeps, h.air_substeps, S.fp64 != 0, prof);
        CU(cudaGetLastError());
        CU(S.launch_err);
        CU(prof->err);
    } else {
        for (uint32_t k = 0; k < n; k++) CU(cudaGraphLaunch(g->exec, S.stream));
        launches = g->launches * n;
    }
    CU(cudaEventRecord(S.ev1, S.stream));
    if ((r = read_state(S)) != NTR_OK) return r;
    float ms = 0.0f;
    CU(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
    S.last_ms = ms;
    S.last_launches = launches;
    S.step_ms = n ? ms / n : 0.0;
    const ntr_state& s = S.h_state->s;
    if (taken) *taken = s.step - before;
    if (s.overflow) return fail(NTR_E_OVERFLOW, "the water needs more than " + std::to_string(h.block_cap) + " grid blocks");
    if (S.h_state->err) return fail(NTR_E_TIMEOUT, "a bounded device-side wait gave up");
    adapt_after_batch(h, s);
    return NTR_OK;
}

// A batch slot's streams and events, kept across the scenes it holds (creating them is a
// driver call each, which admitting a scene would otherwise pay).
struct SimHandles {
    cudaStream_t stream = nullptr, aux = nullptr, aux2 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_fork[3] = {nullptr, nullptr, nullptr}, ev_join[3] = {nullptr, nullptr, nullptr};
    ntr_gpu_params* h_params = nullptr;
};
static ntr_status make_handles(SimHandles& h) {
    CU(cudaMallocHost((void**)&h.h_params, sizeof(ntr_gpu_params)));
    CU(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&h.aux, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&h.aux2, cudaStreamNonBlocking));
    for (int k = 0; k < 3; k++) {
        CU(cudaEventCreateWithFlags(&h.ev_fork[k], cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&h.ev_join[k], cudaEventDisableTiming));
    }
    CU(cudaEventCreate(&h.ev0));
    CU(cudaEventCreate(&h.ev1));
    return NTR_OK;
}
static void free_handles(SimHandles& h) {
    if (h.h_params) cudaFreeHost(h.h_params);
    if (h.ev0) cudaEventDestroy(h.ev0);
    if (h.ev1) cudaEventDestroy(h.ev1);
    for (int k = 0; k < 3; k++) {
        if (h.ev_fork[k]) cudaEventDestroy(h.ev_fork[k]);
        if (h.ev_join[k]) cudaEventDestroy(h.ev_join[k]);
    }
    if (h.aux2) cudaStreamDestroy(h.aux2);
    if (h.aux) cudaStreamDestroy(h.aux);
    if (h.stream) cudaStreamDestroy(h.stream);
    h = SimHandles{};
}

static ntr_status create_from(const World& w, int device, Sim*& out, uint8_t* arena = nullptr, size_t arena_cap = 0,
                              DevState* h_state = nullptr, const SimHandles* borrowed = nullptr) {
    ntr_status r = check_device(device);
    if (r != NTR_OK) return r;
    DeviceScope scope(device);
    if (!scope.ok) return fail(NTR_E_CUDA, "cudaSetDevice failed");
    DevFacts f;
    if ((r = device_facts(device, f)) != NTR_OK) return r;
    if (f.major < 10) return fail(NTR_E_NODEVICE, "this library is built for sm_100a (B200); device is sm_" + std::to_string(f.major * 10 + f.minor));
    std::unique_ptr<Sim> S(new Sim);
    S->device = device;
    S->host.h = w.h;
    S->U = w.h.params;
    S->sms = f.sms;
    S->coop_ctas = f.coop_ctas;
    S->p2g_occ = f.p2g_occ, S->g2p128_occ = f.g2p128_occ, S->g2p256_occ = f.g2p256_occ;
    if (S->coop_ctas < 1) return fail(NTR_E_NODEVICE, "the device cannot hold a solver CTA");
    if (w.h.block_cap > 65535u) return fail(NTR_E_INVALID, "block_cap is at most 65535");
    SimHandles hs;
    if (borrowed) {
        hs = *borrowed;
        S->own_streams = false;
    } else if ((r = make_handles(hs)) != NTR_OK) {
        free_handles(hs);
        return r;
    }
    S->stream = hs.stream, S->aux = hs.aux, S->aux2 = hs.aux2, S->ev0 = hs.ev0, S->ev1 = hs.ev1, S->h_params = hs.h_params;
    for (int k = 0; k < 3; k++) S->ev_fork[k] = hs.ev_fork[k], S->ev_join[k] = hs.ev_join[k];
    if (h_state)
        S->h_state = h_state, S->own_h_state = false;
    else
        CU(cudaMallocHost((void**)&S->h_state, sizeof(DevState)));
    S->arena = arena, S->arena_cap = arena_cap;
    if ((r = allocate(*S)) != NTR_OK) return r;
    if ((r = upload_static(*S, w)) != NTR_OK) return r;
    if ((r = upload_state(*S, w)) != NTR_OK) return r;
    if ((r = push_params(*S)) != NTR_OK) return r;
    if ((r = read_state(*S)) != NTR_OK) return r;
    if (S->host.h.substeps == 0)
        if ((r = measure_rubber(*S)) != NTR_OK) return r;
    out = S.release();
    return NTR_OK;
}

// ---- snapshot -------------------------------------------------------------------------------------
static ntr_status snapshot(Sim& S, std::vector<uint8_t>& blob) {
    Dev& D = S.D;
    ntr_status r = read_state(S);
    if (r != NTR_OK) return r;
    World w;
    w.h = S.host.h;
    w.h.params = S.U;
    const DevState& ds = *S.h_state;
    w.h.state = ds.s;
    w.h.state.rz = (float)ds.rz, w.h.state.alpha = (float)ds.alpha, w.h.state.beta = (float)ds.beta;
    w.h.state.b_norm = (float)ds.b_norm, w.h.state.r_norm = (float)ds.r_norm;
    const uint32_t nb = std::min(ds.s.n_blocks, D.cap_blocks);
    w.h.n_blocks_prev = nb;
    w.h.n_spray = std::min(ds.s.spray_count, D.spray_cap);
    w.shape_sections();
    {
        std::vector<float4> a[5];
        float4* src[5] = {D.pos, D.vel, D.c0, D.c1, D.c2};
        for (int k = 0; k < 5; k++) {
            a[k].resize(D.Np);
            CU(cudaMemcpy(a[k].data(), src[k], (size_t)D.Np * 16, cudaMemcpyDeviceToHost));
        }
        float* p = w.as<float>(NTR_SEC_PARTICLES);
        for (uint32_t i = 0; i < D.Np; i++)
            for (int k = 0; k < 5; k++) std::memcpy(p + 20 * (size_t)i + 4 * k, &a[k][i], 16);
    }
    auto dl = [&](int sec, const void* src) -> ntr_status {
        if (!w.sec[sec].empty()) CU(cudaMemcpy(w.sec[sec].data(), src, w.sec[sec].size(), cudaMemcpyDeviceToHost));
        return NTR_OK;
    };
    if ((r = dl(NTR_SEC_MEM_X, D.mem_x[0])) || (r = dl(NTR_SEC_MEM_V, D.mem_v[0])) || (r = dl(NTR_SEC_MEM_MASS, D.mem_mass)) ||
        (r = dl(NTR_SEC_MEM_WATER, D.mem_water)) || (r = dl(NTR_SEC_MEM_LAYER, D.mem_layer)) || (r = dl(NTR_SEC_MEM_PUSH, D.mem_push)) ||
        (r = dl(NTR_SEC_TRIS, D.tris)) || (r = dl(NTR_SEC_ALIVE, D.alive)) || (r = dl(NTR_SEC_VTRI_OFF, D.vtri_off)) ||
        (r = dl(NTR_SEC_VTRI, D.vtri)) || (r = dl(NTR_SEC_BULLETS, D.bullets)) || (r = dl(NTR_SEC_PATCHES, D.patches)) ||
        (r = dl(NTR_SEC_OUTLINES, D.outlines)) || (r = dl(NTR_SEC_SECTIONS, D.sections)) || (r = dl(NTR_SEC_BULLET_HIT, D.bullet_hit)) ||
        (r = dl(NTR_SEC_POSE_LOG, D.pose_log)) || (r = dl(NTR_SEC_SPRAY, D.spray)) || (r = dl(NTR_SEC_LANDED, D.landed)) ||
        (r = dl(NTR_SEC_TOUCH, D.touch)))
        return r;
    const int cur = (int)(ds.s.step & 1u);
    if (nb) {
        CU(cudaMemcpy(w.sec[NTR_SEC_BLOCKS_PREV].data(), D.block_list[cur], (size_t)nb * 4, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(w.sec[NTR_SEC_BLOCK_ACTIVE].data(), D.block_active, (size_t)nb * 4, cudaMemcpyDeviceToHost));
        float* af = w.as<float>(NTR_SEC_AIR);
        for (uint32_t f = 0; f < NTR_AIR_FIELDS; f++)
            CU(cudaMemcpy(af + (size_t)f * nb * 64, D.air[0] + (size_t)f * D.cap_cells, (size_t)nb * 64 * 4, cudaMemcpyDeviceToHost));
    }
    blob = serialize(w);
    return NTR_OK;
}

}  // namespace ntr

using namespace ntr;

struct ntr_sim {
    Sim* s;
};

#define GUARD(sim)                                             \
    if (!(sim) || !(sim)->s) return fail(NTR_E_INVALID, "null simulation handle"); \
    Sim& S = *(sim)->s;                                        \
    DeviceScope device_scope_(S.device);                       \
    if (!device_scope_.ok) return fail(NTR_E_CUDA, "cudaSetDevice failed")

extern "C" {

NTR_API ntr_status ntr_sim_create_from_world(const void* blob, size_t len, int device, ntr_sim** out) {
    if (!blob || !out) return fail(NTR_E_INVALID, "null argument");
    World w;
    std::string err;
    if (!deserialize(blob, len, w, err)) return fail(NTR_E_INVALID, err);
    Sim* s = nullptr;
    ntr_status r = create_from(w, device, s);
    if (r != NTR_OK) return r;
    *out = new ntr_sim{s};
    clear_error();
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_create(const ntr_sim_params* p, int device, ntr_sim** out) {
    if (!p || !out) return fail(NTR_E_INVALID, "null argument");
    ntr_status r = check_device(device);
    if (r != NTR_OK) return r;
    World w;
    std::string err;
    if (!build_world(*p, w, err)) return fail(NTR_E_INVALID, err);
    Sim* s = nullptr;
    if ((r = create_from(w, device, s)) != NTR_OK) return r;
    *out = new ntr_sim{s};
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_destroy(ntr_sim* sim) {
    if (!sim) return NTR_OK;
    delete sim->s;
    delete sim;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_step(ntr_sim* sim, uint32_t n, uint32_t stop_ns, uint32_t* taken) {
    GUARD(sim);
    if (n == 0) {
        if (taken) *taken = 0;
        return NTR_OK;
    }
    return run_batch(S, n, stop_ns, taken);
}

NTR_API ntr_status ntr_sim_advance(ntr_sim* sim, double t_target, uint32_t budget, uint32_t* taken_out) {
    GUARD(sim);
    ntr_world_header& h = S.host.h;
    uint32_t taken = 0;
    if (!h.started) {
        if (t_target < h.t0) {
            h.t = std::max(t_target, h.t_start);
            if (taken_out) *taken_out = 0;
            return NTR_OK;
        }
        h.started = 1;
        h.t = h.t0;
    }
    const double span = std::min(t_target - h.t0, 4.0);
    const uint32_t stop = (uint32_t)std::llround(std::max(span, 0.0) * 1e9);
    ntr_status r = NTR_OK;
    while (taken < budget && S.h_state->s.t_ns < stop) {
        const ntr_state& s = S.h_state->s;
        uint32_t dt = s.free_dt_ns > 0 ? s.free_dt_ns : (uint32_t)(S.U.fluid[2] * 1e9f);
        if (dt == 0) dt = 1;
        size_t fit = S.step_ms > 0.0 ? (size_t)(4.0 / S.step_ms) : 1;
        if (S.batch_steps) fit = S.batch_steps;
        size_t want = (size_t)((stop - s.t_ns + dt - 1) / dt);
        size_t cap = std::min<size_t>(budget - taken, 256);
        cap = std::min(cap, std::max<size_t>(fit, 1));
        uint32_t n = (uint32_t)std::clamp<size_t>(want, 1, std::max<size_t>(cap, 1));
        uint32_t got = 0;
        if ((r = run_batch(S, n, stop, &got)) != NTR_OK) break;
        taken += got;
        if (got == 0) break;
    }
    h.t = h.t0 + (double)S.h_state->s.t_ns * 1e-9;
    if (taken_out) *taken_out = taken;
    return r;
}

NTR_API ntr_status ntr_sim_read_state(ntr_sim* sim, ntr_state* out) {
    GUARD(sim);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    ntr_status r = read_state(S);
    if (r != NTR_OK) return r;
    *out = S.h_state->s;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_info_get(ntr_sim* sim, ntr_sim_info* out) {
    GUARD(sim);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    const ntr_world_header& h = S.host.h;
    std::memset(out, 0, sizeof *out);
    out->n_particles = h.n_particles, out->n_verts = h.n_verts, out->n_tris = h.n_tris, out->n_shots = h.n_shots;
    for (int k = 0; k < 3; k++) out->dims[k] = S.U.dims[k], out->grid_origin[k] = S.U.origin[k];
    out->block_cap = h.block_cap, out->spray_cap = h.spray_cap;
    out->iters = h.iters, out->substeps = h.substeps, out->air_substeps = h.air_substeps;
    out->dx = h.dx, out->spacing = S.U.fluid[3];
    out->t = h.t, out->t_start = h.t_start, out->t0 = h.t0;
    out->device_bytes = S.device_bytes;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_buffer(ntr_sim* sim, ntr_buf which, void** dev_ptr, size_t* bytes) {
    GUARD(sim);
    Dev& D = S.D;
    const int cur = (int)(S.h_state->s.step & 1u);
    void* p = nullptr;
    size_t b = 0;
    switch (which) {
        case NTR_BUF_PARTICLES: p = D.pos, b = (size_t)D.Np * 80; break;
        case NTR_BUF_STATE: p = D.st, b = sizeof(ntr_state); break;
        case NTR_BUF_MEM_POS: p = D.mem_x[0], b = (size_t)D.Nv * 16; break;
        case NTR_BUF_TRIS: p = (void*)D.tris, b = (size_t)D.Nt * 32; break;
        case NTR_BUF_ALIVE: p = D.alive, b = (size_t)D.Nt * 4; break;
        case NTR_BUF_VTRI_OFF: p = D.vtri_off, b = ((size_t)D.Nv + 1) * 4; break;
        case NTR_BUF_VTRI: p = D.vtri, b = (size_t)S.host.h.n_vtri * 4; break;
        case NTR_BUF_SPRAY: p = D.spray, b = (size_t)D.spray_cap * 48; break;
        case NTR_BUF_TOUCH: p = D.touch, b = (size_t)D.wet_res * D.wet_res * 4; break;
        case NTR_BUF_LANDED: p = D.landed, b = (size_t)D.spray_cap * 16; break;
        case NTR_BUF_BLOCK_LIST: p = D.block_list[cur], b = (size_t)D.cap_blocks * 4; break;
        case NTR_BUF_SORTED: p = D.sorted, b = (size_t)D.Np * 4; break;
        case NTR_BUF_BLOCK_START: p = D.block_start, b = ((size_t)D.cap_blocks + 1) * 4; break;
        case NTR_BUF_ACC: p = D.acc, b = (size_t)NTR_ACC_FIELDS * D.cap_cells * 4; break;
        case NTR_BUF_CF: p = D.cf, b = (size_t)NTR_CELL_FIELDS * D.cap_cells * 4; break;
        case NTR_BUF_AIR: p = D.air[0], b = (size_t)NTR_AIR_FIELDS * D.cap_cells * 4; break;
        case NTR_BUF_BLOCK_NB: p = D.block_nb, b = (size_t)D.cap_blocks * 27 * 4; break;
        default: return fail(NTR_E_INVALID, "unknown buffer");
    }
    if (dev_ptr) *dev_ptr = p;
    if (bytes) *bytes = b;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_download(ntr_sim* sim, ntr_buf which, void* host, size_t bytes) {
    GUARD(sim);
    if (!host) return fail(NTR_E_INVALID, "null argument");
    void* p = nullptr;
    size_t b = 0;
    ntr_status r = ntr_sim_buffer(sim, which, &p, &b);
    if (r != NTR_OK) return r;
    if (which == NTR_BUF_PARTICLES) {
        // Five float4 arrays, each n_particles long.
        Dev& D = S.D;
        float4* src[5] = {D.pos, D.vel, D.c0, D.c1, D.c2};
        size_t each = (size_t)D.Np * 16;
        for (int k = 0; k < 5 && bytes > 0; k++) {
            size_t n = std::min(bytes, each);
            CU(cudaMemcpy((char*)host + k * each, src[k], n, cudaMemcpyDeviceToHost));
            bytes -= n;
        }
        return NTR_OK;
    }
    CU(cudaStreamSynchronize(S.stream));
    CU(cudaMemcpy(host, p, std::min(bytes, b), cudaMemcpyDeviceToHost));
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_snapshot(ntr_sim* sim, void* buf, size_t cap, size_t* len) {
    GUARD(sim);
    std::vector<uint8_t> blob;
    ntr_status r = snapshot(S, blob);
    if (r != NTR_OK) return r;
    if (len) *len = blob.size();
    if (buf) {
        if (cap < blob.size()) return fail(NTR_E_INVALID, "snapshot buffer too small");
        std::memcpy(buf, blob.data(), blob.size());
    }
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_restore(ntr_sim* sim, const void* blob, size_t len) {
    GUARD(sim);
    World w;
    std::string err;
    if (!deserialize(blob, len, w, err)) return fail(NTR_E_INVALID, err);
    const ntr_world_header& a = S.host.h;
    if (w.h.n_particles != a.n_particles || w.h.n_verts != a.n_verts || w.h.n_tris != a.n_tris || w.h.block_cap != a.block_cap ||
        w.h.spray_cap != a.spray_cap || w.h.wet_res != a.wet_res || std::memcmp(w.h.params.bdims, a.params.bdims, 16) != 0)
        return fail(NTR_E_INVALID, "world blob is of a different scene size");
    CU(cudaStreamSynchronize(S.stream));
    S.host.h = w.h;
    S.U = w.h.params;
    ntr_status r;
    if ((r = upload_static(S, w)) != NTR_OK) return r;
    if ((r = upload_state(S, w)) != NTR_OK) return r;
    if ((r = push_params(S)) != NTR_OK) return r;
    if ((r = read_state(S)) != NTR_OK) return r;
    if (S.host.h.substeps == 0)
        if ((r = measure_rubber(S)) != NTR_OK) return r;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_profile(ntr_sim* sim, uint32_t n, uint32_t stop_ns, char* report, size_t cap, size_t* len) {
    GUARD(sim);
    Prof prof;
    uint32_t taken = 0;
    ntr_status r = run_batch(S, n, stop_ns, &taken, &prof);
    if (r != NTR_OK) return r;
    return prof_report(prof, report, cap, len);
}

}  // extern "C"

namespace ntr {
// The profile's events as a report: per kernel name, its launches and device time.
static ntr_status prof_report(Prof& prof, char* report, size_t cap, size_t* len) {
    std::vector<std::string> order;
    std::map<std::string, std::pair<uint64_t, double>> acc;
    for (size_t i = 1; i < prof.next; i++) {
        if (std::strcmp(prof.name[i], "start") == 0) continue;
        float ms = 0.0f;
        CU(cudaEventElapsedTime(&ms, prof.ev[i - 1], prof.ev[i]));
        std::string k = prof.name[i];
        if (!acc.count(k)) order.push_back(k);
        acc[k].first += 1;
        acc[k].second += ms;
    }
    std::string out;
    char line[256];
    for (auto& k : order) {
        snprintf(line, sizeof line, "%s,%llu,%.6f\n", k.c_str(), (unsigned long long)acc[k].first, acc[k].second);
        out += line;
    }
    if (len) *len = out.size();
    if (report) {
        if (cap < out.size() + 1) return fail(NTR_E_INVALID, "report buffer too small");
        std::memcpy(report, out.c_str(), out.size() + 1);
    }
    return NTR_OK;
}
}  // namespace ntr

extern "C" {

NTR_API ntr_status ntr_sim_set_batch_steps(ntr_sim* sim, uint32_t n) {
    GUARD(sim);
    S.batch_steps = n;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_set_precision(ntr_sim* sim, int fp64_reductions) {
    GUARD(sim);
    S.fp64 = fp64_reductions ? 1u : 0u;
    S.D.fp64_dots = S.fp64;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_get_tuning(ntr_sim* sim, ntr_tuning* out) {
    GUARD(sim);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    *out = S.tune;
    if (!out->solve_ctas) out->solve_ctas = S.coop_ctas;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_set_tuning(ntr_sim* sim, const ntr_tuning* t) {
    GUARD(sim);
    if (!t) return fail(NTR_E_INVALID, "null argument");
    ntr_tuning n = *t;
    if (n.solve_ctas > S.coop_ctas) return fail(NTR_E_INVALID, "solve_ctas is at most " + std::to_string(S.coop_ctas) + " (co-resident) on this device");
    if (n.cell_ctas_per_sm > 64 || n.block_ctas_per_sm > 64) return fail(NTR_E_INVALID, "at most 64 CTAs per SM");
    if (!n.cell_ctas_per_sm) n.cell_ctas_per_sm = 8;
    if (!n.block_ctas_per_sm) n.block_ctas_per_sm = SIM_BLOCK_CTAS;
    n.pad = 0;
    CU(cudaStreamSynchronize(S.stream));
    S.tune = n;
    for (auto& kv : S.graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    S.graphs.clear();
    return NTR_OK;
}

// A coordinate search over the launch shapes: block kernels, then cell kernels, then the solve.
// Each candidate starts from the same state and takes one untimed step (its graph) and `steps`
// timed ones.
NTR_API ntr_status ntr_sim_autotune(ntr_sim* sim, uint32_t steps, ntr_tuning* best, double* best_ms) {
    GUARD(sim);
    if (steps == 0) return fail(NTR_E_INVALID, "steps must be positive");
    std::vector<uint8_t> blob;
    ntr_status r = snapshot(S, blob);
    if (r != NTR_OK) return r;
    ntr_tuning cur = S.tune;
    double cur_ms = 1e300;
    auto trial = [&](const ntr_tuning& t, double& ms) -> ntr_status {
        ntr_status q;
        if ((q = ntr_sim_restore(sim, blob.data(), blob.size())) != NTR_OK) return q;
        if ((q = ntr_sim_set_tuning(sim, &t)) != NTR_OK) return q;
        uint32_t got = 0;
        if ((q = run_batch(S, 1, 0xFFFFFFFFu, &got)) != NTR_OK) return q;
        if ((q = run_batch(S, steps, 0xFFFFFFFFu, &got)) != NTR_OK) return q;
        ms = got ? S.last_ms / got : 1e300;
        return NTR_OK;
    };
    if ((r = trial(cur, cur_ms)) != NTR_OK) return r;
    const uint32_t blocks[] = {4, 6, 12, 16}, cells[] = {4, 6, 12, 16};
    const uint32_t solves[] = {S.coop_ctas, S.coop_ctas / 2, (uint32_t)S.sms};
    for (uint32_t v : blocks) {
        ntr_tuning t = cur;
        t.block_ctas_per_sm = v;
        double ms;
        if ((r = trial(t, ms)) != NTR_OK) return r;
        if (ms < cur_ms) cur = t, cur_ms = ms;
    }
    for (uint32_t v : cells) {
        ntr_tuning t = cur;
        t.cell_ctas_per_sm = v;
        double ms;
        if ((r = trial(t, ms)) != NTR_OK) return r;
        if (ms < cur_ms) cur = t, cur_ms = ms;
    }
    for (uint32_t v : solves) {
        if (v == 0 || v > S.coop_ctas) continue;
        ntr_tuning t = cur;
        t.solve_ctas = v;
        double ms;
        if ((r = trial(t, ms)) != NTR_OK) return r;
        if (ms < cur_ms) cur = t, cur_ms = ms;
    }
    if ((r = ntr_sim_restore(sim, blob.data(), blob.size())) != NTR_OK) return r;
    if ((r = ntr_sim_set_tuning(sim, &cur)) != NTR_OK) return r;
    if (best) *best = cur;
    if (best_ms) *best_ms = cur_ms;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_test_barrier(ntr_sim* sim, uint32_t spins, uint32_t skip_cta) {
    GUARD(sim);
    CU(cudaStreamSynchronize(S.stream));
    S.D.bar_spins = spins ? spins : BARRIER_SPINS;
    S.D.bar_skip = skip_cta;
    // The kernels take the pointer table by value: the captured step graphs hold the old one.
    for (auto& kv : S.graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    S.graphs.clear();
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_work(ntr_sim* sim, uint64_t out[NTR_WORK_FIELDS], int reset) {
    GUARD(sim);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    static_assert(sizeof(DevState::work) == NTR_WORK_FIELDS * sizeof(uint64_t), "work counters");
    CU(cudaMemcpyAsync(out, &S.D.st->work[0], sizeof(DevState::work), cudaMemcpyDeviceToHost, S.stream));
    if (reset) CU(cudaMemsetAsync(&S.D.st->work[0], 0, sizeof(DevState::work), S.stream));
    CU(cudaStreamSynchronize(S.stream));
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_last_launches(ntr_sim* sim, uint64_t* launches, double* device_ms) {
    GUARD(sim);
    if (launches) *launches = S.last_launches;
    if (device_ms) *device_ms = S.last_ms;
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_pack_particles(ntr_sim* sim, void* dst, size_t bytes, void* stream) {
    GUARD(sim);
    if (!dst) return fail(NTR_E_INVALID, "null argument");
    if (bytes < (size_t)S.D.Np * 80) return fail(NTR_E_INVALID, "destination smaller than 80 bytes per particle");
    if ((uintptr_t)dst % 16) return fail(NTR_E_INVALID, "destination not 16-byte aligned");
    const uint32_t grid = (uint32_t)std::min<size_t>(((size_t)S.D.Np * 5 + 255) / 256, (size_t)S.sms * 16);
    k_pack_particles<<<std::max(grid, 1u), 256, 0, S.stream>>>(S.D, (float4*)dst);
    CU(cudaGetLastError());
    if (stream) {
        if (!S.ev_out) CU(cudaEventCreateWithFlags(&S.ev_out, cudaEventDisableTiming));
        CU(cudaEventRecord(S.ev_out, S.stream));
        CU(cudaStreamWaitEvent((cudaStream_t)stream, S.ev_out, 0));
    } else {
        CU(cudaStreamSynchronize(S.stream));
    }
    return NTR_OK;
}

NTR_API ntr_status ntr_sim_conservation(ntr_sim* sim, double out[8]) {
    GUARD(sim);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    double* d = nullptr;
    CU(cudaMallocAsync((void**)&d, 64, S.stream));
    CU(cudaMemsetAsync(d, 0, 64, S.stream));
    k_conservation<<<S.sms * 4, 256, 0, S.stream>>>(S.D, d);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out, d, 64, cudaMemcpyDeviceToHost, S.stream));
    CU(cudaFreeAsync(d, S.stream));
    CU(cudaStreamSynchronize(S.stream));
    return NTR_OK;
}

}  // extern "C"

// ---- the shared-memory atomic peak (ntr_probe_shared_atomics) -----------------------------------
// P2G makes 216 shared-memory atomic adds a particle. This kernel measures the rate the SMs
// sustain for them at their best: P2G's CTA shape (256 threads, its tile's 15.2 KB of shared
// memory, as many CTAs an SM as P2G runs), every lane of a warp on its own bank and node, integer adds in a chain of
// `iters` per lane whose sums are kept (so that none is optimised away).
namespace ntr {
__global__ void __launch_bounds__(256, 4) k_probe_shared_atomics(uint32_t iters, int32_t* out) {
    __shared__ int32_t tile[8 * 476];
    for (uint32_t t = threadIdx.x; t < 8 * 476; t += blockDim.x) tile[t] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    int32_t* mine = tile + (warp * 32u) % (8u * 476u - 32u) + lane;
    for (uint32_t k = 0; k < iters; k++) {
        atomicAdd(mine, (int32_t)k);
        atomicAdd(mine + 256, (int32_t)(k ^ lane));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t sum = 0;
        for (uint32_t t = 0; t < 8 * 476; t++) sum += tile[t];
        out[blockIdx.x] = sum;
    }
}
}  // namespace ntr

extern "C" NTR_API ntr_status ntr_probe_shared_atomics(int device, uint32_t iters, double* lane_atomics_per_s) {
    using namespace ntr;
    if (!lane_atomics_per_s || iters == 0) return fail(NTR_E_INVALID, "null argument or no iterations");
    ntr_status r = check_device(device);
    if (r != NTR_OK) return r;
    DeviceScope scope(device);
    if (!scope.ok) return fail(NTR_E_CUDA, "cudaSetDevice failed");
    DevFacts f;
    if ((r = device_facts(device, f)) != NTR_OK) return r;
    const uint32_t grid = (uint32_t)f.sms * f.p2g_occ;  // P2G's CTAs an SM
    int32_t* out = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CU(cudaMallocAsync((void**)&out, sizeof(int32_t) * grid, s));
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    k_probe_shared_atomics<<<grid, 256, 0, s>>>(iters, out);  // warm-up
    CU(cudaEventRecord(e0, s));
    k_probe_shared_atomics<<<grid, 256, 0, s>>>(iters, out);
    CU(cudaEventRecord(e1, s));
    CU(cudaGetLastError());
    CU(cudaEventSynchronize(e1));
    float ms = 0.0f;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    cudaFreeAsync(out, s);
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    *lane_atomics_per_s = (double)grid * 256.0 * 2.0 * iters / (ms * 1e-3);
    return NTR_OK;
}

// ---- sorting by block without allocating (ntr_sort_by_block_noalloc) --------------------------
// For callers that cannot allocate device memory (a framework that has reserved the GPU's
// memory for its own pool, a frame loop that must not make the device-wide synchronising
// cudaMalloc/cudaFree calls): the step's stable radix sort, with its scratch in the file-scope
// device array below instead of a simulation's buffers. The array holds a small state record
// (the kernels' early-exit check and block count), the digit totals, the digit-major
// histogram, and the keys and values between passes. The kernels are the step's own, given a
// pointer table into this array.
namespace ntr {
constexpr size_t NOALLOC_TILES = (NTR_NOALLOC_MAX_KEYS + RADIX_TILE - 1) / RADIX_TILE;
constexpr size_t NOALLOC_STATE_WORDS = 64;
constexpr size_t NOALLOC_OFF_COLTOT = NOALLOC_STATE_WORDS;
constexpr size_t NOALLOC_OFF_HIST = NOALLOC_OFF_COLTOT + 256;
constexpr size_t NOALLOC_OFF_KEY_ALT = NOALLOC_OFF_HIST + 256 * NOALLOC_TILES;
constexpr size_t NOALLOC_OFF_VAL_ALT = NOALLOC_OFF_KEY_ALT + NTR_NOALLOC_MAX_KEYS;
constexpr size_t NOALLOC_OFF_KEY_SORTED = NOALLOC_OFF_VAL_ALT + NTR_NOALLOC_MAX_KEYS;
constexpr size_t NOALLOC_WORDS = NOALLOC_OFF_KEY_SORTED + NTR_NOALLOC_MAX_KEYS;
static_assert(sizeof(DevState) <= NOALLOC_STATE_WORDS * 4, "the state record fits its slot");

// About 13 MB, held on every GPU that loads the library until the process exits.
static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_WORDS];

// Sets what the sort kernels read of the state: a live step (dt_ns != 0) and the block count.
// Everything else of the scratch is written whole by every call before it is read.
__global__ void k_noalloc_prepare(DevState* st, uint32_t n_blocks) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        st->s.dt_ns = 1u;
        st->s.n_blocks = n_blocks;
    }
}

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[64];  // per device: the scratch array's device address
}  // namespace ntr

extern "C" NTR_API ntr_status ntr_sort_by_block_noalloc(const uint32_t* keys, uint32_t n, uint32_t n_blocks, uint32_t* sorted,
                                                        uint32_t* block_start, void* stream) {
    using namespace ntr;
    if (n > NTR_NOALLOC_MAX_KEYS)
        return fail(NTR_E_INVALID, "ntr_sort_by_block_noalloc: " + std::to_string(n) + " keys, at most " + std::to_string(NTR_NOALLOC_MAX_KEYS));
    if (n_blocks > NTR_NOALLOC_MAX_BLOCKS)
        return fail(NTR_E_INVALID, "ntr_sort_by_block_noalloc: " + std::to_string(n_blocks) + " blocks, at most " +
                                       std::to_string(NTR_NOALLOC_MAX_BLOCKS));
    if ((n > 0 && (!keys || !sorted)) || !block_start) return fail(NTR_E_INVALID, "ntr_sort_by_block_noalloc: null device array");
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(NTR_E_INVALID, "ntr_sort_by_block_noalloc: device index out of range");
    void* base = nullptr;
    {
        // Once per device, with that device current. In host code the array's name is only a
        // host-side stand-in; the kernels need its device address.
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            cudaError_t e = cudaGetSymbolAddress(&g_noalloc_addr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_noalloc_addr[dev] = nullptr;
                return fail(NTR_E_CUDA, std::string("cudaGetSymbolAddress of the sort scratch: ") + cudaGetErrorString(e));
            }
        }
        base = g_noalloc_addr[dev];
    }
    uint32_t* w = static_cast<uint32_t*>(base);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Dev D{};
    D.st = reinterpret_cast<DevState*>(w);
    D.Np = n;
    D.cap_blocks = n_blocks;
    D.n_tiles = std::max<uint32_t>(1u, (n + RADIX_TILE - 1) / RADIX_TILE);
    D.coltot = w + NOALLOC_OFF_COLTOT;
    D.hist = w + NOALLOC_OFF_HIST;
    D.key_alt = w + NOALLOC_OFF_KEY_ALT;
    D.val_alt = w + NOALLOC_OFF_VAL_ALT;
    D.key_sorted = w + NOALLOC_OFF_KEY_SORTED;
    D.sorted = sorted;
    D.block_start = block_start;
    const uint32_t P = radix_passes_for(std::max<uint32_t>(n_blocks, 1u));
    k_noalloc_prepare<<<1, 32, 0, s>>>(D.st, n_blocks);
    const uint32_t* kin = keys;
    const uint32_t* vin = nullptr;
    for (uint32_t p = 0; p < P && n > 0; p++) {
        const bool to_final = ((P - 1 - p) % 2) == 0;
        uint32_t* kout = to_final ? D.key_sorted : D.key_alt;
        uint32_t* vout = to_final ? D.sorted : D.val_alt;
        k_radix_hist<<<D.n_tiles, RADIX_T, 0, s>>>(D, D.hist, kin, 8u * p);
        k_radix_scan<<<256, 256, 0, s>>>(D, D.hist);
        k_radix_scatter<<<D.n_tiles, SCAT_T, 0, s>>>(D, D.hist, kin, vin, kout, vout, 8u * p, nullptr);
        kin = kout;
        vin = vout;
    }
    k_block_bounds<<<(n + 1 + 255) / 256, 256, 0, s>>>(D);
    CU(cudaGetLastError());
    return NTR_OK;
}

// ---- batches of scenes (include/natray.h, ntr_batch_*) ------------------------------------------
#include "batch.cuh"

struct ntr_batch {
    Batch* b;
};

#define BGUARD(batch)                                                                   \
    if (!(batch) || !(batch)->b) return fail(NTR_E_INVALID, "null batch handle");        \
    Batch& B = *(batch)->b;                                                             \
    std::unique_lock<std::mutex> batch_lock_(B.mu);                                     \
    B.cv.wait(batch_lock_, [&] { return !B.in_flight; });                               \
    DeviceScope device_scope_(B.device);                                                \
    if (!device_scope_.ok) return fail(NTR_E_CUDA, "cudaSetDevice failed")

constexpr uint32_t BATCH_REJECTED = 0xfffffffeu;

extern "C" {

NTR_API ntr_status ntr_batch_create(int device, uint32_t max_scenes, uint64_t hbm_budget, ntr_batch** out) {
    if (!out) return fail(NTR_E_INVALID, "null argument");
    Batch* b = nullptr;
    ntr_status r = batch_create(device, max_scenes, hbm_budget, b);
    if (r != NTR_OK) return r;
    *out = new ntr_batch{b};
    return NTR_OK;
}

NTR_API ntr_status ntr_batch_destroy(ntr_batch* batch) {
    if (!batch) return NTR_OK;
    delete batch->b;
    delete batch;
    return NTR_OK;
}

NTR_API ntr_status ntr_batch_admit(ntr_batch* batch, const void* blob, size_t len, uint32_t n_steps, uint32_t* slot) {
    if (!batch || !batch->b) return fail(NTR_E_INVALID, "null batch handle");
    if (!blob || !slot) return fail(NTR_E_INVALID, "null argument");
    Batch& B = *batch->b;
    DeviceScope scope(B.device);
    if (!scope.ok) return fail(NTR_E_CUDA, "cudaSetDevice failed");
    return batch_admit_overlapped(B, blob, len, n_steps, *slot);
}

NTR_API ntr_status ntr_world_device_bytes(const void* blob, size_t len, uint64_t* bytes) {
    if (!blob || !bytes) return fail(NTR_E_INVALID, "null argument");
    World w;
    std::string err;
    if (!deserialize(blob, len, w, err)) return fail(NTR_E_INVALID, err);
    return world_device_bytes(w, *bytes);
}

NTR_API ntr_status ntr_batch_enqueue(ntr_batch* batch, const void* blob, size_t len, uint32_t n_steps, uint64_t* ticket) {
    if (!batch || !batch->b) return fail(NTR_E_INVALID, "null batch handle");
    if (!blob || !ticket) return fail(NTR_E_INVALID, "null argument");
    // The blob is checked and copied before the batch's lock is taken (a 1M-particle world is
    // about 93 MB), so a producer thread holds up the stepping thread only for the queue's push.
    {
        World w;
        std::string err;
        if (!deserialize(blob, len, w, err)) return fail(NTR_E_INVALID, err);
    }
    const uint8_t* p = static_cast<const uint8_t*>(blob);
    std::vector<uint8_t> copy(p, p + len);
    Batch& B = *batch->b;
    std::lock_guard<std::mutex> lock(B.mu);
    B.queue.push_back(Batch::Queued{B.next_ticket, std::move(copy), n_steps});
    *ticket = B.next_ticket++;
    return NTR_OK;
}

NTR_API ntr_status ntr_batch_ticket(ntr_batch* batch, uint64_t ticket, uint32_t* slot) {
    BGUARD(batch);
    if (!slot) return fail(NTR_E_INVALID, "null argument");
    auto it = B.placed.find(ticket);
    if (it != B.placed.end()) {
        if (it->second == BATCH_REJECTED) return fail(NTR_E_INVALID, "the queued scene could not be admitted");
        *slot = it->second;
        return NTR_OK;
    }
    for (const auto& q : B.queue)
        if (q.ticket == ticket) {
            *slot = NTR_BATCH_MAX;
            return NTR_OK;
        }
    return fail(NTR_E_INVALID, "unknown ticket");
}

NTR_API ntr_status ntr_batch_profile(ntr_batch* batch, uint32_t n, char* report, size_t cap, size_t* len) {
    BGUARD(batch);
    Prof prof;
    uint32_t active = 0;
    ntr_status r = batch_step(B, n, active, &prof);
    if (r != NTR_OK) return r;
    return prof_report(prof, report, cap, len);
}

NTR_API ntr_status ntr_batch_step(ntr_batch* batch, uint32_t n, uint32_t* active) {
    BGUARD(batch);
    // Queued scenes first, in order, as far as slots and memory allow.
    while (!B.queue.empty()) {
        Batch::Queued& q = B.queue.front();
        uint32_t slot = 0;
        const ntr_status r = batch_admit(B, q.blob.data(), q.blob.size(), q.n_steps, slot);
        if (r == NTR_E_BUSY) break;
        B.placed[q.ticket] = r == NTR_OK ? slot : BATCH_REJECTED;
        B.queue.pop_front();
    }
    uint32_t a = 0;
    ntr_status r = batch_step(B, n, a, nullptr, &batch_lock_);
    if (active) *active = a;
    return r;
}

NTR_API ntr_status ntr_batch_poll(ntr_batch* batch, uint32_t slot, ntr_batch_slot* out) {
    BGUARD(batch);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    if (slot >= B.max_scenes) return fail(NTR_E_INVALID, "slot out of range");
    std::memset(out, 0, sizeof *out);
    const BatchSlot& sl = B.slots[slot];
    if (!sl.sim) return NTR_OK;
    out->in_use = 1;
    out->finished = sl.done >= sl.target ? 1u : 0u;
    out->steps_done = sl.done, out->steps_target = sl.target;
    out->device_bytes = sl.sim->device_bytes;
    out->state = sl.sim->h_state->s;
    return NTR_OK;
}

NTR_API ntr_status ntr_batch_snapshot(ntr_batch* batch, uint32_t slot, void* buf, size_t cap, size_t* len) {
    BGUARD(batch);
    if (slot >= B.max_scenes || !B.slots[slot].sim) return fail(NTR_E_INVALID, "no scene in that slot");
    std::vector<uint8_t> blob;
    ntr_status r = snapshot(*B.slots[slot].sim, blob);
    if (r != NTR_OK) return r;
    if (len) *len = blob.size();
    if (!buf) return NTR_OK;
    if (cap < blob.size()) return fail(NTR_E_INVALID, "snapshot buffer too small");
    std::memcpy(buf, blob.data(), blob.size());
    return NTR_OK;
}

NTR_API ntr_status ntr_batch_retire(ntr_batch* batch, uint32_t slot) {
    BGUARD(batch);
    return batch_retire(B, slot);
}

NTR_API ntr_status ntr_batch_set_tuning(ntr_batch* batch, const ntr_tuning* t) {
    BGUARD(batch);
    if (!t) return fail(NTR_E_INVALID, "null argument");
    ntr_tuning n = *t;
    if (n.solve_ctas > B.ctas) return fail(NTR_E_INVALID, "solve_ctas is at most " + std::to_string(B.ctas) + " (co-resident) on this device");
    if (n.cell_ctas_per_sm > 64 || n.block_ctas_per_sm > 64) return fail(NTR_E_INVALID, "at most 64 CTAs per SM");
    if (!n.cell_ctas_per_sm) n.cell_ctas_per_sm = 8;
    if (!n.block_ctas_per_sm) n.block_ctas_per_sm = 8;
    n.pad = 0;
    B.tune = n;
    for (auto& sl : B.slots)
        if (sl.sim) sl.sim->tune = n;
    return NTR_OK;  // the step graph is captured again at the next step (the shapes are in its key)
}

NTR_API ntr_status ntr_batch_get_tuning(ntr_batch* batch, ntr_tuning* out) {
    BGUARD(batch);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    *out = B.tune;
    if (!out->solve_ctas) out->solve_ctas = B.ctas;
    return NTR_OK;
}

// A coordinate search over the batch's launch shapes, as ntr_sim_autotune's, on the batch's own
// scenes: each candidate takes one untimed batch step (its graph) and `steps` timed ones. The
// scenes are not put back: the tuning steps are steps of theirs (the results do not depend on
// the shapes). The batch keeps the fastest.
NTR_API ntr_status ntr_batch_autotune(ntr_batch* batch, uint32_t steps, ntr_tuning* best, double* best_ms) {
    if (!batch || !batch->b) return fail(NTR_E_INVALID, "null batch handle");
    if (steps == 0) return fail(NTR_E_INVALID, "steps must be positive");
    Batch& B = *batch->b;
    ntr_tuning cur;
    ntr_status r = ntr_batch_get_tuning(batch, &cur);
    if (r != NTR_OK) return r;
    auto trial = [&](const ntr_tuning& t, double& ms) -> ntr_status {
        ntr_status q;
        if ((q = ntr_batch_set_tuning(batch, &t)) != NTR_OK) return q;
        uint32_t active = 0;
        if ((q = ntr_batch_step(batch, 1, &active)) != NTR_OK) return q;
        const auto t0 = std::chrono::steady_clock::now();
        if ((q = ntr_batch_step(batch, steps, &active)) != NTR_OK) return q;
        ms = active ? std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / steps : 1e300;
        return NTR_OK;
    };
    double cur_ms = 1e300;
    if ((r = trial(cur, cur_ms)) != NTR_OK) return r;
    const uint32_t blocks[] = {4, 6, 12, 16}, cells[] = {4, 6, 12, 16};
    const uint32_t solves[] = {B.ctas * 7 / 8, B.ctas * 3 / 4, B.ctas / 2};
    for (uint32_t v : blocks) {
        ntr_tuning t = cur;
        t.block_ctas_per_sm = v;
        double ms;
        if ((r = trial(t, ms)) != NTR_OK) return r;
        if (ms < cur_ms) cur = t, cur_ms = ms;
    }
    for (uint32_t v : cells) {
        ntr_tuning t = cur;
        t.cell_ctas_per_sm = v;
        double ms;
        if ((r = trial(t, ms)) != NTR_OK) return r;
        if (ms < cur_ms) cur = t, cur_ms = ms;
    }
    for (uint32_t v : solves) {
        if (v == 0) continue;
        ntr_tuning t = cur;
        t.solve_ctas = v;
        double ms;
        if ((r = trial(t, ms)) != NTR_OK) return r;
        if (ms < cur_ms) cur = t, cur_ms = ms;
    }
    if ((r = ntr_batch_set_tuning(batch, &cur)) != NTR_OK) return r;
    if (best) *best = cur;
    if (best_ms) *best_ms = cur_ms;
    return NTR_OK;
}

NTR_API ntr_status ntr_batch_info_get(ntr_batch* batch, ntr_batch_info* out) {
    BGUARD(batch);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    std::memset(out, 0, sizeof *out);
    out->max_scenes = B.max_scenes;
    for (const auto& sl : B.slots)
        if (sl.sim) {
            out->in_use++;
            if (sl.done < sl.target) out->active++;
        }
    out->held_bytes = B.held, out->budget_bytes = B.budget, out->steps = B.steps;
    out->captures = B.captures, out->instantiations = B.instantiations;
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) == cudaSuccess) out->free_bytes = f;
    return NTR_OK;
}

}  // extern "C"

// ---- keyframe cache (include/natray.h, ntr_cache_*) ---------------------------------------------
#include "cache.cuh"

struct ntr_cache {
    Cache* c;
};

#define CGUARD(cache)                                                                   \
    if (!(cache) || !(cache)->c) return fail(NTR_E_INVALID, "null cache handle");        \
    Cache& C = *(cache)->c;                                                             \
    DeviceScope device_scope_(C.device);                                                \
    if (!device_scope_.ok) return fail(NTR_E_CUDA, "cudaSetDevice failed")

extern "C" {

NTR_API ntr_status ntr_cache_params_default(const ntr_sim_params* p, ntr_cache_params* out) {
    if (!p || !out) return fail(NTR_E_INVALID, "null argument");
    if (p->n_shots > NTR_MAX_SHOTS) return fail(NTR_E_INVALID, "too many shots");
    std::memset(out, 0, sizeof *out);
    out->page_bytes = 128ull << 20;
    out->pages = 16;
    out->t_end = 1.0;
    // t_hit of src/sim.rs:280-291: each shot's delay after the earliest, f32 difference in ms.
    float first = 3.4028235e38f;
    for (uint32_t k = 0; k < p->n_shots; k++) first = std::min(first, p->shots[k].delay_ms);
    out->n_arrivals = p->n_shots;
    for (uint32_t k = 0; k < p->n_shots; k++) out->arrivals[k] = (double)(p->shots[k].delay_ms - first) * 1e-3;
    return NTR_OK;
}

NTR_API uint64_t ntr_key_bytes(uint32_t n_particles, uint32_t n_verts, uint32_t n_tris, uint32_t spray, uint32_t live) {
    return key_bytes_of(n_particles, n_verts, n_tris, spray, live);
}

NTR_API double ntr_key_next_time(double t, const double* arrivals, uint32_t n_arrivals, double t_end, uint64_t free_bytes,
                                 uint64_t key_bytes) {
    if (!arrivals) n_arrivals = 0;
    return key_next_time(t, arrivals, n_arrivals, t_end, std::max<uint64_t>(free_bytes, 1), key_bytes);
}

static ntr_status cache_check_params(const ntr_cache_params* cp) {
    if (cp->pages == 0 || cp->page_bytes < 256) return fail(NTR_E_INVALID, "the keyframe pool needs at least one page of 256 bytes");
    if (cp->n_arrivals > NTR_MAX_SHOTS) return fail(NTR_E_INVALID, "too many arrivals");
    if (cp->page_bytes > (1ull << 40) / cp->pages) return fail(NTR_E_INVALID, "keyframe pool too large");
    return NTR_OK;
}

NTR_API ntr_status ntr_cache_create(ntr_sim* sim, const ntr_cache_params* cp, ntr_cache** out) {
    if (!out || !cp) return fail(NTR_E_INVALID, "null argument");
    *out = nullptr;
    GUARD(sim);
    ntr_status r = cache_check_params(cp);
    if (r != NTR_OK) return r;
    std::unique_ptr<Cache> c(new Cache);
    c->handle = sim, c->S = &S, c->device = S.device, c->P = *cp;
    c->pool_bytes = cp->page_bytes * cp->pages;
    if (cudaMalloc(&c->pool, c->pool_bytes) != cudaSuccess) {
        cudaGetLastError();
        c->pool = nullptr;
        return fail(NTR_E_NOMEM, "device allocation of the keyframe pool (" + std::to_string(c->pool_bytes) + " bytes) failed");
    }
    CU(cudaMallocHost(&c->h_counts, 16));
    for (cudaEvent_t& e : c->ev) CU(cudaEventCreate(&e));
    if ((r = cache_size_for(*c, S)) != NTR_OK) return r;
    if ((r = cache_restart(*c)) != NTR_OK) return r;
    *out = new ntr_cache{c.release()};
    return NTR_OK;
}

NTR_API ntr_status ntr_cache_rebuild(ntr_cache* cache, ntr_sim* sim) {
    CGUARD(cache);
    if (!sim || !sim->s) return fail(NTR_E_INVALID, "null simulation handle");
    if (sim->s->device != C.device) return fail(NTR_E_INVALID, "the simulation is on another device than the cache");
    C.handle = sim, C.S = sim->s;
    ntr_status r = cache_size_for(C, *C.S);
    if (r != NTR_OK) return r;
    return cache_restart(C);
}

NTR_API ntr_status ntr_cache_destroy(ntr_cache* cache) {
    if (!cache) return NTR_OK;
    delete cache->c;
    delete cache;
    return NTR_OK;
}

NTR_API ntr_status ntr_cache_bake(ntr_cache* cache, uint32_t max_steps, uint32_t* steps) {
    CGUARD(cache);
    return cache_bake(C, max_steps, steps);
}

NTR_API ntr_status ntr_cache_store(ntr_cache* cache) {
    CGUARD(cache);
    if (C.done) return NTR_OK;
    return cache_store(C);
}

NTR_API ntr_status ntr_cache_show(ntr_cache* cache, double t, int* changed) {
    CGUARD(cache);
    return cache_show(C, t, changed);
}

NTR_API ntr_status ntr_cache_info_get(ntr_cache* cache, ntr_cache_info* out) {
    CGUARD(cache);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    std::memset(out, 0, sizeof *out);
    out->keys = (uint32_t)C.keys.size(), out->done = C.done, out->full = C.full, out->shown_spray = C.shown_spray;
    out->used_bytes = C.used(), out->pool_bytes = C.pool_bytes, out->shown_id = C.shown_id;
    out->end = C.end(), out->next_t = C.next_t, out->shown = C.shown;
    return NTR_OK;
}

NTR_API ntr_status ntr_cache_last_times(ntr_cache* cache, double* index_ms, double* pack_ms, double* show_ms) {
    CGUARD(cache);
    float a = 0.f, b = 0.f, c = 0.f;
    if (C.stored) {
        CU(cudaEventSynchronize(C.ev[3]));
        CU(cudaEventElapsedTime(&a, C.ev[0], C.ev[1]));
        CU(cudaEventElapsedTime(&b, C.ev[2], C.ev[3]));
    }
    if (C.showed) {
        CU(cudaEventSynchronize(C.ev[5]));
        CU(cudaEventElapsedTime(&c, C.ev[4], C.ev[5]));
    }
    if (index_ms) *index_ms = a;
    if (pack_ms) *pack_ms = b;
    if (show_ms) *show_ms = c;
    return NTR_OK;
}

NTR_API ntr_status ntr_cache_key(ntr_cache* cache, uint32_t k, ntr_key_info* out) {
    CGUARD(cache);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    if (k >= C.keys.size()) return fail(NTR_E_INVALID, "keyframe index out of range");
    const KeyRec& r = C.keys[k];
    std::memset(out, 0, sizeof *out);
    out->t = r.t, out->offset = r.offset, out->bytes = r.bytes, out->page = r.page, out->spray = r.spray, out->live = r.live;
    return NTR_OK;
}

NTR_API ntr_status ntr_cache_key_buffer(ntr_cache* cache, uint32_t k, void** dev_ptr, size_t* bytes) {
    CGUARD(cache);
    if (k >= C.keys.size()) return fail(NTR_E_INVALID, "keyframe index out of range");
    if (dev_ptr) *dev_ptr = C.key_ptr(C.keys[k]);
    if (bytes) *bytes = C.keys[k].bytes;
    return NTR_OK;
}

static ntr_status cache_buffer(Cache& C, uint32_t which, void** p, size_t* b) {
    switch (which) {
        case NTR_SHOWN_PARTICLES: *p = C.shown_p, *b = (size_t)C.np * 32; break;
        case NTR_SHOWN_SPRAY: *p = C.shown_drops, *b = (size_t)C.spray_cap * 32; break;
        case NTR_SHOWN_MEM_POS: *p = C.shown_mem, *b = (size_t)C.nv * 16; break;
        case NTR_SHOWN_ALIVE: *p = C.shown_alive, *b = (size_t)C.nt * 4; break;
        case NTR_SHOWN_WET: *p = C.shown_wet, *b = (size_t)C.wet_res * C.wet_res * 4; break;
        case NTR_SHOWN_SPRAY_W: *p = C.spray_w, *b = (size_t)C.spray_cap * 8; break;
        default:
            if (which - NTR_SHOWN_COUNT >= C.keys.size()) return fail(NTR_E_INVALID, "unknown cache buffer");
            *p = C.key_ptr(C.keys[which - NTR_SHOWN_COUNT]), *b = C.keys[which - NTR_SHOWN_COUNT].bytes;
    }
    return NTR_OK;
}

NTR_API ntr_status ntr_cache_buffer(ntr_cache* cache, ntr_shown which, void** dev_ptr, size_t* bytes) {
    CGUARD(cache);
    if ((uint32_t)which >= NTR_SHOWN_COUNT) return fail(NTR_E_INVALID, "unknown shown buffer");
    void* p = nullptr;
    size_t b = 0;
    ntr_status r = cache_buffer(C, (uint32_t)which, &p, &b);
    if (r != NTR_OK) return r;
    if (dev_ptr) *dev_ptr = p;
    if (bytes) *bytes = b;
    return NTR_OK;
}

NTR_API ntr_status ntr_cache_download(ntr_cache* cache, uint32_t which, void* host, size_t bytes) {
    CGUARD(cache);
    if (!host && bytes) return fail(NTR_E_INVALID, "null argument");
    void* p = nullptr;
    size_t b = 0;
    ntr_status r = cache_buffer(C, which, &p, &b);
    if (r != NTR_OK) return r;
    if (bytes > b) return fail(NTR_E_INVALID, "download larger than the buffer");
    CU(cudaStreamSynchronize(C.S->stream));
    CU(cudaMemcpy(host, p, bytes, cudaMemcpyDeviceToHost));
    return NTR_OK;
}

}  // extern "C"

// ---- debug statistics (include/natray.h, ntr_sim_stats) -----------------------------------------
#include "stats.cuh"

extern "C" NTR_API ntr_status ntr_sim_stats(ntr_sim* sim, ntr_stats* out) {
    GUARD(sim);
    if (!out) return fail(NTR_E_INVALID, "null argument");
    Dev& D = S.D;
    cudaStream_t s = S.stream;
    const uint32_t n_cta_tri = std::max((D.Nt + 255u) / 256u, 1u);
    const size_t acc_bytes = (sizeof(StatsAcc) + 255) & ~(size_t)255;
    const size_t cand_bytes = ((size_t)n_cta_tri * 3 * sizeof(TensionCand) + 255) & ~(size_t)255;
    const size_t cell_bytes = (size_t)D.cap_cells * 4;
    if (!S.stats_mem) {
        if (cudaMalloc(&S.stats_mem, acc_bytes + cand_bytes + cell_bytes) != cudaSuccess) {
            cudaGetLastError();
            S.stats_mem = nullptr;
            return fail(NTR_E_NOMEM, "device allocation of the statistics' scratch failed");
        }
    }
    StatsAcc* A = (StatsAcc*)S.stats_mem;
    TensionCand* cand = (TensionCand*)((uint8_t*)S.stats_mem + acc_bytes);
    uint32_t* cells = (uint32_t*)((uint8_t*)S.stats_mem + acc_bytes + cand_bytes);
    ntr_status r = read_state(S);
    if (r != NTR_OK) return r;
    const uint32_t nb = std::min(S.h_state->s.n_blocks, D.cap_blocks);
    StatsAcc init{};
    for (int k = 0; k < 3; k++) init.lo[k] = init.mlo[k] = 0xffffffffu, init.hi[k] = init.mhi[k] = 0u;
    init.fill_min = init.plo = 0xffffffffu;
    CU(cudaMemcpyAsync(A, &init, sizeof init, cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(cells, 0, (size_t)nb * 64 * 4, s));
    k_stats_particles<<<std::max((D.Np + 255u) / 256u, 1u), 256, 0, s>>>(D, A, cells);
    k_stats_cells<<<std::max((nb * 64u + 255u) / 256u, 1u), 256, 0, s>>>(D, A, cells);
    k_stats_verts<<<std::max((D.Nv + 255u) / 256u, 1u), 256, 0, s>>>(D, A);
    k_stats_tris<<<n_cta_tri, 256, 0, s>>>(D, A, cand);
    CU(cudaGetLastError());
    StatsAcc a{};
    std::vector<TensionCand> c((size_t)n_cta_tri * 3);
    std::vector<DBullet> bl(NTR_MAX_SHOTS);
    CU(cudaMemcpyAsync(&a, A, sizeof a, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(c.data(), cand, c.size() * sizeof(TensionCand), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(bl.data(), D.bullets, bl.size() * sizeof(DBullet), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    float4 fast_p = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t fast_i = ~(uint32_t)(a.fastest & 0xffffffffull);
    if (a.water && fast_i < D.Np) CU(cudaMemcpy(&fast_p, D.pos + fast_i, 16, cudaMemcpyDeviceToHost));

    std::memset(out, 0, sizeof *out);
    const double dx = S.host.h.dx, dx3 = dx * dx * dx, spacing = 0.5 * dx;
    out->water = a.water, out->n_particles = D.Np;
    const double n = (double)std::max(a.water, 1u);
    for (int k = 0; k < 3; k++) {
        out->lo[k] = a.water ? fkey_inv(a.lo[k]) : 0.f, out->hi[k] = a.water ? fkey_inv(a.hi[k]) : 0.f;
        out->mean[k] = a.sum_x[k] / n, out->vmean[k] = a.sum_v[k] / n;
        out->mem_lo[k] = D.Nv ? fkey_inv(a.mlo[k]) : 0.f, out->mem_hi[k] = D.Nv ? fkey_inv(a.mhi[k]) : 0.f;
    }
    out->vmax = a.water ? fkey_inv((uint32_t)(a.fastest >> 32)) : 0.f;
    out->fastest[0] = fast_p.x, out->fastest[1] = fast_p.y, out->fastest[2] = fast_p.z;
    out->volume_l = (double)a.full_cells * dx3 * 1e3;
    out->inside_l = a.inside * 1e3;
    out->free_verts = a.free_verts, out->on_water = a.on_water, out->torn = a.torn;
    out->fill_min = a.free_verts ? fkey_inv(a.fill_min) : 0.f;
    out->fill_mean = a.free_verts ? (float)(a.fill_sum / (double)a.free_verts) : 0.f;
    out->rubber_vmax = D.Nv ? fkey_inv(a.rubber_vmax) : 0.f;
    // The three most tense over all CTAs' candidates: by tension, then by triangle.
    std::vector<TensionCand> best;
    for (const TensionCand& q : c)
        if (q.tri != NONE && q.tension >= 0.0) best.push_back(q);
    std::sort(best.begin(), best.end(), [](const TensionCand& x, const TensionCand& y) {
        return x.tension > y.tension || (x.tension == y.tension && x.tri < y.tri);
    });
    out->n_tension = (uint32_t)std::min<size_t>(best.size(), 3);
    for (uint32_t k = 0; k < out->n_tension; k++) {
        out->tension[k] = best[k].tension, out->tension_tri[k] = best[k].tri;
        out->stretch[k][0] = best[k].l1, out->stretch[k][1] = best[k].l2;
    }
    out->air_cells = a.air_cells, out->vapour_cells = a.vapour;
    out->gauge_lo = a.air_cells ? fkey_inv(a.plo) : 0.f, out->gauge_hi = a.air_cells ? fkey_inv(a.phi) : 0.f;
    out->air_umax = a.air_cells ? fkey_inv(a.umax) : 0.f;
    // Energies (src/sim.rs:847-857): a particle's mass is the water in its spacing cube.
    out->water_j = a.ke * (1000.0 * (spacing * spacing * spacing));
    const double cavity = (double)a.vapour * dx3;
    out->vapour_cm3 = cavity * 1e6, out->vapour_j = cavity * 101325.0;
    out->n_bullets = std::min<uint32_t>(S.U.mem[3], NTR_MAX_SHOTS);
    for (uint32_t k = 0; k < out->n_bullets; k++) {
        const DBullet& b = bl[k];
        ntr_stats_bullet& o = out->bullets[k];
        o.state = b.info.z, o.sections = b.info.w;
        o.x[0] = b.x.x, o.x[1] = b.x.y, o.x[2] = b.x.z;
        const float vx = b.v.x, vy = b.v.y, vz = b.v.z;
        const float vsq = vx * vx + vy * vy + vz * vz;
        o.speed = std::sqrt(vsq);
        // The axis: the body's z rotated by its orientation quaternion (x, y, z, w).
        const double qx = b.q.x, qy = b.q.y, qz = b.q.z, qw = b.q.w;
        const double ax = 2.0 * (qx * qz + qw * qy), ay = 2.0 * (qy * qz - qw * qx), az = 1.0 - 2.0 * (qx * qx + qy * qy);
        const double al = std::sqrt(ax * ax + ay * ay + az * az), vl = std::sqrt((double)vsq);
        const double cs = al > 0.0 && vl > 0.0 ? std::clamp((ax * vx + ay * vy + az * vz) / (al * vl), -1.0, 1.0) : 1.0;
        o.yaw_deg = (float)(std::acos(cs) * (180.0 / 3.14159265358979323846));
        const double spin = (ax * b.l.x + ay * b.l.y + az * b.l.z) / (double)b.shape.x;
        o.spin_rev_s = (float)(spin / (2.0 * 3.14159265358979323846));
        o.kinetic_j = 0.5 * (double)b.x.w * (double)vsq;
        out->bullets_j += o.kinetic_j;
    }
    return NTR_OK;
}
