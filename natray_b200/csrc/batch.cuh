// Batches of independent scenes on one GPU (include/natray.h, ntr_batch_*): the serving engine.
//
// Every admitted scene keeps its own device-resident state (a Sim in a slot's memory region).
// A batch step runs the step of EVERY scene with one launch per kernel: each launch gives each
// scene a contiguous range of its CTAs (the scene's own grid for that kernel, sized to the
// scene), and every CTA finds its scene's pointer table through a prefix table of first CTAs
// (Multi, multi_cta). The pressure systems of all scenes are solved by ONE cooperative launch
// that splits the GPU's CTAs over the scenes by their block counts (k_solve_batch). The launch
// sequence is the one-scene step's, on the same three streams, captured once as a CUDA graph
// for the batch's current scenes and shapes and replayed per step; scenes differ in their
// rubber and air substep counts (each scene's kernels skip the substeps past its own) and in
// how many steps they take in a call (each scene's step budget stops it, as a stop time would).
// A call moves its host data in one copy each way: the pointer tables, grid prefixes, each
// scene's parameters and step budget go up together (k_batch_begin puts the parameters and
// budgets in place), and k_batch_end gathers the scenes' states into one buffer that comes
// back. The host then adapts each scene's solver iterations and substeps as ntr_sim_step does,
// so a scene's results are those of the scene run alone with the same chunks of steps.
//
// Included at the end of sim.cu (it uses the Sim internals there).
#pragma once

#include <chrono>
#include <deque>

namespace ntr {

// The kinds of per-scene grids a step's launches use (enqueue_step's grid expressions).
enum GridKind { GK_ONE, GK_CELL, GK_WORDS, GK_MARK, GK_SCAN, GK_TILES, GK_RSCAN, GK_BOUNDS, GK_BLK, GK_SHOTS, GK_PATCH,
                GK_VERT, GK_VERT4, GK_TRI, GK_COUNT };

// A scene's parameters for a batch call (Sim::run sets the same before a one-scene call).
struct BatchJobIn {
    ntr_gpu_params U;
    uint32_t budget, pad[3];
};

// Each scene's parameters and step budget into place, and its solver counters of the call
// (iters_max, unconverged) cleared: one CTA a scene.
__global__ void k_batch_begin(const Dev* __restrict__ jobs, const BatchJobIn* __restrict__ in) {
    const Dev& D = jobs[blockIdx.x];
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&in[blockIdx.x].U);
    uint32_t* dst = reinterpret_cast<uint32_t*>(const_cast<ntr_gpu_params*>(D.U));
    for (uint32_t t = threadIdx.x; t < sizeof(ntr_gpu_params) / 4; t += blockDim.x) dst[t] = src[t];
    if (threadIdx.x == 0) {
        D.st->step_budget = in[blockIdx.x].budget;
        D.st->s.iters_max = 0u;
        D.st->s.unconverged = 0u;
    }
}

// After a call's steps: a scene parked for the end of the call gets its last step length back
// (its state is then what its own last step left, as after ntr_sim_step of its steps), its
// budget goes back to no limit, and its state is gathered into out[scene].
__global__ void k_batch_end(const Dev* __restrict__ jobs, DevState* __restrict__ out) {
    DevState* st = jobs[blockIdx.x].st;
    if (threadIdx.x == 0) {
        if (st->parked) {
            st->s.dt_ns = st->parked_dt;
            st->parked = 0u;
        }
        st->step_budget = 0xFFFFFFFFu;
    }
    __syncthreads();
    const uint32_t* src = reinterpret_cast<const uint32_t*>(st);
    uint32_t* dst = reinterpret_cast<uint32_t*>(out + blockIdx.x);
    for (uint32_t t = threadIdx.x; t < sizeof(DevState) / 4; t += blockDim.x) dst[t] = src[t];
}

struct BatchSlot {
    std::unique_ptr<Sim> sim;
    uint32_t target = 0, done = 0;
    // The slot's device region and pinned state buffer, kept across the scenes it holds; the
    // region grows (and only then is reallocated) when a scene needs more.
    uint8_t* arena = nullptr;
    size_t arena_cap = 0;
    DevState* h_state = nullptr;
    SimHandles hs;  // its scenes' streams and events, made at its first scene
    bool reserved = false;  // a scene is being created in it (ntr_batch_admit, outside the lock)
};

struct Batch {
    int device = 0;
    uint32_t max_scenes = 0;
    uint64_t budget = 0;   // bytes the batch may hold; 0: no limit
    uint64_t reserve = 0;  // free device memory that admission leaves
    uint64_t held = 0;
    uint64_t steps = 0;
    uint32_t ctas = 0;  // CTAs of the joint solve (every co-resident one)
    // Launch shapes of every scene's grids and the joint solve (ntr_batch_set_tuning): the
    // per-SM caps of the cell and transfer kernels, and the joint solve's CTAs (0: all).
    ntr_tuning tune{0u, 8u, 8u, 0u};
    std::vector<BatchSlot> slots;
    cudaStream_t solve_stream = nullptr;  // the batch step's main stream
    cudaStream_t aux = nullptr, aux2 = nullptr;  // its side streams (as a one-scene step's)
    cudaEvent_t ev_fork[3] = {nullptr, nullptr, nullptr}, ev_join[3] = {nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> ev_sub;
    // What a call sends up, in one buffer on each side (pinned on the host): the pointer tables
    // of the scenes in the current step's order, per kind of grid the scenes' first CTAs
    // (GK_COUNT x (max_scenes + 1)), and each scene's parameters; and what comes back: the
    // scenes' states.
    uint8_t* d_stage = nullptr;
    uint8_t* h_stage = nullptr;
    size_t off_first = 0, off_in = 0, stage_bytes = 0;
    Dev* d_jobs = nullptr;
    uint32_t* d_first = nullptr;
    BatchJobIn* d_in = nullptr;
    DevState* d_out = nullptr;
    DevState* h_out = nullptr;
    uint32_t n_jobs_cap = 0;
    uint32_t captures = 0;        // step graphs captured (a new set of scenes or shapes)
    uint32_t instantiations = 0;  // of them, those that needed a new executable graph
    // The captured step of the current scenes and shapes, and what it was captured for.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<uint32_t> graph_key;
    // Every call on the batch holds this lock: calls from several host threads take turns. A
    // batch step lets it go while it waits for the GPU (in_flight): then only admissions, which
    // touch free slots alone, may proceed; every other call waits for the step to end.
    std::mutex mu;
    std::condition_variable cv;
    bool in_flight = false;
    // Scenes queued by any thread (ntr_batch_enqueue), admitted in order at the start of the
    // next ntr_batch_step; where each ticket went (a slot, or BATCH_REJECTED).
    struct Queued {
        uint64_t ticket;
        std::vector<uint8_t> blob;
        uint32_t n_steps;
    };
    std::deque<Queued> queue;
    uint64_t next_ticket = 1;
    std::map<uint64_t, uint32_t> placed;

    ~Batch() {
        DeviceScope scope(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (int k = 0; k < 3; k++) {
            if (ev_fork[k]) cudaEventDestroy(ev_fork[k]);
            if (ev_join[k]) cudaEventDestroy(ev_join[k]);
        }
        for (cudaEvent_t e : ev_sub)
            if (e) cudaEventDestroy(e);
        if (aux) cudaStreamDestroy(aux);
        if (aux2) cudaStreamDestroy(aux2);
        for (auto& s : slots) {
            s.sim.reset();
            free_handles(s.hs);
            if (s.arena) cudaFree(s.arena);
            if (s.h_state) cudaFreeHost(s.h_state);
        }
        slots.clear();
        if (d_stage) cudaFree(d_stage);
        if (h_stage) cudaFreeHost(h_stage);
        if (d_out) cudaFree(d_out);
        if (h_out) cudaFreeHost(h_out);
        if (solve_stream) cudaStreamDestroy(solve_stream);
    }
};

// Device bytes a world would take as a Sim (the allocation of `allocate`, counted, not made).
static ntr_status world_device_bytes(const World& w, uint64_t& bytes) {
    Sim S;
    S.dry = true;
    S.host.h = w.h;
    S.U = w.h.params;
    ntr_status r = allocate(S);
    bytes = S.device_bytes;
    return r;
}

static ntr_status batch_create(int device, uint32_t max_scenes, uint64_t budget, Batch*& out) {
    ntr_status r = check_device(device);
    if (r != NTR_OK) return r;
    if (max_scenes == 0 || max_scenes > NTR_BATCH_MAX) return fail(NTR_E_INVALID, "max_scenes is 1.." + std::to_string(NTR_BATCH_MAX));
    DeviceScope scope(device);
    if (!scope.ok) return fail(NTR_E_CUDA, "cudaSetDevice failed");
    DevFacts f;
    if ((r = device_facts(device, f)) != NTR_OK) return r;
    if (f.major < 10) return fail(NTR_E_NODEVICE, "this library is built for sm_100a (B200)");
    // Each system of the joint solve takes at most 256 CTAs (the residues of the reference's
    // summation tree); together they may use every CTA the device holds at once.
    const uint32_t ctas = f.coop_all;
    // Every scene needs a CTA of the joint solve.
    if (max_scenes > ctas) return fail(NTR_E_INVALID, "max_scenes is at most " + std::to_string(ctas) + " on this device");
    std::unique_ptr<Batch> B(new Batch);
    B->device = device;
    B->max_scenes = max_scenes;
    B->ctas = ctas;
    B->budget = budget;
    B->reserve = (uint64_t)1 << 30;
    B->slots.resize(max_scenes);
    CU(cudaStreamCreateWithFlags(&B->solve_stream, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&B->aux, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&B->aux2, cudaStreamNonBlocking));
    for (int k = 0; k < 3; k++) {
        CU(cudaEventCreateWithFlags(&B->ev_fork[k], cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&B->ev_join[k], cudaEventDisableTiming));
    }
    for (auto& s : B->slots) {
        CU(cudaMallocHost((void**)&s.h_state, sizeof(DevState)));
    }
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    B->off_first = up16(sizeof(Dev) * max_scenes);
    B->off_in = up16(B->off_first + sizeof(uint32_t) * GK_COUNT * (max_scenes + 1));
    B->stage_bytes = B->off_in + sizeof(BatchJobIn) * max_scenes;
    CU(cudaMalloc((void**)&B->d_stage, B->stage_bytes));
    CU(cudaMallocHost((void**)&B->h_stage, B->stage_bytes));
    B->d_jobs = reinterpret_cast<Dev*>(B->d_stage);
    B->d_first = reinterpret_cast<uint32_t*>(B->d_stage + B->off_first);
    B->d_in = reinterpret_cast<BatchJobIn*>(B->d_stage + B->off_in);
    CU(cudaMalloc((void**)&B->d_out, sizeof(DevState) * max_scenes));
    CU(cudaMallocHost((void**)&B->h_out, sizeof(DevState) * max_scenes));
    B->n_jobs_cap = max_scenes;
    out = B.release();
    return NTR_OK;
}

// Picks and prepares a free slot for a scene of `need` device bytes (its region grown if it must
// be, its streams made): a free slot whose region already holds the scene (the smallest such),
// else the free slot with the largest region. Under the batch's lock.
static ntr_status batch_reserve(Batch& B, uint64_t need, uint32_t& slot) {
    uint32_t free_slot = NONE, fits = NONE;
    for (uint32_t i = 0; i < B.max_scenes; i++) {
        const BatchSlot& c = B.slots[i];
        if (c.sim || c.reserved) continue;
        if (c.arena_cap >= need && (fits == NONE || c.arena_cap < B.slots[fits].arena_cap)) fits = i;
        if (free_slot == NONE || c.arena_cap > B.slots[free_slot].arena_cap) free_slot = i;
    }
    if (fits != NONE) free_slot = fits;
    if (free_slot == NONE) return fail(NTR_E_BUSY, "every slot of the batch is in use");
    BatchSlot& sl = B.slots[free_slot];
    const uint64_t grow = need > sl.arena_cap ? need + need / 4 - sl.arena_cap : 0;  // 25 % headroom
    if (B.budget && B.held + grow > B.budget) return fail(NTR_E_BUSY, "the scene's " + std::to_string(need) + " bytes exceed the batch's budget now");
    if (grow) {
        // The free device memory is asked only when the slot's region must grow (the query
        // takes milliseconds).
        size_t free_b = 0, total_b = 0;
        CU(cudaMemGetInfo(&free_b, &total_b));
        if ((uint64_t)free_b < grow + B.reserve) return fail(NTR_E_BUSY, "the scene's " + std::to_string(need) + " bytes do not fit the free device memory now");
    }
    if (grow) {
        if (sl.arena) CU(cudaFree(sl.arena));
        B.held -= sl.arena_cap;
        sl.arena = nullptr, sl.arena_cap = 0;
        CU(cudaMalloc((void**)&sl.arena, need + need / 4));
        sl.arena_cap = need + need / 4;
        B.held += sl.arena_cap;
    }
    ntr_status r;
    if (!sl.hs.stream && (r = make_handles(sl.hs)) != NTR_OK) {
        free_handles(sl.hs);
        return r;
    }
    slot = free_slot;
    return NTR_OK;
}

// Admission with the batch's lock held throughout (the queued scenes of a batch step).
static ntr_status batch_admit(Batch& B, const void* blob, size_t len, uint32_t n_steps, uint32_t& slot) {
    CU(cudaSetDevice(B.device));
    World w;
    std::string err;
    if (!deserialize(blob, len, w, err)) return fail(NTR_E_INVALID, err);
    uint64_t need = 0;
    ntr_status r = world_device_bytes(w, need);
    if (r != NTR_OK) return r;
    uint32_t k = 0;
    if ((r = batch_reserve(B, need, k)) != NTR_OK) return r;
    BatchSlot& sl = B.slots[k];
    Sim* s = nullptr;
    if ((r = create_from(w, B.device, s, sl.arena, sl.arena_cap, sl.h_state, &sl.hs)) != NTR_OK) return r;
    s->tune = B.tune;
    sl.sim.reset(s);
    sl.target = n_steps;
    sl.done = 0;
    slot = k;
    return NTR_OK;
}

// Admission from any thread, beside a batch step: the world is checked and sized without the
// lock, a slot reserved under it, the scene created in the slot without it (its uploads and
// measuring substep on the slot's own stream, overlapping the step's work on the GPU), and the
// scene placed under it again. Only the reservation and the placing wait for the lock, which a
// batch step lets go while it waits for the GPU.
static ntr_status batch_admit_overlapped(Batch& B, const void* blob, size_t len, uint32_t n_steps, uint32_t& slot) {
    World w;
    std::string err;
    if (!deserialize(blob, len, w, err)) return fail(NTR_E_INVALID, err);
    uint64_t need = 0;
    ntr_status r = world_device_bytes(w, need);
    if (r != NTR_OK) return r;
    uint32_t k = 0;
    {
        std::lock_guard<std::mutex> lk(B.mu);
        if ((r = batch_reserve(B, need, k)) != NTR_OK) return r;
        B.slots[k].reserved = true;
    }
    BatchSlot& sl = B.slots[k];
    Sim* s = nullptr;
    r = create_from(w, B.device, s, sl.arena, sl.arena_cap, sl.h_state, &sl.hs);
    std::lock_guard<std::mutex> lk(B.mu);
    sl.reserved = false;
    if (r != NTR_OK) return r;
    s->tune = B.tune;
    sl.sim.reset(s);
    sl.target = n_steps;
    sl.done = 0;
    slot = k;
    return NTR_OK;
}

static ntr_status batch_retire(Batch& B, uint32_t slot) {
    if (slot >= B.max_scenes || !B.slots[slot].sim) return fail(NTR_E_INVALID, "no scene in that slot");
    CU(cudaSetDevice(B.device));
    B.slots[slot].sim.reset();  // the slot keeps its device region for the next scene
    B.slots[slot].target = B.slots[slot].done = 0;
    return NTR_OK;
}


static void scene_grids(const Sim& S, uint32_t g[GK_COUNT]) {
    const Dev& D = S.D;
    const Grids gr = launch_grids(S);
    g[GK_ONE] = 1;
    g[GK_CELL] = gr.cell;
    g[GK_WORDS] = std::max((D.nwords + 255) / 256, 1u);
    g[GK_MARK] = (uint32_t)(((uint64_t)warp_round(D.Np) + warp_round(D.cap_blocks) + warp_round(D.Nv) + 255) / 256);
    g[GK_SCAN] = D.scan_ctas;
    g[GK_TILES] = D.n_tiles;
    g[GK_RSCAN] = 256;
    g[GK_BOUNDS] = (D.Np + 1 + 255) / 256;
    g[GK_BLK] = gr.blk;
    g[GK_SHOTS] = S.U.mem[3] ? S.U.mem[3] : 1;
    g[GK_PATCH] = (NTR_MAX_PATCHES + BULLET_PW - 1) / BULLET_PW;
    g[GK_VERT] = (D.Nv + 255) / 256 ? (D.Nv + 255) / 256 : 1;
    g[GK_VERT4] = (uint32_t)(((uint64_t)D.Nv * 4 + 255) / 256);
    g[GK_TRI] = std::max((D.Nt + 255) / 256, 1u);
}

// The step of every scene of the batch, one launch per kernel over all of them: the launch
// sequence of enqueue_step (on the same three streams), with each scene's own grid within each
// launch. `tot` is each kind's CTAs over all scenes.
// With `prof`, every launch goes to the main stream in order with an event after it (the batch's
// kernel-by-kernel profile, ntr_batch_profile).
static uint64_t enqueue_step_multi(Batch& B, uint32_t n_jobs, const uint32_t* tot, uint32_t max_shots, uint32_t n_mem,
                                   uint32_t n_air, bool fp64, Sim& S0, Prof* prof = nullptr) {
    cudaStream_t s = B.solve_stream, a = prof ? s : B.aux, a2 = prof ? s : B.aux2;
    uint64_t nl = 0;
    auto M = [&](int kind) { return Multi{B.d_jobs, B.d_first + (size_t)kind * (B.max_scenes + 1), n_jobs}; };
#define LM(kern, kind, threads, strm, ...)                                              \
    do {                                                                                \
        if (tot[kind]) kern<<<tot[kind], (threads), 0, (strm)>>>(M(kind), ##__VA_ARGS__); \
        nl++;                                                                           \
        if (prof) prof->mark(#kern, s);                                                 \
    } while (0)
    if (prof) prof->mark("start", s);
    auto fork = [&](int k, cudaStream_t to) {
        if (to == s) return;
        cudaEventRecord(B.ev_fork[k], s);
        cudaStreamWaitEvent(to, B.ev_fork[k], 0);
    };
    auto join = [&](int k, cudaStream_t from) {
        if (from == s) return;
        cudaEventRecord(B.ev_join[k], from);
        cudaStreamWaitEvent(s, B.ev_join[k], 0);
    };
    LM(k_begin_step_m, GK_ONE, 32, s);
    fork(0, a);
    LM(k_clear_acc_m, GK_CELL, 256, a);
    LM(k_spray_update_m, GK_CELL, 256, a);  // beside the sort, as in enqueue_step
    LM(k_clear_mask_m, GK_WORDS, 256, s);
    LM(k_mark_m, GK_MARK, 256, s);
    LM(k_scan_words_a_m, GK_SCAN, SCAN_T, s);
    LM(k_scan_words_b_m, GK_SCAN, SCAN_T, s);
    cudaEventRecord(B.ev_fork[1], s);
    cudaStreamWaitEvent(a, B.ev_fork[1], 0);
    LM(k_mem_splat_m, GK_VERT, 256, a);
    LM(k_air_carry_m, GK_CELL, 256, a);
    LM(k_keys_hist_m, GK_TILES, KEYS_T, s);
    for (uint32_t p = 0; p < 2; p++) {  // at most two passes below 65,536 blocks
        if (p >= 2) LM(k_radix_hist_m, GK_TILES, RADIX_T, s, p);
        LM(k_radix_scan_m, GK_RSCAN, 256, s, p);
        LM(k_radix_scatter_m, GK_TILES, SCAT_T, s, p);
    }
    LM(k_block_bounds_m, GK_BOUNDS, 256, s);
    LM(k_p2g_m, GK_BLK, P2G_T, s);
    join(0, a);
    LM(k_gather_prep_m, GK_CELL, 256, s);
    LM(k_air_fill_m, GK_CELL, 256, s);
    LM(k_bullet_prep_m, GK_SHOTS, 32, s);
    if (tot[GK_PATCH]) k_bullet_patch_m<<<dim3(tot[GK_PATCH], max_shots), BULLET_PW * 32, 0, s>>>(M(GK_PATCH));
    nl++;
    if (prof) prof->mark("k_bullet_patch_m", s);
    LM(k_bullet_finish_m, GK_SHOTS, 256, s);
    LM(k_bullet_apply_m, GK_CELL, 256, s);
    // Every scene's grid barrier counter starts from zero (k_solve_batch keeps one per scene).
    LM(k_solve_reset_m, GK_ONE, 32, s);
    // Every scene needs a CTA of the joint solve.
    const uint32_t solve_ctas = B.tune.solve_ctas ? std::min(B.ctas, std::max(B.tune.solve_ctas, n_jobs)) : B.ctas;
    nl += enqueue_solve(S0, s, B.d_jobs, n_jobs, fp64, prof, solve_ctas);
    LM(k_project_m, GK_CELL, 256, s);
    LM(k_extend_1_m, GK_CELL, 256, s);
    LM(k_extend_2_m, GK_CELL, 256, s);
    const uint32_t n_sub = std::max(n_mem, n_air);
    while (B.ev_sub.size() < 2 * (size_t)n_sub) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) S0.launch_err = cudaErrorMemoryAllocation;
        B.ev_sub.push_back(e);
    }
    fork(1, a);
    fork(2, a2);
    LM(k_mem_sample_m, GK_VERT4, 256, a);
    for (uint32_t i = 0; i < n_sub; i++) {
        if (i < n_mem) {
            if (a != s && i >= 1 && i - 1 < n_air) cudaStreamWaitEvent(a, B.ev_sub[2 * (i - 1) + 1], 0);
            // (enqueue_step makes substep 0's beside the sort; here, beside 64 scenes' sorts, that
            // was slower: 2.932 s against 2.917 for the 64-scene run.)
            LM(k_mem_tri_m, GK_TRI, 256, a, i, (int)(i % 2));
            LM(k_mem_substep_m, GK_VERT, 256, a, i, (int)(i % 2));
            if (a != s) cudaEventRecord(B.ev_sub[2 * i], a);
        }
        if (i < n_air) {
            if (a2 != s && i >= 1 && i - 1 < n_mem) cudaStreamWaitEvent(a2, B.ev_sub[2 * (i - 1)], 0);
            LM(k_air_substep_m, GK_CELL, 256, a2, i, (int)(i % 2));
            if (a2 != s) cudaEventRecord(B.ev_sub[2 * i + 1], a2);
        }
    }
    LM(k_g2p_m<128>, GK_BLK, 128, s);
    LM(k_spray_scan_m, GK_ONE, 1024, s);
    LM(k_spray_emit_m, GK_CELL, 256, s);
    join(1, a);
    join(2, a2);
#undef LM
    return nl;
}

// n steps of every unfinished scene: each scene takes min(n, its steps left) (its step budget
// stops it after those), all of them in the same replays of the batch's step graph.
// `lk` (the batch's lock, held by the caller) is let go while the step waits for the GPU.
static ntr_status batch_step(Batch& B, uint32_t n, uint32_t& active, Prof* prof = nullptr, std::unique_lock<std::mutex>* lk = nullptr) {
    std::vector<uint32_t> order;
    std::vector<uint32_t> todo(B.max_scenes, 0u);
    for (uint32_t i = 0; i < B.max_scenes; i++) {
        BatchSlot& sl = B.slots[i];
        if (!sl.sim || sl.done >= sl.target) continue;
        todo[i] = std::min(n, sl.target - sl.done);
        order.push_back(i);
    }
    active = (uint32_t)order.size();
    if (order.empty() || n == 0) return NTR_OK;
    const uint32_t n_jobs = (uint32_t)order.size();
    cudaStream_t s = B.solve_stream;
    // Each scene's parameters for this call (Sim::run) and its step budget, the pointer tables
    // and the grids of the scenes in order, staged in the pinned buffer and sent in one copy.
    Dev* jobs = reinterpret_cast<Dev*>(B.h_stage);
    uint32_t* first = reinterpret_cast<uint32_t*>(B.h_stage + B.off_first);
    BatchJobIn* in = reinterpret_cast<BatchJobIn*>(B.h_stage + B.off_in);
    std::fill(first, first + (size_t)GK_COUNT * (B.max_scenes + 1), 0u);
    uint32_t tot[GK_COUNT] = {};
    std::vector<uint32_t> key;
    uint32_t fp64 = B.slots[order[0]].sim->fp64, max_shots = 1, n_mem = 0, n_air = 0, steps = 0;
    for (uint32_t j = 0; j < n_jobs; j++) {
        Sim& S = *B.slots[order[j]].sim;
        if (S.fp64 != fp64) return fail(NTR_E_INVALID, "the scenes of a batch step must use the same solver precision");
        ntr_world_header& h = S.host.h;
        S.U.limits[2] = h.iters;
        S.U.limits[3] = 0xFFFFFFFFu;
        S.U.mem[1] = h.substeps;
        S.U.mem[2] = h.air_substeps;
        in[j].U = S.U;
        in[j].budget = todo[order[j]];
        S.size_class = size_class_of(std::max(S.h_state->s.n_blocks, S.h_state->s.n_blocks_prev));
        jobs[j] = S.D;
        uint32_t g[GK_COUNT];
        scene_grids(S, g);
        for (int k = 0; k < GK_COUNT; k++) {
            first[(size_t)k * (B.max_scenes + 1) + j] = tot[k];
            tot[k] += g[k];
        }
        max_shots = std::max(max_shots, g[GK_SHOTS]);
        n_mem = std::max(n_mem, h.substeps);
        n_air = std::max(n_air, h.air_substeps);
        steps = std::max(steps, todo[order[j]]);
        key.push_back(order[j]);
        key.push_back(S.size_class);
    }
    for (int k = 0; k < GK_COUNT; k++) first[(size_t)k * (B.max_scenes + 1) + n_jobs] = tot[k];
    key.insert(key.end(), {n_jobs, fp64, max_shots, n_mem, n_air, B.tune.cell_ctas_per_sm, B.tune.block_ctas_per_sm, B.tune.solve_ctas});
    CU(cudaMemcpyAsync(B.d_stage, B.h_stage, B.off_in + sizeof(BatchJobIn) * n_jobs, cudaMemcpyHostToDevice, s));
    k_batch_begin<<<n_jobs, 64, 0, s>>>(B.d_jobs, B.d_in);
    CU(cudaGetLastError());
    // The step graph of these scenes and shapes (captured again when they change).
    Sim& S0 = *B.slots[order[0]].sim;
    if (!prof && (!B.exec || key != B.graph_key)) {
        if (B.graph) cudaGraphDestroy(B.graph), B.graph = nullptr;
        S0.launch_err = cudaSuccess;
        CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        enqueue_step_multi(B, n_jobs, tot, max_shots, n_mem, n_air, fp64 != 0, S0);
        cudaError_t le = cudaGetLastError();
        cudaError_t ce = cudaStreamEndCapture(s, &B.graph);
        if (S0.launch_err != cudaSuccess) le = S0.launch_err;
        if (le != cudaSuccess) {
            if (B.graph) cudaGraphDestroy(B.graph), B.graph = nullptr;
            if (B.exec) cudaGraphExecDestroy(B.exec), B.exec = nullptr;
            return fail(NTR_E_CUDA, std::string("kernel launch during capture: ") + cudaGetErrorString(le));
        }
        if (ce != cudaSuccess) {
            if (B.exec) cudaGraphExecDestroy(B.exec), B.exec = nullptr;
            return fail(NTR_E_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce));
        }
        // Most changes are only of grid sizes (a scene's size class): the executable graph
        // takes the new launch shapes in place. A changed sequence (substep counts, an empty
        // grid) needs a new one.
        bool updated = false;
        if (B.exec) {
            cudaGraphExecUpdateResultInfo info;
            updated = cudaGraphExecUpdate(B.exec, B.graph, &info) == cudaSuccess;
            if (!updated) {
                cudaGetLastError();
                cudaGraphExecDestroy(B.exec), B.exec = nullptr;
            }
        }
        if (!updated) CU(cudaGraphInstantiate(&B.exec, B.graph, 0));
        B.graph_key = key;
        B.captures++;
        B.instantiations += updated ? 0u : 1u;
    }
    std::vector<uint32_t> before(n_jobs);
    for (uint32_t j = 0; j < n_jobs; j++) before[j] = B.slots[order[j]].sim->h_state->s.step;
    if (prof) {
        S0.launch_err = cudaSuccess;
        for (uint32_t k = 0; k < steps; k++) enqueue_step_multi(B, n_jobs, tot, max_shots, n_mem, n_air, fp64 != 0, S0, prof);
        CU(cudaGetLastError());
        CU(S0.launch_err);
        CU(prof->err);
    } else {
        for (uint32_t k = 0; k < steps; k++) CU(cudaGraphLaunch(B.exec, s));
    }
    B.steps += steps;
    // The states back in one copy (parked scenes' step lengths restored, budgets back to no
    // limit on the device), then the host control of each scene (Sim::run).
    k_batch_end<<<n_jobs, 64, 0, s>>>(B.d_jobs, B.d_out);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(B.h_out, B.d_out, sizeof(DevState) * n_jobs, cudaMemcpyDeviceToHost, s));
    {
        // Admissions may reserve and fill free slots meanwhile; every other call waits.
        if (lk) {
            B.in_flight = true;
            lk->unlock();
        }
        const cudaError_t e = cudaStreamSynchronize(s);
        if (lk) {
            lk->lock();
            B.in_flight = false;
            B.cv.notify_all();
        }
        CU(e);
    }
    ntr_status first_err = NTR_OK;
    for (uint32_t j = 0; j < n_jobs; j++) {
        BatchSlot& sl = B.slots[order[j]];
        Sim& S = *sl.sim;
        *S.h_state = B.h_out[j];
        const ntr_state& st = S.h_state->s;
        sl.done += st.step - before[j];
        if (st.overflow && first_err == NTR_OK)
            first_err = fail(NTR_E_OVERFLOW, "a scene needs more than " + std::to_string(S.host.h.block_cap) + " grid blocks");
        if (S.h_state->err && first_err == NTR_OK) first_err = fail(NTR_E_TIMEOUT, "a bounded device-side wait gave up");
        if (!st.overflow && !S.h_state->err) adapt_after_batch(S.host.h, st);
    }
    return first_err;
}

}  // namespace ntr
