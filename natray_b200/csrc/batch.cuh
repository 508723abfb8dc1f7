// Batches of independent scenes on one GPU (include/natray.h, ntr_batch_*): the serving engine.
//
// Every admitted scene is a Sim of its own (device-resident state, its own streams and cached
// graphs). A batch step runs, per scene, the step's part before the pressure solve on the
// scene's stream; then ONE cooperative launch solves every scene's system, the GPU's CTAs split
// over the scenes by their block counts (k_solve, solve_split); then each scene's part after the
// solve, again on its own stream, so the scenes' work overlaps on the device. The host reads the
// scenes' states back once per ntr_batch_step call and adapts each one's solver iterations and
// substeps as ntr_sim_step does, so a scene's results are those of the scene run alone.
//
// Included at the end of sim.cu (it uses the Sim internals there).
#pragma once

#include <chrono>
#include <deque>

namespace ntr {

struct BatchSlot {
    std::unique_ptr<Sim> sim;
    uint32_t target = 0, done = 0;
    cudaEvent_t ev_pre = nullptr;  // the scene's part before the solve is done
    // The slot's device region and pinned state buffer, kept across the scenes it holds; the
    // region grows (and only then is reallocated) when a scene needs more.
    uint8_t* arena = nullptr;
    size_t arena_cap = 0;
    DevState* h_state = nullptr;
};

struct Batch {
    int device = 0;
    uint32_t max_scenes = 0;
    uint64_t budget = 0;   // bytes the batch may hold; 0: no limit
    uint64_t reserve = 0;  // free device memory that admission leaves
    uint64_t held = 0;
    uint64_t steps = 0;
    uint32_t ctas = 0;  // CTAs of the joint solve
    std::vector<BatchSlot> slots;
    cudaStream_t solve_stream = nullptr;
    cudaEvent_t ev_solve = nullptr;
    Dev* d_jobs = nullptr;  // the pointer tables of the scenes in the current step's order
    uint32_t n_jobs_cap = 0;
    // Every call on the batch holds this lock: calls from several host threads take turns.
    std::mutex mu;
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
        for (auto& s : slots) {
            s.sim.reset();
            if (s.ev_pre) cudaEventDestroy(s.ev_pre);
            if (s.arena) cudaFree(s.arena);
            if (s.h_state) cudaFreeHost(s.h_state);
        }
        slots.clear();
        if (d_jobs) cudaFree(d_jobs);
        if (ev_solve) cudaEventDestroy(ev_solve);
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
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(NTR_E_NODEVICE, "this library is built for sm_100a (B200)");
    int occ_a = 0, occ_b = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, k_solve_batch<true>, SOLVE_T, 0));
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, k_solve_batch<false>, SOLVE_T, 0));
    const uint32_t ctas = (uint32_t)std::min(256, prop.multiProcessorCount * std::min(occ_a, occ_b));
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
    CU(cudaEventCreateWithFlags(&B->ev_solve, cudaEventDisableTiming));
    for (auto& s : B->slots) {
        CU(cudaEventCreateWithFlags(&s.ev_pre, cudaEventDisableTiming));
        CU(cudaMallocHost((void**)&s.h_state, sizeof(DevState)));
    }
    CU(cudaMalloc((void**)&B->d_jobs, sizeof(Dev) * max_scenes));
    B->n_jobs_cap = max_scenes;
    out = B.release();
    return NTR_OK;
}

static ntr_status batch_admit(Batch& B, const void* blob, size_t len, uint32_t n_steps, uint32_t& slot) {
    CU(cudaSetDevice(B.device));
    World w;
    std::string err;
    if (!deserialize(blob, len, w, err)) return fail(NTR_E_INVALID, err);
    uint64_t need = 0;
    ntr_status r = world_device_bytes(w, need);
    if (r != NTR_OK) return r;
    // A free slot whose region already holds the scene (the smallest such), else the free slot
    // with the largest region.
    uint32_t free_slot = NONE, fits = NONE;
    for (uint32_t i = 0; i < B.max_scenes; i++) {
        const BatchSlot& c = B.slots[i];
        if (c.sim) continue;
        if (c.arena_cap >= need && (fits == NONE || c.arena_cap < B.slots[fits].arena_cap)) fits = i;
        if (free_slot == NONE || c.arena_cap > B.slots[free_slot].arena_cap) free_slot = i;
    }
    if (fits != NONE) free_slot = fits;
    if (free_slot == NONE) return fail(NTR_E_BUSY, "every slot of the batch is in use");
    size_t free_b = 0, total_b = 0;
    CU(cudaMemGetInfo(&free_b, &total_b));
    BatchSlot& sl = B.slots[free_slot];
    const uint64_t grow = need > sl.arena_cap ? need + need / 4 - sl.arena_cap : 0;  // 25 % headroom
    if (B.budget && B.held + grow > B.budget) return fail(NTR_E_BUSY, "the scene's " + std::to_string(need) + " bytes exceed the batch's budget now");
    if (grow && (uint64_t)free_b < grow + B.reserve) return fail(NTR_E_BUSY, "the scene's " + std::to_string(need) + " bytes do not fit the free device memory now");
    if (grow) {
        if (sl.arena) CU(cudaFree(sl.arena));
        B.held -= sl.arena_cap;
        sl.arena = nullptr, sl.arena_cap = 0;
        CU(cudaMalloc((void**)&sl.arena, need + need / 4));
        sl.arena_cap = need + need / 4;
        B.held += sl.arena_cap;
    }
    Sim* s = nullptr;
    if ((r = create_from(w, B.device, s, sl.arena, sl.arena_cap, sl.h_state)) != NTR_OK) return r;
    sl.sim.reset(s);
    sl.target = n_steps;
    sl.done = 0;
    slot = free_slot;
    return NTR_OK;
}

static ntr_status batch_retire(Batch& B, uint32_t slot) {
    if (slot >= B.max_scenes || !B.slots[slot].sim) return fail(NTR_E_INVALID, "no scene in that slot");
    CU(cudaSetDevice(B.device));
    B.slots[slot].sim.reset();  // the slot keeps its device region for the next scene
    B.slots[slot].target = B.slots[slot].done = 0;
    return NTR_OK;
}

// n steps of every unfinished scene. The scenes are ordered by the steps they take in this call,
// longest first, so the scenes that still step at step k are a prefix of the jobs table, and
// one table serves every step of the call.
static ntr_status batch_step(Batch& B, uint32_t n, uint32_t& active) {
    CU(cudaSetDevice(B.device));
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
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return todo[a] > todo[b]; });
    // The scenes' pointer tables, and each scene's parameters for this call (Sim::run).
    std::vector<Dev> jobs(order.size());
    ntr_status r;
    uint32_t fp64 = B.slots[order[0]].sim->fp64;
    for (size_t j = 0; j < order.size(); j++) {
        Sim& S = *B.slots[order[j]].sim;
        if (S.fp64 != fp64) return fail(NTR_E_INVALID, "the scenes of a batch step must use the same solver precision");
        jobs[j] = S.D;
        ntr_world_header& h = S.host.h;
        S.U.limits[2] = h.iters;
        S.U.limits[3] = 0xFFFFFFFFu;
        S.U.mem[1] = h.substeps;
        S.U.mem[2] = h.air_substeps;
        if ((r = push_params(S)) != NTR_OK) return r;
        CU(cudaMemsetAsync(&S.D.st->s.iters_max, 0, 8, S.stream));
    }
    CU(cudaMemcpyAsync(B.d_jobs, jobs.data(), sizeof(Dev) * jobs.size(), cudaMemcpyHostToDevice, B.solve_stream));
    std::vector<StepGraph*> pre(order.size()), post(order.size());
    for (size_t j = 0; j < order.size(); j++) {
        Sim& S = *B.slots[order[j]].sim;
        if ((r = get_graph(S, pre[j], PART_PRE)) != NTR_OK) return r;
        if ((r = get_graph(S, post[j], PART_POST)) != NTR_OK) return r;
    }
    std::vector<uint32_t> before(order.size());
    for (size_t j = 0; j < order.size(); j++) before[j] = B.slots[order[j]].sim->h_state->s.step;
    Sim& S0 = *B.slots[order[0]].sim;
    S0.launch_err = cudaSuccess;
    for (uint32_t k = 0; k < todo[order[0]]; k++) {
        uint32_t n_k = 0;  // scenes that take step k
        for (size_t j = 0; j < order.size(); j++) {
            if (todo[order[j]] <= k) break;
            Sim& S = *B.slots[order[j]].sim;
            CU(cudaGraphLaunch(pre[j]->exec, S.stream));
            CU(cudaEventRecord(B.slots[order[j]].ev_pre, S.stream));
            CU(cudaStreamWaitEvent(B.solve_stream, B.slots[order[j]].ev_pre, 0));
            n_k++;
        }
        enqueue_solve(S0, B.solve_stream, B.d_jobs, n_k, fp64 != 0, nullptr, B.ctas);
        CU(S0.launch_err);
        CU(cudaEventRecord(B.ev_solve, B.solve_stream));
        for (uint32_t j = 0; j < n_k; j++) {
            Sim& S = *B.slots[order[j]].sim;
            CU(cudaStreamWaitEvent(S.stream, B.ev_solve, 0));
            CU(cudaGraphLaunch(post[j]->exec, S.stream));
        }
    }
    B.steps += todo[order[0]];
    // States back, one copy per scene, then the host control of each (Sim::run).
    for (size_t j = 0; j < order.size(); j++) {
        Sim& S = *B.slots[order[j]].sim;
        CU(cudaMemcpyAsync(S.h_state, S.D.st, sizeof(DevState), cudaMemcpyDeviceToHost, S.stream));
    }
    ntr_status first = NTR_OK;
    for (size_t j = 0; j < order.size(); j++) {
        BatchSlot& sl = B.slots[order[j]];
        Sim& S = *sl.sim;
        CU(cudaStreamSynchronize(S.stream));
        const ntr_state& st = S.h_state->s;
        sl.done += st.step - before[j];
        if (st.overflow && first == NTR_OK)
            first = fail(NTR_E_OVERFLOW, "a scene needs more than " + std::to_string(S.host.h.block_cap) + " grid blocks");
        if (S.h_state->err && first == NTR_OK) first = fail(NTR_E_TIMEOUT, "a bounded device-side wait gave up");
        if (!st.overflow && !S.h_state->err) adapt_after_batch(S.host.h, st);
    }
    return first;
}

}  // namespace ntr
