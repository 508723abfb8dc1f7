// Host-side world: the parsed form of a world blob (include/natray.h), and the scene builder
// that makes the initial one. CPU only.
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "natray.h"

namespace ntr {

// Element size and count of each section, from the header's counts.
struct SectionShape {
    size_t elem;   // bytes per element
    size_t count;  // elements
};
SectionShape section_shape(const ntr_world_header& h, int sec);

struct World {
    ntr_world_header h{};
    std::vector<uint8_t> sec[NTR_SEC_COUNT];

    template <class T>
    T* as(int s) { return reinterpret_cast<T*>(sec[s].data()); }
    template <class T>
    const T* as(int s) const { return reinterpret_cast<const T*>(sec[s].data()); }
    // Resizes every section to what the header's counts say, every byte zero.
    void shape_sections();
};

std::vector<uint8_t> serialize(const World& w);
// Writes the blob into `out` (when not null) and returns its size in bytes.
size_t serialize_into(const World& w, void* out);
// Returns false with a message on a malformed blob.
bool deserialize(const void* blob, size_t len, World& w, std::string& err);

// Scene construction, src/balloon.rs:343-464 and src/sim.rs:208-441 (before the measuring
// substep, which the creator of the simulation runs).
bool build_world(const ntr_sim_params& p, World& w, std::string& err);
bool flights(const ntr_sim_params& p, std::vector<ntr_flight>& out, std::string& err);

// `inflate` of src/balloon.rs:170-248 with `Latex::new(shear, thick)`.
bool inflate_profile(double shear, double thick, double rest_r, double volume, double rho_g, ntr_profile& out, std::string& err);

// Params helpers, src/params.rs and src/presets.rs.
void params_default(ntr_sim_params& p);
bool params_set(ntr_sim_params& p, const char* key, const char* value, std::string& err);
bool params_preset(ntr_sim_params& p, const char* name, std::string& err);

// Enough substeps, with a little to spare, that a step of `dt` isn't cut short by them. Even.
// src/sim.rs:96-105.
uint32_t substeps_for(float dt, float sub_dt);

// Host adaptation after a batch, src/sim.rs:634-647. Returns false on block overflow.
void adapt_after_batch(ntr_world_header& h, const ntr_state& s);

}  // namespace ntr
