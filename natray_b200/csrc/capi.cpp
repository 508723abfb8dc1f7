// The CPU half of the C ABI: errors, parameters and world construction.
#include <cstdlib>
#include <cstring>
#include <string>

#include "capi_util.hpp"
#include "world.hpp"

namespace ntr {
static thread_local std::string g_last_error;
ntr_status fail(ntr_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}
void clear_error() { g_last_error.clear(); }
}  // namespace ntr

using namespace ntr;

extern "C" {

NTR_API size_t ntr_last_error(char* buf, size_t cap) {
    size_t n = g_last_error.size();
    if (buf && cap) {
        size_t k = n < cap - 1 ? n : cap - 1;
        std::memcpy(buf, g_last_error.data(), k);
        buf[k] = 0;
    }
    return n;
}

NTR_API const char* ntr_version(void) { return "natray-b200 0.1 (sm_100a)"; }

NTR_API void ntr_free(void* p) { std::free(p); }

NTR_API ntr_status ntr_params_default(ntr_sim_params* p) {
    if (!p) return fail(NTR_E_INVALID, "null params");
    params_default(*p);
    return NTR_OK;
}

NTR_API ntr_status ntr_params_set(ntr_sim_params* p, const char* key, const char* value) {
    if (!p || !key) return fail(NTR_E_INVALID, "null argument");
    std::string err;
    if (!params_set(*p, key, value, err)) return fail(NTR_E_INVALID, err);
    return NTR_OK;
}

NTR_API ntr_status ntr_params_preset(ntr_sim_params* p, const char* name) {
    if (!p || !name) return fail(NTR_E_INVALID, "null argument");
    std::string err;
    if (!params_preset(*p, name, err)) return fail(NTR_E_INVALID, err);
    return NTR_OK;
}

NTR_API ntr_status ntr_inflate(double shear_modulus, double thickness, double rest_radius, double volume, double rho_g, ntr_profile* out) {
    if (!out) return fail(NTR_E_INVALID, "null argument");
    if (!(shear_modulus > 0) || !(thickness > 0) || !(rest_radius > 0) || !(volume > 0) || !(rho_g >= 0))
        return fail(NTR_E_INVALID, "inflation parameters out of range");
    std::string err;
    if (!inflate_profile(shear_modulus, thickness, rest_radius, volume, rho_g, *out, err)) return fail(NTR_E_INVALID, err);
    return NTR_OK;
}

NTR_API ntr_status ntr_world_build(const ntr_sim_params* p, void** blob, size_t* len) {
    if (!p || !blob || !len) return fail(NTR_E_INVALID, "null argument");
    World w;
    std::string err;
    if (!build_world(*p, w, err)) return fail(NTR_E_INVALID, err);
    const size_t n = serialize_into(w, nullptr);
    void* out = std::malloc(n);
    if (!out) return fail(NTR_E_NOMEM, "host allocation of the world blob failed");
    serialize_into(w, out);
    *blob = out;
    *len = n;
    return NTR_OK;
}

NTR_API ntr_status ntr_shot_flights(const ntr_sim_params* p, ntr_flight* out, uint32_t cap, uint32_t* n) {
    if (!p || (!out && cap)) return fail(NTR_E_INVALID, "null argument");
    std::vector<ntr_flight> v;
    std::string err;
    if (!flights(*p, v, err)) return fail(NTR_E_INVALID, err);
    if (n) *n = (uint32_t)v.size();
    for (uint32_t k = 0; k < v.size() && k < cap; k++) out[k] = v[k];
    return NTR_OK;
}

}  // extern "C"
