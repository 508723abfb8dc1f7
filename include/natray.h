/*
 * natray.h - C ABI of the B200 simulation step of natray (a water balloon shot by bullets).
 *
 * This header is the drop-in boundary that replaces the wgpu dispatch layer of the reference
 * (src/gpu.rs:60-214) and the `Sim` surface built on it (src/sim.rs:149-689). A Rust host
 * binds it through a thin FFI crate; this repository binds it from Python through ctypes.
 *
 * Conventions
 *   - Every call returns an ntr_status. Nothing aborts across the ABI; the message of the last
 *     failure on the calling thread is available from ntr_last_error().
 *   - Plain pointers and sizes only. Device pointers are lent by ntr_sim_buffer() and stay
 *     valid until ntr_sim_destroy() or ntr_sim_restore().
 *   - One ntr_sim per host thread at a time; each owns its own CUDA stream.
 *
 * World blob
 *   A "world" is the complete description of a simulation: parameters, the static scene (mesh,
 *   bullet surfaces) and all state that lives across steps. It is one contiguous byte blob: an
 *   ntr_world_header followed by sections at the offsets the header lists. It is produced on the
 *   CPU by ntr_world_build() (no GPU needed), consumed by ntr_sim_create_from_world(), and
 *   written back by ntr_sim_snapshot(). The same format is the fixture format of the tests.
 *   Block lists in a world are in canonical order: ascending block slot.
 */
#ifndef NATRAY_H
#define NATRAY_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define NTR_API __declspec(dllexport)
#else
#define NTR_API __attribute__((visibility("default")))
#endif

/* Errors. The reference panics on these (src/sim.rs:635, src/gpu.rs:63-69, src/balloon.rs:225). */
typedef enum ntr_status {
    NTR_OK = 0,
    NTR_E_INVALID = 1,     /* bad argument, bad parameter value, malformed world blob */
    NTR_E_NOMEM = 2,       /* device or host allocation refused */
    NTR_E_OVERFLOW = 3,    /* more grid blocks needed than the block capacity holds */
    NTR_E_UNCONVERGED = 4, /* warning: a step ran out of solver iterations */
    NTR_E_TIMEOUT = 5,     /* a bounded device-side wait gave up */
    NTR_E_CUDA = 6,        /* CUDA runtime error */
    NTR_E_NODEVICE = 7,    /* no CUDA device, or the library was built without one */
    NTR_E_BUSY = 8         /* admission refused for lack of free memory or slots */
} ntr_status;

#define NTR_MAX_SHOTS 4
#define NTR_MAX_PATCHES 576
#define NTR_N_SEC 32
#define NTR_LOG_CAP 256
#define NTR_OUTLINE 33
#define NTR_HIT_FIELDS 13
#define NTR_ACC_FIELDS 19
#define NTR_CELL_FIELDS 11
#define NTR_AIR_FIELDS 5
#define NTR_LAYER_MODES 6
#define NTR_MAX_VALENCE 64 /* triangles per membrane vertex, at most */

/* One bullet fired at the balloon. Mirrors `Shot` (src/params.rs:205-264). `bullet` indexes
 * the table of loads (src/params.rs:193-201): 0 .22 LR, 1 9 mm, 2 .45 ACP, 3 M855, 4 .308,
 * 5 wadcutter, 6 BB. */
typedef struct ntr_shot {
    uint32_t bullet;
    float speed;
    float caliber_mm;
    float mass_g;
    float spin_rpm;
    float range_m;
    float muzzle_yaw_deg;
    float azimuth_deg;
    float elevation_deg;
    float impact_offset_cm;
    float impact_side_cm;
    float delay_ms;
} ntr_shot;

/* Mirrors `SimParams` (src/params.rs:266-314), plus the knobs the reference hard-codes. */
typedef struct ntr_sim_params {
    uint32_t n_shots;
    ntr_shot shots[NTR_MAX_SHOTS];
    float balloon_diameter_cm;
    float balloon_height;
    float rubber_modulus_mpa;
    float rubber_rest_diameter_cm;
    float rubber_break_stretch;
    float rubber_thickness_mm;
    float gravity;
    float spray_amount;
    float mist_amount;
    uint32_t resolution;
    /* Hard-coded in the reference, exposed here. Defaults reproduce the reference. */
    uint32_t mesh_level;  /* icosphere subdivisions (src/balloon.rs:357: 6) */
    float dt_max;         /* longest step in s (src/sim.rs:19: 1e-3); 2e-6 gives a fixed step */
    uint64_t seed;        /* 0: the reference jitter state 0x9E3779B97F4A7C15 (src/balloon.rs:359) */
    uint32_t block_cap;   /* grid block capacity, 0 = sized from the particle count */
    uint32_t spray_cap;   /* spray slots (src/sim.rs:13: 1,200,000) */
    uint32_t max_iters;   /* solver iteration ceiling (src/sim.rs:21: 4096) */
    float solve_tol;      /* relative residual (src/sim.rs:20: 1e-5) */
} ntr_sim_params;

/* The per-step uniform, field for field `Params` of src/sim.rs:49-64 / shaders/sim_defs.wgsl:8-21. */
typedef struct ntr_gpu_params {
    float origin[4];    /* domain corner, w = cell size h */
    uint32_t dims[4];   /* domain size in cells, w = particle count */
    uint32_t bdims[4];  /* domain size in 4^3 blocks, w = block capacity */
    float gravity[4];   /* xyz, w = sound speed in water */
    float fluid[4];     /* water density, CFL, longest step, particle spacing */
    float wet[4];       /* x = wet map half size */
    uint32_t limits[4]; /* wet map resolution, spray capacity, solver iterations, stop (ns) */
    float solve[4];     /* x = relative tolerance */
    uint32_t mem[4];    /* rubber verts, rubber substeps, air substeps, bullets */
    float rubber[4];    /* Ogden moduli (Pa), uninflated thickness */
    float rubber2[4];   /* ground friction, break stretch */
    float knot[4];      /* where the neck is tied, w = neck radius */
} ntr_gpu_params;

/* The GPU clock and counters, word for word `State` of src/sim.rs:66-94 /
 * shaders/sim_defs.wgsl:24-58. f32 fields that the device lowers with atomicMin are f32. */
typedef struct ntr_state {
    uint32_t t_ns;
    uint32_t dt_ns;
    uint32_t step;
    uint32_t n_blocks;
    float max_speed;
    uint32_t n_blocks_prev;
    uint32_t overflow;
    uint32_t solve_iters;
    float rz;
    float alpha;
    float b_norm;
    float r_norm;
    uint32_t free_dt_ns;
    uint32_t iters_max;
    uint32_t unconverged;
    float beta;
    uint32_t spray_count;
    float mem_dt;
    float cap_dt;
    float mem_dt_seen;
    float dt_flow;
    float air_dt;
    float air_dt_seen;
    uint32_t mem_ticket;
} ntr_state;

/* Sections of a world blob. Element layouts (all little-endian, 4-byte words):
 *   PARTICLES   n_particles x 20 f32: pos.xyzw, vel.xyz + alive (w), c0 (w = pressure Pa),
 *               c1 (w = thin age s), c2 (w = scratch)           -- `Particle`, sim_defs.wgsl:61
 *   MEM_X/V     n_verts x 4 f32 (v.w = 1 where a bullet holds it)
 *   MEM_MASS    n_verts f32 (0 where the knot holds it)
 *   MEM_WATER   n_verts x 4 f32 (water velocity, fill)
 *   MEM_LAYER   n_verts x 6 x 4 f32 (Stokes-layer modes)
 *   MEM_PUSH    n_verts x 2 f32 (push on the water N, area m^2)
 *   TRIS        n_tris x (3 u32, rest_area f32, dm_inv 4 f32)    -- `GpuTri`, balloon.rs:23-29
 *   ALIVE       n_tris u32
 *   VTRI_OFF    (n_verts + 1) u32;  VTRI  n_vtri u32
 *   BULLETS     4 x 28 words (`Bullet`, bullet.wgsl:16-34)
 *   PATCHES     4 x 576 x 8 f32;  OUTLINES 4 x 33 x 2 f32;  SECTIONS 4 x 32 x 12 f32
 *   BULLET_HIT  4 x 13 i32;  POSE_LOG 4 x 256 x 12 f32
 *   BLOCKS_PREV n_blocks_prev u32 block slots, ascending
 *   BLOCK_ACTIVE n_blocks_prev u32
 *   AIR         5 fields x (64 n_blocks_prev) f32, field-major (rho, m.xyz, E)
 *   SPRAY       n_spray x 12 f32 (pos + r, vel + weight, air);  LANDED n_spray x 4 f32
 *   TOUCH       wet_res^2 u32 (f32 bits of the first wet time) */
typedef enum ntr_section {
    NTR_SEC_PARTICLES = 0,
    NTR_SEC_MEM_X,
    NTR_SEC_MEM_V,
    NTR_SEC_MEM_MASS,
    NTR_SEC_MEM_WATER,
    NTR_SEC_MEM_LAYER,
    NTR_SEC_MEM_PUSH,
    NTR_SEC_TRIS,
    NTR_SEC_ALIVE,
    NTR_SEC_VTRI_OFF,
    NTR_SEC_VTRI,
    NTR_SEC_BULLETS,
    NTR_SEC_PATCHES,
    NTR_SEC_OUTLINES,
    NTR_SEC_SECTIONS,
    NTR_SEC_BULLET_HIT,
    NTR_SEC_POSE_LOG,
    NTR_SEC_BLOCKS_PREV,
    NTR_SEC_BLOCK_ACTIVE,
    NTR_SEC_AIR,
    NTR_SEC_SPRAY,
    NTR_SEC_LANDED,
    NTR_SEC_TOUCH,
    NTR_SEC_COUNT
} ntr_section;

#define NTR_WORLD_MAGIC 0x5752544Eu /* "NTRW" */
#define NTR_WORLD_VERSION 1u

typedef struct ntr_world_header {
    uint32_t magic;
    uint32_t version;
    uint32_t n_particles;
    uint32_t n_verts;
    uint32_t n_tris;
    uint32_t n_vtri;
    uint32_t n_shots;
    uint32_t n_blocks_prev;
    uint32_t n_spray;
    uint32_t wet_res;
    uint32_t spray_cap;
    uint32_t block_cap;
    /* Host-side control that src/sim.rs:186-198 keeps between batches. */
    uint32_t iters;
    uint32_t substeps;
    uint32_t air_substeps;
    uint32_t unconverged;
    uint32_t started;
    uint32_t max_iters;
    double t;
    double t_start;
    double t0;
    double dx;
    ntr_gpu_params params;
    ntr_state state;
    uint64_t offset[NTR_SEC_COUNT];
    uint64_t bytes[NTR_SEC_COUNT];
} ntr_world_header;

/* Buffers a renderer or keyframe packer reads (src/sim.rs:149-205 pub fields). */
typedef enum ntr_buf {
    NTR_BUF_PARTICLES = 0, /* SoA: 5 arrays of n_particles float4 (pos, vel, c0, c1, c2) */
    NTR_BUF_STATE,         /* one ntr_state */
    NTR_BUF_MEM_POS,       /* n_verts float4 */
    NTR_BUF_TRIS,
    NTR_BUF_ALIVE,
    NTR_BUF_VTRI_OFF,
    NTR_BUF_VTRI,
    NTR_BUF_SPRAY,         /* spray_cap x 48 B */
    NTR_BUF_TOUCH,
    NTR_BUF_LANDED,
    NTR_BUF_BLOCK_LIST,    /* this step's block slots, ascending */
    NTR_BUF_SORTED,        /* particle indices grouped by block, ascending within a block */
    NTR_BUF_BLOCK_START,   /* n_blocks + 1 u32 */
    NTR_BUF_ACC,           /* 19 fields x block_cap*64 i32, field-major */
    NTR_BUF_CF,            /* 11 fields x block_cap*64 f32, field-major */
    NTR_BUF_AIR,           /* 5 fields x block_cap*64 f32, field-major */
    NTR_BUF_BLOCK_NB,      /* n_blocks x 27 u32 */
    NTR_BUF_COUNT
} ntr_buf;

typedef struct ntr_sim_info {
    uint32_t n_particles;
    uint32_t n_verts;
    uint32_t n_tris;
    uint32_t n_shots;
    uint32_t dims[3];
    uint32_t block_cap;
    uint32_t spray_cap;
    uint32_t iters;
    uint32_t substeps;
    uint32_t air_substeps;
    double dx;
    double spacing;
    float grid_origin[3];
    float pad;
    double t;
    double t_start;
    double t0;
    uint64_t device_bytes;
} ntr_sim_info;

typedef struct ntr_sim ntr_sim;

/* Message of the last failure on this thread (empty if none). Returns the message length. */
NTR_API size_t ntr_last_error(char* buf, size_t cap);
NTR_API const char* ntr_version(void);
NTR_API void ntr_free(void* p);

/* --- Parameters (CPU only) -------------------------------------------------------------- */
/* SimParams::default (src/params.rs:297-314). */
NTR_API ntr_status ntr_params_default(ntr_sim_params* p);
/* A `key=value` override, `set_kv` of src/params.rs:361-423 (look keys are accepted and
 * ignored: they only change the renderer). */
NTR_API ntr_status ntr_params_set(ntr_sim_params* p, const char* key, const char* value);
/* A named scene, `presets::named` of src/presets.rs:110-116. */
NTR_API ntr_status ntr_params_preset(ntr_sim_params* p, const char* name);

/* The filled balloon's axisymmetric shape, `Profile` of src/balloon.rs:73-110. */
#define NTR_PROFILE_SAMPLES 402
typedef struct ntr_profile {
    uint32_t n_samples;
    uint32_t pad;
    double neck_angle;
    double z_neck;
    double neck_r;
    double volume;
    double z_centroid;
    double stretch;
    double r_max;
    double samples[NTR_PROFILE_SAMPLES][3]; /* (angle on the uninflated sphere, r, z) */
} ntr_profile;

/* --- World construction (CPU only) ------------------------------------------------------- */
/* `inflate` of src/balloon.rs:170-248: Ogden latex of the given small-strain shear modulus
 * (Pa) and thickness (m), uninflated radius rest_radius (m), filled with `volume` (m^3) of
 * water under rho*g = rho_g (Pa/m). */
NTR_API ntr_status ntr_inflate(double shear_modulus, double thickness, double rest_radius, double volume, double rho_g,
                               ntr_profile* out);
/* Builds the scene and the initial state, as `Sim::new` does before its first dispatch
 * (src/sim.rs:208-494, scene from src/balloon.rs:343-464 and src/bullet.rs:56-132), including
 * the zero-length measuring substep of src/sim.rs:524-541. The blob is allocated here and
 * released with ntr_free(). */
NTR_API ntr_status ntr_world_build(const ntr_sim_params* p, void** blob, size_t* len);

/* A shot's flight through still air to the balloon (Flight::new, src/flight.rs:404-471): the
 * launch from the muzzle that puts the tip on the target at the shot's speed, the state at
 * which the simulation takes the bullet over (LOOKAHEAD = 5 cm short of the balloon), and the
 * report at impact. */
typedef struct ntr_flight {
    double x[3], u[3], n[3], h[3]; /* hand-over: centre of mass (m), velocity (m/s), nose axis, angular momentum */
    double roll;
    double t_read;         /* when the simulation takes over (s, reference timeline: 0 = first arrival) */
    double t_hit;          /* when the tip reaches the balloon */
    double v_impact;       /* speed there (m/s) */
    double sg_air;         /* gyroscopic stability there (infinite for a ball) */
    double yaw_impact_deg; /* angle between the axis and the velocity there */
    double twist;          /* rifling turns per metre */
    double muzzle_x[3], muzzle_u[3]; /* the launch */
} ntr_flight;
/* The flights of the scene's shots (as many as p->n_shots; the first `cap` are written). CPU only. */
NTR_API ntr_status ntr_shot_flights(const ntr_sim_params* p, ntr_flight* out, uint32_t cap, uint32_t* n);

/* --- Simulation on one GPU ---------------------------------------------------------------- */
/* Sim::new (src/sim.rs:208). */
NTR_API ntr_status ntr_sim_create(const ntr_sim_params* p, int device, ntr_sim** out);
/* A simulation from a world blob (a fixture, or a snapshot). */
NTR_API ntr_status ntr_sim_create_from_world(const void* blob, size_t len, int device, ntr_sim** out);
NTR_API ntr_status ntr_sim_destroy(ntr_sim* s);
/* Sim::run (src/sim.rs:585-648): one batch of up to n steps that stops at stop_ns, one state
 * read back, then the host's adaptation of solver iterations and substeps. */
NTR_API ntr_status ntr_sim_step(ntr_sim* s, uint32_t n, uint32_t stop_ns, uint32_t* taken);
/* Sim::advance (src/sim.rs:498-522). */
NTR_API ntr_status ntr_sim_advance(ntr_sim* s, double t_target, uint32_t budget, uint32_t* taken);
NTR_API ntr_status ntr_sim_read_state(ntr_sim* s, ntr_state* out);
NTR_API ntr_status ntr_sim_info_get(ntr_sim* s, ntr_sim_info* out);
/* Lends a device buffer. */
NTR_API ntr_status ntr_sim_buffer(ntr_sim* s, ntr_buf which, void** dev_ptr, size_t* bytes);
/* Copies a device buffer (or its first `bytes`) to host memory. */
NTR_API ntr_status ntr_sim_download(ntr_sim* s, ntr_buf which, void* host, size_t bytes);
/* The whole state as a world blob. With buf == NULL only *len is set. */
NTR_API ntr_status ntr_sim_snapshot(ntr_sim* s, void* buf, size_t cap, size_t* len);
/* Replaces the state with a world blob of the same scene sizes. */
NTR_API ntr_status ntr_sim_restore(ntr_sim* s, const void* blob, size_t len);
/* FP64 accumulation of the solver's inner products and residual (default on). */
NTR_API ntr_status ntr_sim_set_precision(ntr_sim* s, int fp64_reductions);
/* What `Sim::debug_stats` (src/sim.rs:691-863) prints, computed on the device (ntr_sim_stats).
 * Sums are FP64 (the reference's means are sequential FP32 sums); counts, minima and maxima are
 * exact. The clock, block count, solver and substep figures the reference prints beside these
 * are in ntr_state and ntr_sim_info. */
typedef struct ntr_stats_bullet {
    uint32_t state;    /* the bullet's phase (Bullet.info[2]) */
    uint32_t sections; /* cavity sections recorded (Bullet.info[3]) */
    float x[3];
    float speed;       /* m/s */
    float yaw_deg;     /* angle between the axis and the velocity */
    float spin_rev_s;
    double kinetic_j;
} ntr_stats_bullet;
typedef struct ntr_stats {
    /* water: particles with vel.w > 0.5 */
    uint32_t water, n_particles;
    float lo[3], hi[3];
    double mean[3], vmean[3];
    float vmax, fastest[3];     /* the fastest particle's speed and position (the first of equals) */
    double volume_l;            /* cells holding 4 or more particles, times their volume, litres */
    /* rubber */
    double inside_l;            /* volume the membrane encloses, litres */
    float mem_lo[3], mem_hi[3];
    uint32_t free_verts, on_water, torn, n_tension;
    float fill_min, fill_mean, rubber_vmax, pad0;
    double tension[3];          /* N/m, the most tense intact triangles, most tense first */
    uint32_t tension_tri[3], pad1;
    float stretch[3][2];        /* their principal stretches */
    /* air of the step's cells typed air */
    uint32_t air_cells, vapour_cells;  /* vapour: gauge below -90 kPa */
    float gauge_lo, gauge_hi, air_umax, pad2;
    /* energies */
    double water_j, bullets_j, vapour_cm3, vapour_j;
    uint32_t n_bullets, pad3;
    ntr_stats_bullet bullets[NTR_MAX_SHOTS];
} ntr_stats;
/* The statistics of the simulation's current state. The first call allocates its scratch on
 * the device (4 bytes per cell of the block capacity, and a few KB); it synchronises with the
 * simulation's stream. */
NTR_API ntr_status ntr_sim_stats(ntr_sim* s, ntr_stats* out);

/* The number of steps ntr_sim_advance puts in one batch. 0 (the default) is the reference's
 * rule: as many as fit in 4 ms of the measured step time, at most 256 (src/sim.rs:505-516).
 * The host adapts the solver's iterations and the substeps between batches, so where batches
 * end changes the results, and with the default that depends on the GPU's timing; a fixed
 * count makes runs repeat bit for bit. */
NTR_API ntr_status ntr_sim_set_batch_steps(ntr_sim* s, uint32_t n);
/* One batch as ntr_sim_step runs it, but launched kernel by kernel outside the step's graph
 * with an event after each, and a report of device time per kernel, one text line per kernel
 * name "name,launches,total_ms" (the reference's NATRAY_PROF, src/sim.rs:594-614, 670-689).
 * With report == NULL only *len (the report's length) is set. */
NTR_API ntr_status ntr_sim_profile(ntr_sim* s, uint32_t n, uint32_t stop_ns, char* report, size_t cap, size_t* len);
/* The work the steps did since the simulation was created or restored, or since the last call
 * with reset != 0, counted on the device by the steps themselves (out[k] for NTR_WORK_*): steps
 * taken; cells of their blocks (64 per block, summed over the steps); water cells times solver
 * iterations; rubber substeps; free-gas cells times air substeps; spray slots in use. The
 * algorithmic bytes of those steps follow from them (160 per particle and step, 160 per cell,
 * 48 per water cell and iteration, 256 per vertex and 32 per triangle and rubber substep, 44 per
 * gas cell and air substep, 48 per spray slot): the per-step quantities the reference's
 * profiler sees through its State readback (src/sim.rs:594-689). Waits for the stream. */
#define NTR_WORK_FIELDS 6
enum { NTR_WORK_STEPS = 0, NTR_WORK_CELLS, NTR_WORK_WATER_ITERS, NTR_WORK_MEM_SUBSTEPS, NTR_WORK_GAS_SUBSTEPS, NTR_WORK_SPRAY };
NTR_API ntr_status ntr_sim_work(ntr_sim* s, uint64_t out[NTR_WORK_FIELDS], int reset);
/* For tests of the failure path; no counterpart in the reference (whose solver loop is host
 * dispatches, fluid.wgsl:572-577, src/sim.rs:634-647). The persistent pressure solve's grid
 * barriers give up after `spins` polls (0: the default, 2^24), setting an error that the step
 * reports as NTR_E_TIMEOUT, and CTA `skip_cta` of the solve (0xFFFFFFFF: none) skips its first
 * arrival, so that every other CTA's wait runs out. Every CTA then returns: the kernel ends, the
 * context stays usable, and the state is that of a failed step (restore a snapshot). */
NTR_API ntr_status ntr_sim_test_barrier(ntr_sim* s, uint32_t spins, uint32_t skip_cta);
/* Kernel launches made by the last ntr_sim_step call, and its device time in ms. */
NTR_API ntr_status ntr_sim_last_launches(ntr_sim* s, uint64_t* launches, double* device_ms);
/* The particles in the reference's layout (`Particle`, sim_defs.wgsl:61: 20 f32 each, pos.xyzw,
 * vel.xyz + alive, c0, c1, c2), written into a device buffer the caller owns (16-byte aligned,
 * at least n_particles * 80 bytes): for a renderer or packer written against that layout, which
 * this library keeps as five arrays. Ordered after the simulation's work so far. With
 * stream != NULL (a cudaStream_t) the call is asynchronous and that stream's later work sees the
 * result; with NULL it returns once the buffer is written. */
NTR_API ntr_status ntr_sim_pack_particles(ntr_sim* s, void* dst_device, size_t bytes, void* stream);
/* Conservation sums over live particles, accumulated in FP64 on the device:
 * out[0] = live count, out[1..3] = momentum per particle mass, out[4] = kinetic energy per
 * particle mass, out[5..7] = sum of positions. */
NTR_API ntr_status ntr_sim_conservation(ntr_sim* s, double out[8]);

/* The device's sustained rate of shared-memory atomic adds (lane additions per second) at their
 * best, in P2G's CTA shape: the peak against which P2G's 216 such adds a particle are measured.
 * No counterpart in the reference. */
NTR_API ntr_status ntr_probe_shared_atomics(int device, uint32_t iters, double* lane_atomics_per_s);

/* --- Launch shapes and their autotuner ----------------------------------------------------
 * No counterpart in the reference (wgpu picks nothing of the kind). How many CTAs the step's
 * kernels use; the results do not depend on it, bit for bit. Zero fields take the defaults.
 * ntr_sim_autotune times `steps` steps of the simulation's own scene per candidate (restoring
 * its state before each and at the end, so the simulation is where it was), keeps the fastest
 * in the simulation and returns it. */
typedef struct {
    uint32_t solve_ctas;        /* CTAs of the cooperative pressure solve, 1..256 (default: all that fit, at most 256) */
    uint32_t cell_ctas_per_sm;  /* CTAs of 256 threads per SM of the per-cell kernels (default 8) */
    uint32_t block_ctas_per_sm; /* CTAs per SM of the per-block transfer kernels P2G and G2P (default 8 in a batch, 5 in
                                   a simulation: its step takes at most what an SM holds at once, its CTAs taking blocks as
                                   they come free, and 5 leaves G2P room for the rubber's kernels beside it) */
    uint32_t pad;
} ntr_tuning;
NTR_API ntr_status ntr_sim_get_tuning(ntr_sim* s, ntr_tuning* out);
NTR_API ntr_status ntr_sim_set_tuning(ntr_sim* s, const ntr_tuning* t);
NTR_API ntr_status ntr_sim_autotune(ntr_sim* s, uint32_t steps, ntr_tuning* best, double* best_ms_per_step);

/* --- Batches of independent scenes --------------------------------------------------------
 * No counterpart in the reference (it runs one Sim at a time, src/sim.rs:149-205): a serving
 * engine for many scenes of uneven size on one GPU. Each admitted scene keeps its state on the
 * device in its own slot. ntr_batch_step advances every unfinished scene by n steps: per step
 * one launch per kernel covers every scene (each its own range of CTAs, sized to it), and the
 * pressure systems of all of them are solved by ONE cooperative launch that splits the GPU
 * over them; the step is a CUDA graph, captured again only when the set of scenes or their
 * size classes change. A scene's results are bit for bit those of the same scene run alone
 * with ntr_sim_step(n) calls of the same n.
 *
 *   ntr_batch_create  max_scenes (at most NTR_BATCH_MAX) slots; hbm_budget bytes the batch may
 *                     hold on the device (0: no limit but the free memory)
 *   ntr_batch_admit   a world blob (ntr_world_build, ntr_sim_snapshot) into a free slot, to run
 *                     n_steps steps; NTR_E_BUSY when no slot is free or the scene's device memory
 *                     does not fit the budget or the free HBM (less a reserve): admit it later.
 *                     From any thread, also while another thread's ntr_batch_step runs: the
 *                     scene is created in a reserved slot outside the batch's lock, its uploads
 *                     on the slot's own stream beside the step's work
 *   ntr_batch_step    n steps of every unfinished scene (fewer for a scene that reaches its
 *                     target); *active (may be NULL) = scenes that stepped
 *   ntr_batch_poll    a slot's state and progress
 *   ntr_batch_snapshot  a slot's world blob, as ntr_sim_snapshot
 *   ntr_batch_retire  frees a slot; it keeps its device region for the next scene it takes, so
 *                     admitting and retiring make no device-wide synchronising allocation calls
 *                     unless a scene needs a bigger region */
#define NTR_BATCH_MAX 128u
typedef struct ntr_batch ntr_batch;
typedef struct {
    uint32_t in_use;      /* the slot holds a scene */
    uint32_t finished;    /* it has taken its steps */
    uint32_t steps_done, steps_target;
    uint64_t device_bytes;
    ntr_state state;
} ntr_batch_slot;
typedef struct {
    uint32_t max_scenes, in_use, active;
    uint32_t captures;     /* step graphs captured (for a new set of scenes or shapes) */
    uint64_t held_bytes;   /* device memory the slots hold (a slot keeps its region for its next scene) */
    uint64_t budget_bytes;
    uint64_t free_bytes;   /* free device memory now */
    uint64_t steps;        /* batch steps taken */
    uint32_t instantiations; /* of the captures, those that needed a new executable graph (the
                                others updated the last one in place) */
    uint32_t pad;
} ntr_batch_info;
NTR_API ntr_status ntr_batch_create(int device, uint32_t max_scenes, uint64_t hbm_budget, ntr_batch** out);
NTR_API ntr_status ntr_batch_destroy(ntr_batch* b);
NTR_API ntr_status ntr_batch_admit(ntr_batch* b, const void* world_blob, size_t len, uint32_t n_steps, uint32_t* slot);
NTR_API ntr_status ntr_batch_step(ntr_batch* b, uint32_t n, uint32_t* active);
/* ntr_batch_step's n steps launched kernel by kernel outside the batch's graph, one stream, an
 * event after each, and a report of device time per kernel, "name,launches,total_ms" a line (as
 * ntr_sim_profile; the reference's NATRAY_PROF, src/sim.rs:594-614, for one scene). With
 * report == NULL only *len is set. The scenes advance as with ntr_batch_step. */
NTR_API ntr_status ntr_batch_profile(ntr_batch* b, uint32_t n, char* report, size_t cap, size_t* len);
NTR_API ntr_status ntr_batch_poll(ntr_batch* b, uint32_t slot, ntr_batch_slot* out);
NTR_API ntr_status ntr_batch_snapshot(ntr_batch* b, uint32_t slot, void* buf, size_t cap, size_t* len);
NTR_API ntr_status ntr_batch_retire(ntr_batch* b, uint32_t slot);
NTR_API ntr_status ntr_batch_info_get(ntr_batch* b, ntr_batch_info* out);
/* The batch's launch shapes (ntr_tuning: the per-SM caps of every scene's cell and transfer
 * kernel grids, and the CTAs of the joint solve, at least one per scene; zero fields take the
 * defaults), for every scene in it and every scene it admits; a scene's results do not depend
 * on them. ntr_batch_autotune searches them as ntr_sim_autotune does, on the batch's own scenes:
 * one untimed and `steps` timed batch steps per candidate, which are steps of the scenes (they
 * are not put back), and keeps the fastest. */
NTR_API ntr_status ntr_batch_set_tuning(ntr_batch* b, const ntr_tuning* t);
NTR_API ntr_status ntr_batch_get_tuning(ntr_batch* b, ntr_tuning* out);
NTR_API ntr_status ntr_batch_autotune(ntr_batch* b, uint32_t steps, ntr_tuning* best, double* best_ms_per_step);
/* The device memory a simulation of this world takes (what admission to a batch checks against
 * its budget and the free memory; a server placing scenes on GPUs uses it). CPU only. */
NTR_API ntr_status ntr_world_device_bytes(const void* world_blob, size_t len, uint64_t* bytes);
/* Admission from any thread. Every ntr_batch_* call holds the batch's lock, so calls from
 * several host threads take turns (a call waits at most for the one in progress, such as a
 * batch step), except that a batch step lets the lock go while it waits for the GPU, during
 * which only ntr_batch_admit proceeds, and ntr_batch_admit holds it only to reserve a slot and
 * to place the scene. ntr_batch_enqueue checks the world blob, queues a copy and returns a ticket; the
 * queued scenes are admitted in order at the start of the next ntr_batch_step, as far as slots
 * and memory allow (a scene that does not fit yet stays at the head of the queue).
 * ntr_batch_ticket gives the ticket's slot once admitted, NTR_BATCH_MAX while it waits, and
 * NTR_E_INVALID if its admission failed. */
NTR_API ntr_status ntr_batch_enqueue(ntr_batch* b, const void* world_blob, size_t len, uint32_t n_steps, uint64_t* ticket);
NTR_API ntr_status ntr_batch_ticket(ntr_batch* b, uint64_t ticket, uint32_t* slot);

/* --- Sorting particles by block without allocating ------------------------------------------
 * No counterpart in the reference: an addition for callers that cannot allocate device
 * memory, such as a host application whose framework has reserved the GPU's memory for its
 * own pool, or a frame loop that must not make the device-wide synchronising cudaMalloc and
 * cudaFree calls. The same stable radix sort the step uses (particles grouped by block index,
 * ascending particle index within a block), with its scratch in a fixed array inside this
 * library: NTR_NOALLOC_MAX_KEYS keys, NTR_NOALLOC_MAX_BLOCKS blocks (about 13 MB, held on every
 * GPU that loads the library until the process exits).
 *
 *   keys         device array of n block indices (< n_blocks), or 0xFFFFFFFF for a particle
 *                that takes no part
 *   sorted       device array of n: the particle indices, grouped by block; the first
 *                block_start[n_blocks] entries are meaningful
 *   block_start  device array of n_blocks + 1: where each block's particles start in sorted
 *   stream       a cudaStream_t (NULL: the default stream); the call is asynchronous on it
 *
 * The first call on a device looks up the scratch array's device address for that device; make
 * that first call before any stream capture. Every call shares the one scratch array, so calls
 * whose work overlaps on the GPU (different streams, or different host threads) race: order
 * them. n > NTR_NOALLOC_MAX_KEYS or n_blocks > NTR_NOALLOC_MAX_BLOCKS is NTR_E_INVALID. */
#define NTR_NOALLOC_MAX_KEYS 1048576u
#define NTR_NOALLOC_MAX_BLOCKS 65535u
NTR_API ntr_status ntr_sort_by_block_noalloc(const uint32_t* keys, uint32_t n, uint32_t n_blocks, uint32_t* sorted,
                                             uint32_t* block_start, void* stream);

/* --- Keyframe cache: `Cache` of src/cache.rs ------------------------------------------------
 * The simulation runs ahead and stores compact keyframes in a fixed device pool; playback
 * blends between two of them into the buffers a renderer reads. A keyframe is, in u32 words
 * (shaders/keys.wgsl:1-10): the spray slot count, the live spray count and two zero words;
 * two words per water particle and per membrane vertex (21 bits per axis inside the 8 m box
 * [-4, 4] x [-0.5, 7.5] x [-4, 4], the top bit of the second word set for a live particle); one
 * alive bit per triangle; then, for the spray, one live bit per slot, the live count before each
 * word of bits, and three words (position, radius bits) per live slot in slot order. A
 * keyframe is rounded up to 256 bytes and never spans two pool pages.
 *
 * The cache borrows the simulation: it steps it in ntr_cache_bake and reads its buffers, and
 * the simulation must outlive the cache (or be replaced with ntr_cache_rebuild). Every device
 * buffer is allocated in ntr_cache_create; bake and show never allocate. */
#define NTR_KEY_HEAD 4u        /* header words (src/cache.rs:20) */
#define NTR_KEY_SPRAY_WORDS 3u /* words per live spray slot (src/cache.rs:21) */
#define NTR_KEY_Q_MAX 2097151u /* position steps per axis over the 8 m box (shaders/keys.wgsl:18-20) */

typedef struct ntr_cache ntr_cache;

typedef struct ntr_cache_params {
    uint64_t page_bytes; /* 128 MiB (src/cache.rs:16) */
    uint32_t pages;      /* 16 (src/cache.rs:17) */
    uint32_t n_arrivals; /* entries of `arrivals` in use, at most NTR_MAX_SHOTS */
    double t_end;        /* end of the timeline, 1 s (src/cache.rs:14) */
    double arrivals[NTR_MAX_SHOTS]; /* each shot's arrival time `flight.t_hit` (src/cache.rs:257) */
} ntr_cache_params;

/* One stored keyframe (`Key`, src/cache.rs:58-66). */
typedef struct ntr_key_info {
    double t;        /* simulated time */
    uint64_t offset; /* bytes into its page */
    uint64_t bytes;  /* its size (ntr_key_bytes) */
    uint32_t page;
    uint32_t spray;  /* spray slots in use */
    uint32_t live;   /* of those, live */
    uint32_t pad;
} ntr_key_info;

typedef struct ntr_cache_info {
    uint32_t keys, done, full, shown_spray;
    uint64_t used_bytes, pool_bytes, shown_id;
    double end;    /* time of the newest keyframe */
    double next_t; /* when the next keyframe is due */
    double shown;  /* time of the shown state; NaN until the first ntr_cache_show */
} ntr_cache_info;

/* The buffers ntr_cache_show fills (src/cache.rs:393-408), plus the spray weights. */
typedef enum ntr_shown {
    NTR_SHOWN_PARTICLES = 0, /* n_particles x 2 float4: position (w 1), velocity (w 1 live, 0 not) */
    NTR_SHOWN_SPRAY,         /* spray_cap x 2 float4: position + radius, velocity + weight (negative
                                while the drop is still part of the crown sheet) */
    NTR_SHOWN_MEM_POS,       /* n_verts float4 (w 0) */
    NTR_SHOWN_ALIVE,         /* n_tris u32, 1 for an intact triangle */
    NTR_SHOWN_WET,           /* wet_res^2 u32: water on the ground, 1e-3 mm^3 per cell */
    NTR_SHOWN_SPRAY_W,       /* spray_cap float2: weight, time the drop tears loose */
    NTR_SHOWN_COUNT
} ntr_shown;

/* Cache parameters for a scene: the reference's pool and timeline, and the shots' arrival
 * times as Sim::new computes them (src/sim.rs:280-291: delay minus the earliest delay). CPU only. */
NTR_API ntr_status ntr_cache_params_default(const ntr_sim_params* p, ntr_cache_params* out);
/* Bytes of a keyframe with `spray` slots of which `live` are in use (`key_bytes`,
 * src/cache.rs:412-421). CPU only. */
NTR_API uint64_t ntr_key_bytes(uint32_t n_particles, uint32_t n_verts, uint32_t n_tris, uint32_t spray, uint32_t live);
/* When the keyframe after one stored at `t` is due (src/cache.rs:249-264): 2% of the time since
 * the last arrival, between 10 us and 4 ms, stretched when the keys still to come at that
 * spacing would overrun the free pool, and never past the next arrival or t_end. CPU only. */
NTR_API double ntr_key_next_time(double t, const double* arrivals, uint32_t n_arrivals, double t_end,
                                 uint64_t free_bytes, uint64_t key_bytes);

/* Cache::new without the Sim::new: allocates the pool and the shown buffers, takes the
 * simulation to its start (Sim::advance(0, 0)) and stores the first keyframe. */
NTR_API ntr_status ntr_cache_create(ntr_sim* s, const ntr_cache_params* cp, ntr_cache** out);
/* Cache::rebuild: starts over on another simulation (or the same one restored), reusing the
 * pool. The shown buffers are reallocated when the scene sizes change. */
NTR_API ntr_status ntr_cache_rebuild(ntr_cache* c, ntr_sim* s);
NTR_API ntr_status ntr_cache_destroy(ntr_cache* c);
/* Cache::bake: up to max_steps simulation steps, storing keyframes when they are due. */
NTR_API ntr_status ntr_cache_bake(ntr_cache* c, uint32_t max_steps, uint32_t* steps);
/* Stores a keyframe of the simulation's current state now (what bake does when one is due;
 * the schedule of later keys follows from it). */
NTR_API ntr_status ntr_cache_store(ntr_cache* c);
/* Cache::show: fills the shown buffers for time t (clamped to what was simulated). *changed
 * is 0 when t is what is shown already. Asynchronous on the simulation's stream. */
NTR_API ntr_status ntr_cache_show(ntr_cache* c, double t, int* changed);
NTR_API ntr_status ntr_cache_info_get(ntr_cache* c, ntr_cache_info* out);
/* Device time (ms) of the last keyframe store, in its two parts (the spray index, then the
 * packing; the host's read of the spray counts between them is in neither), and of the last
 * show, measured with events on the simulation's stream; 0 before the first. Any pointer may be
 * NULL. Waits for the timed work to finish. */
NTR_API ntr_status ntr_cache_last_times(ntr_cache* c, double* index_ms, double* pack_ms, double* show_ms);
NTR_API ntr_status ntr_cache_key(ntr_cache* c, uint32_t k, ntr_key_info* out);
/* Lends keyframe k's words (valid until the cache restarts or is destroyed). */
NTR_API ntr_status ntr_cache_key_buffer(ntr_cache* c, uint32_t k, void** dev_ptr, size_t* bytes);
/* Lends a shown buffer (valid until rebuild or destroy). */
NTR_API ntr_status ntr_cache_buffer(ntr_cache* c, ntr_shown which, void** dev_ptr, size_t* bytes);
/* Copies the first `bytes` of a shown buffer, or of keyframe k's words when which is
 * NTR_SHOWN_COUNT + k, to host memory (synchronous). */
NTR_API ntr_status ntr_cache_download(ntr_cache* c, uint32_t which, void* host, size_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* NATRAY_H */
