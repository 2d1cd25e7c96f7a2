/*
 * ivp.h -- C ABI of the B200 implicit velocity projection (IP) pressure step.
 *
 * Drop-in boundary for the reference's IP pressure-solver plugin
 * (medialab-ku/ImplicitVelocityProjection).  Every entry point names the
 * reference interface it replaces.  Memory is owned by the caller (PyTorch
 * tensors in the Python host layer): the engine receives raw device pointers,
 * counts and a CUDA stream, and allocates no device memory after
 * ivp_engine_create.  No C++ exceptions cross this boundary; every call
 * returns an ivp_status.
 *
 * Streams are passed as `void*` holding a cudaStream_t (NULL = legacy default
 * stream).  Calls are stream-ordered and asynchronous unless stated.  One
 * host thread drives an engine at a time; engines are independent.
 */
#ifndef IVP_H
#define IVP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference raises RuntimeError for NOT_SPD
 * (scripts/sim/forces/pressure/ip.py:308-309) and NOT_CONVERGED
 * (scripts/sim/forces/pressure/pressure_base.py:487-495). */
typedef enum {
    IVP_OK = 0,
    IVP_ERR_NOT_SPD = 1,        /* CG saw p^T A p < 0 */
    IVP_ERR_NOT_CONVERGED = 2,  /* outer-iteration cap reached above densityErrorTol */
    IVP_ERR_NBR_OVERFLOW = 3,   /* truncated neighbour lists (more neighbours than neighborCacheSize) dropped
                                   more pairs than the engine's transpose-correction storage holds; lists
                                   are truncated as the reference does (neighbour_search.py:38-51) and
                                   solved with its exact transpose otherwise (ip.py:110-121) */
    IVP_ERR_BAD_ARG = 4,
    IVP_ERR_CUDA = 5,
    IVP_ERR_TIMEOUT = 6,
    IVP_ERR_NOT_BOUND = 7,      /* particle arrays not bound */
    IVP_ERR_DEVICE_CHECK = 8    /* a device-side bounds check failed (index out of range) */
} ivp_status;

/* One independent scene.  Its particles occupy [particle_offset,
 * particle_offset + n_particles) of the bound arrays.  Field meanings follow
 * the reference's configuration keys (scripts/io/config_builder.py:10-115,
 * ip.py:228-229, pressure_base.py:314-317, simulation_data.py:157). */
typedef struct {
    int32_t particle_offset;
    int32_t n_particles;
    int32_t n_dynamic;          /* particles with is_dynamic == 1 in the range */
    float particle_radius;      /* r: d = 2r, support radius h = 4r */
    float domain_size[3];       /* domain [0, L) per axis (boundary clamp, grid) */
    float dt;                   /* timeStepSize */
    float gravity[3];           /* gravitation */
    float omega;                /* IP omega (default 10) */
    double tol_pcg;             /* absolute ||r||^2 tolerance of CG (default 1e-6) */
    double density_error_tol;   /* densityErrorTol (default 1e-3) */
    int32_t max_outer_iters;    /* maxOuterIters (default 1000) */
    int32_t max_iteration_pcg;  /* CG cap (reference hard-codes 1000) */
    int32_t fixed_outer_iters;  /* fixedOuterIters (0/1) */
    int32_t cache_size;         /* neighborCacheSize (default 60) */
    float viscosity_coeff;      /* kinematic viscosity for Weiler18 (viscosityMethod 1) */
    int32_t viscosity_method;   /* 0 off, 1 Weiler 2018 implicit */
    int32_t surface_tension_method;  /* 0 off, 1 Jeske 2023 implicit (surfaceTensionMethod) */
    float surface_tension_coeff;     /* sigma (surfaceTensionCoeff) */
    int32_t pressure_solver;         /* IVP_SOLVER_IP (0, pressureMethod 1) or IVP_SOLVER_PRJ (1, pressureMethod 0) */
    int32_t reserved[1];
} ivp_scene_desc;

typedef struct {
    int32_t lanes_per_particle;   /* 1, 2, 4 or 8 lanes share one particle's neighbour sum; 0 (default):
                                     chosen from the scenes (ivp_resolve_options) */
    int32_t particles_per_block;  /* particles per CTA in the neighbour-sum kernels; 0: chosen with
                                     the lane count */
    int32_t list_stride;          /* neighbour-list row stride: even, >= every scene's cache_size */
    int32_t max_hist;             /* per-scene stats history length (outer iterations) */
    int32_t use_graphs;           /* 1: whole steps as CUDA graphs (device-side control, no host sync) */
    int32_t persistent;           /* 1: the IP solve as one persistent cooperative kernel with grid barriers;
                                     0: one launch per phase, loops as conditional graph nodes */
    int32_t row_format;           /* neighbour-row entries: 0 default (= 1), 1 full {m_j gradW_ij, j}
                                     (16 B), 2 compact {j, w_ij} (8 B, gradient rebuilt from the
                                     positions: half the list memory, slower; bit-identical to 1),
                                     3 bf16 (4 B id + the gradient in 3 bf16: the reduced-precision
                                     variant, 10 B per entry) */
    int32_t build_kernel;         /* neighbour build: 1 one thread per particle walking its 27-cell
                                     window, 2 one warp per cell sharing each candidate among 4
                                     particles; the same lists in the same order.  0 (default):
                                     chosen from the scenes (1 from 256 dynamic particles per SM) */
} ivp_options;

/* Device arrays in the reference's layout and particle order
 * (scripts/sim/simulation_data.py:165-212).  vec3 arrays are float[N][3]. */
typedef struct {
    float* x;              /* positions (read; written by ivp_advect / ivp_step) */
    float* v;              /* velocities (read/write) */
    const float* m;        /* masses (static particles carry the reference's x10) */
    const float* density0; /* rest densities */
    const int32_t* is_dynamic;
    const int32_t* material;
    float* density;        /* out: SPH density (ps.density) */
    float* kdiag;          /* out: k = 1/(Aii + eps) (PressureBase.k) */
    float* divergence;     /* out, may be NULL: max(J v, 0) (ps.divergence) */
    int32_t n_total;       /* particles in the arrays (sum over scenes) */
} ivp_particles;

/* Per-scene results of the last IP solve (pressure_base.py:331-339). */
typedef struct {
    int32_t status;
    int32_t outer_iters;          /* stats_outer_iters */
    int32_t n_density_errors;     /* entries of stats_density_errors */
    int32_t overflow_particles;   /* particles whose neighbour count exceeded cache_size */
    double final_density_error;   /* stats_final_density_error */
    double last_density_error;
    int32_t total_pcg_iters;      /* CG iterations of the last solve */
    /* counters since ivp_reset_counters (kept on the device, no host sync per step) */
    int32_t solves;
    int32_t failed_solves;
    int32_t last_failure;         /* status of the last failed solve */
    int64_t sum_outer_iters;
    int64_t sum_pcg_iters;
    double max_final_density_error;
    int64_t neighbour_pairs;      /* pairs in the scene's current neighbour lists */
    int64_t sum_visc_iters;       /* implicit-viscosity CG iterations */
    int64_t sum_st_iters;         /* implicit surface-tension CG iterations */
    double last_pap;              /* p^T A p of the last CG iteration (the value the reference prints
                                     with its non-positive-definite error, ip.py:308-309) */
    int32_t last_cg_iter;         /* CG iterations completed in the last PCG call when it stopped */
    int32_t fixup_entries;        /* transpose corrections of the scene's last build (non-zero only when
                                     some list was truncated at cache_size) */
} ivp_solve_stats;

/* Pressure solvers (ivp_scene_desc.pressure_solver). */
enum { IVP_SOLVER_IP = 0, IVP_SOLVER_PRJ = 1 };

/* Kernel ids reported by ivp_profile_step. */
enum {
    IVP_K_GRAVITY = 0, IVP_K_SOLVE_BEGIN, IVP_K_PACK, IVP_K_RHS, IVP_K_CG_A, IVP_K_CG_B, IVP_K_SOLVE_END,
    IVP_K_DIVERGENCE, IVP_K_ADVECT, IVP_K_KEYS, IVP_K_SCAN_LOCAL, IVP_K_SCAN_ADD, IVP_K_PLACE, IVP_K_ORDER,
    IVP_K_NBR_BUILD, IVP_K_STATIC_OUT, IVP_K_VISC, IVP_K_PERSISTENT, IVP_K_SURFACE_TENSION, IVP_K_PRJ,
    IVP_K_COUNT = 24
};

typedef struct ivp_engine ivp_engine;

/* Defaults for ivp_options: engine settings with no counterpart in the
 * reference (its solver settings are per scene, in ivp_scene_desc). */
void ivp_default_options(ivp_options* opt);

/* The options an engine over these scenes runs with: a lane count of 0
 * becomes 4 lanes x 64 particles per CTA while the scenes' dynamic
 * particles fill at most 16 such tiles per SM of the current device, else 2
 * lanes x 128 particles (many tiles per CTA: fewer, larger tiles per phase);
 * a particles-per-block of 0 follows the lane count (256 threads).  Other
 * fields are copied.  ivp_workspace_bytes and ivp_engine_create resolve the
 * options the same way.  No counterpart in the reference (Warp picks its own
 * launch shapes). */
int ivp_resolve_options(const ivp_scene_desc* scenes, int32_t n_scenes, const ivp_options* opt, ivp_options* out);

/* Workspace bytes for a set of scenes (no allocation).  Replaces the
 * solver's own allocations at particle_max_num (ip.py:232-242,
 * pressure_base.py:290-302) with one caller-owned workspace. */
int ivp_workspace_bytes(const ivp_scene_desc* scenes, int32_t n_scenes, const ivp_options* opt, size_t* bytes);

/* Creates an engine over a caller-owned device workspace of
 * ivp_workspace_bytes bytes (256-byte aligned).  Builds the scene tables on
 * the device.  Replaces the construction of SimulationData / NeighbourSearch
 * / IP (scripts/sim/simulation_data.py:118-212, neighbour_search.py:93-114,
 * ip.py:225-242). */
int ivp_engine_create(const ivp_scene_desc* scenes, int32_t n_scenes, const ivp_options* opt, void* workspace,
                      size_t workspace_bytes, void* stream, ivp_engine** out);
int ivp_engine_destroy(ivp_engine* e);

/* Updates the run-time parameters of one scene (dt, gravity, omega, tolerances,
 * iteration caps, viscosity coefficient) -- the attributes the reference's
 * GUI and Framework change between steps (gui.py:435-473, IP.solve(dt)).
 * Geometry fields (particle counts, radius, domain, cache size) must be
 * unchanged.  Stream-ordered. */
int ivp_update_scene(ivp_engine* e, int32_t scene, const ivp_scene_desc* desc, void* stream);

/* Binds the particle arrays (replaces the SimulationData arrays). */
int ivp_engine_bind(ivp_engine* e, const ivp_particles* p);

/* NeighbourSearch.build + build_cache (neighbour_search.py:116-155) fused with
 * PressureBase.compute_density and compute_Aii (pressure_base.py:341-365):
 * cell hash, counting sort by cell, reordered particle copies, compact
 * neighbour lists, density and k.  Also writes density/kdiag of the bound
 * arrays. */
int ivp_neighbour_build(ivp_engine* e, void* stream);

/* PressureBase.compute_density / compute_Aii (pressure_base.py:341-365) from
 * the current lists and the bound positions/masses. */
int ivp_compute_density(ivp_engine* e, void* stream);
int ivp_compute_aii(ivp_engine* e, void* stream);

/* IP.solve(dt) (ip.py:331-404) for every scene: outer loop, CG, v = d/dt,
 * stats.  Asynchronous; read results with ivp_read_stats. */
int ivp_ip_solve(ivp_engine* e, void* stream);

/* Weiler18.solve(coeff, dt) (scripts/sim/forces/non_pressure/viscosity/
 * weiler18.py:371-401): implicit viscosity with block-Jacobi PCG for every
 * scene whose viscosity_method is 1 and viscosity_coeff > 0; updates the bound
 * velocities.  Uses the current neighbour lists and densities. */
int ivp_viscosity_solve(ivp_engine* e, void* stream);

/* Jeske23.solve(sigma, sigma, dt) (scripts/sim/forces/non_pressure/
 * surface_tension/jeske23.py:585-655): implicit surface tension with Jacobi
 * PCG for every scene whose surface_tension_method is 1 and
 * surface_tension_coeff > 0; updates the bound velocities.  Uses the current
 * neighbour lists and densities.  ivp_step runs it after gravity and before
 * the viscosity (framework.py:400-421). */
int ivp_surface_tension_solve(ivp_engine* e, void* stream);

/* PRJ.solve(dt) (scripts/sim/forces/pressure/prj.py:296-340): projected
 * Jacobi on the constant-density constraint (IISPH-style, omega 0.5, no warm
 * start, no divergence-free pass) for every scene whose pressure_solver is
 * IVP_SOLVER_PRJ; v = dt_v / dt unless the scene does not converge.  Stats as
 * for the IP solve (stats_outer_iters = passes). */
int ivp_prj_solve(ivp_engine* e, void* stream);

/* apply_gravity (framework.py:26-41). */
int ivp_apply_gravity(ivp_engine* e, void* stream);

/* advect_position + enforce_boundary (framework.py:117-136, boundary.py:27-91). */
int ivp_advect(ivp_engine* e, void* stream);

/* n_steps of Framework.forward() with IP (framework.py:423-544): gravity,
 * implicit viscosity where a scene enables it, IP solve, advect + clamp,
 * neighbour rebuild, density, Aii.  The engine must have been built once
 * (ivp_neighbour_build), as Framework.initialize does (framework.py:323-330). */
int ivp_step(ivp_engine* e, int32_t n_steps, void* stream);

/* One ivp_step whose particle state comes from and goes back to host memory,
 * as a caller of Framework.forward() that keeps x and v on the host would copy
 * it around each step (framework.py:423-544 works on device arrays): x_in /
 * v_in (float[count][3], particles [first, first + count) of the bound
 * arrays) are uploaded and x_out / v_out downloaded inside the step,
 * overlapped with its kernels -- v before the first force, x beside the
 * solves (the advection is its first reader), both downloads beside the next
 * step's neighbour build (the advection is the last writer of x and v).
 * Inputs and outputs may alias (the upload of x lands before the advection,
 * the downloads start after it).  Any pointer may be NULL (that copy is
 * skipped).  Host buffers must be page-locked (IVP_ERR_BAD_ARG otherwise).
 * The outputs are complete when the stream has passed the step. */
int ivp_step_io(ivp_engine* e, const float* x_in, const float* v_in, float* x_out, float* v_out, int64_t first,
                int64_t count, void* stream);

/* Zeroes the counters reported in ivp_solve_stats (stream-ordered). */
int ivp_reset_counters(ivp_engine* e, void* stream);

/* Runs n_steps of ivp_step with host-driven launches (no graphs) and CUDA
 * events around every kernel; accumulates per-kernel device milliseconds and
 * launch counts into ms[IVP_K_COUNT] and launches[IVP_K_COUNT].  Synchronous.
 * Same results as ivp_step.  The reference times only whole solves
 * (stats_total_cost_ms, pressure_base.py:331-339); no per-kernel counterpart. */
int ivp_profile_step(ivp_engine* e, int32_t n_steps, void* stream, double* ms, int32_t* launches);

/* Builds and instantiates the engine's neighbour-build and step graphs
 * without launching them, so that the first ivp_neighbour_build / ivp_step
 * of a new engine spends no host time on graph construction (the served form
 * prepares the next batch's engine while the current one runs).  Host only;
 * the particle arrays must be bound.  No counterpart in the reference. */
int ivp_prepare(ivp_engine* e);

/* ivp_read_stats of every scene (out[n_scenes]) with one stream
 * synchronisation: the per-scene statistics attributes after a batched step
 * (pressure_base.py:331-339). */
int ivp_read_stats_all(ivp_engine* e, void* stream, ivp_solve_stats* out);

/* Synchronises the stream and copies one scene's stats of the last solve:
 * the statistics attributes of IP / PressureBase (pressure_base.py:331-339). */
int ivp_read_stats(ivp_engine* e, int32_t scene, void* stream, ivp_solve_stats* out);

/* Copies up to `cap` per-outer-iteration density errors / CG iteration counts
 * of the last solve (stats_density_errors, stats_pcg_iters,
 * pressure_base.py:331-339).  Synchronous. */
int ivp_read_history(ivp_engine* e, int32_t scene, void* stream, double* errors, int32_t* pcg_iters, int32_t cap,
                     int32_t* n_errors, int32_t* n_pcg);

/* ivp_read_stats and ivp_read_history of one scene with a single stream
 * synchronisation: everything IP.solve leaves in its statistics attributes
 * after a solve (pressure_base.py:331-339, ip.py:394-404), as read after
 * every Framework.forward(). */
int ivp_read_solve(ivp_engine* e, int32_t scene, void* stream, ivp_solve_stats* out, double* errors,
                   int32_t* pcg_iters, int32_t cap, int32_t* n_errors, int32_t* n_pcg);

/* Exports the neighbour lists of one scene in the reference's cache layout
 * (neighbor_count[N], neighbor_ids[N*cache]) with original particle indices,
 * for parity checks.  Synchronous, device pointers. */
int ivp_export_neighbours(ivp_engine* e, int32_t scene, int32_t* count, int32_t* ids, int32_t cache, void* stream);

/* Test hook, no counterpart in the reference (whose launches never wait on
 * one another).  Sets how long any wait of the engine's persistent kernels on
 * a grid barrier may last before the kernel gives up, sets the timeout flag
 * and returns (default 2 s; ns <= 0 restores it).  A solve cut short this way
 * reports IVP_ERR_TIMEOUT until ivp_reset_counters clears the flag.  Host
 * only: rebuilds the engine's graphs at their next launch. */
int ivp_set_wait_limit(ivp_engine* e, int64_t ns);

/* Limits of ivp_density_aii_noalloc. */
#define IVP_NOALLOC_MAX_PARTICLES 65536
#define IVP_NOALLOC_MAX_CELLS 262144

/* No counterpart in the reference.  SPH density and k = 1/(Aii + 1e-3) of
 * every dynamic particle of one scene (k = 0 for static particles), for
 * callers that cannot allocate device memory: code living inside another
 * runtime's memory arena (whose GPU memory another allocator owns), or
 * real-time loops that cannot take the device synchronisation of
 * cudaMalloc/cudaFree.  It allocates nothing and
 * needs no workspace: its scratch is one fixed device array inside the
 * library (about 6.3 MB, held on every GPU that loads the library until the
 * process exits).  Results equal those of ivp_neighbour_build for the same
 * particles.  Inputs: x float[n][3], m float[n], is_dynamic int[n] (caller
 * order, device pointers); outputs density[n], kdiag[n] (density of static
 * particles is left untouched).  At most IVP_NOALLOC_MAX_PARTICLES particles
 * and IVP_NOALLOC_MAX_CELLS cells of size h = 4 r over the domain; larger
 * inputs return IVP_ERR_BAD_ARG without touching the device.  All calls share
 * the scratch array: calls whose GPU work overlaps (other streams or host
 * threads) race and must be serialised by the caller.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current; make that first call before any stream capture. */
int ivp_density_aii_noalloc(const float* x, const float* m, const int32_t* is_dynamic, int32_t n_particles,
                            float particle_radius, const float* domain_size, int32_t cache_size, float* density,
                            float* kdiag, void* stream);

const char* ivp_status_string(int32_t status);
/* Last CUDA error string seen by the engine (thread-local). */
const char* ivp_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* IVP_H */
