// ivp_device.cuh -- device data layout and helpers of the IP pressure step.
//
// Layout in HBM (one engine = one or more independent scenes):
//   * bound particle arrays, caller order (SimulationData layout): x, v, m,
//     density0, is_dynamic, material; outputs density, k;
//   * slots: every particle gets one slot per rebuild; slots are ordered by
//     (scene, dynamic-before-static, cell, particle id).  Scene s owns slots
//     [s_begin, s_end), its dynamic particles [s_begin, s_dyn_end).  Because
//     of that order "j is dynamic" is `j < s_dyn_end` (no load), and the
//     vector arrays of the solver hold exact zeros at static slots, which
//     makes the reference's `[dyn j]` branches (ip.py:55-58, 160-163,
//     209-213) branch-free with identical rounding;
//   * per-slot arrays: xm (float4 x,y,z,m), rest density, density, k, c, and
//     the solver vectors as float4 (16-byte gathers);
//   * neighbour rows, one per dynamic particle, `stride` entries of float4
//     {J_ij, neighbour slot}: J_ij = m_j grad W_ij, the per-pair vector the
//     reference forms from its cache (J_ij / val_ij in pressure_base.py:81
//     and ip.py:54; spiky gradient of sph_kernel.py:52-61).  Every
//     neighbour sum then streams its row and gathers only the neighbour's
//     operand: mass-weighted terms use (m_j a_i + m_i a_j) grad W_ij =
//     (a_i + m_i (a_j / m_j)) J_ij with a_j / m_j stored per particle;
//   * tiles: (scene, first slot, end slot, first row) -- a tile never spans
//     two scenes, so per-scene reductions are per-tile FP64 partials summed
//     in one fixed association over the scene's tiles (128 logical lanes,
//     then a fixed tree), whichever CTA or launch produced them: the same
//     bits in the persistent and per-phase paths and for a scene alone or
//     in a batch.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ivp {

constexpr int kMaxHistDefault = 128;
constexpr int SOLVER_IP = 0, SOLVER_PRJ = 1;

struct SceneParams {
    int p_begin, p_end;        // particle range in the bound arrays
    int s_begin, s_dyn_end, s_end;
    int n_dyn;
    int row_base;              // first neighbour row of this scene
    int key_base;              // keys [key_base, key_base + 2*ncell): dynamic cells, then static cells
    int dims[3];
    int ncell;
    float cell_inv;            // 1/h (cell size = support radius, neighbour_search.py:105-107)
    float h;
    float dt, inv_dt, omega, padding;
    float domain[3];
    float gravity[3];
    float r2_max;              // largest FP32 d2 with sqrtf(d2) < h: `d2 <= r2_max` is the strict `|r| < h` test
    float inv_h;
    float W0;                  // cubic_kernel(0, h)
    float cubic_k;             // 8/pi / h^3 (sph_kernel.py:14-15)
    float spiky_k;             // 45 / (pi h^6) (sph_kernel.py:55)
    float visc_coeff;
    int visc_method;
    float st_coeff;            // Jeske 2023 surface tension sigma
    int st_method;
    float st_d;                // particle diameter d (W^st clamps r at d)
    float st_h;                // surface-tension support h_st = 2 d (jeske23.py:455)
    int solver;                // SOLVER_IP or SOLVER_PRJ
    int max_outer, max_pcg, fixed_iters, cache;
    int tile_begin, tile_end;
    int hist_base;
    double tol_opt, tol_pcg;
};

// Per-scene solver control block, written by the CTA that decides a phase
// (the scene's last CTA of a per-phase launch; in a persistent kernel CTA 0
// or the last CTA to arrive at the barrier) and read by every CTA of the next
// phase.
struct SceneCtl {
    double err;          // last average density error
    double rr_old;
    double pap;
    double alpha;
    double beta;
    double final_err;
    double rr0;
    int outer_it;        // updates applied (stats_outer_iters)
    int cg_it;
    int outer_active;
    int solve_pending;
    int cg_active;
    int status;
    int n_err;
    int total_cg;
    // implicit non-pressure CG, shared by the surface tension (Jeske 2023,
    // jeske23.py:520-579) and viscosity (Weiler 2018, weiler18.py:298-365)
    // solves, which run one after the other
    double v_rz;         // r.z of the current iterate
    double v_alpha;
    double v_beta;
    double v_pap;
    int v_active;        // CG running
    int v_it;            // CG iterations of this solve
    int v_total;         // CG iterations of the last step (stats)
    int v_on;            // the force being solved is enabled for this scene (set at its start)
    int v_max;           // CG iteration cap of that force (100 surface tension, 1000 viscosity)
    int v_pad;
    // sticky counters since the last reset (ivp_reset_counters)
    double acc_max_final_err;
    int acc_solves;
    int acc_outer;
    int acc_cg;
    int acc_failed;
    int acc_last_failure;
    int acc_visc;        // viscosity CG iterations
    int acc_st;          // surface-tension CG iterations
};

static_assert(sizeof(SceneCtl) % sizeof(double) == 0, "SceneCtl is read as doubles");

struct Flags {
    int any_outer, any_solve, any_cg, bad;
    int any_visc, pad_v;
    int bad_index, bad_where;
    // loop guard: decision launches of the current solve and their budget;
    // past the budget every active scene stops with IVP_ERR_TIMEOUT, so a
    // control-flow fault cannot keep a conditional graph loop running
    int launches, limit;
    int timeout, pad0, pad1, pad2;
};

// Byte layout of the statistics staging block: the scene's control block,
// overflow count, the flags, pair count, correction count, then its error and
// CG-count histories (max_hist entries each).
struct StatStage {
    size_t ctl, ovf, flags, pairs, fix, err, pcg, total;
    __host__ __device__ static size_t up8(size_t b) { return (b + 7) & ~size_t(7); }
    __host__ __device__ explicit StatStage(int hist);
};

struct Dev {
    // bound arrays (caller order)
    float* x;
    float* v;
    const float* m;
    const float* rho0;
    const int* dyn;
    const int* material;
    float* density_out;
    float* k_out;
    float* div_out;
    int n_total;
    // tables
    const SceneParams* scenes;
    int n_scenes;
    SceneCtl* ctl;
    const int4* tiles;       // (scene, slot begin, slot end, row begin)
    const int4* segs;        // neighbour-build cell segments (scene, cy, cz, x_lo)
    int n_segs;
    int* live_segs;          // segments holding dynamic particles in the current build (any order)
    int* seg_ctr;            // [0] live segment count
    int n_tiles;
    const int* pscene;       // scene of each particle
    // sort
    int* key;
    int* rank;
    int* cell_count;
    int* cell_start;         // n_keys + 1
    int* block_sums;
    int n_keys;
    int* placed;             // slot -> particle (unstable within a cell)
    int* pid;                // slot -> particle (stable)
    int* inv;                // particle -> slot
    int* overflow;           // per scene
    unsigned long long* pairs;  // per scene: neighbour pairs of the last build
    // neighbour-cache overflow (a dynamic particle with more than cache_size
    // neighbours): its row is rebuilt with the reference's first cache_size
    // hits, and CG phase B adds the transpose terms the gather form gets
    // wrong for pairs that appear in only one of the two rows (the
    // reference's scatter form, ip.py:110-121, is the exact transpose)
    int* ovf_list;           // [n_dyn] slots whose lists were truncated in the current build
    int* ovf_ctr;            // [0] truncated particles, [1] dropped dynamic pairs
    int2* drop;              // [drop_cap] (o, k): dynamic k within h of o, left out of o's row
    float4* drop_w;          // [drop_cap] J_ko of k's row entry for o, .w = 1; .w = 0 if o is not in k's row
    int drop_cap;
    int* fix_cnt;            // [n_total] corrections per target slot (all zero outside the fix-up)
    int* fix_off;            // [n_total + 1] CSR offsets of the corrections by target slot
    int* fix_bsums;          // scan block sums of fix_cnt
    float4* fix_w;           // [2 drop_cap] {w, source slot}: phase B adds -omega y_source w
    int* fix_fail;           // [n_scenes] 1: more dropped pairs than drop_cap (the IP solve stops
                             // with IVP_ERR_NBR_OVERFLOW)
    int* fix_scene;          // [n_scenes] corrections of the scene in the current build
    unsigned long long h_fix;  // graph conditional: the build sets it when a list was truncated
    // per slot
    float4* xm;
    float* rho0s;
    float* dens;
    float* kd;
    float* c;
    float4* d0;
    float4* d1;
    float4* sol;
    float4* e;               // IP: d - sol of own slots (rhs, every CG-B), gathered by the next pack
    float4* r;               // viscosity residual (own slot only)
    // CG records, two float4 per slot (one 32-byte sector): [2i] the vector
    // the next direction is formed from (IP residual r, or the viscosity
    // preconditioned residual z with .w = 1/rho of fluid slots), [2i+1] the
    // previous direction.  Iteration k reads cg[k & 1] and writes
    // cg[(k + 1) & 1], so a neighbour gather takes one sector.
    float4* cg0;
    float4* cg1;
    // IP CG, per slot: the residual r (gathered by phase A), the direction p
    // (own slot) and J p of the last phase A (own slot, for the recurrence
    // J p_k = J r_k + beta J p_(k-1))
    float4* rip;
    float4* pip;
    float* jp;
    // viscosity and surface-tension CG, per slot (own): the direction p and
    // the neighbour sum of the last phase A (L(p) or S(p), carried by the
    // recurrence L(p_k) = L(z_k) + beta L(p_(k-1)))
    float4* vpp;
    float4* vlp;
    float4* stz;             // surface-tension CG: z per slot (gathered by phase A)
    float* y;
    float* s;
    float* fk;
    float* inv_m;            // 1/m of dynamic slots (0 for static)
    float* rflu;             // 1/rho of fluid slots (0 for non-fluid): viscosity neighbour weight
    float4* vs;              // viscosity: slot-ordered velocity
    float4* vap;             // viscosity: A p
    float4* pinv;            // viscosity: 3x3 block-Jacobi inverse, 3 rows per slot
    float2* st_w;            // surface tension: {j, m_bar_ij g~_ij} per neighbour-row entry (same indexing)
    float4* st_rec;          // surface tension, two float4 per slot: {v, div} {rho, 1/rho if fluid, 0, 0}
    float* st_inv;           // surface tension: Jacobi inverse per slot (jeske23.py:295-350)
    float* q;                // fk / m
    float* z;                // y / m
    // neighbour rows
    // neighbour rows, by row_fmt: ROW_FULL float4 {J, j}; ROW_COMPACT float2
    // {j, w}; ROW_BF16 int j here and the gradient as 3 bf16 in nbr_g
    float4* nbr;
    unsigned short* nbr_g;
    int row_fmt;
    int row_stream;          // 1: the rows exceed L2 (row loads hint L2 evict-first)
    int* nbr_cnt;
    int stride;
    // reductions
    double* partial;
    int* scene_counter;
    int* launch_counter;
    Flags* flags;
    double* err_hist;
    int* pcg_hist;
    // one scene's statistics gathered for a single device-to-host copy
    // (StatStage layout)
    unsigned char* stage;
    int hist_len;
    // graph conditionals (0 = not inside a conditional graph)
    unsigned long long h_outer, h_solve, h_cg, h_visc;
    // advect leaves scenes whose last solve raised where they are (the
    // reference raises before advecting, framework.py:483-513)
    int advect_skip_failed;
    // the viscosity kernel applies the step's gravity in its prologue (set on
    // step launches whose first force is the viscosity; k_gravity is then skipped)
    int fold_gravity;
    // the persistent solve runs the viscosity phases (set on step launches)
    int visc_enabled;
    int force;               // implicit non-pressure solve of this launch: 0 viscosity, 1 surface tension
    int bar_all_reduce;      // persistent solve: every CTA reduces the (few) partials itself
    // persistent solve: grid-barrier words and the phase budget
    unsigned* bar_count;
    unsigned* bar_gen;
    long long phase_limit;
    unsigned long long bar_limit_ns;  // longest wait on a grid barrier before giving up (default 2 s)
};

// ------------------------------------------------------------------ math

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 scale3(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }

// sph_kernel.py:8-25 (cubic spline, FP32 operation order of the reference)
__device__ __forceinline__ float cubic_W(float r, float h, float k) {
    float res = 0.0f;
    float q = r / h;
    if (q <= 1.0f) {
        if (q <= 0.5f) {
            float q2 = q * q;
            float q3 = q2 * q;
            res = k * (6.0f * q3 - 6.0f * q2 + 1.0f);
        } else {
            float f = 1.0f - q;
            res = k * 2.0f * f * f * f;
        }
    }
    return res;
}

// sph_kernel.py:52-61 as a weight: grad W(r) = w * r with
// w = -k (h - |r|)^2 / max(|r|, 1e-6)
__device__ __forceinline__ float spiky_w(float rn, float h, float k) {
    float rc = rn < 1e-6f ? 1e-6f : rn;
    float t = h - rc;
    return (-k * (t * t)) / rc;
}

// |r|^2 rounded exactly as the reference's wp.length computes it before the
// square root: ((x*x + y*y) + z*z), every product and sum rounded (no FMA).
__device__ __forceinline__ float norm2_rn(float3 r) {
    return __fadd_rn(__fadd_rn(__fmul_rn(r.x, r.x), __fmul_rn(r.y, r.y)), __fmul_rn(r.z, r.z));
}

// cubic spline from q = r/h (sph_kernel.py:8-25)
__device__ __forceinline__ float cubic_Wq(float q, float k) {
    float res = 0.0f;
    if (q <= 1.0f) {
        if (q <= 0.5f) {
            const float q2 = q * q;
            res = k * (6.0f * (q2 * q) - 6.0f * q2 + 1.0f);
        } else {
            const float f = 1.0f - q;
            res = k * 2.0f * f * f * f;
        }
    }
    return res;
}

__device__ __forceinline__ int cell_coord(float v, float inv, int dim) {
    float c = floorf(v * inv);
    c = fmaxf(c, 0.0f);                       // NaN -> 0
    c = fminf(c, (float)(dim - 1));
    return (int)c;
}

// Sum over the G lanes of a group that may have diverged from the rest of
// the warp (only the group's lanes take part).
template <int G>
__device__ __forceinline__ float group_sum_masked(float v, unsigned gmask) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gmask, v, o);
    return v;
}

template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

constexpr int ROW_FULL = 0, ROW_COMPACT = 1, ROW_BF16 = 2;

__device__ __forceinline__ float bf16_lo(unsigned w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(unsigned w) { return __uint_as_float(w & 0xffff0000u); }
__device__ __forceinline__ unsigned short bf16_bits(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }

// Entry k of a neighbour row in any layout: full rows hold {J_ij, j},
// compact rows {j, w_ij} with J_ij = w_ij (x_i - x_j), bf16 rows j and J_ij
// rounded to bf16.
__device__ __forceinline__ int row_j(const Dev& D, int row, int k) {
    const size_t e = (size_t)row * D.stride + k;
    if (D.row_fmt == ROW_FULL) return __float_as_int(D.nbr[e].w);
    if (D.row_fmt == ROW_COMPACT) return __float_as_int(reinterpret_cast<const float2*>(D.nbr)[e].x);
    return reinterpret_cast<const int*>(D.nbr)[e];
}

__device__ __forceinline__ float3 row_J(const Dev& D, int row, int k, float3 xi, int* j) {
    const size_t e = (size_t)row * D.stride + k;
    if (D.row_fmt == ROW_FULL) {
        const float4 v = D.nbr[e];
        *j = __float_as_int(v.w);
        return f3(v);
    }
    if (D.row_fmt == ROW_BF16) {
        *j = reinterpret_cast<const int*>(D.nbr)[e];
        const unsigned short* g = D.nbr_g + 3 * e;
        return make_float3(__uint_as_float((unsigned)g[0] << 16), __uint_as_float((unsigned)g[1] << 16),
                           __uint_as_float((unsigned)g[2] << 16));
    }
    const float2 v = reinterpret_cast<const float2*>(D.nbr)[e];
    *j = __float_as_int(v.x);
    const float3 r = sub3(xi, f3(D.xm[*j]));
    return make_float3(__fmul_rn(v.y, r.x), __fmul_rn(v.y, r.y), __fmul_rn(v.y, r.z));
}

// One 32-byte CG record (two float4, 32-byte aligned) in a single 256-bit
// load: one L1 request per lane instead of two for a neighbour gather.  The
// records of a tile's neighbourhood are gathered by many of its particles,
// so they are kept in L1 ahead of streamed data.
__device__ __forceinline__ void ld_rec(const float4* p, float4& a, float4& b) {
    asm volatile("ld.global.L1::evict_last.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
                 : "l"(p));
}

// One 16-byte per-slot vector written in an earlier phase of the same
// launch, gathered for a neighbour (kept in L1 ahead of streamed data; the
// fence after each grid barrier orders it after the writes).
__device__ __forceinline__ float4 ld_vec(const float4* p) {
    float4 a;
    asm volatile("ld.global.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w)
                 : "l"(p));
    return a;
}

// Two consecutive neighbour-list entries (32-byte aligned, read-only for the
// launch) in one 256-bit load through the non-coherent path.  A row is read
// once per pass, so it does not allocate in L1, which keeps L1 for the
// neighbour records that the particles of a tile share.
__device__ __forceinline__ void ld_rec_nc(const float4* p, float4& a, float4& b) {
    asm volatile("ld.global.nc.L1::no_allocate.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
                 : "l"(p));
}

// The same load with an L2 evict-first hint, for rows that exceed L2 and so
// stream from DRAM in every pass anyway: the hint keeps L2 for the neighbour
// records the gathers reuse.  (Where the rows fit in L2 they are reused from
// it by every pass, and the hint would evict them.)
__device__ __forceinline__ void ld_rec_nc_stream(const float4* p, float4& a, float4& b) {
    asm volatile("ld.global.nc.L1::no_allocate.L2::evict_first.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
                 : "l"(p));
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum (fixed tree), result valid in every thread.
template <int BLOCK>
__device__ __forceinline__ double block_sum_d(double v, double* sh) {
    v = warp_sum_d(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        t = (l < BLOCK / 32) ? sh[l] : 0.0;
        t = warp_sum_d(t);
        if (l == 0) sh[0] = t;
    }
    __syncthreads();
    return sh[0];
}

__host__ __device__ inline StatStage::StatStage(int hist) {
    ctl = 0;
    ovf = up8(sizeof(SceneCtl));
    flags = ovf + 8;
    pairs = up8(flags + sizeof(Flags));
    fix = pairs + 8;
    err = fix + 8;
    pcg = err + sizeof(double) * (size_t)hist;
    total = up8(pcg + sizeof(int) * (size_t)hist);
}

}  // namespace ivp
