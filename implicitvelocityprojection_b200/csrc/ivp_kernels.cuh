// ivp_kernels.cuh -- CUDA kernels of the IP pressure step (sm_100a).
//
// Bandwidth-bound sparse neighbour sums on CUDA cores (no tensor cores: the
// operator is a gather over ~30 neighbours per particle, ~1 flop/byte).
// Every neighbour-sum kernel maps G lanes to one particle: lane l takes the
// list entries 2l, 2l+1, then 2l+2G, ... (two entries per 256-bit row read)
// and the group reduces with shuffles.  Reductions across particles are FP64
// per-tile partials, summed per scene in one fixed association.  With one
// launch per phase, the last CTA of each scene sums them and runs the
// scene's solver control (outer loop / CG decisions of ip.py:346-392 and
// ip.py:283-329), and the last CTA of the launch sets the CUDA-graph
// conditional variables, so a whole step runs without a host round trip.  The
// persistent kernels sum them at each grid barrier (every CTA when there are
// one or two scenes, else the last CTA to arrive).
#pragma once
#include "ivp_device.cuh"
#include "ivp_scan.cuh"

namespace ivp {

// K_V_*: the implicit non-pressure CG (surface tension or viscosity, the
// launch's Dev::force); K_ST_DIV: the surface-tension divergence pass before
// its setup (no reduction)
// K_PJ_*: the two passes of a PRJ iteration (head without a reduction)
enum Kind {
    K_PACK = 0, K_RHS = 1, K_CG_A = 2, K_CG_B = 3, K_V_SETUP = 4, K_V_A = 5, K_V_B = 6, K_ST_DIV = 7,
    K_PJ_HEAD = 8, K_PJ_TAIL = 9
};
constexpr int FORCE_VISC = 0, FORCE_ST = 1;
constexpr int MODE_IP = 0, MODE_FORCE = 1, MODE_PRJ = 3;

constexpr int IVP_OK_ = 0, IVP_NOT_SPD_ = 1, IVP_NOT_CONVERGED_ = 2, IVP_NBR_OVERFLOW_ = 3, IVP_TIMEOUT_ = 6;

__device__ __forceinline__ void set_cond(unsigned long long h, unsigned v) {
    if (h) cudaGraphSetConditional((cudaGraphConditionalHandle)h, v);
}

__device__ __forceinline__ void flag_bad(const Dev& D, int idx, int where) {
    if (atomicExch(&D.flags->bad, 1) == 0) {
        D.flags->bad_index = idx;
        D.flags->bad_where = where;
    }
}

// ---------------------------------------------------------------- control

// Scene-level decision after a reduction (one thread).  `s` is the FP64 sum
// over the scene's dynamic particles.  `C` is the scene's control block (in
// global memory for the launch-per-phase path, a per-CTA shared-memory copy
// for the persistent path); history is written when `hist` is set.
// Weiler 2018 CG caps (weiler18.py:208-209)
constexpr int kViscMaxIter = 1000;
constexpr double kViscTol = 1e-5;

__device__ __forceinline__ bool visc_on(const SceneParams& P) { return P.visc_method == 1 && P.visc_coeff > 0.0f; }
__device__ __forceinline__ bool st_enabled(const SceneParams& P) { return P.st_method == 1 && P.st_coeff > 0.0f; }

// Start of an implicit non-pressure solve of force D.force for one scene.
__device__ __forceinline__ void force_begin(const Dev& D, const SceneParams& P, SceneCtl& C) {
    const bool on = D.force == FORCE_ST ? st_enabled(P) : visc_on(P);
    C.v_on = (on && P.n_dyn > 0) ? 1 : 0;
    C.v_max = D.force == FORCE_ST ? 100 : kViscMaxIter;  // jeske23.py:470, weiler18.py:208
    C.v_active = 0;
    C.v_total = 0;
}

// End of that solve: its CG iterations into the sticky counters.
__device__ __forceinline__ void force_account(const Dev& D, SceneCtl& C) {
    if (D.force == FORCE_ST) C.acc_st += C.v_total;
    else C.acc_visc += C.v_total;
}

__device__ void scene_decide(const Dev& D, const SceneParams& P, SceneCtl& C, int kind, double s, bool hist,
                             double s2 = 0.0) {
    if (kind == K_V_SETUP) {
        // weiler18.py:327-330: iterate only if r.z > 1e-12
        C.v_rz = s;
        C.v_it = 0;
        C.v_beta = 0.0;
        C.v_total = 0;
        C.v_active = s > 1e-12 ? 1 : 0;
        return;
    }
    if (kind == K_V_A) {
        // weiler18.py:332-338 (pAp <= 0 ends the solve without an error)
        C.v_pap = s;
        if (s <= 0.0) C.v_active = 0;
        else C.v_alpha = C.v_rz / (s > 1e-12 ? s : 1e-12);
        return;
    }
    if (kind == K_V_B) {
        // weiler18.py:349-365 and jeske23.py:553-567: s = r.r (stop test),
        // s2 = r.z (beta); both use tol 1e-5, caps 1000 and 100 (v_max)
        C.v_it += 1;
        C.v_total = C.v_it;
        if ((s < kViscTol && C.v_it >= 2) || C.v_it >= C.v_max) {
            C.v_active = 0;
        } else {
            C.v_beta = s2 / (C.v_rz > 1e-12 ? C.v_rz : 1e-12);
            C.v_rz = s2;
        }
        return;
    }
    if (kind == K_PJ_TAIL) {
        // prj.py:175-187: the pass index is the update count
        const double err = P.n_dyn > 0 ? s / (double)P.n_dyn : 0.0;
        C.err = err;
        if (hist && C.n_err < D.hist_len) D.err_hist[P.hist_base + C.n_err] = err;
        C.n_err += 1;
        const bool converged = err < P.tol_opt && !P.fixed_iters;
        if ((converged && C.outer_it >= 1) || C.outer_it >= P.max_outer) {
            C.outer_active = 0;
            C.final_err = err;
            if (!P.fixed_iters && err >= P.tol_opt && C.outer_it >= P.max_outer) C.status = IVP_NOT_CONVERGED_;
        } else {
            C.outer_it += 1;
        }
        return;
    }
    if (kind == K_PACK) {
        // pressure_base.py:405-423 average, ip.py:364-370 stopping rule
        const double err = P.n_dyn > 0 ? s / (double)P.n_dyn : 0.0;
        C.err = err;
        if (hist && C.n_err < D.hist_len) D.err_hist[P.hist_base + C.n_err] = err;
        C.n_err += 1;
        const bool converged = err < P.tol_opt && !P.fixed_iters;
        if ((converged && C.outer_it >= 1) || C.outer_it >= P.max_outer) {
            C.outer_active = 0;
            C.solve_pending = 0;
            C.final_err = err;
            // check_converged (pressure_base.py:487-495)
            if (!P.fixed_iters && err >= P.tol_opt && C.outer_it >= P.max_outer) C.status = IVP_NOT_CONVERGED_;
        } else {
            C.solve_pending = 1;
        }
    } else if (kind == K_RHS) {
        // ip.py:293-304: r = b, rr = r.r, iterate only if rr > 1e-30
        C.rr0 = s;
        C.rr_old = s;
        C.cg_it = 0;
        C.beta = 0.0;
        if (s > 1e-30) {
            C.cg_active = 1;
        } else {
            C.cg_active = 0;
            if (hist && C.outer_it < D.hist_len) D.pcg_hist[P.hist_base + C.outer_it] = 0;
            C.outer_it += 1;
            C.solve_pending = 0;
        }
    } else if (kind == K_CG_A) {
        // ip.py:307-311
        C.pap = s;
        if (s < 0.0) {
            C.status = IVP_NOT_SPD_;
            C.cg_active = 0;
            C.outer_active = 0;
            C.solve_pending = 0;
            C.final_err = C.err;
        } else {
            C.alpha = C.rr_old / (s > 1e-30 ? s : 1e-30);
        }
    } else if (kind == K_CG_B) {
        // ip.py:317-327
        const double rr_new = s;
        C.cg_it += 1;
        C.total_cg += 1;
        if ((rr_new < P.tol_pcg && C.cg_it >= 2) || C.cg_it >= P.max_pcg) {
            C.cg_active = 0;
            if (hist && C.outer_it < D.hist_len) D.pcg_hist[P.hist_base + C.outer_it] = C.cg_it;
            C.outer_it += 1;
            C.solve_pending = 0;
        } else {
            C.beta = rr_new / (C.rr_old > 1e-30 ? C.rr_old : 1e-30);
            C.rr_old = rr_new;
        }
    }
}

__device__ void scene_finalize(const Dev& D, int sc, int kind, double s) {
    scene_decide(D, D.scenes[sc], D.ctl[sc], kind, s, true);
}

// A scene's sum of its tile partials, with one fixed association that depends
// only on the scene's tile count: 128 logical lanes, lane L adding tiles
// L, L+128, L+256, ... in order onto 0.0, then the tree v[L] += v[L + off] for
// off = 64, 32, 16, ..., 1.  scene_sum_block runs the lanes on four warps of
// a CTA, scene_sum_warp on one warp (logical lanes l, l+32, l+64, l+96 in lane
// l); both execute the same floating-point operations, so every path and every
// batch composition produce the same bits.  Out-of-range slots add +0.0, which
// leaves a sum started at +0.0 unchanged.
constexpr int kSumChunk = 16;

__device__ __forceinline__ double lane_sum128(const double* __restrict__ p, int t, int te) {
    double s = 0.0;
    for (; t < te; t += kSumChunk * 128) {
        double v[kSumChunk];
#pragma unroll
        for (int m = 0; m < kSumChunk; ++m) v[m] = t + 128 * m < te ? __ldcg(p + t + 128 * m) : 0.0;
#pragma unroll
        for (int m = 0; m < kSumChunk; ++m) s += v[m];
    }
    return s;
}

// Tail of the tree for lanes 0..31 holding v[L] + v[L + 32] (after off = 64
// and 32): shuffle-down steps 16..1, result in lane 0, broadcast.
__device__ __forceinline__ double tree32(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, 0);
}

__device__ __forceinline__ double scene_sum_warp(const double* __restrict__ partial, int tb, int te) {
    const int l = threadIdx.x & 31;
    // a[k] is logical lane l + 32 k; its q-th tile is tb + l + 32 (k + 4 q)
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = tb + l; t < te; t += kSumChunk * 32) {
        double v[kSumChunk];
#pragma unroll
        for (int m = 0; m < kSumChunk; ++m) v[m] = t + 32 * m < te ? __ldcg(partial + t + 32 * m) : 0.0;
#pragma unroll
        for (int m = 0; m < kSumChunk; ++m) a[m & 3] += v[m];
    }
    return tree32((a[0] + a[2]) + (a[1] + a[3]));
}

// All threads of the CTA call it (BLOCK >= 128); `sh` holds 128 doubles.
// Result valid in every thread.
template <int BLOCK>
__device__ __forceinline__ double scene_sum_block(const double* __restrict__ partial, int tb, int te, double* sh) {
    static_assert(BLOCK >= 128, "scene_sum_block needs four warps");
    const int t = threadIdx.x;
    __syncthreads();
    if (t < 128) sh[t] = lane_sum128(partial, tb + t, te);
    __syncthreads();
    if (t < 64) sh[t] = sh[t] + sh[t + 64];
    __syncthreads();
    double v = 0.0;
    if (t < 32) {
        v = tree32(sh[t] + sh[t + 32]);
        if (t == 0) sh[0] = v;
    }
    __syncthreads();
    v = sh[0];
    __syncthreads();
    return v;
}

// Budget of decision launches for one solve sequence (per-phase path): past
// it launch_finalize stops every scene with IVP_ERR_TIMEOUT.  The timeout
// flag stays set until the host clears it (ivp_reset_counters).
__device__ __forceinline__ void guard_begin(const Dev& D) {
    long lim = 64;
    for (int s = 0; s < D.n_scenes; ++s)
        lim += (long)(D.scenes[s].max_outer + 1) * (long)(2 * D.scenes[s].max_pcg + 3) + 2 * kViscMaxIter + 4;
    D.flags->limit = lim > 0x3fffffff ? 0x3fffffff : (int)lim;
    D.flags->launches = 0;
}

// Control-block reset at the start of IP.solve (reset_stats,
// pressure_base.py:497-502).
__device__ __forceinline__ void ctl_begin(const SceneParams& P, SceneCtl& C, int solver = SOLVER_IP) {
    C.err = 0.0;
    C.rr_old = C.pap = C.alpha = C.beta = C.rr0 = 0.0;
    C.final_err = 0.0;
    C.outer_it = 0;
    C.cg_it = 0;
    C.outer_active = (P.n_dyn > 0 && P.solver == solver) ? 1 : 0;
    C.solve_pending = 0;
    C.cg_active = 0;
    C.status = IVP_OK_;
    C.n_err = 0;
    C.total_cg = 0;
}

// ctl_begin of an IP scene; a scene whose truncated lists need more
// corrections than the workspace holds stops at once with
// IVP_ERR_NBR_OVERFLOW instead of solving with a wrong operator.
__device__ __forceinline__ void ip_ctl_begin(const Dev& D, int s) {
    SceneCtl& C = D.ctl[s];
    ctl_begin(D.scenes[s], C);
    if (C.outer_active && D.fix_fail[s]) {
        C.status = IVP_NBR_OVERFLOW_;
        C.outer_active = 0;
    }
}

// Launch-level decision (one thread of the last CTA of the launch).
__device__ void launch_finalize(const Dev& D, int kind) {
    volatile Flags* F = D.flags;
    F->launches = F->launches + 1;
    if (F->launches > F->limit) {
        F->timeout = 1;
        for (int s = 0; s < D.n_scenes; ++s) {
            volatile SceneCtl* C = D.ctl + s;
            if (C->outer_active || C->cg_active || C->solve_pending || C->v_active) {
                C->status = IVP_TIMEOUT_;
                C->outer_active = 0;
                C->solve_pending = 0;
                C->cg_active = 0;
                C->v_active = 0;
            }
        }
    }
    int any_outer = 0, any_solve = 0, any_cg = 0, any_visc = 0;
    // other CTAs wrote these during this launch: read past L1
    for (int s = 0; s < D.n_scenes; ++s) {
        const volatile SceneCtl* C = D.ctl + s;
        any_outer |= C->outer_active;
        any_solve |= C->solve_pending;
        any_cg |= C->cg_active;
        any_visc |= C->v_active;
    }
    D.flags->any_outer = any_outer;
    D.flags->any_solve = any_solve;
    D.flags->any_cg = any_cg;
    D.flags->any_visc = any_visc;
    if (kind == K_PACK) {
        set_cond(D.h_outer, any_outer);
        set_cond(D.h_solve, any_solve);
    } else if (kind == K_PJ_TAIL) {
        set_cond(D.h_outer, any_outer);
    } else if (kind == K_RHS || kind == K_CG_B) {
        set_cond(D.h_cg, any_cg);
    } else if (kind == K_V_SETUP || kind == K_V_B) {
        set_cond(D.h_visc, any_visc);
    }
}

// Reduce `part` over the CTA, hand it to the scene (last CTA of the scene
// sums the scene's partials in tile order) and to the launch.
template <int BLOCK>
__device__ void block_finish(const Dev& D, int sc, bool active, double part, int kind, double part2 = 0.0) {
    __shared__ double sh[128];
    __shared__ int sh_last;
    const double total = block_sum_d<BLOCK>(part, sh);
    const double total2 = kind == K_V_B ? block_sum_d<BLOCK>(part2, sh) : 0.0;
    const SceneParams& P = D.scenes[sc];
    if (threadIdx.x == 0) {
        sh_last = 0;
        if (active) {
            D.partial[blockIdx.x] = total;
            D.partial[D.n_tiles + blockIdx.x] = total2;
            __threadfence();
            const int ntiles = P.tile_end - P.tile_begin;
            if (atomicAdd(&D.scene_counter[sc], 1) == ntiles - 1) sh_last = 1;
        }
    }
    __syncthreads();
    if (sh_last) {  // uniform over the CTA
        __threadfence();
        const double s = scene_sum_block<BLOCK>(D.partial, P.tile_begin, P.tile_end, sh);
        const double s2 =
            kind == K_V_B ? scene_sum_block<BLOCK>(D.partial + D.n_tiles, P.tile_begin, P.tile_end, sh) : 0.0;
        if (threadIdx.x == 0) {
            D.scene_counter[sc] = 0;
            scene_decide(D, D.scenes[sc], D.ctl[sc], kind, s, true, s2);
            __threadfence();
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(D.launch_counter, 1) == (int)gridDim.x - 1) {
            __threadfence();
            *D.launch_counter = 0;
            launch_finalize(D, kind);
            __threadfence();
        }
    }
}

// ------------------------------------------------------------- rebuild

// Cell key and rank within the cell for every particle (neighbour_search.py:116-129,
// the HashGrid build, as a counting sort).
__device__ __forceinline__ void cell_key(const Dev& D, int p, int sc, float px, float py, float pz) {
    const SceneParams& P = D.scenes[sc];
    const int cx = cell_coord(px, P.cell_inv, P.dims[0]);
    const int cy = cell_coord(py, P.cell_inv, P.dims[1]);
    const int cz = cell_coord(pz, P.cell_inv, P.dims[2]);
    const int cell = (cz * P.dims[1] + cy) * P.dims[0] + cx;
    const int key = P.key_base + (D.dyn[p] ? 0 : P.ncell) + cell;
    D.key[p] = key;
    D.rank[p] = atomicAdd(&D.cell_count[key], 1);
}

__global__ void k_keys(const Dev D) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= D.n_total) return;
    cell_key(D, p, D.pscene[p], D.x[3 * p], D.x[3 * p + 1], D.x[3 * p + 2]);
}

// Build segments: kSegW cells along x of one (y, z) cell row of a scene.
constexpr int kSegW = 8;

// Places every particle (thread p < n_total) and, once the cell starts are
// known, appends the build segments that hold dynamic particles (thread
// g < n_segs) to D.live_segs in any order, one atomic per warp; D.seg_ctr[0]
// (zeroed before) ends as their count.  Most segments of a scene's grid are
// empty (air above the fluid), so the build then runs only CTAs that work.
__global__ void k_place(const Dev D) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < D.n_total) {
        const int key = D.key[p];
        D.placed[D.cell_start[key] + D.rank[p]] = p;
        // the scan has consumed the counts: every nonzero count belongs to
        // some particle's key, so this leaves cell_count all zero for the
        // next build (the workspace starts zeroed)
        D.cell_count[key] = 0;
    }
    bool live = false;
    if (p < D.n_segs) {
        const int4 seg = D.segs[p];
        const SceneParams& P = D.scenes[seg.x];
        const int dimx = P.dims[0];
        const int x_hi = min(seg.w + kSegW, dimx) - 1;
        const int kd0 = P.key_base + (seg.z * P.dims[1] + seg.y) * dimx;
        live = D.cell_start[kd0 + x_hi + 1] > D.cell_start[kd0 + seg.w];
    }
    const unsigned ball = __ballot_sync(0xffffffffu, live);
    if (!ball) return;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0) base = atomicAdd(D.seg_ctr, __popc(ball));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (live) D.live_segs[base + __popc(ball & ((1u << lane) - 1u))] = p;
}

// Stable order inside each cell (by particle id), then gather the particle
// copies into slot order.
__global__ void k_order(const Dev D) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= D.n_total) return;
    const int p = D.placed[s];
    const int key = D.key[p];
    const int b = D.cell_start[key], e = D.cell_start[key + 1];
    int before = 0;
    for (int q = b; q < e; ++q) before += (D.placed[q] < p);
    const int slot = b + before;
    // the caller's n_dynamic must match is_dynamic: dynamic particles land in
    // [s_begin, s_dyn_end) of their scene
    const SceneParams& P = D.scenes[D.pscene[p]];
    if ((slot < P.s_dyn_end) != (D.dyn[p] != 0) || slot < P.s_begin || slot >= P.s_end) flag_bad(D, p, 10);
    D.pid[slot] = p;
    D.inv[p] = slot;
    const float m = D.m[p];
    D.xm[slot] = make_float4(D.x[3 * p], D.x[3 * p + 1], D.x[3 * p + 2], m);
    D.rho0s[slot] = D.rho0[p];
    D.inv_m[slot] = D.dyn[p] ? __frcp_rn(m) : 0.0f;  // the reference's m_inv (simulation_data.py:53-56)
    if (!D.dyn[p]) D.k_out[p] = 0.0f;  // static k is zero (pressure_base.py:65-67); the build writes dynamic k
}

// Neighbour lists of every dynamic particle (build_neighbor_cache,
// neighbour_search.py:10-51: j != i, |x_i - x_j| < h strict, first
// cache_size kept) fused with the density sum (pressure_base.py:12-46), the
// diagonal k = 1/(Aii + 1e-3) (pressure_base.py:49-87) and the constraint
// c = rho - rho0 (pressure_base.py:169-184).
//
// Cell-tiled: one CTA per build segment that holds dynamic particles (CTA b
// takes D.live_segs[b]; the grid covers every segment and the CTAs past the
// live count return at once).  The CTA stages the candidates of the 9
// neighbouring rows x {dynamic, static} -- 18 contiguous slot ranges covering
// x_lo-1 .. x_hi+1 -- into shared memory with coalesced loads, together with
// their cell starts.
//
// One warp per cell: the particles of a cell share their 27-cell candidate
// window, so a warp takes up to PP particles of one cell and walks the window
// once.  Each lane loads one candidate per round and tests it against all PP
// particles; one warp ballot per particle orders that round's hits by
// candidate, so each list keeps the sequential candidate order (rows dz, dy
// ascending; dynamic cells before static cells; slots ascending) and the
// first-cache_size truncation of the sequential scan.  The window is the
// concatenation of the cell's 18 slot ranges, so rounds run over all 32
// lanes across range ends; a lane finds its range by a binary search over
// the range starts.  The dense pass (J, density, Aii) then runs 32/PP lanes
// per particle.  Segments whose neighbourhood exceeds the staging capacity
// read the candidates from global memory instead.
constexpr int kStageCap = 2048;  // staged candidates per CTA (32 KB): with PP = 4, static + dynamic shared stay under 48 KB
constexpr int kBuildPP = 4;      // particles per warp

template <int PP>
__global__ void __launch_bounds__(256, 4) k_nbr_build(const Dev D) {
    constexpr int NW = 8;          // warps per CTA
    constexpr int NC = kSegW + 3;  // cell starts x_lo-1 .. x_hi+2
    constexpr int HB = 64;         // hit buffer per particle (cap <= 64)
    constexpr int LPP = 32 / PP;   // lanes per particle in the dense pass
    static_assert(PP == 2 || PP == 4, "PP: 2 or 4 particles per warp (shared memory stays under 48 KB)");
    extern __shared__ float4 stage[];
    __shared__ int sh_cs[18][NC];
    __shared__ int sh_off[18], sh_base[18];
    __shared__ int sh_total, sh_pairs;
    __shared__ int sh_vst[NW][32];  // per warp: window offset of each range, INT_MAX past the 18th
    __shared__ int sh_rj[NW][18];   // first slot of each range in the window
    __shared__ int sh_rs[NW][18];   // its stage index
    __shared__ int hit_j[NW][PP][HB];
    __shared__ short hit_s[NW][PP][HB];
    if ((int)blockIdx.x >= D.seg_ctr[0]) return;  // past the live segments (block-uniform)
    const int4 seg = D.segs[D.live_segs[blockIdx.x]];  // (scene, cy, cz, x_lo)
    const int sc = seg.x, cy = seg.y, cz = seg.z, x_lo = seg.w;
    const SceneParams& P = D.scenes[sc];
    const int dimx = P.dims[0];
    const int x_hi = min(x_lo + kSegW, dimx) - 1;
    const int kd0 = P.key_base + (cz * P.dims[1] + cy) * dimx;
    const int s0 = __ldg(D.cell_start + kd0 + x_lo), s1 = __ldg(D.cell_start + kd0 + x_hi + 1);
    if (s0 == s1) return;  // no dynamic particle in this segment (block-uniform)
    for (int e = threadIdx.x; e < 18 * NC; e += blockDim.x) {
        const int q = e / NC, c = e % NC;
        const int rr = q >> 1, pass = q & 1;
        const int z = cz + rr / 3 - 1, y = cy + rr % 3 - 1;
        const int x = x_lo - 1 + c;
        int v = -1;
        if (z >= 0 && z < P.dims[2] && y >= 0 && y < P.dims[1] && x >= 0 && x <= dimx)
            v = __ldg(D.cell_start + P.key_base + (pass ? P.ncell : 0) + (z * P.dims[1] + y) * dimx + x);
        sh_cs[q][c] = v;
    }
    if (threadIdx.x == 0) sh_pairs = 0;
    __syncthreads();
    const int ca = (x_lo > 0 ? x_lo - 1 : 0) - (x_lo - 1);
    const int cb = (x_hi < dimx - 1 ? x_hi + 1 : dimx - 1) + 1 - (x_lo - 1);
    if (threadIdx.x < 32) {
        const int q = threadIdx.x;
        int len = 0, b = 0;
        if (q < 18) {
            b = sh_cs[q][ca];
            const int e = sh_cs[q][cb];
            len = (b >= 0 && e >= b) ? e - b : 0;
        }
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (q >= o) incl += t;
        }
        if (q < 18) {
            sh_off[q] = incl - len;
            sh_base[q] = b;
        }
        if (q == 31) sh_total = incl;
    }
    __syncthreads();
    const bool staged = sh_total <= kStageCap;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (staged) {
        // one flat pass over the staged candidates (every thread's loads are
        // independent); a binary search over the range offsets finds each
        // candidate's range
        const int total = sh_total;
#pragma unroll 4
        for (int k = threadIdx.x; k < total; k += blockDim.x) {
            int q = 0;
#pragma unroll
            for (int st = 16; st > 0; st >>= 1)
                if (q + st < 18 && sh_off[q + st] <= k) q += st;
            stage[k] = __ldg(D.xm + sh_base[q] + (k - sh_off[q]));
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const float h = P.h, inv_h = P.inv_h, r2max = P.r2_max, spk = P.spiky_k, ck = P.cubic_k;
    const int dyn_end = P.s_dyn_end;
    const int cap = min(min(P.cache, D.stride), HB);
    const int ncell = x_hi - x_lo + 1;
    // work items: (cell, run of up to PP of its dynamic particles), dealt to
    // the warps round-robin; the segment's own cells are row q = 8
    // (dz = dy = 0, dynamic), columns 1 .. ncell + 1
    int nitems = 0;
    for (int k = 0; k < ncell; ++k) nitems += (sh_cs[8][k + 2] - sh_cs[8][k + 1] + PP - 1) / PP;
    int my_pairs = 0;
    for (int it = w; it < nitems; it += NW) {
        int k = 0, acc = 0, pb = 0, pe = 0;
        for (; k < ncell; ++k) {
            const int b = sh_cs[8][k + 1], e = sh_cs[8][k + 2];
            const int nch = (e - b + PP - 1) / PP;
            if (it < acc + nch) {
                pb = b + (it - acc) * PP;
                pe = min(pb + PP, e);
                break;
            }
            acc += nch;
        }
        const int cx = x_lo + k;
        const int c0 = (cx > 0 ? cx - 1 : 0) - (x_lo - 1);
        const int c1 = (cx < dimx - 1 ? cx + 1 : dimx - 1) + 1 - (x_lo - 1);
        // the cell's window: 18 ranges, concatenated in scan order
        int L;
        {
            int len = 0, jb = 0, so = 0;
            if (lane < 18) {
                jb = sh_cs[lane][c0];
                const int je = sh_cs[lane][c1];
                len = (jb >= 0 && je > jb) ? je - jb : 0;
                so = sh_off[lane] + (jb - sh_base[lane]);
            }
            int incl = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            sh_vst[w][lane] = lane < 18 ? incl - len : INT_MAX;
            if (lane < 18) {
                sh_rj[w][lane] = jb;
                sh_rs[w][lane] = so;
            }
            L = __shfl_sync(0xffffffffu, incl, 31);
            __syncwarp();
        }
        const int np = pe - pb;
        float3 xi[PP];
        int cnt[PP];
#pragma unroll
        for (int p = 0; p < PP; ++p) {
            xi[p] = f3(D.xm[pb + (p < np ? p : 0)]);
            cnt[p] = 0;
        }
        // phase 1: filter
        for (int base = 0; base < L; base += 32) {
            const int v = base + lane;
            const bool valid = v < L;
            const int vv = valid ? v : L - 1;
            int q = 0;
#pragma unroll
            for (int st = 16; st > 0; st >>= 1)
                if (sh_vst[w][q + st] <= vv) q += st;
            const int off = vv - sh_vst[w][q];
            const int j = sh_rj[w][q] + off;
            const int s = sh_rs[w][q] + off;
            const float4 xj4 = staged ? stage[s] : __ldg(D.xm + j);
            const float3 xj = f3(xj4);
            const int jr = j - pb;
#pragma unroll
            for (int p = 0; p < PP; ++p) {
                if (p < np) {
                    const bool hit = valid && jr != p && norm2_rn(sub3(xi[p], xj)) <= r2max;
                    const unsigned ball = __ballot_sync(0xffffffffu, hit);
                    const int pos = cnt[p] + __popc(ball & lt);
                    if (hit && pos < cap) {
                        hit_j[w][p][pos] = j;
                        hit_s[w][p][pos] = (short)s;
                    }
                    cnt[p] += __popc(ball);
                }
            }
        }
        __syncwarp();
        // phase 2: dense over the hits, LPP lanes per particle
        const int p = lane / LPP, sub = lane % LPP;
        int found = 0;
#pragma unroll
        for (int t = 0; t < PP; ++t)
            if (t == p) found = cnt[t];
        const bool act = p < np;
        const int n_hit = act ? min(found, cap) : 0;
        const int i = pb + (act ? p : 0);
        const float4 xi4 = D.xm[i];
        const float3 xs = f3(xi4);
        const int row = P.row_base + (i - P.s_begin);
        float4* out = D.nbr + (size_t)row * D.stride;
        float2* out2 = reinterpret_cast<float2*>(D.nbr) + (size_t)row * D.stride;
        float rho = 0.0f, aii = 0.0f;
        float3 jii = make_float3(0.0f, 0.0f, 0.0f);
        for (int kk = sub; kk < n_hit; kk += LPP) {
            const int j = hit_j[w][p][kk];
            const float4 xj4 = staged ? stage[hit_s[w][p][kk]] : __ldg(D.xm + j);
            const float3 r = sub3(xs, f3(xj4));
            // spiky gradient (sph_kernel.py:52-61): -k (h - |r|)^2 r / |r|
            const float rn = sqrtf(norm2_rn(r));
            const float rc = rn < 1e-6f ? 1e-6f : rn;
            const float t = h - rc;
            const float sg = -spk * (t * t);
            const float ir = __frcp_rn(rc);
            const float mj = xj4.w;
            const float wgt = mj * (sg * ir);
            const float3 J = make_float3(__fmul_rn(wgt, r.x), __fmul_rn(wgt, r.y), __fmul_rn(wgt, r.z));
            if (D.row_fmt == ROW_FULL) {
                out[kk] = make_float4(J.x, J.y, J.z, __int_as_float(j));
            } else if (D.row_fmt == ROW_COMPACT) {
                out2[kk] = make_float2(__int_as_float(j), wgt);
            } else {
                const size_t e = (size_t)row * D.stride + kk;
                reinterpret_cast<int*>(D.nbr)[e] = j;
                unsigned short* gb = D.nbr_g + 3 * e;
                gb[0] = bf16_bits(J.x);
                gb[1] = bf16_bits(J.y);
                gb[2] = bf16_bits(J.z);
            }
            rho += mj * cubic_Wq(rn * inv_h, ck);
            if (j < dyn_end) aii += dot3(J, J) * __frcp_rn(mj);
            jii = sub3(jii, J);
        }
#pragma unroll
        for (int o = LPP / 2; o > 0; o >>= 1) {
            rho += __shfl_xor_sync(0xffffffffu, rho, o);
            aii += __shfl_xor_sync(0xffffffffu, aii, o);
            jii.x += __shfl_xor_sync(0xffffffffu, jii.x, o);
            jii.y += __shfl_xor_sync(0xffffffffu, jii.y, o);
            jii.z += __shfl_xor_sync(0xffffffffu, jii.z, o);
        }
        if (act && sub == 0) {
            const float mi = xi4.w;
            float dens = 0.0f;
            dens = dens + mi * P.W0;
            dens += rho;
            aii += dot3(jii, jii) * __frcp_rn(mi);
            const float kd = __frcp_rn(aii + 1e-3f);
            D.nbr_cnt[row] = n_hit;
            D.dens[i] = dens;
            D.kd[i] = kd;
            D.c[i] = dens - D.rho0s[i];
            const int pid = D.pid[i];
            D.rflu[i] = D.material[pid] == 1 ? __frcp_rn(dens) : 0.0f;
            D.density_out[pid] = dens;
            D.k_out[pid] = kd;
            if (found > cap) {
                // truncated list: the fix-up rebuilds the row in the
                // reference's candidate order and adds transpose corrections
                atomicAdd(&D.overflow[sc], 1);
                D.ovf_list[atomicAdd(&D.ovf_ctr[0], 1)] = i;
                set_cond(D.h_fix, 1u);
            }
            my_pairs += n_hit;
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) my_pairs += __shfl_xor_sync(0xffffffffu, my_pairs, o);
    if (lane == 0 && my_pairs) atomicAdd(&sh_pairs, my_pairs);
    __syncthreads();
    if (threadIdx.x == 0 && sh_pairs) atomicAdd(&D.pairs[sc], (unsigned long long)sh_pairs);
}

// Neighbour lists, density, Aii, k, c and 1/rho of every dynamic particle,
// one thread per particle (one CTA per tile of dynamic slots).  The thread
// walks its 27-cell window in the same sequential candidate order as
// k_nbr_build -- (y, z) rows with dz outer and dy inner, in each row the
// dynamic then the static slots of the x-adjacent cells, slots ascending --
// so it keeps the same first cache_size hits.  Two passes: the filter loop
// only appends each kept hit to the thread's list in shared memory as 16 bits
// (which of the 18 slot ranges, and the offset in it; hit k of thread t at
// [k * blockDim + t], so two neighbouring threads share a 4-byte bank word:
// at most 2-way conflicts), then a dense pass rebuilds each hit's
// slot and computes its row entry, density and Aii terms.  The filter, which
// runs for every candidate, stays short even though the lanes of a warp hit
// on different iterations; the small list leaves most of L1 to the candidate
// positions that neighbouring threads (neighbouring slots) share.  A range
// offset that does not fit the 10 bits (more than 1,023 slots in three cells
// of one row) sets the scene's fix-up failure flag, so its IP solve stops
// with IVP_ERR_NBR_OVERFLOW instead of using a wrong list.
constexpr int kTppMaxThreads = 128;
constexpr int kTppHits = 64;  // >= every cache_size (the row stride caps it)
constexpr int kTppOffBits = 10;

__global__ void __launch_bounds__(kTppMaxThreads) k_nbr_build_tpp(const Dev D) {
    extern __shared__ unsigned short hit_q[];
    const int nt = blockDim.x;
    const int4 tile = __ldg(D.tiles + blockIdx.x);
    const int sc = tile.x;
    const SceneParams& P = D.scenes[sc];
    const int tid = threadIdx.x;
    const int i = tile.y + tid;
    const bool act = i < tile.z;
    int n_hit = 0;
    if (act) {
        const float4 xi4 = D.xm[i];
        const float3 xi = f3(xi4);
        const int dimx = P.dims[0];
        const int cx = cell_coord(xi.x, P.cell_inv, dimx);
        const int cy = cell_coord(xi.y, P.cell_inv, P.dims[1]);
        const int cz = cell_coord(xi.z, P.cell_inv, P.dims[2]);
        const int x0 = cx > 0 ? cx - 1 : 0, x1 = cx < dimx - 1 ? cx + 1 : dimx - 1;
        const float r2max = P.r2_max;
        const int cap = min(min(P.cache, D.stride), kTppHits);
        int found = 0;
        bool too_wide = false;
        // filter, one dz plane (six slot ranges) at a time: the twelve range
        // bounds of a plane load together, so a thread waits on three rounds
        // of cell-start loads instead of eighteen
        for (int dz = 0; dz < 3; ++dz) {
            const int z = cz + dz - 1;
            int rb[6], re[6];
#pragma unroll
            for (int u = 0; u < 6; ++u) {
                const int y = cy + (u >> 1) - 1, pass = u & 1;
                rb[u] = re[u] = 0;
                if (z >= 0 && z < P.dims[2] && y >= 0 && y < P.dims[1]) {
                    const int kb = P.key_base + (pass ? P.ncell : 0) + (z * P.dims[1] + y) * dimx;
                    rb[u] = __ldg(D.cell_start + kb + x0);
                    re[u] = __ldg(D.cell_start + kb + x1 + 1);
                }
            }
#pragma unroll
            for (int u = 0; u < 6; ++u) {
                const int q = dz * 6 + u, jb = rb[u], je = re[u];
#pragma unroll 4
                for (int j = jb; j < je; ++j) {
                    const float3 r = sub3(xi, f3(__ldg(D.xm + j)));
                    if (j != i && norm2_rn(r) <= r2max) {
                        const int off = j - jb;
                        too_wide |= off >= (1 << kTppOffBits);
                        if (found < cap) hit_q[found * nt + tid] = (unsigned short)((q << kTppOffBits) | (off & 1023));
                        ++found;
                    }
                }
            }
        }
        n_hit = min(found, cap);
        if (too_wide) D.fix_fail[sc] = 1;
        // dense pass: the build's arithmetic for every kept hit, in order;
        // two hits at a time, so their position loads are in flight together
        // (four: 80 registers, slower on the larger scenes)
        const float h = P.h, inv_h = P.inv_h, spk = P.spiky_k, ck = P.cubic_k;
        const int dyn_end = P.s_dyn_end;
        const int row = P.row_base + (i - P.s_begin);
        float4* out = D.nbr + (size_t)row * D.stride;
        float2* out2 = reinterpret_cast<float2*>(D.nbr) + (size_t)row * D.stride;
        float rho = 0.0f, aii = 0.0f;
        float3 jii = make_float3(0.0f, 0.0f, 0.0f);
        int q_cur = -1, jb_cur = 0;
        for (int k0 = 0; k0 < n_hit; k0 += 2) {
            int jj[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                jj[u] = i;
                if (k0 + u < n_hit) {
                    const unsigned hq = hit_q[(k0 + u) * nt + tid];
                    const int q = (int)(hq >> kTppOffBits);
                    if (q != q_cur) {  // hits come in range order: one cell-start load per range
                        q_cur = q;
                        const int rr = q >> 1, pass = q & 1;
                        const int z = cz + rr / 3 - 1, y = cy + rr % 3 - 1;
                        jb_cur = __ldg(D.cell_start + P.key_base + (pass ? P.ncell : 0) + (z * P.dims[1] + y) * dimx + x0);
                    }
                    jj[u] = jb_cur + (int)(hq & 1023u);
                }
            }
            float4 xq[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) xq[u] = __ldg(D.xm + jj[u]);
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int k = k0 + u;
                if (k >= n_hit) break;
                const int j = jj[u];
                const float4 xj4 = xq[u];
                const float3 r = sub3(xi, f3(xj4));
                const float rn = sqrtf(norm2_rn(r));
                const float rc = rn < 1e-6f ? 1e-6f : rn;
                const float t = h - rc;
                const float sg = -spk * (t * t);
                const float ir = __frcp_rn(rc);
                const float mj = xj4.w;
                const float wgt = mj * (sg * ir);
                const float3 J = make_float3(__fmul_rn(wgt, r.x), __fmul_rn(wgt, r.y), __fmul_rn(wgt, r.z));
                if (D.row_fmt == ROW_FULL) {
                    out[k] = make_float4(J.x, J.y, J.z, __int_as_float(j));
                } else if (D.row_fmt == ROW_COMPACT) {
                    out2[k] = make_float2(__int_as_float(j), wgt);
                } else {
                    const size_t e = (size_t)row * D.stride + k;
                    reinterpret_cast<int*>(D.nbr)[e] = j;
                    unsigned short* gb = D.nbr_g + 3 * e;
                    gb[0] = bf16_bits(J.x);
                    gb[1] = bf16_bits(J.y);
                    gb[2] = bf16_bits(J.z);
                }
                rho += mj * cubic_Wq(rn * inv_h, ck);
                if (j < dyn_end) aii += dot3(J, J) * __frcp_rn(mj);
                jii = sub3(jii, J);
            }
        }
        const float mi = xi4.w;
        float dens = 0.0f;
        dens = dens + mi * P.W0;
        dens += rho;
        aii += dot3(jii, jii) * __frcp_rn(mi);
        const float kd = __frcp_rn(aii + 1e-3f);
        D.nbr_cnt[row] = n_hit;
        D.dens[i] = dens;
        D.kd[i] = kd;
        D.c[i] = dens - D.rho0s[i];
        const int pid = D.pid[i];
        D.rflu[i] = D.material[pid] == 1 ? __frcp_rn(dens) : 0.0f;
        D.density_out[pid] = dens;
        D.k_out[pid] = kd;
        if (found > cap) {
            atomicAdd(&D.overflow[sc], 1);
            D.ovf_list[atomicAdd(&D.ovf_ctr[0], 1)] = i;
            set_cond(D.h_fix, 1u);
        }
    }
    // pair count of the scene (a tile never spans scenes): one atomic per CTA
    int pairs = n_hit;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    __shared__ int sh_pairs;
    if (threadIdx.x == 0) sh_pairs = 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && pairs) atomicAdd(&sh_pairs, pairs);
    __syncthreads();
    if (threadIdx.x == 0 && sh_pairs) atomicAdd(&D.pairs[sc], (unsigned long long)sh_pairs);
}

// ---- neighbour-cache overflow: rows of truncated lists and the transpose
// corrections (only when some dynamic particle has more than cache_size
// neighbours; a graph conditional runs these kernels in that build only)

constexpr int kOvfHits = 256;  // hits one warp ranks per truncated particle

// Rows of the truncated particles in the reference's candidate order.  The
// reference walks the 3x3x3 cells around x_i with z outermost and x
// innermost, each cell in increasing particle index (Warp's hash grid,
// neighbour_search.py:38-51, with cells of size h from the domain origin),
// and keeps the first cache_size hits: the hits with the smallest
// (linear cell index, particle index) keys.  One warp per truncated
// particle re-scans its window, ranks every hit by that key, writes the
// first cache_size in key order and recomputes density, Aii, k, c and 1/rho
// over them exactly as the build does.  Dropped dynamic neighbours are
// recorded for the corrections.
__global__ void __launch_bounds__(256) k_ovf_rows(const Dev D) {
    __shared__ unsigned long long hk[8][kOvfHits];
    __shared__ int hj[8][kOvfHits];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int n_ovf = D.ovf_ctr[0];
    for (int o = blockIdx.x * 8 + w; o < n_ovf; o += gridDim.x * 8) {
        const int i = D.ovf_list[o];
        const int sc = D.pscene[D.pid[i]];
        const SceneParams& P = D.scenes[sc];
        const float4 xi4 = D.xm[i];
        const float3 xi = f3(xi4);
        const int dimx = P.dims[0];
        const int cx = cell_coord(xi.x, P.cell_inv, dimx);
        const int cy = cell_coord(xi.y, P.cell_inv, P.dims[1]);
        const int cz = cell_coord(xi.z, P.cell_inv, P.dims[2]);
        const int x0 = cx > 0 ? cx - 1 : 0, x1 = cx < dimx - 1 ? cx + 1 : dimx - 1;
        int H = 0;
        for (int dz = -1; dz <= 1; ++dz) {
            const int z = cz + dz;
            if (z < 0 || z >= P.dims[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int y = cy + dy;
                if (y < 0 || y >= P.dims[1]) continue;
                const int cb = (z * P.dims[1] + y) * dimx;
                for (int pass = 0; pass < 2; ++pass) {
                    const int kb = P.key_base + (pass ? P.ncell : 0) + cb;
                    const int jb = D.cell_start[kb + x0], je = D.cell_start[kb + x1 + 1];
                    const int s1 = x0 + 1 <= x1 ? D.cell_start[kb + x0 + 1] : je;
                    const int s2 = x0 + 2 <= x1 ? D.cell_start[kb + x0 + 2] : je;
                    for (int base = jb; base < je; base += 32) {
                        const int j = base + lane;
                        bool hit = false;
                        unsigned long long key = 0ull;
                        if (j < je && j != i) {
                            hit = norm2_rn(sub3(xi, f3(D.xm[j]))) <= P.r2_max;
                            if (hit) {
                                const int c = j >= s2 ? x0 + 2 : (j >= s1 ? x0 + 1 : x0);
                                key = ((unsigned long long)(unsigned)(cb + c) << 32) | (unsigned)D.pid[j];
                            }
                        }
                        const unsigned ball = __ballot_sync(0xffffffffu, hit);
                        const int pos = H + __popc(ball & lt);
                        if (hit && pos < kOvfHits) {
                            hk[w][pos] = key;
                            hj[w][pos] = j;
                        }
                        H += __popc(ball);
                    }
                }
            }
        }
        __syncwarp();
        if (H > kOvfHits) {
            // more hits than one warp ranks: stop the scene's IP solve loudly
            if (lane == 0) D.fix_fail[sc] = 1;
            continue;
        }
        const int cap = min(min(P.cache, D.stride), 64);
        const int row = P.row_base + (i - P.s_begin);
        float4* out = D.nbr + (size_t)row * D.stride;
        float2* out2 = reinterpret_cast<float2*>(D.nbr) + (size_t)row * D.stride;
        float rho = 0.0f, aii = 0.0f;
        float3 jii = make_float3(0.0f, 0.0f, 0.0f);
        for (int h = lane; h < H; h += 32) {
            const unsigned long long kh = hk[w][h];
            int r = 0;
            for (int q = 0; q < H; ++q) r += hk[w][q] < kh ? 1 : 0;
            const int j = hj[w][h];
            if (r >= cap) {
                if (j < P.s_dyn_end) {
                    const int d = atomicAdd(&D.ovf_ctr[1], 1);
                    if (d < D.drop_cap) D.drop[d] = make_int2(i, j);
                    else D.fix_fail[sc] = 1;
                }
                continue;
            }
            // the build's dense-pass arithmetic for entry r
            const float4 xj4 = D.xm[j];
            const float3 rv = sub3(xi, f3(xj4));
            const float rn = sqrtf(norm2_rn(rv));
            const float rc = rn < 1e-6f ? 1e-6f : rn;
            const float t = P.h - rc;
            const float sg = -P.spiky_k * (t * t);
            const float ir = __frcp_rn(rc);
            const float mj = xj4.w;
            const float wgt = mj * (sg * ir);
            const float3 J = make_float3(__fmul_rn(wgt, rv.x), __fmul_rn(wgt, rv.y), __fmul_rn(wgt, rv.z));
            if (D.row_fmt == ROW_FULL) {
                out[r] = make_float4(J.x, J.y, J.z, __int_as_float(j));
            } else if (D.row_fmt == ROW_COMPACT) {
                out2[r] = make_float2(__int_as_float(j), wgt);
            } else {
                const size_t e = (size_t)row * D.stride + r;
                reinterpret_cast<int*>(D.nbr)[e] = j;
                unsigned short* gb = D.nbr_g + 3 * e;
                gb[0] = bf16_bits(J.x);
                gb[1] = bf16_bits(J.y);
                gb[2] = bf16_bits(J.z);
            }
            rho += mj * cubic_Wq(rn * P.inv_h, P.cubic_k);
            if (j < P.s_dyn_end) aii += dot3(J, J) * __frcp_rn(mj);
            jii = sub3(jii, J);
        }
#pragma unroll
        for (int q = 16; q > 0; q >>= 1) {
            rho += __shfl_xor_sync(0xffffffffu, rho, q);
            aii += __shfl_xor_sync(0xffffffffu, aii, q);
            jii.x += __shfl_xor_sync(0xffffffffu, jii.x, q);
            jii.y += __shfl_xor_sync(0xffffffffu, jii.y, q);
            jii.z += __shfl_xor_sync(0xffffffffu, jii.z, q);
        }
        if (lane == 0) {
            const float mi = xi4.w;
            float dens = 0.0f;
            dens = dens + mi * P.W0;
            dens += rho;
            aii += dot3(jii, jii) * __frcp_rn(mi);
            const float kd = __frcp_rn(aii + 1e-3f);
            D.nbr_cnt[row] = cap;
            D.dens[i] = dens;
            D.kd[i] = kd;
            D.c[i] = dens - D.rho0s[i];
            const int pid = D.pid[i];
            D.rflu[i] = D.material[pid] == 1 ? __frcp_rn(dens) : 0.0f;
            D.density_out[pid] = dens;
            D.k_out[pid] = kd;
        }
        __syncwarp();
    }
}

// Each dropped pair (o, k): k is within h of o but not in o's row.  When o
// is in k's row, the pair appears in one row only: k's gather-form phase B
// counts a transpose term the reference does not (k is not in o's row), and
// o's misses the reference's term from k's row.  Both get a correction;
// counted per target slot here, placed by k_ovf_fill.
__global__ void k_ovf_pairs(const Dev D) {
    const int n = min(D.ovf_ctr[1], D.drop_cap);
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
        const int2 pr = D.drop[d];
        const int o = pr.x, k = pr.y;
        const int sc = D.pscene[D.pid[k]];
        const SceneParams& P = D.scenes[sc];
        const int rowk = P.row_base + (k - P.s_begin);
        const int cnt = D.nbr_cnt[rowk];
        int q = -1;
        for (int e = 0; e < cnt; ++e)
            if (row_j(D, rowk, e) == o) {
                q = e;
                break;
            }
        if (q < 0) {
            D.drop_w[d] = make_float4(0.f, 0.f, 0.f, 0.f);  // in neither row: nothing to correct
            continue;
        }
        int jj;
        const float3 J = row_J(D, rowk, q, f3(D.xm[k]), &jj);
        D.drop_w[d] = make_float4(J.x, J.y, J.z, 1.0f);
        atomicAdd(&D.fix_cnt[o], 1);
        atomicAdd(&D.fix_cnt[k], 1);
        atomicAdd(&D.fix_scene[sc], 2);
    }
}

// Places the corrections by target slot (fix_off from the scan of fix_cnt,
// which this pass counts back down to zero for the next build):
//   target o, source k: the reference's term -omega y_k J_ko, which o's
//     gather misses (w = J_ko);
//   target k, source o: the gather's term omega m_k (y_o / m_o) J_ko, which
//     the reference does not have (w = (m_k / m_o) J_ko, subtracted).
__global__ void k_ovf_fill(const Dev D) {
    const int n = min(D.ovf_ctr[1], D.drop_cap);
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
        const float4 w = D.drop_w[d];
        if (w.w == 0.0f) continue;
        const int2 pr = D.drop[d];
        const int o = pr.x, k = pr.y;
        const int po = D.fix_off[o] + atomicSub(&D.fix_cnt[o], 1) - 1;
        D.fix_w[po] = make_float4(w.x, w.y, w.z, __int_as_float(k));
        const float s = D.xm[k].w * D.inv_m[o];
        const int pk = D.fix_off[k] + atomicSub(&D.fix_cnt[k], 1) - 1;
        D.fix_w[pk] = make_float4(s * w.x, s * w.y, s * w.z, __int_as_float(o));
    }
}

// Corrections of each target in increasing source slot, so phase B adds them
// in a fixed order (deterministic results).
__global__ void k_ovf_sort(const Dev D) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= D.n_total) return;
    const int b = D.fix_off[t], e = D.fix_off[t + 1];
    for (int a = b + 1; a < e; ++a) {
        const float4 v = D.fix_w[a];
        const int key = __float_as_int(v.w);
        int c = a - 1;
        while (c >= b && __float_as_int(D.fix_w[c].w) > key) {
            D.fix_w[c + 1] = D.fix_w[c];
            --c;
        }
        D.fix_w[c + 1] = v;
    }
}

// Static particles: the reference zeroes their k (pressure_base.py:65-67) and
// leaves their density untouched.
__global__ void k_static_outputs(const Dev D) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= D.n_total) return;
    const int p = D.pid[s];
    if (!D.dyn[p]) D.k_out[p] = 0.0f;
}

// Standalone PressureBase.compute_density from the lists and the bound
// positions (pressure_base.py:12-46).
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_density(const Dev D) {
    const int4 tile = D.tiles[blockIdx.x];
    const SceneParams& P = D.scenes[tile.x];
    const int g = threadIdx.x / G, lane = threadIdx.x % G;
    const int i = tile.y + g;
    const bool valid = i < tile.z;
    const int row = tile.w + g;
    const int cnt = valid ? D.nbr_cnt[row] : 0;
    float3 xi = make_float3(0.f, 0.f, 0.f);
    int pi = 0;
    if (valid) {
        pi = D.pid[i];
        xi = make_float3(D.x[3 * pi], D.x[3 * pi + 1], D.x[3 * pi + 2]);
    }
    float acc = 0.0f;
    for (int k = lane; k < cnt; k += G) {
        const int j = row_j(D, row, k);
        const int pj = D.pid[j];
        const float3 r = sub3(xi, make_float3(D.x[3 * pj], D.x[3 * pj + 1], D.x[3 * pj + 2]));
        acc += D.m[pj] * cubic_W(sqrtf(dot3(r, r)), P.h, P.cubic_k);
    }
    acc = group_sum<G>(acc);
    if (valid && lane == 0) {
        float rho = 0.0f;
        rho = rho + D.m[pi] * P.W0;
        rho += acc;
        D.dens[i] = rho;
        D.c[i] = rho - D.rho0s[i];
        D.density_out[pi] = rho;
        D.rflu[i] = D.material[pi] == 1 ? __frcp_rn(rho) : 0.0f;
    }
}

// Standalone PressureBase.compute_Aii (pressure_base.py:49-87).
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_aii(const Dev D) {
    const int4 tile = D.tiles[blockIdx.x];
    const SceneParams& P = D.scenes[tile.x];
    const int g = threadIdx.x / G, lane = threadIdx.x % G;
    const int i = tile.y + g;
    const bool valid = i < tile.z;
    const int row = tile.w + g;
    const int cnt = valid ? D.nbr_cnt[row] : 0;
    const float4 xi4 = valid ? D.xm[i] : make_float4(0.f, 0.f, 0.f, 1.f);
    float aii = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
    for (int k = lane; k < cnt; k += G) {
        int j;
        const float3 J = row_J(D, row, k, f3(xi4), &j);
        if (j < P.s_dyn_end) aii += dot3(J, J) * __frcp_rn(D.xm[j].w);
        jx -= J.x;
        jy -= J.y;
        jz -= J.z;
    }
    aii = group_sum<G>(aii);
    jx = group_sum<G>(jx);
    jy = group_sum<G>(jy);
    jz = group_sum<G>(jz);
    if (valid && lane == 0) {
        const float3 jii = make_float3(jx, jy, jz);
        aii += dot3(jii, jii) * __frcp_rn(xi4.w);
        const float kd = __frcp_rn(aii + 1e-3f);
        D.kd[i] = kd;
        D.k_out[D.pid[i]] = kd;
    }
}

// ------------------------------------------------------------- glue

// apply_gravity (framework.py:26-41)
__global__ void k_gravity(const Dev D) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= D.n_total || !D.dyn[p]) return;
    const SceneParams& P = D.scenes[D.pscene[p]];
    const float gx = P.gravity[0] * P.dt, gy = P.gravity[1] * P.dt, gz = P.gravity[2] * P.dt;
    D.v[3 * p] = D.v[3 * p] + gx;
    D.v[3 * p + 1] = D.v[3 * p + 1] + gy;
    D.v[3 * p + 2] = D.v[3 * p + 2] + gz;
}

// IP.solve prologue: d = dt v (ip.py:343) into slot order; resets the
// scene's control block (reset_stats, pressure_base.py:497-502).
__global__ void k_solve_begin(const Dev D) {
    const int4 tile = D.tiles[blockIdx.x];
    const SceneParams& P = D.scenes[tile.x];
    if (blockIdx.x == 0 && threadIdx.x == 0) guard_begin(D);
    if (blockIdx.x == P.tile_begin && threadIdx.x == 0) ip_ctl_begin(D, tile.x);
    if (P.solver != SOLVER_IP) return;
    const int i = tile.y + threadIdx.x;
    if (i >= tile.z) return;
    const int p = D.pid[i];
    const float dt = P.dt;
    D.d0[i] = make_float4(dt * D.v[3 * p], dt * D.v[3 * p + 1], dt * D.v[3 * p + 2], 0.0f);
}

// IP.solve epilogue (ip.py:394-398): v = d / dt for scenes that did not
// raise; the final density error of the reference (pressure_base.py:438-447)
// equals the error of the last pack, which evaluated J d + c at the same d.
__global__ void k_solve_end(const Dev D) {
    const int4 tile = D.tiles[blockIdx.x];
    const SceneParams& P = D.scenes[tile.x];
    if (P.solver != SOLVER_IP) return;
    const SceneCtl& C = D.ctl[tile.x];
    if (blockIdx.x == P.tile_begin && threadIdx.x == 0) {
        SceneCtl& W = D.ctl[tile.x];
        W.acc_solves += 1;
        W.acc_outer += C.outer_it;
        W.acc_cg += C.total_cg;
        if (C.final_err > W.acc_max_final_err) W.acc_max_final_err = C.final_err;
        if (C.status != IVP_OK_) {
            W.acc_failed += 1;
            W.acc_last_failure = C.status;
        }
    }
    const int i = tile.y + threadIdx.x;
    if (i >= tile.z || C.status != IVP_OK_) return;
    const float4 d = (C.outer_it & 1) ? D.d1[i] : D.d0[i];
    const int p = D.pid[i];
    const float s = P.inv_dt;
    D.v[3 * p] = s * d.x;
    D.v[3 * p + 1] = s * d.y;
    D.v[3 * p + 2] = s * d.z;
}

// advect_position (framework.py:117-136) + enforce_boundary (boundary.py:27-91)
__device__ __forceinline__ void advect_particle(const Dev& D, int p, int sc, float pos_out[3]) {
    const SceneParams& P = D.scenes[sc];
    float* x = D.x + 3 * p;
    float* v = D.v + 3 * p;
    const bool dyn = D.dyn[p] != 0;
    float vx = v[0], vy = v[1], vz = v[2];
    if (!dyn) {
        vx = vy = vz = 0.0f;
        v[0] = v[1] = v[2] = 0.0f;
    }
    float pos[3] = {x[0] + P.dt * vx, x[1] + P.dt * vy, x[2] + P.dt * vz};
    if (dyn) {
        float n[3] = {0.0f, 0.0f, 0.0f};
        const float pad = P.padding;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (pos[a] > P.domain[a] - pad) {
                n[a] += 1.0f;
                pos[a] = P.domain[a] - pad;
            }
            if (pos[a] <= pad) {
                n[a] += -1.0f;
                pos[a] = pad;
            }
        }
        const float nl = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nl > 1e-6f) {
            const float ux = n[0] / nl, uy = n[1] / nl, uz = n[2] / nl;
            const float vn = vx * ux + vy * uy + vz * uz;
            v[0] = vx - (1.0f + 0.5f) * vn * ux;
            v[1] = vy - (1.0f + 0.5f) * vn * uy;
            v[2] = vz - (1.0f + 0.5f) * vn * uz;
        }
    }
    x[0] = pos[0];
    x[1] = pos[1];
    x[2] = pos[2];
    pos_out[0] = pos[0];
    pos_out[1] = pos[1];
    pos_out[2] = pos[2];
}

__global__ void k_advect(const Dev D) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= D.n_total) return;
    const int sc = D.pscene[p];
    if (D.advect_skip_failed && D.ctl[sc].status != IVP_OK_) return;
    float pos[3];
    advect_particle(D, p, sc, pos);
}

// The end of a step: advection fused with the first pass of the next
// neighbour build (the cell key and in-cell rank of the moved particle),
// and the zeroing of the build's per-scene counters.
// Particles of a scene whose solve failed keep their positions, as in
// k_advect with advect_skip_failed.
__global__ void k_advect_keys(const Dev D) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    // the build's per-scene counters start from zero (read from k_place on)
    if (p < D.n_scenes) {
        D.overflow[p] = 0;
        D.pairs[p] = 0ull;
        D.fix_fail[p] = 0;
        D.fix_scene[p] = 0;
    }
    if (p == 0) {
        D.seg_ctr[0] = 0;
        D.ovf_ctr[0] = 0;
        D.ovf_ctr[1] = 0;
    }
    if (p >= D.n_total) return;
    const int sc = D.pscene[p];
    float pos[3];
    if (D.ctl[sc].status != IVP_OK_) {
        pos[0] = D.x[3 * p];
        pos[1] = D.x[3 * p + 1];
        pos[2] = D.x[3 * p + 2];
    } else {
        advect_particle(D, p, sc, pos);
    }
    cell_key(D, p, sc, pos[0], pos[1], pos[2]);
}

// ------------------------------------------------------------- IP solve

// Pair-loop unroll: each lane loads PU list entries before gathering, so PU
// independent gather chains are in flight.  The entries come in 32-byte
// pairs: in a batch of G * PU entries starting at a multiple of G * PU, lane
// l takes entries 2l + 2Gu and 2l + 2Gu + 1 (u < PU / 2), one 256-bit load
// each.  Rows start on 1 KB boundaries and the list stride is even, so the
// second entry of a pair is inside the row whenever the first is below the
// count.  Entries past the row end become (self, w = 0), which contributes
// exactly 0; entries outside the scene are redirected to self and reported
// once after the loop.
#ifndef IVP_PAIR_UNROLL
#define IVP_PAIR_UNROLL 4
#endif
constexpr int PU = IVP_PAIR_UNROLL;
static_assert(PU % 2 == 0, "entries are loaded in pairs");

struct PairBatch {
    int j[PU];
    float3 J[PU];
    unsigned live;  // bit u: entry u is a neighbour (not a masked slot past the row end)
};

__device__ __forceinline__ void pair_entry(const float4& e, bool in, int self, int lo, int hi, int& j, float3& J,
                                           bool& bad, unsigned& live, int u) {
    const int jj = __float_as_int(e.w);
    const bool ok = jj >= lo && jj < hi;
    bad |= in && !ok;
    j = (in && ok) ? jj : self;
    J = (in && ok) ? f3(e) : make_float3(0.f, 0.f, 0.f);
    live |= (in && ok) ? (1u << u) : 0u;
}

// k0 = 2 * lane + (batch start); xi is the row particle's position (the
// compact rows recompute J_ij = w_ij (x_i - x_j) from it).
template <int G>
__device__ __forceinline__ bool load_pairs(const Dev& D, int row, float3 xi, int k0, int cnt, int self, int lo,
                                           int hi, PairBatch& b) {
    bool bad = false;
    b.live = 0u;
    if (D.row_fmt == ROW_BF16) {
        // entries k, k+1 (k even): ids as one 8-byte load, gradients as
        // three 4-byte words of bf16 pairs
        const int2* __restrict__ ids = reinterpret_cast<const int2*>(reinterpret_cast<const int*>(D.nbr) +
                                                                     (size_t)row * D.stride);
        const unsigned* __restrict__ gw =
            reinterpret_cast<const unsigned*>(D.nbr_g + 3 * (size_t)row * D.stride);
#pragma unroll
        for (int u = 0; u < PU / 2; ++u) {
            const int k = k0 + u * 2 * G;
            int2 jj = make_int2(self, self);
            unsigned w0 = 0u, w1 = 0u, w2 = 0u;
            if (k < cnt) {
                jj = __ldg(ids + (k >> 1));
                const unsigned* p = gw + (3 * k >> 1);
                w0 = __ldg(p);
                w1 = __ldg(p + 1);
                w2 = __ldg(p + 2);
            }
            const float4 e0 = make_float4(bf16_lo(w0), bf16_hi(w0), bf16_lo(w1), __int_as_float(jj.x));
            const float4 e1 = make_float4(bf16_hi(w1), bf16_lo(w2), bf16_hi(w2), __int_as_float(jj.y));
            pair_entry(e0, k < cnt, self, lo, hi, b.j[2 * u], b.J[2 * u], bad, b.live, 2 * u);
            pair_entry(e1, k + 1 < cnt, self, lo, hi, b.j[2 * u + 1], b.J[2 * u + 1], bad, b.live, 2 * u + 1);
        }
    } else if (D.row_fmt == ROW_FULL) {
        const float4* __restrict__ nb = D.nbr + (size_t)row * D.stride;
#pragma unroll
        for (int u = 0; u < PU / 2; ++u) {
            const int k = k0 + u * 2 * G;
            float4 e0 = make_float4(0.f, 0.f, 0.f, 0.f), e1 = e0;
            if (k < cnt) {
                if (D.row_stream) ld_rec_nc_stream(nb + k, e0, e1);
                else ld_rec_nc(nb + k, e0, e1);
            }
            pair_entry(e0, k < cnt, self, lo, hi, b.j[2 * u], b.J[2 * u], bad, b.live, 2 * u);
            pair_entry(e1, k + 1 < cnt, self, lo, hi, b.j[2 * u + 1], b.J[2 * u + 1], bad, b.live, 2 * u + 1);
        }
    } else {
        const float4* __restrict__ nb =
            reinterpret_cast<const float4*>(reinterpret_cast<const float2*>(D.nbr) + (size_t)row * D.stride);
#pragma unroll
        for (int u = 0; u < PU / 2; ++u) {
            const int k = k0 + u * 2 * G;
            float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < cnt) e = __ldg(nb + (k >> 1));  // entries k, k+1: {j, w, j, w}
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int jj = __float_as_int(h ? e.z : e.x);
                const float w = h ? e.w : e.y;
                const bool in = k + h < cnt;
                const bool ok = jj >= lo && jj < hi;
                bad |= in && !ok;
                const int j = (in && ok) ? jj : self;
                const float3 r = sub3(xi, f3(__ldg(D.xm + j)));
                b.j[2 * u + h] = j;
                b.live |= (in && ok) ? (1u << (2 * u + h)) : 0u;
                b.J[2 * u + h] = (in && ok) ? make_float3(__fmul_rn(w, r.x), __fmul_rn(w, r.y), __fmul_rn(w, r.z))
                                            : make_float3(0.f, 0.f, 0.f);
            }
        }
    }
    return bad;
}

// The pair loop of one row: batches of PU entries per lane, `body(b)`
// consuming one batch.  (Requesting batch k+1's entries before batch k's
// gathers spills at the persistent kernels' 64-register budget and measured
// 20-35 % slower.)
template <int G, class Body>
__device__ __forceinline__ bool pair_loop(const Dev& D, int row, float3 xi, int cnt, int lane, int self, int lo,
                                          int hi, Body&& body) {
    bool bad = false;
    for (int k0 = 2 * lane; k0 < cnt; k0 += G * PU) {
        PairBatch b;
        bad |= load_pairs<G>(D, row, xi, k0, cnt, self, lo, hi, b);
        body(b);
    }
    return bad;
}

// Shared prologue of the neighbour-sum kernels: tile, scene, particle.
struct TileCtx {
    int4 tile;
    int sc;
    int g, lane, i, row;
    bool valid;
};

template <int G>
__device__ __forceinline__ TileCtx tile_ctx(const Dev& D, int t) {
    TileCtx c;
    c.tile = __ldg(D.tiles + t);
    c.sc = c.tile.x;
    c.g = threadIdx.x / G;
    c.lane = threadIdx.x % G;
    c.i = c.tile.y + c.g;
    c.row = c.tile.w + c.g;
    c.valid = c.i < c.tile.z;
    return c;
}

// L1 prefetch of a slot's own values that a tile body reads only after its
// neighbour sum, so that read finds them in L1 instead of waiting on L2.
__device__ __forceinline__ void pf_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// ---- per-tile bodies (return this thread's contribution to the FP64 partial)

// ip_pack_fused (ip.py:124-171) + coef_wise_div + the average density error
// (pressure_base.py:187-203), with the previous outer update d -= sol
// (ip.py:389) applied on the fly (it = updates applied so far).  Writes
// s = dfdt k and fk = f k for the rhs and CG phases.
template <int G>
__device__ __forceinline__ double pack_tile(const Dev& D, const SceneParams& P, const TileCtx& T, int it) {
    const bool upd = it >= 1;
    const float4* src = (upd && ((it - 1) & 1)) ? D.d1 : D.d0;
    float4* dst = (it & 1) ? D.d1 : D.d0;
    // after an update the displacement is d - sol, which rhs and every CG-B
    // stored per slot in D.e (one gather per neighbour instead of two)
    const float4* dsrc = upd ? D.e : src;
    if (T.valid && T.lane == 0) {
        pf_l1(D.c + T.i);
        pf_l1(D.kd + T.i);
        pf_l1(D.inv_m + T.i);
        pf_l1(D.rho0s + T.i);
    }
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    float3 xi = make_float3(0.f, 0.f, 0.f), di = xi;
    if (T.valid) {
        xi = f3(D.xm[T.i]);
        di = f3(dsrc[T.i]);
    }
    float acc = 0.0f;
    bool bad = false;
    const int self = T.valid ? T.i : P.s_begin;
    for (int k0 = 2 * T.lane; k0 < cnt; k0 += G * PU) {
        PairBatch b;
        bad |= load_pairs<G>(D, T.row, xi, k0, cnt, self, P.s_begin, P.s_end, b);
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const float3 dj = f3(dsrc[b.j[u]]);
            acc += dot3(sub3(di, dj), b.J[u]);
        }
    }
    if (bad) flag_bad(D, T.i, 1);
    acc = group_sum<G>(acc);
    double part = 0.0;
    if (T.valid && T.lane == 0) {
        if (upd) dst[T.i] = make_float4(di.x, di.y, di.z, 0.0f);
        const float t = acc + D.c[T.i];
        const float f = t > 0.0f ? t : 0.0f;
        const float kd = D.kd[T.i];
        D.s[T.i] = (t >= 1e-6f) ? kd : 0.0f;
        const float fk = f * kd;
        D.fk[T.i] = fk;
        D.q[T.i] = fk * D.inv_m[T.i];
        const float r0 = D.rho0s[T.i];
        const float q = f / (r0 < 1e-6f ? 1e-6f : r0);
        part = (double)(q > 0.0f ? q : 0.0f);
    }
    return part;
}

// ip_rhs_fused (ip.py:174-215) fused with the CG start: sol = 0 (ip.py:384),
// r = rhs, p_prev = 0, rr = r.r (ip.py:293-296).
template <int G>
__device__ __forceinline__ double rhs_tile(const Dev& D, const SceneParams& P, const TileCtx& T,
                                           const float4* __restrict__ dcur) {
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    float3 xi = make_float3(0.f, 0.f, 0.f);
    float fki = 0.0f, mi = 0.0f;
    if (T.valid) {
        const float4 a = D.xm[T.i];
        xi = f3(a);
        mi = a.w;
        fki = D.fk[T.i];
    }
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    bool bad = false;
    const int self = T.valid ? T.i : P.s_begin;
    for (int k0 = 2 * T.lane; k0 < cnt; k0 += G * PU) {
        PairBatch b;
        bad |= load_pairs<G>(D, T.row, xi, k0, cnt, self, P.s_begin, P.s_end, b);
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const float wgt = fki + mi * D.q[b.j[u]];
            ax += wgt * b.J[u].x;
            ay += wgt * b.J[u].y;
            az += wgt * b.J[u].z;
        }
    }
    if (bad) flag_bad(D, T.i, 2);
    ax = group_sum<G>(ax);
    ay = group_sum<G>(ay);
    az = group_sum<G>(az);
    double part = 0.0;
    if (T.valid && T.lane == 0) {
        const float om = P.omega;
        const float4 rhs = make_float4(om * ax, om * ay, om * az, 0.0f);
        D.rip[T.i] = rhs;
        D.pip[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
        D.jp[T.i] = 0.0f;
        D.sol[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
        D.e[T.i] = dcur[T.i];  // d - 0
        part = (double)dot3(f3(rhs), f3(rhs));
    }
    return part;
}

// CG phase A: p = r + beta p_prev (ip.py:323-327) for the own slot, and
// J p (compute_Jx_pcg, ip.py:19-60) by the recurrence
//   J p_k = J r_k + beta J p_(k-1),
// exact for the linear J, so the neighbour pass gathers only r_j (16 B from a
// dense array) instead of r_j and p_prev_j; J p of the own slot is kept for
// the next iteration.  y = dfdt k (J p), and the FP64 partials of
// p^T A p = sum m |p|^2 + omega sum y (J p) (the value dot(p, A p) of
// ip.py:307: phase B applies the exact transpose of J).
template <int G>
__device__ __forceinline__ double cga_tile(const Dev& D, const SceneParams& P, const TileCtx& T, float beta,
                                           int cg_it) {
    if (T.valid && T.lane == 0) {
        pf_l1(D.pip + T.i);
        pf_l1(D.jp + T.i);
        pf_l1(D.s + T.i);
        pf_l1(D.inv_m + T.i);
    }
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    float3 xi = make_float3(0.f, 0.f, 0.f), ri = xi;
    if (T.valid) {
        xi = f3(D.xm[T.i]);
        ri = f3(D.rip[T.i]);
    }
    float acc = 0.0f;
    const int self = T.valid ? T.i : P.s_begin;
    const bool bad = pair_loop<G>(D, T.row, xi, cnt, T.lane, self, P.s_begin, P.s_end, [&](const PairBatch& b) {
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const float3 rj = f3(ld_vec(D.rip + b.j[u]));
            acc += dot3(sub3(ri, rj), b.J[u]);
        }
    });
    if (bad) flag_bad(D, T.i, 3);
    acc = group_sum<G>(acc);
    double part = 0.0;
    if (T.valid && T.lane == 0) {
        const float mi = D.xm[T.i].w;
        const float4 qi = D.pip[T.i];
        const float3 pi = make_float3(ri.x + beta * qi.x, ri.y + beta * qi.y, ri.z + beta * qi.z);
        const float jp = cg_it > 0 ? acc + beta * D.jp[T.i] : acc;
        D.jp[T.i] = jp;
        const float yi = jp * D.s[T.i];
        D.y[T.i] = yi;
        D.z[T.i] = yi * D.inv_m[T.i];
        D.pip[T.i] = make_float4(pi.x, pi.y, pi.z, 0.0f);
        part = (double)(mi * dot3(pi, pi)) + (double)P.omega * (double)yi * (double)jp;
    }
    return part;
}

// Sum of y_source w over slot i's transpose corrections (k_ovf_fill), in
// increasing source slot.  Kept out of line: it runs only in scenes with a
// truncated list and must not take registers from the pair loop.
__device__ __noinline__ float3 ovf_correction(const int* __restrict__ fix_off, const float4* __restrict__ fix_w,
                                               const float* __restrict__ y, int i) {
    float3 c = make_float3(0.0f, 0.0f, 0.0f);
    const int fb = fix_off[i], fe = fix_off[i + 1];
    for (int f = fb; f < fe; ++f) {
        const float4 w = fix_w[f];
        const float ys = y[__float_as_int(w.w)];
        c.x += ys * w.x;
        c.y += ys * w.y;
        c.z += ys * w.z;
    }
    return c;
}

// CG phase B: Ap = m p + omega J^T y in gather form (compute_Ax_part1/2,
// ip.py:63-121, as pressure_base.py:130-166 writes J^T), x += alpha p,
// r -= alpha Ap (pcg_update_x_r_scalar, math_utils.py:181-195), rr = r.r.
template <int G>
__device__ __forceinline__ double cgb_tile(const Dev& D, const SceneParams& P, const TileCtx& T, float alpha,
                                           int cg_it, const float4* __restrict__ dcur) {
    if (T.valid && T.lane == 0) {
        pf_l1(D.pip + T.i);
        pf_l1(D.sol + T.i);
        pf_l1(D.rip + T.i);
        pf_l1(dcur + T.i);
    }
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    float3 xi = make_float3(0.f, 0.f, 0.f);
    float mi = 0.0f, yi = 0.0f;
    if (T.valid) {
        const float4 a = D.xm[T.i];
        xi = f3(a);
        mi = a.w;
        yi = D.y[T.i];
    }
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    const int self = T.valid ? T.i : P.s_begin;
    const bool bad = pair_loop<G>(D, T.row, xi, cnt, T.lane, self, P.s_begin, P.s_end, [&](const PairBatch& b) {
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const float wgt = yi + mi * D.z[b.j[u]];
            ax += wgt * b.J[u].x;
            ay += wgt * b.J[u].y;
            az += wgt * b.J[u].z;
        }
    });
    if (bad) flag_bad(D, T.i, 4);
    ax = group_sum<G>(ax);
    ay = group_sum<G>(ay);
    az = group_sum<G>(az);
    double part = 0.0;
    if (T.valid && T.lane == 0) {
        if (D.overflow[T.sc] > 0) {
            // truncated lists: the transpose terms of pairs held in one row
            // only (k_ovf_fill), in a fixed order
            const float3 c = ovf_correction(D.fix_off, D.fix_w, D.y, T.i);
            ax -= c.x;
            ay -= c.y;
            az -= c.z;
        }
        const float om = P.omega;
        const float4 p4 = D.pip[T.i];
        const float3 ap = make_float3(mi * p4.x + om * ax, mi * p4.y + om * ay, mi * p4.z + om * az);
        float4 xs = D.sol[T.i], rs = D.rip[T.i];
        xs.x = xs.x + alpha * p4.x;
        xs.y = xs.y + alpha * p4.y;
        xs.z = xs.z + alpha * p4.z;
        rs.x = rs.x - alpha * ap.x;
        rs.y = rs.y - alpha * ap.y;
        rs.z = rs.z - alpha * ap.z;
        D.sol[T.i] = xs;
        const float4 dd = dcur[T.i];
        D.e[T.i] = make_float4(dd.x - xs.x, dd.y - xs.y, dd.z - xs.z, 0.0f);
        D.rip[T.i] = rs;
        part = (double)dot3(f3(rs), f3(rs));
    }
    return part;
}

// compute_divergence (pressure_base.py:449-457): max(J v, 0) with v = d/dt.
template <int G>
__device__ __forceinline__ void div_tile(const Dev& D, const SceneParams& P, const TileCtx& T, int outer_it) {
    const float4* dc = (outer_it & 1) ? D.d1 : D.d0;
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    const float s = P.inv_dt;
    float3 xi = make_float3(0.f, 0.f, 0.f), vi = xi;
    if (T.valid) {
        xi = f3(D.xm[T.i]);
        vi = scale3(s, f3(dc[T.i]));
    }
    float acc = 0.0f;
    for (int k = T.lane; k < cnt; k += G) {
        int j;
        const float3 J = row_J(D, T.row, k, xi, &j);
        const float3 vj = scale3(s, f3(dc[j]));
        acc += dot3(sub3(vi, vj), J);
    }
    acc = group_sum<G>(acc);
    if (T.valid && T.lane == 0 && D.div_out) D.div_out[D.pid[T.i]] = acc > 0.0f ? acc : 0.0f;
}

// ---- Weiler 2018 implicit viscosity (weiler18.py:21-401), slot order

// L_i(u) over fluid neighbours (weiler18.py:150-169):
//   d (m_j / rho_j) (u_ij . x_ij) / (|x_ij|^2 + 0.01 h^2) grad W_ij
// = d (1/rho_j) (u_ij . x_ij) / (|x_ij|^2 + 0.01 h^2) J_ij,  d = 10;
// rflu_j = 1/rho_j for fluid j, 0 otherwise (the reference's `continue`).
__device__ __forceinline__ float visc_factor(const Dev& D, const SceneParams& P, int i) {
    const float mu = P.visc_coeff * D.rho0s[i];  // weiler18.py:146
    return P.dt * mu / D.dens[i];
}

// Setup (weiler18.py:381-396): 3x3 block-Jacobi inverse M_i^-1 of
// I - dt mu_i/rho_i L_ii (weiler18.py:21-85), rhs = v - A v, r = rhs,
// z = M^-1 r, dv = 0, p_prev = 0; partial r.z.
template <int G>
__device__ __forceinline__ double visc_setup_tile(const Dev& D, const SceneParams& P, const TileCtx& T) {
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    const bool fluid = T.valid && D.rflu[T.i] != 0.0f;
    float3 xi = make_float3(0.f, 0.f, 0.f), vi = xi;
    // vs holds every slot's {v, 1/rho if fluid} (written before the setup)
    if (T.valid) {
        xi = f3(D.xm[T.i]);
        vi = f3(D.vs[T.i]);
    }
    const float eps2 = 0.01f * P.h * P.h;
    float L[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) L[q] = 0.0f;
    float lx = 0.0f, ly = 0.0f, lz = 0.0f;
    bool bad = false;
    const int self = T.valid ? T.i : P.s_begin;
    for (int k0 = 2 * T.lane; k0 < (fluid ? cnt : 0); k0 += G * PU) {
        PairBatch b;
        bad |= load_pairs<G>(D, T.row, xi, k0, cnt, self, P.s_begin, P.s_end, b);
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const int j = b.j[u];
            const float3 xij = sub3(xi, f3(__ldg(D.xm + j)));
            const float4 vj = D.vs[j];
            const float3 vij = sub3(vi, f3(vj));
            const float rsq = dot3(xij, xij);
            const float c = (10.0f * vj.w) * __frcp_rn(rsq + eps2);
            const float3 J = b.J[u];
            const float Jv[3] = {J.x, J.y, J.z}, Xv[3] = {xij.x, xij.y, xij.z};
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int q = 0; q < 3; ++q) L[3 * r + q] += c * (Jv[r] * Xv[q]);
            const float s = c * dot3(vij, xij);
            lx += s * J.x;
            ly += s * J.y;
            lz += s * J.z;
        }
    }
    if (bad) flag_bad(D, T.i, 5);
#pragma unroll
    for (int q = 0; q < 9; ++q) L[q] = group_sum<G>(L[q]);
    lx = group_sum<G>(lx);
    ly = group_sum<G>(ly);
    lz = group_sum<G>(lz);
    double part = 0.0;
    if (T.valid && T.lane == 0) {
        float M[9];
        float3 av = vi;
        if (fluid) {
            const float f = visc_factor(D, P, T.i);
#pragma unroll
            for (int q = 0; q < 9; ++q) M[q] = ((q % 4 == 0) ? 1.0f : 0.0f) - f * L[q];
            av = make_float3(vi.x - f * lx, vi.y - f * ly, vi.z - f * lz);
        } else {
#pragma unroll
            for (int q = 0; q < 9; ++q) M[q] = (q % 4 == 0) ? 1.0f : 0.0f;
        }
        // inverse by the adjugate (wp.inverse)
        const float c00 = M[4] * M[8] - M[5] * M[7], c01 = M[5] * M[6] - M[3] * M[8], c02 = M[3] * M[7] - M[4] * M[6];
        const float id = 1.0f / (M[0] * c00 + M[1] * c01 + M[2] * c02);
        const float4 r0 = make_float4(c00 * id, (M[2] * M[7] - M[1] * M[8]) * id, (M[1] * M[5] - M[2] * M[4]) * id, 0.f);
        const float4 r1 = make_float4(c01 * id, (M[0] * M[8] - M[2] * M[6]) * id, (M[2] * M[3] - M[0] * M[5]) * id, 0.f);
        const float4 r2 = make_float4(c02 * id, (M[1] * M[6] - M[0] * M[7]) * id, (M[0] * M[4] - M[1] * M[3]) * id, 0.f);
        D.pinv[3 * T.i] = r0;
        D.pinv[3 * T.i + 1] = r1;
        D.pinv[3 * T.i + 2] = r2;
        const float3 rh = make_float3(vi.x + (-1.0f) * av.x, vi.y + (-1.0f) * av.y, vi.z + (-1.0f) * av.z);
        const float3 z = make_float3(dot3(f3(r0), rh), dot3(f3(r1), rh), dot3(f3(r2), rh));
        D.r[T.i] = make_float4(rh.x, rh.y, rh.z, 0.f);
        // the record a neighbour gathers: {z | 1/rho} and {x}; the position
        // half is the same in both ping-pong buffers for the whole solve
        D.cg0[2 * T.i] = make_float4(z.x, z.y, z.z, D.rflu[T.i]);
        D.cg0[2 * T.i + 1] = make_float4(xi.x, xi.y, xi.z, 0.f);
        D.cg1[2 * T.i + 1] = make_float4(xi.x, xi.y, xi.z, 0.f);
        D.vpp[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
        D.vlp[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
        D.sol[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
        part = (double)dot3(rh, z);
    }
    return part;
}

// CG phase A (weiler18.py:332-333, 361-364): p = z + beta p_prev for the own
// slot, A p = p - dt mu/rho L(p) with L(p) by the recurrence
//   L(p_k) = L(z_k) + beta L(p_(k-1))
// (exact for the linear L), so a neighbour contributes one 32-byte record
// {z_j | 1/rho_j, x_j}; partial p.Ap.
template <int G>
__device__ __forceinline__ double visc_a_tile(const Dev& D, const SceneParams& P, const TileCtx& T, float beta,
                                              int it) {
    // {z | 1/rho, x}.  Only dynamic slots' records are ever written; a
    // static neighbour's record keeps the zeros of ivp_engine_create's
    // workspace clear, so its 1/rho = 0 removes it from the sum (the
    // reference's fluid-only `continue`) with finite arithmetic.
    const float4* cc = (it & 1) ? D.cg1 : D.cg0;
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    const bool fluid = T.valid && D.rflu[T.i] != 0.0f;
    float3 xi = make_float3(0.f, 0.f, 0.f), zi = xi;
    if (T.valid) {
        xi = f3(D.xm[T.i]);
        zi = f3(cc[2 * T.i]);
    }
    const float eps2 = 0.01f * P.h * P.h;
    float lx = 0.0f, ly = 0.0f, lz = 0.0f;
    bool bad = false;
    const int self = T.valid ? T.i : P.s_begin;
    for (int k0 = 2 * T.lane; k0 < (fluid ? cnt : 0); k0 += G * PU) {
        PairBatch b;
        bad |= load_pairs<G>(D, T.row, xi, k0, cnt, self, P.s_begin, P.s_end, b);
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            float4 zj, xj;
            ld_rec(cc + 2 * b.j[u], zj, xj);
            const float3 xij = sub3(xi, f3(xj));
            const float rsq = dot3(xij, xij);
            const float s = (10.0f * zj.w) * __frcp_rn(rsq + eps2) * dot3(sub3(zi, f3(zj)), xij);
            lx += s * b.J[u].x;
            ly += s * b.J[u].y;
            lz += s * b.J[u].z;
        }
    }
    if (bad) flag_bad(D, T.i, 6);
    lx = group_sum<G>(lx);
    ly = group_sum<G>(ly);
    lz = group_sum<G>(lz);
    double part = 0.0;
    if (T.valid && T.lane == 0) {
        const float4 qi = D.vpp[T.i];
        const float3 pi = make_float3(zi.x + beta * qi.x, zi.y + beta * qi.y, zi.z + beta * qi.z);
        float3 ap = pi;
        if (fluid) {
            if (it > 0) {
                const float4 lp = D.vlp[T.i];
                lx = lx + beta * lp.x;
                ly = ly + beta * lp.y;
                lz = lz + beta * lp.z;
            }
            D.vlp[T.i] = make_float4(lx, ly, lz, 0.f);
            const float f = visc_factor(D, P, T.i);
            ap = make_float3(pi.x - f * lx, pi.y - f * ly, pi.z - f * lz);
        }
        D.vpp[T.i] = make_float4(pi.x, pi.y, pi.z, 0.f);
        D.vap[T.i] = make_float4(ap.x, ap.y, ap.z, 0.f);
        part = (double)dot3(pi, ap);
    }
    return part;
}

// CG phase B (weiler18.py:340-359), no neighbours: dv += alpha p,
// r -= alpha Ap, z = M^-1 r; partials r.r and r.z.
template <int G>
__device__ __forceinline__ void visc_b_tile(const Dev& D, const TileCtx& T, float alpha, int it, double* part,
                                            double* part2) {
    *part = 0.0;
    *part2 = 0.0;
    if (!(T.valid && T.lane == 0)) return;
    float4* cn = (it & 1) ? D.cg0 : D.cg1;  // receives the new z
    const float4 p4 = D.vpp[T.i], ap = D.vap[T.i];
    float4 x = D.sol[T.i], r = D.r[T.i];
    x.x = x.x + alpha * p4.x;
    x.y = x.y + alpha * p4.y;
    x.z = x.z + alpha * p4.z;
    const float na = -alpha;
    r.x = r.x + na * ap.x;
    r.y = r.y + na * ap.y;
    r.z = r.z + na * ap.z;
    D.sol[T.i] = x;
    D.r[T.i] = r;
    const float3 rr = f3(r);
    const float3 z = make_float3(dot3(f3(D.pinv[3 * T.i]), rr), dot3(f3(D.pinv[3 * T.i + 1]), rr),
                                 dot3(f3(D.pinv[3 * T.i + 2]), rr));
    cn[2 * T.i] = make_float4(z.x, z.y, z.z, D.rflu[T.i]);
    *part = (double)dot3(rr, rr);
    *part2 = (double)dot3(rr, z);
}

// End (weiler18.py:398-401): v += dv, back to the caller's order.
__device__ __forceinline__ void visc_end_tile(const Dev& D, const TileCtx& T) {
    if (!(T.valid && T.lane == 0)) return;
    const int p = D.pid[T.i];
    const float4 dv = D.sol[T.i];
    D.v[3 * p] = D.v[3 * p] + 1.0f * dv.x;
    D.v[3 * p + 1] = D.v[3 * p + 1] + 1.0f * dv.y;
    D.v[3 * p + 2] = D.v[3 * p + 2] + 1.0f * dv.z;
}


// ---- Jeske 2023 implicit surface tension (jeske23.py), over fluid pairs

// compute_Wst (jeske23.py:26-44): theta W_cubic(max(r, d); h_st), theta = 10/7
__device__ __forceinline__ float st_W(float r, float d, float h) {
    const float theta = 10.0f / 7.0f;
    const float rc = r > d ? r : d;
    const float q = rc / h;
    const float norm = 8.0f / (3.14159265358979f * h * h * h);
    float fq = 0.0f;
    if (q <= 0.5f) {
        fq = 1.0f - 6.0f * q * q + 6.0f * q * q * q;
    } else if (q <= 1.0f) {
        const float t = 1.0f - q;
        fq = 2.0f * t * t * t;
    }
    return theta * norm * fq;
}

// compute_grad_Wst (jeske23.py:47-67): zero for r <= d, else theta grad W_cubic
__device__ __forceinline__ float3 st_gradW(float3 xij, float r, float d, float h) {
    if (r <= d || r < 1.0e-12f) return make_float3(0.f, 0.f, 0.f);
    const float q = r / h;
    if (q > 1.0f) return make_float3(0.f, 0.f, 0.f);
    const float theta = 10.0f / 7.0f;
    const float norm = 8.0f / (3.14159265358979f * h * h * h);
    float fpq;
    if (q <= 0.5f) {
        fpq = -12.0f * q + 18.0f * q * q;
    } else {
        const float t = 1.0f - q;
        fpq = -6.0f * t * t;
    }
    const float s = theta * norm * (1.0f / h) * fpq;
    return make_float3(s * (xij.x / r), s * (xij.y / r), s * (xij.z / r));
}

// Slot-ordered velocity for the surface-tension passes: vs = {v, 1/rho of
// fluid slots (0 otherwise)}, one 16-byte gather per neighbour.
__global__ void k_slot_velocity(const Dev D) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= D.n_total) return;
    const int s = D.inv[p];
    D.vs[s] = make_float4(D.v[3 * p], D.v[3 * p + 1], D.v[3 * p + 2], D.dyn[p] ? D.rflu[s] : 0.0f);
}

// compute_divergence_jeske23 (jeske23.py:74-115): div_i = sum over fluid j of
// m_j v_ij . grad W_ij = J_ij . v_ij.  Stores the slot's record for the
// setup's neighbour gathers: {v, div} {rho, 1/rho if fluid}.
template <int G>
__device__ __forceinline__ void st_div_tile(const Dev& D, const SceneParams& P, const TileCtx& T) {
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    float3 xi = make_float3(0.f, 0.f, 0.f), vi = xi;
    float rfi = 0.0f;
    if (T.valid) {
        xi = f3(D.xm[T.i]);
        const float4 v4 = D.vs[T.i];
        vi = f3(v4);
        rfi = v4.w;
    }
    const bool fluid = T.valid && rfi != 0.0f;
    float acc = 0.0f;
    bool bad = false;
    const int self = T.valid ? T.i : P.s_begin;
    for (int k0 = 2 * T.lane; k0 < (fluid ? cnt : 0); k0 += G * PU) {
        PairBatch b;
        bad |= load_pairs<G>(D, T.row, xi, k0, cnt, self, P.s_begin, P.s_end, b);
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const float4 vj = D.vs[b.j[u]];
            const bool use = ((b.live >> u) & 1u) && vj.w != 0.0f;
            acc += use ? dot3(sub3(vi, f3(vj)), b.J[u]) : 0.0f;
        }
    }
    if (bad) flag_bad(D, T.i, 7);
    acc = group_sum<G>(acc);
    if (T.valid && T.lane == 0) {
        D.st_rec[2 * T.i] = make_float4(vi.x, vi.y, vi.z, fluid ? acc : 0.0f);
        D.st_rec[2 * T.i + 1] = make_float4(D.dens[T.i], rfi, 0.f, 0.f);
    }
}

// Setup (jeske23.py:612-649): g~_ij (compute_g_tilde_jeske23,
// jeske23.py:118-188) kept as the list {j, w_ij = m_bar_ij g~_ij} per row
// entry (the CG operator streams only that), the extra right-hand side b
// (jeske23.py:190-237), the Jacobi inverse (jeske23.py:295-350),
// rhs = v - M v + b, then r = rhs, z = M^-1 r, dv = 0, p_prev = 0; partial r.z.
template <int G>
__device__ __forceinline__ double st_setup_tile(const Dev& D, const SceneParams& P, const TileCtx& T) {
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    float3 xi = make_float3(0.f, 0.f, 0.f), vi = xi;
    float mi = 1.0f, rhoi = 1.0f, divi = 0.0f, rfi = 0.0f;
    if (T.valid) {
        const float4 a = D.xm[T.i];
        xi = f3(a);
        mi = a.w;
        float4 r0, r1;
        ld_rec(D.st_rec + 2 * T.i, r0, r1);
        vi = f3(r0);
        divi = r0.w;
        rhoi = r1.x;
        rfi = r1.y;
    }
    const bool fluid = T.valid && rfi != 0.0f;
    const float d = P.st_d, hs = P.st_h, dt = P.dt;
    float bx = 0.f, by = 0.f, bz = 0.f, sx = 0.f, sy = 0.f, sz = 0.f, ds = 0.f;
    bool bad = false;
    const int self = T.valid ? T.i : P.s_begin;
    float2* wrow = D.st_w + (size_t)T.row * D.stride;
    for (int k0 = 2 * T.lane; k0 < (fluid ? cnt : 0); k0 += G * PU) {
        PairBatch b;
        bad |= load_pairs<G>(D, T.row, xi, k0, cnt, self, P.s_begin, P.s_end, b);
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const int k = k0 + (u >> 1) * 2 * G + (u & 1);
            const int j = b.j[u];
            const float4 xj4 = __ldg(D.xm + j);
            float4 q0, q1;
            ld_rec(D.st_rec + 2 * j, q0, q1);
            const bool use = ((b.live >> u) & 1u) && q1.y != 0.0f;
            const float3 xij = sub3(xi, f3(xj4));
            const float r = sqrtf(norm2_rn(xij));
            float gt = 0.0f;
            float3 vij = make_float3(0.f, 0.f, 0.f);
            if (use && r < hs) {
                vij = sub3(vi, f3(q0));
                const float rbar = 0.5f * (rhoi + q1.x);
                const float W = st_W(r, d, hs);
                const float3 gw = st_gradW(xij, r, d, hs);
                const float gij = W / rbar;
                const float tk = dot3(gw, vij) / rbar;
                const float td = W / (2.0f * rbar * rbar) * (divi + q0.w);
                gt = gij + dt * (tk - td);
            }
            const float mbar = 0.5f * (mi + xj4.w);
            const float w = mbar * gt;
            if (k < cnt) wrow[k] = make_float2(__int_as_float(j), use ? w : 0.0f);
            if (use) {
                ds += w;
                if (gt != 0.0f) {
                    bx += (mbar * xij.x) * gt;
                    by += (mbar * xij.y) * gt;
                    bz += (mbar * xij.z) * gt;
                    sx += w * vij.x;
                    sy += w * vij.y;
                    sz += w * vij.z;
                }
            }
        }
    }
    if (bad) flag_bad(D, T.i, 8);
    bx = group_sum<G>(bx);
    by = group_sum<G>(by);
    bz = group_sum<G>(bz);
    sx = group_sum<G>(sx);
    sy = group_sum<G>(sy);
    sz = group_sum<G>(sz);
    ds = group_sum<G>(ds);
    double part = 0.0;
    if (T.valid && T.lane == 0) {
        float3 bb = make_float3(0.f, 0.f, 0.f), mv = vi;
        float inv = 1.0f;
        if (fluid) {
            const float sig = P.st_coeff;
            const float fb = -dt * sig / mi;
            bb = make_float3(fb * bx, fb * by, fb * bz);
            const float f = dt * dt * sig / mi;
            float dg = 1.0f + f * ds;
            if (dg < 1.0e-12f) dg = 1.0e-12f;
            inv = 1.0f / dg;
            mv = make_float3(vi.x + f * sx, vi.y + f * sy, vi.z + f * sz);
        }
        float3 rh = make_float3(vi.x + (-1.0f) * mv.x, vi.y + (-1.0f) * mv.y, vi.z + (-1.0f) * mv.z);
        rh = make_float3(rh.x + 1.0f * bb.x, rh.y + 1.0f * bb.y, rh.z + 1.0f * bb.z);
        const float3 z = make_float3(inv * rh.x, inv * rh.y, inv * rh.z);
        D.st_inv[T.i] = inv;
        D.r[T.i] = make_float4(rh.x, rh.y, rh.z, 0.f);
        D.stz[T.i] = make_float4(z.x, z.y, z.z, 0.f);
        D.vpp[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
        D.vlp[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
        D.sol[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
        part = (double)dot3(rh, z);
    }
    return part;
}

// CG phase A (jeske23.py:540-545, 570-577): p = z + beta p_prev for the own
// slot, (M p)_i = p_i + dt^2 sigma / m_i S_i(p) with S_i(p) = sum w_ij p_ij
// (compute_Av_jeske23, jeske23.py:240-292) by the recurrence
// S(p_k) = S(z_k) + beta S(p_(k-1)) (exact for the linear S), so a neighbour
// contributes one 16-byte z_j from a dense array; partial p.Mp.
template <int G>
__device__ __forceinline__ double st_a_tile(const Dev& D, const SceneParams& P, const TileCtx& T, float beta,
                                            int it) {
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    const bool fluid = T.valid && D.rflu[T.i] != 0.0f;
    float3 zi = make_float3(0.f, 0.f, 0.f);
    float mi = 1.0f;
    if (T.valid) {
        mi = D.xm[T.i].w;
        zi = f3(D.stz[T.i]);
    }
    float sx = 0.f, sy = 0.f, sz = 0.f;
    const int self = T.valid ? T.i : P.s_begin;
    // list entries k, k+1 as one 16-byte load {j, w, j, w} (rows start on
    // 512-byte boundaries and k is even)
    const float4* wrow = reinterpret_cast<const float4*>(D.st_w + (size_t)T.row * D.stride);
    for (int k0 = 2 * T.lane; k0 < (fluid ? cnt : 0); k0 += G * PU) {
        int jj[PU];
        float ww[PU];
#pragma unroll
        for (int u = 0; u < PU / 2; ++u) {
            const int k = k0 + u * 2 * G;
            float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < cnt) e = wrow[k >> 1];
            const bool in0 = k < cnt, in1 = k + 1 < cnt;
            jj[2 * u] = in0 ? __float_as_int(e.x) : self;
            ww[2 * u] = in0 ? e.y : 0.0f;
            jj[2 * u + 1] = in1 ? __float_as_int(e.z) : self;
            ww[2 * u + 1] = in1 ? e.w : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const int j = (jj[u] >= P.s_begin && jj[u] < P.s_end) ? jj[u] : self;
            const float3 zj = f3(ld_vec(D.stz + j));
            const float w = ww[u];
            if (w != 0.0f) {
                sx += w * (zi.x - zj.x);
                sy += w * (zi.y - zj.y);
                sz += w * (zi.z - zj.z);
            }
        }
    }
    sx = group_sum<G>(sx);
    sy = group_sum<G>(sy);
    sz = group_sum<G>(sz);
    double part = 0.0;
    if (T.valid && T.lane == 0) {
        const float4 qi = D.vpp[T.i];
        const float3 pi = make_float3(zi.x + beta * qi.x, zi.y + beta * qi.y, zi.z + beta * qi.z);
        float3 ap = pi;
        if (fluid) {
            if (it > 0) {
                const float4 sp = D.vlp[T.i];
                sx = sx + beta * sp.x;
                sy = sy + beta * sp.y;
                sz = sz + beta * sp.z;
            }
            D.vlp[T.i] = make_float4(sx, sy, sz, 0.f);
            const float f = P.dt * P.dt * P.st_coeff / mi;
            ap = make_float3(pi.x + f * sx, pi.y + f * sy, pi.z + f * sz);
        }
        D.vpp[T.i] = make_float4(pi.x, pi.y, pi.z, 0.f);
        D.vap[T.i] = make_float4(ap.x, ap.y, ap.z, 0.f);
        part = (double)dot3(pi, ap);
    }
    return part;
}

// CG phase B (jeske23.py:547-567), no neighbours: dv += alpha p,
// r -= alpha M p, z = M^-1 r; partials r.r and r.z.
template <int G>
__device__ __forceinline__ void st_b_tile(const Dev& D, const TileCtx& T, float alpha, int it, double* part,
                                          double* part2) {
    *part = 0.0;
    *part2 = 0.0;
    if (!(T.valid && T.lane == 0)) return;
    const float4 p4 = D.vpp[T.i], ap = D.vap[T.i];
    float4 x = D.sol[T.i], r = D.r[T.i];
    x.x = x.x + alpha * p4.x;
    x.y = x.y + alpha * p4.y;
    x.z = x.z + alpha * p4.z;
    const float na = -alpha;
    r.x = r.x + na * ap.x;
    r.y = r.y + na * ap.y;
    r.z = r.z + na * ap.z;
    D.sol[T.i] = x;
    D.r[T.i] = r;
    const float inv = D.st_inv[T.i];
    const float3 rr = f3(r);
    const float3 z = make_float3(inv * rr.x, inv * rr.y, inv * rr.z);
    D.stz[T.i] = make_float4(z.x, z.y, z.z, 0.f);
    *part = (double)dot3(rr, rr);
    *part2 = (double)dot3(rr, z);
}


// ---- PRJ: projected Jacobi on the constant-density constraint (prj.py)
//
// Slot arrays: r = dt v (dt_v_0, own), d0 = dt_v (gathered by the tail),
// fk = dt^2 lambda (own), q = dt^2 lambda / m (gathered by the head; zero at
// static slots), c = rho - rho0 and k = D^-1 from the build.

// pj_head_fused (prj.py:17-55): dt_v = dt_v_0 - dt^2 J^T lambda / max(m, 1e-6),
// J^T lambda in gather form (m_j l_i + m_i l_j) grad W = (l_i + m_i q_j) J_ij.
template <int G>
__device__ __forceinline__ void pj_head_tile(const Dev& D, const SceneParams& P, const TileCtx& T) {
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    float3 xi = make_float3(0.f, 0.f, 0.f);
    float li = 0.0f, mi = 1.0f;
    if (T.valid) {
        const float4 a = D.xm[T.i];
        xi = f3(a);
        mi = a.w;
        li = D.fk[T.i];
    }
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    const int self = T.valid ? T.i : P.s_begin;
    const bool bad = pair_loop<G>(D, T.row, xi, cnt, T.lane, self, P.s_begin, P.s_end, [&](const PairBatch& b) {
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const float wgt = li + mi * D.q[b.j[u]];
            ax += wgt * b.J[u].x;
            ay += wgt * b.J[u].y;
            az += wgt * b.J[u].z;
        }
    });
    if (bad) flag_bad(D, T.i, 11);
    ax = group_sum<G>(ax);
    ay = group_sum<G>(ay);
    az = group_sum<G>(az);
    if (T.valid && T.lane == 0) {
        const float den = mi < 1e-6f ? 1e-6f : mi;
        const float4 v0 = D.r[T.i];
        D.d0[T.i] = make_float4(v0.x - ax / den, v0.y - ay / den, v0.z - az / den, 0.0f);
    }
}

// pj_tail_fused (prj.py:58-117): r = dt J dt_v + c, lambda = max(lambda +
// omega r D^-1, 0); partial max(r / max(rho0, 1e-6), 0).
template <int G>
__device__ __forceinline__ double pj_tail_tile(const Dev& D, const SceneParams& P, const TileCtx& T) {
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    float3 xi = make_float3(0.f, 0.f, 0.f), vi = xi;
    if (T.valid) {
        xi = f3(D.xm[T.i]);
        vi = f3(D.d0[T.i]);
    }
    float acc = 0.0f;
    const int self = T.valid ? T.i : P.s_begin;
    const bool bad = pair_loop<G>(D, T.row, xi, cnt, T.lane, self, P.s_begin, P.s_end, [&](const PairBatch& b) {
#pragma unroll
        for (int u = 0; u < PU; ++u) acc += dot3(sub3(vi, f3(D.d0[b.j[u]])), b.J[u]);
    });
    if (bad) flag_bad(D, T.i, 12);
    acc = group_sum<G>(acc);
    double part = 0.0;
    if (T.valid && T.lane == 0) {
        const float r = acc + D.c[T.i];
        const float l = D.fk[T.i] + P.omega * r * D.kd[T.i];
        const float lc = l > 0.0f ? l : 0.0f;
        D.fk[T.i] = lc;
        D.q[T.i] = lc * D.inv_m[T.i];
        const float r0 = D.rho0s[T.i];
        const float e = r / (r0 < 1e-6f ? 1e-6f : r0);
        part = (double)(e > 0.0f ? e : 0.0f);
    }
    return part;
}

// PRJ.solve prologue (prj.py:307-330): dt_v_0 = dt v, dt_v = dt_v_0,
// lambda = 0, for the slots of one tile.
__device__ __forceinline__ void pj_begin_tile(const Dev& D, const SceneParams& P, int4 tile, int first, int step) {
    for (int i = tile.y + first; i < tile.z; i += step) {
        const int p = D.pid[i];
        const float dt = P.dt;
        const float4 v0 = make_float4(dt * D.v[3 * p], dt * D.v[3 * p + 1], dt * D.v[3 * p + 2], 0.0f);
        D.r[i] = v0;
        D.d0[i] = v0;
        D.fk[i] = 0.0f;
        D.q[i] = 0.0f;
    }
}

// v = dt_v / dt (prj.py:332-336) for a scene that did not raise.
__device__ __forceinline__ void pj_end_slot(const Dev& D, const SceneParams& P, int i) {
    const float4 d = D.d0[i];
    const int p = D.pid[i];
    const float s = P.inv_dt;
    D.v[3 * p] = s * d.x;
    D.v[3 * p + 1] = s * d.y;
    D.v[3 * p + 2] = s * d.z;
}

// Statistics of a finished solve into the sticky counters.
__device__ __forceinline__ void solve_account(SceneCtl& c) {
    c.acc_solves += 1;
    c.acc_outer += c.outer_it;
    c.acc_cg += c.total_cg;
    if (c.final_err > c.acc_max_final_err) c.acc_max_final_err = c.final_err;
    if (c.status != IVP_OK_) {
        c.acc_failed += 1;
        c.acc_last_failure = c.status;
    }
}

// ---- PRJ, one launch per phase
__global__ void k_prj_begin(const Dev D) {
    const int4 tile = D.tiles[blockIdx.x];
    const SceneParams& P = D.scenes[tile.x];
    if (blockIdx.x == 0 && threadIdx.x == 0) guard_begin(D);
    if (P.solver != SOLVER_PRJ) return;
    if (blockIdx.x == P.tile_begin && threadIdx.x == 0) ctl_begin(P, D.ctl[tile.x], SOLVER_PRJ);
    pj_begin_tile(D, P, tile, threadIdx.x, blockDim.x);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_pj_head(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    if (D.ctl[T.sc].outer_active) pj_head_tile<G>(D, D.scenes[T.sc], T);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_pj_tail(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    __shared__ int sh_active;
    if (threadIdx.x == 0) sh_active = D.ctl[T.sc].outer_active;
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active) part = pj_tail_tile<G>(D, D.scenes[T.sc], T);
    block_finish<BLOCK>(D, T.sc, active, part, K_PJ_TAIL);
}

__global__ void k_prj_end(const Dev D) {
    const int4 tile = D.tiles[blockIdx.x];
    const SceneParams& P = D.scenes[tile.x];
    if (P.solver != SOLVER_PRJ) return;
    SceneCtl& C = D.ctl[tile.x];
    if (blockIdx.x == P.tile_begin && threadIdx.x == 0) solve_account(C);
    if (C.status != IVP_OK_) return;
    for (int i = tile.y + threadIdx.x; i < tile.z; i += blockDim.x) pj_end_slot(D, P, i);
}

// ---- one launch per phase (device-side control through graph conditionals)

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_pack(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    __shared__ int sh_active, sh_it;
    if (threadIdx.x == 0) {
        sh_active = D.ctl[T.sc].outer_active;
        sh_it = D.ctl[T.sc].outer_it;
    }
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active) part = pack_tile<G>(D, D.scenes[T.sc], T, sh_it);
    block_finish<BLOCK>(D, T.sc, active, part, K_PACK);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_rhs(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    __shared__ int sh_active;
    __shared__ int sh_outer;
    if (threadIdx.x == 0) {
        sh_active = D.ctl[T.sc].solve_pending;
        sh_outer = D.ctl[T.sc].outer_it;
    }
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active) part = rhs_tile<G>(D, D.scenes[T.sc], T, (sh_outer & 1) ? D.d1 : D.d0);
    block_finish<BLOCK>(D, T.sc, active, part, K_RHS);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cg_a(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    __shared__ int sh_active, sh_it;
    __shared__ float sh_beta;
    if (threadIdx.x == 0) {
        const SceneCtl& C = D.ctl[T.sc];
        sh_active = C.cg_active;
        sh_it = C.cg_it;
        sh_beta = (float)C.beta;
    }
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active) part = cga_tile<G>(D, D.scenes[T.sc], T, sh_beta, sh_it);
    block_finish<BLOCK>(D, T.sc, active, part, K_CG_A);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cg_b(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    __shared__ int sh_active, sh_it, sh_outer;
    __shared__ float sh_alpha;
    if (threadIdx.x == 0) {
        const SceneCtl& C = D.ctl[T.sc];
        sh_active = C.cg_active;
        sh_it = C.cg_it;
        sh_alpha = (float)C.alpha;
        sh_outer = C.outer_it;
    }
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active) part = cgb_tile<G>(D, D.scenes[T.sc], T, sh_alpha, sh_it, (sh_outer & 1) ? D.d1 : D.d0);
    block_finish<BLOCK>(D, T.sc, active, part, K_CG_B);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_divergence(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    const SceneParams& P = D.scenes[T.sc];
    div_tile<G>(D, P, T, P.solver == SOLVER_PRJ ? 0 : D.ctl[T.sc].outer_it);
}

// viscosity, one launch per phase
__global__ void k_visc_begin(const Dev D) {
    const int4 tile = D.tiles[blockIdx.x];
    const SceneParams& P = D.scenes[tile.x];
    if (blockIdx.x == 0 && threadIdx.x == 0) guard_begin(D);
    if (blockIdx.x == P.tile_begin && threadIdx.x == 0) {
        SceneCtl& C = D.ctl[tile.x];
        force_begin(D, P, C);
    }
}

// Surface-tension divergence pass (one launch, no reduction).
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_st_div(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    if (D.ctl[T.sc].v_on) st_div_tile<G>(D, D.scenes[T.sc], T);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_visc_setup(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    __shared__ int sh_active;
    if (threadIdx.x == 0) sh_active = D.ctl[T.sc].v_on;
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active)
        part = D.force == FORCE_ST ? st_setup_tile<G>(D, D.scenes[T.sc], T) : visc_setup_tile<G>(D, D.scenes[T.sc], T);
    block_finish<BLOCK>(D, T.sc, active, part, K_V_SETUP);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_visc_a(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    __shared__ int sh_active, sh_it;
    __shared__ float sh_beta;
    if (threadIdx.x == 0) {
        const SceneCtl& C = D.ctl[T.sc];
        sh_active = C.v_active;
        sh_it = C.v_it;
        sh_beta = (float)C.v_beta;
    }
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active)
        part = D.force == FORCE_ST ? st_a_tile<G>(D, D.scenes[T.sc], T, sh_beta, sh_it)
                                   : visc_a_tile<G>(D, D.scenes[T.sc], T, sh_beta, sh_it);
    block_finish<BLOCK>(D, T.sc, active, part, K_V_A);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_visc_b(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    __shared__ int sh_active, sh_it;
    __shared__ float sh_alpha;
    if (threadIdx.x == 0) {
        const SceneCtl& C = D.ctl[T.sc];
        sh_active = C.v_active;
        sh_it = C.v_it;
        sh_alpha = (float)C.v_alpha;
    }
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0, part2 = 0.0;
    if (active) {
        if (D.force == FORCE_ST) st_b_tile<G>(D, T, sh_alpha, sh_it, &part, &part2);
        else visc_b_tile<G>(D, T, sh_alpha, sh_it, &part, &part2);
    }
    block_finish<BLOCK>(D, T.sc, active, part, K_V_B, part2);
}

template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_visc_end(const Dev D) {
    const TileCtx T = tile_ctx<G>(D, blockIdx.x);
    SceneCtl& C = D.ctl[T.sc];
    if (!C.v_on) return;
    visc_end_tile(D, T);
    if (blockIdx.x == D.scenes[T.sc].tile_begin && threadIdx.x == 0) force_account(D, C);
}

// ---- the whole IP.solve in one persistent cooperative launch

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier of a co-resident (cooperative) grid, fused with the
// phase's reduction: the last CTA to arrive sums every active scene's tile
// partials (the same association as the per-phase path), runs the scene
// decisions (one thread per scene) on its own copies of the control blocks
// (current: every CTA refreshes them after each barrier), writes them back and
// only then releases the others.  Every CTA executes a gpu-scope fence after
// the barrier, which orders its later plain loads (the L1-cached neighbour
// gathers) after every write of the previous phase.  The wait is bounded: after
// D.bar_limit_ns (kBarrierLimitNs unless a test shortens it) a CTA sets the
// timeout flag and reports failure, so a fault can never keep the kernel
// spinning.
constexpr unsigned long long kBarrierLimitNs = 2000000000ull;

__device__ __forceinline__ bool phase_active(const SceneCtl& C, int kind) {
    switch (kind) {
        case K_PACK:
        case K_PJ_HEAD:
        case K_PJ_TAIL: return C.outer_active != 0;
        case K_RHS: return C.solve_pending != 0;
        case K_CG_A:
        case K_CG_B: return C.cg_active != 0;
        case K_V_SETUP:
        case K_ST_DIV: return C.v_on != 0;
        default: return C.v_active != 0;
    }
}

__device__ __forceinline__ SceneCtl ctl_load(const SceneCtl* p) {
    SceneCtl c;
    const double* ds = reinterpret_cast<const double*>(p);
    double* dd = reinterpret_cast<double*>(&c);
#pragma unroll
    for (int k = 0; k < (int)(sizeof(SceneCtl) / sizeof(double)); ++k) dd[k] = __ldcg(ds + k);
    return c;
}

// Scenes up to this count are summed one after another by the whole CTA;
// more are spread over the warps, one scene per warp.
constexpr int kBlockSumScenes = 2;

// Scene sums of a phase's tile partials (`partial`, second partial at
// `partial + n_tiles`) into sum_sh / sum_sh2, then every active scene's
// decision on the CTA's control-block copies.  `publish`: this CTA writes the
// decided blocks (and the history) to global memory.
template <int BLOCK>
__device__ void reduce_and_decide(const Dev& D, int kind, const double* partial, double* sum_sh, double* sum_sh2,
                                  SceneCtl* sc_sh, double* red_sh, bool publish) {
    const int ns = D.n_scenes;
    if (ns <= kBlockSumScenes) {
        for (int s = 0; s < ns; ++s) {
            if (!phase_active(sc_sh[s], kind)) continue;
            const SceneParams& P = D.scenes[s];
            const double v = scene_sum_block<BLOCK>(partial, P.tile_begin, P.tile_end, red_sh);
            const double v2 =
                kind == K_V_B ? scene_sum_block<BLOCK>(partial + D.n_tiles, P.tile_begin, P.tile_end, red_sh) : 0.0;
            if (threadIdx.x == 0) {
                sum_sh[s] = v;
                sum_sh2[s] = v2;
            }
        }
    } else {
        const int warp = threadIdx.x >> 5;
        for (int s = warp; s < ns; s += BLOCK / 32) {
            if (!phase_active(sc_sh[s], kind)) continue;
            const SceneParams& P = D.scenes[s];
            const double v = scene_sum_warp(partial, P.tile_begin, P.tile_end);
            const double v2 = kind == K_V_B ? scene_sum_warp(partial + D.n_tiles, P.tile_begin, P.tile_end) : 0.0;
            if ((threadIdx.x & 31) == 0) {
                sum_sh[s] = v;
                sum_sh2[s] = v2;
            }
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < ns; s += BLOCK) {
        SceneCtl& c = sc_sh[s];
        if (!phase_active(c, kind)) continue;
        scene_decide(D, D.scenes[s], c, kind, sum_sh[s], publish, sum_sh2[s]);
        if (publish) {
            D.ctl[s] = c;
            __threadfence();
        }
    }
    __syncthreads();
}

// Barrier in which every CTA reduces: after all CTAs arrived (one monotonic
// arrival counter, `target` = this barrier's count), each CTA sums the
// partials and runs the decisions itself -- same inputs, same code, same
// bits -- so no control block has to travel back.  CTA 0 publishes them.
// Used when the partials are few (one or two scenes); the partials alternate
// between two buffers by barrier parity, so a CTA that runs ahead into the
// next phase never overwrites partials another CTA is still reading.
template <int BLOCK>
__device__ bool grid_all_reduce_barrier(const Dev& D, int kind, const double* partial, int* sh_flag,
                                        double* sum_sh, double* sum_sh2, SceneCtl* sc_sh, double* red_sh,
                                        unsigned target) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(D.bar_count, 1u);
        volatile unsigned* cnt = D.bar_count;
        int ok = 1;
        const unsigned long long t0 = globaltimer_ns();
        while ((int)(*cnt - target) < 0) {
            __nanosleep(32);
            if (globaltimer_ns() - t0 > D.bar_limit_ns) {
                ok = 0;
                D.flags->timeout = 1;
                break;
            }
        }
        __threadfence();
        sh_flag[1] = ok;
    }
    __syncthreads();
    if (!sh_flag[1]) return false;
    if (kind >= 0) reduce_and_decide<BLOCK>(D, kind, partial, sum_sh, sum_sh2, sc_sh, red_sh, blockIdx.x == 0);
    return true;
}

template <int BLOCK>
__device__ bool grid_reduce_barrier(const Dev& D, int kind, const double* partial, int* sh_flag, double* sum_sh,
                                    double* sum_sh2, SceneCtl* sc_sh, double* red_sh) {
    unsigned g = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        g = *((volatile unsigned*)D.bar_gen);
        __threadfence();
        sh_flag[0] = atomicAdd(D.bar_count, 1u) == gridDim.x - 1;
        sh_flag[1] = 1;
    }
    __syncthreads();
    if (sh_flag[0]) {
        __threadfence();
        if (kind >= 0) reduce_and_decide<BLOCK>(D, kind, partial, sum_sh, sum_sh2, sc_sh, red_sh, true);
        __syncthreads();
        if (threadIdx.x == 0) {
            *D.bar_count = 0;
            __threadfence();
            atomicAdd(D.bar_gen, 1u);
        }
    } else if (threadIdx.x == 0) {
        // the generation advances only after every CTA arrived, so g (read
        // before arriving) is the current one
        volatile unsigned* gen = D.bar_gen;
        const unsigned long long t0 = globaltimer_ns();
        while (*gen == g) {
            __nanosleep(32);
            if (globaltimer_ns() - t0 > D.bar_limit_ns) {
                sh_flag[1] = 0;
                D.flags->timeout = 1;
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
    return sh_flag[1] != 0;
}

// Tiles whose partials a persistent CTA collects before one combining pass.
constexpr int kFlushTiles = 16;

// Phase driver shared by the persistent kernels: tiles dealt round-robin over
// the CTAs, local copies of the control blocks, one grid barrier + reduction
// per phase.
template <int G, int BLOCK>
struct Phaser {
    const Dev& D;
    double* sum_sh;
    double* sum_sh2;
    SceneCtl* sc_sh;
    double* red_sh;
    int* flag_sh;
    int* any_sh;
    long long phases;

    int* act_sh;   // [n_scenes + 1] exclusive prefix of the phase's active tile counts
    int* tb_sh;    // [n_scenes] first tile of each scene
    int* tn_sh;    // [n_scenes] tile count of each scene

    __device__ Phaser(const Dev& d, double* dyn, double* red, int* flag, int* anyp)
        : D(d), red_sh(red), flag_sh(flag), any_sh(anyp), phases(0) {
        sum_sh = dyn;
        sum_sh2 = dyn + D.n_scenes;
        sc_sh = reinterpret_cast<SceneCtl*>(dyn + 2 * D.n_scenes);
        act_sh = reinterpret_cast<int*>(sc_sh + D.n_scenes);
        tb_sh = act_sh + D.n_scenes + 1;
        tn_sh = tb_sh + D.n_scenes;
        for (int s = threadIdx.x; s < D.n_scenes; s += BLOCK) {
            tb_sh[s] = D.scenes[s].tile_begin;
            tn_sh[s] = D.scenes[s].tile_end - D.scenes[s].tile_begin;
        }
        __syncthreads();
    }

    // Exclusive prefix of the tile counts of the scenes active in `kind`
    // (warp 0, 32 scenes per pass).
    __device__ void active_prefix(int kind) {
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            int carry = 0;
            for (int base = 0; base < D.n_scenes; base += 32) {
                const int s = base + lane;
                const int v = (s < D.n_scenes && phase_active(sc_sh[s], kind)) ? tn_sh[s] : 0;
                int inc = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += u;
                }
                if (s < D.n_scenes) act_sh[s] = carry + inc - v;
                carry += __shfl_sync(0xffffffffu, inc, 31);
            }
            if (lane == 0) act_sh[D.n_scenes] = carry;
        }
        __syncthreads();
    }

    // Last scene s with act_sh[s] <= a: the active scene holding active tile a.
    __device__ int scene_of(int a) const {
        int lo = 0, hi = D.n_scenes;  // act_sh[lo] <= a < act_sh[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (act_sh[mid] <= a) lo = mid;
            else hi = mid;
        }
        return lo;
    }

    unsigned nbar = 0;  // barriers passed by this launch (the same count in every CTA)

    // this phase's partial buffer (two per tile, alternating by barrier parity)
    __device__ double* partials() const { return D.partial + (size_t)(nbar & 1u) * 2u * (size_t)D.n_tiles; }

    __device__ bool barrier(int kind) {
        const double* part = partials();
        ++nbar;
        if (D.bar_all_reduce)
            return grid_all_reduce_barrier<BLOCK>(D, kind, part, flag_sh, sum_sh, sum_sh2, sc_sh, red_sh,
                                                  nbar * gridDim.x);
        return grid_reduce_barrier<BLOCK>(D, kind, part, flag_sh, sum_sh, sum_sh2, sc_sh, red_sh);
    }

    __device__ void refresh() {
        for (int s = threadIdx.x; s < D.n_scenes; s += BLOCK) sc_sh[s] = ctl_load(D.ctl + s);
        __syncthreads();
    }

    __device__ bool any(int kind) {
        if (threadIdx.x == 0) {
            int a = 0;
            for (int s = 0; s < D.n_scenes; ++s) a |= phase_active(sc_sh[s], kind) ? 1 : 0;
            *any_sh = a;
        }
        __syncthreads();
        const bool r = *any_sh != 0;
        __syncthreads();
        return r;
    }

    // VISC selects the phase family compiled into this kernel (each
    // persistent kernel keeps its own register budget)
    // The phase's active tiles (those of the scenes active in `kind`) are
    // split evenly over the grid, so scenes that converged early leave no CTA
    // idle while others work through a converging scene's tiles.
    // MODE selects the phase family compiled into the kernel: MODE_IP, or a
    // non-pressure force (FORCE_VISC / FORCE_ST as MODE_FORCE + force); each
    // persistent kernel keeps its own register budget
    template <int MODE>
    __device__ bool run(int kind) {
        active_prefix(kind);
        const int A = act_sh[D.n_scenes];
        // active tiles dealt round-robin: at any moment the CTAs work on one
        // window of consecutive tiles, whose rows and neighbour records are
        // close in memory (L2 reuse of the gathers), as in a launch of one CTA
        // per tile
        // Tile partials: each warp sums its lanes (warp_sum_d) and parks the
        // warp sum; every kFlushTiles tiles (and at the end) one CTA barrier,
        // then warp s combines the parked sums of tile s exactly as
        // block_sum_d does.  Warps run ahead into the next tile instead of
        // waiting for a CTA-wide reduction after every tile.
        constexpr int NW = BLOCK / 32;
        __shared__ double ws_sh[2][kFlushTiles][NW];
        __shared__ int wt_sh[kFlushTiles];
        const int wid = threadIdx.x >> 5, wl = threadIdx.x & 31;
        int nb = 0;
        auto flush = [&]() {
            __syncthreads();
            double* pb = partials();
            for (int s = wid; s < nb; s += NW) {
                double t1 = wl < NW ? ws_sh[0][s][wl] : 0.0;
                t1 = warp_sum_d(t1);
                double t2 = 0.0;
                if (kind == K_V_B) {
                    t2 = wl < NW ? ws_sh[1][s][wl] : 0.0;
                    t2 = warp_sum_d(t2);
                }
                if (wl == 0) {
                    pb[wt_sh[s]] = t1;
                    pb[D.n_tiles + wt_sh[s]] = t2;
                    __threadfence();
                }
            }
            __syncthreads();
            nb = 0;
        };
        int sc = (int)blockIdx.x < A ? scene_of(blockIdx.x) : 0;
        for (int a = blockIdx.x; a < A; a += gridDim.x) {
            while (a >= act_sh[sc + 1]) ++sc;
            const int t = tb_sh[sc] + (a - act_sh[sc]);
            const SceneParams& P = D.scenes[sc];
            TileCtx T;
            {
                // the context computed from the scene's layout instead of
                // loaded (one dependent load less per tile): the engine cuts
                // each scene's dynamic slots into tiles of TS particles in
                // order, tile k holding slots s_begin + k TS .. min(s_begin +
                // (k + 1) TS, s_dyn_end) and rows row_base + k TS ..
                constexpr int TS = BLOCK / G;
                const int b = (t - tb_sh[sc]) * TS;
                T.tile = make_int4(sc, P.s_begin + b, min(P.s_begin + b + TS, P.s_dyn_end), P.row_base + b);
                T.sc = sc;
                T.g = threadIdx.x / G;
                T.lane = threadIdx.x % G;
                T.i = T.tile.y + T.g;
                T.row = T.tile.w + T.g;
                T.valid = T.i < T.tile.z;
            }
            const SceneCtl& C = sc_sh[T.sc];
            double part = 0.0, part2 = 0.0;
            if constexpr (MODE == MODE_FORCE + FORCE_ST) {
                if (kind == K_ST_DIV) {
                    st_div_tile<G>(D, P, T);
                    continue;  // no reduction
                }
                if (kind == K_V_SETUP) part = st_setup_tile<G>(D, P, T);
                else if (kind == K_V_A) part = st_a_tile<G>(D, P, T, (float)C.v_beta, C.v_it);
                else st_b_tile<G>(D, T, (float)C.v_alpha, C.v_it, &part, &part2);
            } else if constexpr (MODE == MODE_PRJ) {
                if (kind == K_PJ_HEAD) {
                    pj_head_tile<G>(D, P, T);
                    continue;  // no reduction
                }
                part = pj_tail_tile<G>(D, P, T);
            } else if constexpr (MODE == MODE_FORCE + FORCE_VISC) {
                if (kind == K_V_SETUP) part = visc_setup_tile<G>(D, P, T);
                else if (kind == K_V_A) part = visc_a_tile<G>(D, P, T, (float)C.v_beta, C.v_it);
                else visc_b_tile<G>(D, T, (float)C.v_alpha, C.v_it, &part, &part2);
            } else {
                if (kind == K_PACK) part = pack_tile<G>(D, P, T, C.outer_it);
                else if (kind == K_RHS) part = rhs_tile<G>(D, P, T, (C.outer_it & 1) ? D.d1 : D.d0);
                else if (kind == K_CG_A) part = cga_tile<G>(D, P, T, (float)C.beta, C.cg_it);
                else part = cgb_tile<G>(D, P, T, (float)C.alpha, C.cg_it, (C.outer_it & 1) ? D.d1 : D.d0);
            }
            const double w1 = warp_sum_d(part);
            const double w2 = kind == K_V_B ? warp_sum_d(part2) : 0.0;
            if (wl == 0) {
                ws_sh[0][nb][wid] = w1;
                ws_sh[1][nb][wid] = w2;
            }
            if (threadIdx.x == 0) wt_sh[nb] = t;
            if (++nb == kFlushTiles) flush();
        }
        if (nb) flush();  // nb is the same in every thread
        if (!barrier((kind == K_ST_DIV || kind == K_PJ_HEAD) ? -1 : kind)) return false;
        if (++phases > D.phase_limit) {
            // guard: every CTA reaches the same count; CTA 0 stops the scenes,
            // a barrier publishes it
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                for (int s = 0; s < D.n_scenes; ++s) {
                    SceneCtl c = ctl_load(D.ctl + s);
                    if (c.outer_active || c.solve_pending || c.cg_active || c.v_active) {
                        c.status = IVP_TIMEOUT_;
                        c.outer_active = c.solve_pending = c.cg_active = c.v_active = 0;
                        D.ctl[s] = c;
                    }
                }
                D.flags->timeout = 1;
            }
            if (!barrier(-1)) return false;
            refresh();
            return true;
        }
        // the all-reduce barrier decided on this CTA's own copies already
        if (!D.bar_all_reduce) refresh();
        return true;
    }
};

// Register budget of the persistent kernels: room for IVP_PERSIST_THREADS
// resident threads per SM (the occupancy sets how many tiles each CTA walks
// through one after another in every phase).
#ifndef IVP_PERSIST_THREADS
#define IVP_PERSIST_THREADS 1024
#endif
template <int BLOCK>
constexpr int persist_min_blocks() { return IVP_PERSIST_THREADS / BLOCK > 0 ? IVP_PERSIST_THREADS / BLOCK : 1; }

// One implicit non-pressure solve of every scene that enables it, in one
// persistent cooperative launch: Weiler 2018 viscosity (weiler18.py:371-401)
// or Jeske 2023 surface tension (jeske23.py:585-655); D.force == FORCE.
template <int G, int BLOCK, int FORCE>
__global__ void __launch_bounds__(BLOCK, persist_min_blocks<BLOCK>()) k_force_persistent(const Dev D) {
    constexpr int M = MODE_FORCE + FORCE;
    extern __shared__ double dyn_sh[];
    __shared__ double red_sh[128];
    __shared__ int flag_sh[2], any_sh;
    Phaser<G, BLOCK> ph(D, dyn_sh, red_sh, flag_sh, &any_sh);
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int s = 0; s < D.n_scenes; ++s) {
            SceneCtl c = ctl_load(D.ctl + s);
            force_begin(D, D.scenes[s], c);
            D.ctl[s] = c;
        }
    if constexpr (FORCE == FORCE_VISC) {
        // slot-ordered {v, 1/rho if fluid} of every slot for the setup's
        // neighbour gathers (the surface-tension solve gets the same record
        // from k_slot_velocity)
        for (int s = blockIdx.x * BLOCK + threadIdx.x; s < D.n_total; s += gridDim.x * BLOCK) {
            const int p = D.pid[s];
            const bool dyn = D.dyn[p] != 0;
            float vx = D.v[3 * p], vy = D.v[3 * p + 1], vz = D.v[3 * p + 2];
            if (D.fold_gravity && dyn) {
                // apply_gravity (framework.py:26-41), as k_gravity computes it
                const SceneParams& P = D.scenes[D.pscene[p]];
                const float gx = P.gravity[0] * P.dt, gy = P.gravity[1] * P.dt, gz = P.gravity[2] * P.dt;
                vx = vx + gx;
                vy = vy + gy;
                vz = vz + gz;
                D.v[3 * p] = vx;
                D.v[3 * p + 1] = vy;
                D.v[3 * p + 2] = vz;
            }
            D.vs[s] = make_float4(vx, vy, vz, dyn ? D.rflu[s] : 0.0f);
        }
    }
    if (!ph.barrier(-1)) return;
    ph.refresh();
    if (!ph.any(K_V_SETUP)) return;
    if (FORCE == FORCE_ST && !ph.template run<M>(K_ST_DIV)) return;
    if (!ph.template run<M>(K_V_SETUP)) return;
    while (ph.any(K_V_A)) {
        if (!ph.template run<M>(K_V_A)) return;
        if (!ph.any(K_V_B)) break;
        if (!ph.template run<M>(K_V_B)) return;
    }
    for (int t = blockIdx.x; t < D.n_tiles; t += gridDim.x) {
        const TileCtx T = tile_ctx<G>(D, t);
        if (ph.sc_sh[T.sc].v_on) visc_end_tile(D, T);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int s = 0; s < D.n_scenes; ++s) {
            SceneCtl& c = D.ctl[s];
            if (ph.sc_sh[s].v_on) {
                c.v_total = ph.sc_sh[s].v_total;
                force_account(D, c);
            }
        }
}

// The whole IP.solve of every scene in one persistent cooperative launch.
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK, persist_min_blocks<BLOCK>()) k_ip_persistent(const Dev D) {
    extern __shared__ double dyn_sh[];
    __shared__ double red_sh[128];
    __shared__ int flag_sh[2], any_sh;
    Phaser<G, BLOCK> ph(D, dyn_sh, red_sh, flag_sh, &any_sh);
    // CTA 0 starts every scene's control block (reset_stats); the first
    // barrier publishes it
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int s = 0; s < D.n_scenes; ++s) ip_ctl_begin(D, s);
    // d = dt v (ip.py:343) for the owned particles
    for (int t = blockIdx.x; t < D.n_tiles; t += gridDim.x) {
        const int4 tile = __ldg(D.tiles + t);
        const SceneParams& P = D.scenes[tile.x];
        for (int i = tile.y + threadIdx.x; i < tile.z; i += BLOCK) {
            const int p = D.pid[i];
            const float dt = P.dt;
            D.d0[i] = make_float4(dt * D.v[3 * p], dt * D.v[3 * p + 1], dt * D.v[3 * p + 2], 0.0f);
        }
    }
    if (!ph.barrier(-1)) return;
    ph.refresh();
    while (ph.any(K_PACK)) {
        if (!ph.template run<MODE_IP>(K_PACK)) return;
        if (!ph.any(K_RHS)) break;
        if (!ph.template run<MODE_IP>(K_RHS)) return;
        while (ph.any(K_CG_A)) {
            if (!ph.template run<MODE_IP>(K_CG_A)) return;
            if (!ph.any(K_CG_B)) break;
            if (!ph.template run<MODE_IP>(K_CG_B)) return;
        }
    }
    // epilogue (ip.py:394-404): v = d/dt for scenes that did not raise,
    // divergence, statistics
    for (int t = blockIdx.x; t < D.n_tiles; t += gridDim.x) {
        const TileCtx T = tile_ctx<G>(D, t);
        const SceneCtl& C = ph.sc_sh[T.sc];
        const SceneParams& P = D.scenes[T.sc];
        if (P.solver != SOLVER_IP) continue;
        if (C.status == IVP_OK_ && T.lane == 0 && T.valid) {
            const float4 d = (C.outer_it & 1) ? D.d1[T.i] : D.d0[T.i];
            const int p = D.pid[T.i];
            const float s = P.inv_dt;
            D.v[3 * p] = s * d.x;
            D.v[3 * p + 1] = s * d.y;
            D.v[3 * p + 2] = s * d.z;
        }
        if (D.div_out) div_tile<G>(D, P, T, C.outer_it);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int s = 0; s < D.n_scenes; ++s) {
            if (D.scenes[s].solver != SOLVER_IP) continue;
            SceneCtl c = ctl_load(D.ctl + s);
            solve_account(c);
            D.ctl[s] = c;
        }
    }
}

// The whole PRJ.solve of every PRJ scene in one persistent cooperative
// launch: passes of head (no reduction) and tail (error, decision).
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK, persist_min_blocks<BLOCK>()) k_prj_persistent(const Dev D) {
    extern __shared__ double dyn_sh[];
    __shared__ double red_sh[128];
    __shared__ int flag_sh[2], any_sh;
    Phaser<G, BLOCK> ph(D, dyn_sh, red_sh, flag_sh, &any_sh);
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int s = 0; s < D.n_scenes; ++s)
            if (D.scenes[s].solver == SOLVER_PRJ) ctl_begin(D.scenes[s], D.ctl[s], SOLVER_PRJ);
    for (int t = blockIdx.x; t < D.n_tiles; t += gridDim.x) {
        const int4 tile = __ldg(D.tiles + t);
        const SceneParams& P = D.scenes[tile.x];
        if (P.solver == SOLVER_PRJ) pj_begin_tile(D, P, tile, threadIdx.x, BLOCK);
    }
    if (!ph.barrier(-1)) return;
    ph.refresh();
    while (ph.any(K_PJ_HEAD)) {
        if (!ph.template run<MODE_PRJ>(K_PJ_HEAD)) return;
        if (!ph.template run<MODE_PRJ>(K_PJ_TAIL)) return;
    }
    for (int t = blockIdx.x; t < D.n_tiles; t += gridDim.x) {
        const TileCtx T = tile_ctx<G>(D, t);
        const SceneParams& P = D.scenes[T.sc];
        if (P.solver != SOLVER_PRJ) continue;
        const SceneCtl& C = ph.sc_sh[T.sc];
        if (C.status == IVP_OK_ && T.lane == 0 && T.valid) pj_end_slot(D, P, T.i);
        if (D.div_out) div_tile<G>(D, P, T, 0);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int s = 0; s < D.n_scenes; ++s) {
            if (D.scenes[s].solver != SOLVER_PRJ) continue;
            SceneCtl c = ctl_load(D.ctl + s);
            solve_account(c);
            D.ctl[s] = c;
        }
    }
}

__global__ void k_reset_counters(const Dev D) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= D.n_scenes) return;
    SceneCtl& C = D.ctl[s];
    C.acc_max_final_err = 0.0;
    C.acc_solves = C.acc_outer = C.acc_cg = C.acc_failed = C.acc_last_failure = C.acc_visc = C.acc_st = 0;
    if (s == 0) D.flags->timeout = 0;
}

// Neighbour lists of one scene in the reference layout, original indices.
// One scene's statistics and histories gathered into the staging block
// (StatStage), so the host reads them with one copy.  One CTA, 4-byte words
// (every part is a multiple of 4 bytes).
__device__ __forceinline__ void copy_words(unsigned char* dst, const void* src, size_t bytes) {
    const unsigned* s = static_cast<const unsigned*>(src);
    unsigned* d = reinterpret_cast<unsigned*>(dst);
    for (size_t k = threadIdx.x; k < bytes / 4; k += blockDim.x) d[k] = s[k];
}

__global__ void k_stage_stats(const Dev D, int scene, int hist) {
    const StatStage L(hist);
    copy_words(D.stage + L.ctl, D.ctl + scene, sizeof(SceneCtl));
    copy_words(D.stage + L.ovf, D.overflow + scene, sizeof(int));
    copy_words(D.stage + L.flags, D.flags, sizeof(Flags));
    copy_words(D.stage + L.pairs, D.pairs + scene, sizeof(unsigned long long));
    copy_words(D.stage + L.fix, D.fix_scene + scene, sizeof(int));
    copy_words(D.stage + L.err, D.err_hist + (size_t)scene * hist, sizeof(double) * (size_t)hist);
    copy_words(D.stage + L.pcg, D.pcg_hist + (size_t)scene * hist, sizeof(int) * (size_t)hist);
}

__global__ void k_export(const Dev D, int scene, int* count, int* ids, int cache) {
    const SceneParams& P = D.scenes[scene];
    const int i = P.s_begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.s_dyn_end) return;
    const int row = P.row_base + (i - P.s_begin);
    const int p = D.pid[i] - P.p_begin;
    const int cnt = D.nbr_cnt[row];
    count[p] = cnt;
    for (int k = 0; k < cnt && k < cache; ++k) ids[(size_t)p * cache + k] = D.pid[row_j(D, row, k)] - P.p_begin;
}

}  // namespace ivp
