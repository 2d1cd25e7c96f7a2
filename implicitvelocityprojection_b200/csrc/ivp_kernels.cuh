// ivp_kernels.cuh -- CUDA kernels of the IP pressure step (sm_100a).
//
// Bandwidth-bound sparse neighbour sums on CUDA cores (no tensor cores: the
// operator is a gather over ~30 neighbours per particle, ~1 flop/byte).
// Every neighbour-sum kernel maps G lanes to one particle: lane l takes list
// entries l, l+G, ... (coalesced 8-byte row reads) and the group reduces
// with shuffles.  Reductions across particles are FP64 per-CTA partials,
// summed in a fixed order by the last CTA of each scene, which also runs the
// scene's solver control (outer loop / CG decisions of ip.py:346-392 and
// ip.py:283-329); the last CTA of the launch sets the CUDA-graph conditional
// variables, so a whole step runs without a host round trip.
#pragma once
#include "ivp_device.cuh"

namespace ivp {

enum Kind { K_PACK = 0, K_RHS = 1, K_CG_A = 2, K_CG_B = 3, K_FINAL = 4 };

constexpr int IVP_OK_ = 0, IVP_NOT_SPD_ = 1, IVP_NOT_CONVERGED_ = 2, IVP_TIMEOUT_ = 6;

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

// Scene-level decision after a reduction (runs in one thread of the scene's
// last CTA).  `s` is the FP64 sum over the scene's dynamic particles.
__device__ void scene_finalize(const Dev& D, int sc, int kind, double s) {
    const SceneParams& P = D.scenes[sc];
    SceneCtl& C = D.ctl[sc];
    if (kind == K_PACK) {
        // pressure_base.py:405-423 average, ip.py:364-370 stopping rule
        const double err = P.n_dyn > 0 ? s / (double)P.n_dyn : 0.0;
        C.err = err;
        if (C.n_err < D.hist_len) D.err_hist[P.hist_base + C.n_err] = err;
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
            if (C.outer_it < D.hist_len) D.pcg_hist[P.hist_base + C.outer_it] = 0;
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
            if (C.outer_it < D.hist_len) D.pcg_hist[P.hist_base + C.outer_it] = C.cg_it;
            C.outer_it += 1;
            C.solve_pending = 0;
        } else {
            C.beta = rr_new / (C.rr_old > 1e-30 ? C.rr_old : 1e-30);
            C.rr_old = rr_new;
        }
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
            if (C->outer_active || C->cg_active || C->solve_pending) {
                C->status = IVP_TIMEOUT_;
                C->outer_active = 0;
                C->solve_pending = 0;
                C->cg_active = 0;
            }
        }
    }
    int any_outer = 0, any_solve = 0, any_cg = 0;
    // other CTAs wrote these during this launch: read past L1
    for (int s = 0; s < D.n_scenes; ++s) {
        const volatile SceneCtl* C = D.ctl + s;
        any_outer |= C->outer_active;
        any_solve |= C->solve_pending;
        any_cg |= C->cg_active;
    }
    D.flags->any_outer = any_outer;
    D.flags->any_solve = any_solve;
    D.flags->any_cg = any_cg;
    if (kind == K_PACK) {
        set_cond(D.h_outer, any_outer);
        set_cond(D.h_solve, any_solve);
    } else if (kind == K_RHS || kind == K_CG_B) {
        set_cond(D.h_cg, any_cg);
    }
}

// Reduce `part` over the CTA, hand it to the scene (last CTA of the scene
// sums the scene's partials in tile order) and to the launch.
template <int BLOCK>
__device__ void block_finish(const Dev& D, int sc, bool active, double part, int kind) {
    __shared__ double sh[32];
    __shared__ int sh_last;
    const double total = block_sum_d<BLOCK>(part, sh);
    const SceneParams& P = D.scenes[sc];
    if (threadIdx.x == 0) {
        sh_last = 0;
        if (active) {
            D.partial[blockIdx.x] = total;
            __threadfence();
            const int ntiles = P.tile_end - P.tile_begin;
            if (atomicAdd(&D.scene_counter[sc], 1) == ntiles - 1) sh_last = 1;
        }
    }
    __syncthreads();
    if (sh_last) {
        __threadfence();
        double s = 0.0;
        for (int t = P.tile_begin + (int)threadIdx.x; t < P.tile_end; t += BLOCK) s += __ldcg(&D.partial[t]);
        s = block_sum_d<BLOCK>(s, sh);
        if (threadIdx.x == 0) {
            D.scene_counter[sc] = 0;
            scene_finalize(D, sc, kind, s);
            __threadfence();
        }
    }
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
__global__ void k_keys(const Dev D) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= D.n_total) return;
    const int sc = D.pscene[p];
    const SceneParams& P = D.scenes[sc];
    const float px = D.x[3 * p], py = D.x[3 * p + 1], pz = D.x[3 * p + 2];
    const int cx = cell_coord(px, P.cell_inv, P.dims[0]);
    const int cy = cell_coord(py, P.cell_inv, P.dims[1]);
    const int cz = cell_coord(pz, P.cell_inv, P.dims[2]);
    const int cell = (cz * P.dims[1] + cy) * P.dims[0] + cx;
    const int key = P.key_base + (D.dyn[p] ? 0 : P.ncell) + cell;
    D.key[p] = key;
    D.rank[p] = atomicAdd(&D.cell_count[key], 1);
}

// Exclusive scan, pass 1: per-block scan of 4 elements per thread.
constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_local(const int* __restrict__ in, int* __restrict__ out,
                                                          int* __restrict__ block_sums, int n) {
    __shared__ int warp_tot[SCAN_BLOCK / 32];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int tsum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        tsum += v[k];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
        int t = warp_tot[lane];
        int ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += u;
        }
        warp_tot[lane] = ti - t;  // exclusive warp offsets
        if (lane == 31) block_sums[blockIdx.x] = ti;
    }
    __syncthreads();
    int run = warp_tot[w] + incl - tsum;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

// Exclusive scan, pass 2: add the sum of the preceding blocks; block 0 also
// writes the total at out[n].
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_add(int* __restrict__ out, const int* __restrict__ block_sums,
                                                        int n, int n_blocks) {
    __shared__ int sh_off;
    __shared__ int warp_tot[SCAN_BLOCK / 32];
    int acc = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += SCAN_BLOCK) acc += block_sums[b];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < SCAN_BLOCK / 32; ++w) t += warp_tot[w];
        sh_off = t;
        if (blockIdx.x == n_blocks - 1) out[n] = t + block_sums[blockIdx.x];
    }
    __syncthreads();
    const int off = sh_off;
    if (off == 0) return;
    const int base = blockIdx.x * SCAN_TILE;
    for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_BLOCK)
        if (base + k < n) out[base + k] += off;
}

__global__ void k_place(const Dev D) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= D.n_total) return;
    D.placed[D.cell_start[D.key[p]] + D.rank[p]] = p;
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
    D.xm[slot] = make_float4(D.x[3 * p], D.x[3 * p + 1], D.x[3 * p + 2], D.m[p]);
    D.rho0s[slot] = D.rho0[p];
}

// Neighbour lists of every dynamic particle (build_neighbor_cache,
// neighbour_search.py:10-51: j != i, |x_i - x_j| < h strict, first
// cache_size kept) fused with the density sum (pressure_base.py:12-46), the
// diagonal k = 1/(Aii + 1e-3) (pressure_base.py:49-87) and the constraint
// c = rho - rho0 (pressure_base.py:169-184).  One thread per particle; the
// 3 x-adjacent cells of a (y, z) row are one contiguous slot range.
__global__ void k_nbr_build(const Dev D) {
    const int4 tile = D.tiles[blockIdx.x];
    const int i = tile.y + threadIdx.x;
    if (i >= tile.z) return;
    const int sc = tile.x;
    const SceneParams& P = D.scenes[sc];
    const float4 xi4 = D.xm[i];
    const float3 xi = f3(xi4);
    const float mi = xi4.w;
    const float h = P.h;
    const int cx = cell_coord(xi.x, P.cell_inv, P.dims[0]);
    const int cy = cell_coord(xi.y, P.cell_inv, P.dims[1]);
    const int cz = cell_coord(xi.z, P.cell_inv, P.dims[2]);
    const int row = tile.w + threadIdx.x;
    int2* out = D.nbr + (size_t)row * D.stride;
    const int cap = P.cache < D.stride ? P.cache : D.stride;
    float rho = 0.0f;
    rho = rho + mi * P.W0;
    float aii = 0.0f;
    float3 jii = make_float3(0.0f, 0.0f, 0.0f);
    int cnt = 0, found = 0;
    const int x0 = cx > 0 ? cx - 1 : 0;
    const int x1 = cx < P.dims[0] - 1 ? cx + 1 : P.dims[0] - 1;
    for (int dz = -1; dz <= 1; ++dz) {
        const int z = cz + dz;
        if (z < 0 || z >= P.dims[2]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int yy = cy + dy;
            if (yy < 0 || yy >= P.dims[1]) continue;
            const int cb = (z * P.dims[1] + yy) * P.dims[0];
#pragma unroll 1
            for (int pass = 0; pass < 2; ++pass) {
                const int kb = P.key_base + (pass ? P.ncell : 0) + cb;
                const int jb = D.cell_start[kb + x0], je = D.cell_start[kb + x1 + 1];
                for (int j = jb; j < je; ++j) {
                    if (j == i) continue;
                    const float4 xj4 = D.xm[j];
                    const float3 r = sub3(xi, f3(xj4));
                    const float rn = sqrtf(dot3(r, r));
                    if (rn < h) {
                        ++found;
                        if (cnt < cap) {
                            const float w = spiky_w(rn, h, P.spiky_k);
                            out[cnt] = make_int2(j, __float_as_int(w));
                            const float mj = xj4.w;
                            rho += mj * cubic_W(rn, h, P.cubic_k);
                            const float3 g = scale3(w, r);
                            const float3 J = scale3(mj, g);
                            if (j < P.s_dyn_end) aii += dot3(J, J) * (1.0f / mj);
                            jii = sub3(jii, J);
                            ++cnt;
                        }
                    }
                }
            }
        }
    }
    aii += dot3(jii, jii) * (1.0f / mi);
    const float kd = 1.0f / (aii + 1e-3f);
    D.nbr_cnt[row] = cnt;
    D.dens[i] = rho;
    D.kd[i] = kd;
    D.c[i] = rho - D.rho0s[i];
    const int p = D.pid[i];
    D.density_out[p] = rho;
    D.k_out[p] = kd;
    if (found > cap) atomicAdd(&D.overflow[sc], 1);
    atomicAdd(&D.pairs[sc], (unsigned long long)cnt);
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
    const int2* nb = D.nbr + (size_t)row * D.stride;
    float3 xi = make_float3(0.f, 0.f, 0.f);
    int pi = 0;
    if (valid) {
        pi = D.pid[i];
        xi = make_float3(D.x[3 * pi], D.x[3 * pi + 1], D.x[3 * pi + 2]);
    }
    float acc = 0.0f;
    for (int k = lane; k < cnt; k += G) {
        const int j = nb[k].x;
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
    const int2* nb = D.nbr + (size_t)row * D.stride;
    const float4 xi4 = valid ? D.xm[i] : make_float4(0.f, 0.f, 0.f, 1.f);
    float aii = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
    for (int k = lane; k < cnt; k += G) {
        const int2 e = nb[k];
        const float4 xj = D.xm[e.x];
        const float3 gw = scale3(__int_as_float(e.y), sub3(f3(xi4), f3(xj)));
        const float3 J = scale3(xj.w, gw);
        if (e.x < P.s_dyn_end) aii += dot3(J, J) * (1.0f / xj.w);
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
        aii += dot3(jii, jii) * (1.0f / xi4.w);
        const float kd = 1.0f / (aii + 1e-3f);
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
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        long lim = 64;
        for (int s = 0; s < D.n_scenes; ++s)
            lim += (long)(D.scenes[s].max_outer + 1) * (long)(2 * D.scenes[s].max_pcg + 3);
        D.flags->limit = lim > 0x3fffffff ? 0x3fffffff : (int)lim;
        D.flags->launches = 0;
        D.flags->timeout = 0;
    }
    if (blockIdx.x == P.tile_begin && threadIdx.x == 0) {
        SceneCtl& C = D.ctl[tile.x];
        C.err = 0.0;
        C.rr_old = C.pap = C.alpha = C.beta = C.rr0 = 0.0;
        C.final_err = 0.0;
        C.outer_it = 0;
        C.cg_it = 0;
        C.outer_active = P.n_dyn > 0 ? 1 : 0;
        C.solve_pending = 0;
        C.cg_active = 0;
        C.status = IVP_OK_;
        C.n_err = 0;
        C.total_cg = 0;
    }
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
__global__ void k_advect(const Dev D) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= D.n_total) return;
    const int sc = D.pscene[p];
    if (D.advect_skip_failed && D.ctl[sc].status != IVP_OK_) return;
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
}

// ------------------------------------------------------------- IP solve

// Shared prologue of the neighbour-sum kernels: tile, scene, activity flag.
struct TileCtx {
    int4 tile;
    int sc;
    int g, lane, i, row;
    bool valid;
};

template <int G>
__device__ __forceinline__ TileCtx tile_ctx(const Dev& D) {
    TileCtx t;
    t.tile = D.tiles[blockIdx.x];
    t.sc = t.tile.x;
    t.g = threadIdx.x / G;
    t.lane = threadIdx.x % G;
    t.i = t.tile.y + t.g;
    t.row = t.tile.w + t.g;
    t.valid = t.i < t.tile.z;
    return t;
}

// ip_pack_fused (ip.py:124-171) + coef_wise_div + the average density error
// (pressure_base.py:187-203), with the previous outer update d -= sol
// (ip.py:389) applied on the fly.  Writes s = dfdt k and fk = f k for the
// rhs and CG kernels.
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_pack(const Dev D) {
    const TileCtx T = tile_ctx<G>(D);
    __shared__ int sh_active, sh_it;
    if (threadIdx.x == 0) {
        sh_active = D.ctl[T.sc].outer_active;
        sh_it = D.ctl[T.sc].outer_it;
    }
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active) {
        const SceneParams& P = D.scenes[T.sc];
        const int it = sh_it;
        const bool upd = it >= 1;
        const float4* src = (upd && ((it - 1) & 1)) ? D.d1 : D.d0;
        float4* dst = (it & 1) ? D.d1 : D.d0;
        const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
        const int2* nb = D.nbr + (size_t)T.row * D.stride;
        float3 xi = make_float3(0.f, 0.f, 0.f), di = xi;
        if (T.valid) {
            xi = f3(D.xm[T.i]);
            di = f3(src[T.i]);
            if (upd) di = sub3(di, f3(D.sol[T.i]));
        }
        float acc = 0.0f;
        for (int k = T.lane; k < cnt; k += G) {
            const int2 e = nb[k];
            const int j = e.x;
            if (j < P.s_begin || j >= P.s_end) { flag_bad(D, j, 1); continue; }
            const float4 xj = D.xm[j];
            const float3 gw = scale3(__int_as_float(e.y), sub3(xi, f3(xj)));
            float3 dj = f3(src[j]);
            if (upd) dj = sub3(dj, f3(D.sol[j]));
            acc += xj.w * dot3(sub3(di, dj), gw);
        }
        acc = group_sum<G>(acc);
        if (T.valid && T.lane == 0) {
            if (upd) dst[T.i] = make_float4(di.x, di.y, di.z, 0.0f);
            const float t = acc + D.c[T.i];
            const float f = t > 0.0f ? t : 0.0f;
            const float kd = D.kd[T.i];
            D.s[T.i] = (t >= 1e-6f) ? kd : 0.0f;
            D.fk[T.i] = f * kd;
            const float r0 = D.rho0s[T.i];
            const float q = f / (r0 < 1e-6f ? 1e-6f : r0);
            part = (double)(q > 0.0f ? q : 0.0f);
        }
    }
    block_finish<BLOCK>(D, T.sc, active, part, K_PACK);
}

// ip_rhs_fused (ip.py:174-215) fused with the CG start: sol = 0 (ip.py:384),
// r = rhs, p_prev = 0, rr = r.r (ip.py:293-296).
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_rhs(const Dev D) {
    const TileCtx T = tile_ctx<G>(D);
    __shared__ int sh_active;
    if (threadIdx.x == 0) sh_active = D.ctl[T.sc].solve_pending;
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active) {
        const SceneParams& P = D.scenes[T.sc];
        const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
        const int2* nb = D.nbr + (size_t)T.row * D.stride;
        float3 xi = make_float3(0.f, 0.f, 0.f);
        float fki = 0.0f, mi = 0.0f;
        if (T.valid) {
            const float4 a = D.xm[T.i];
            xi = f3(a);
            mi = a.w;
            fki = D.fk[T.i];
        }
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
        for (int k = T.lane; k < cnt; k += G) {
            const int2 e = nb[k];
            const int j = e.x;
            if (j < P.s_begin || j >= P.s_end) { flag_bad(D, j, 2); continue; }
            const float4 xj = D.xm[j];
            const float3 gw = scale3(__int_as_float(e.y), sub3(xi, f3(xj)));
            const float wgt = xj.w * fki + mi * D.fk[j];
            ax += wgt * gw.x;
            ay += wgt * gw.y;
            az += wgt * gw.z;
        }
        ax = group_sum<G>(ax);
        ay = group_sum<G>(ay);
        az = group_sum<G>(az);
        if (T.valid && T.lane == 0) {
            const float om = P.omega;
            const float4 rhs = make_float4(om * ax, om * ay, om * az, 0.0f);
            D.r[T.i] = rhs;
            D.sol[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
            D.p0[T.i] = make_float4(0.f, 0.f, 0.f, 0.f);
            part = (double)dot3(f3(rhs), f3(rhs));
        }
    }
    block_finish<BLOCK>(D, T.sc, active, part, K_RHS);
}

// CG launch A: p = r + beta p_prev (ip.py:323-327, formed on the fly for the
// neighbours too), y = dfdt k (J p) (compute_Jx_pcg, ip.py:19-60), and the
// FP64 partials of p^T A p = sum m |p|^2 + omega sum y (J p) (the value
// dot(p, A p) of ip.py:307, using that the gather-form transpose is the exact
// transpose of J for symmetric lists).
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cg_a(const Dev D) {
    const TileCtx T = tile_ctx<G>(D);
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
    if (active) {
        const SceneParams& P = D.scenes[T.sc];
        const float beta = sh_beta;
        const float4* pp = (sh_it & 1) ? D.p1 : D.p0;
        float4* pn = (sh_it & 1) ? D.p0 : D.p1;
        const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
        const int2* nb = D.nbr + (size_t)T.row * D.stride;
        float3 xi = make_float3(0.f, 0.f, 0.f), pi = xi;
        float mi = 0.0f;
        if (T.valid) {
            const float4 a = D.xm[T.i];
            xi = f3(a);
            mi = a.w;
            const float4 ri = D.r[T.i], qi = pp[T.i];
            pi = make_float3(ri.x + beta * qi.x, ri.y + beta * qi.y, ri.z + beta * qi.z);
        }
        float acc = 0.0f;
        for (int k = T.lane; k < cnt; k += G) {
            const int2 e = nb[k];
            const int j = e.x;
            if (j < P.s_begin || j >= P.s_end) { flag_bad(D, j, 3); continue; }
            const float4 xj = D.xm[j];
            const float3 gw = scale3(__int_as_float(e.y), sub3(xi, f3(xj)));
            const float4 rj = D.r[j], qj = pp[j];
            const float3 pj = make_float3(rj.x + beta * qj.x, rj.y + beta * qj.y, rj.z + beta * qj.z);
            acc += dot3(sub3(pi, pj), scale3(xj.w, gw));
        }
        acc = group_sum<G>(acc);
        if (T.valid && T.lane == 0) {
            const float yi = acc * D.s[T.i];
            D.y[T.i] = yi;
            pn[T.i] = make_float4(pi.x, pi.y, pi.z, 0.0f);
            part = (double)(mi * dot3(pi, pi)) + (double)P.omega * (double)yi * (double)acc;
        }
    }
    block_finish<BLOCK>(D, T.sc, active, part, K_CG_A);
}

// CG launch B: Ap = m p + omega J^T y in gather form (compute_Ax_part1/2,
// ip.py:63-121, as pressure_base.py:130-166 writes J^T), x += alpha p,
// r -= alpha Ap (pcg_update_x_r_scalar, math_utils.py:181-195), rr = r.r.
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cg_b(const Dev D) {
    const TileCtx T = tile_ctx<G>(D);
    __shared__ int sh_active, sh_it;
    __shared__ float sh_alpha;
    if (threadIdx.x == 0) {
        const SceneCtl& C = D.ctl[T.sc];
        sh_active = C.cg_active;
        sh_it = C.cg_it;
        sh_alpha = (float)C.alpha;
    }
    __syncthreads();
    const bool active = sh_active != 0;
    double part = 0.0;
    if (active) {
        const SceneParams& P = D.scenes[T.sc];
        const float4* pc = (sh_it & 1) ? D.p0 : D.p1;
        const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
        const int2* nb = D.nbr + (size_t)T.row * D.stride;
        float3 xi = make_float3(0.f, 0.f, 0.f);
        float mi = 0.0f, yi = 0.0f;
        if (T.valid) {
            const float4 a = D.xm[T.i];
            xi = f3(a);
            mi = a.w;
            yi = D.y[T.i];
        }
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
        for (int k = T.lane; k < cnt; k += G) {
            const int2 e = nb[k];
            const int j = e.x;
            if (j < P.s_begin || j >= P.s_end) { flag_bad(D, j, 4); continue; }
            const float4 xj = D.xm[j];
            const float3 gw = scale3(__int_as_float(e.y), sub3(xi, f3(xj)));
            const float wgt = xj.w * yi + mi * D.y[j];
            ax += wgt * gw.x;
            ay += wgt * gw.y;
            az += wgt * gw.z;
        }
        ax = group_sum<G>(ax);
        ay = group_sum<G>(ay);
        az = group_sum<G>(az);
        if (T.valid && T.lane == 0) {
            const float om = P.omega, alpha = sh_alpha;
            const float4 p4 = pc[T.i];
            const float3 ap = make_float3(mi * p4.x + om * ax, mi * p4.y + om * ay, mi * p4.z + om * az);
            float4 xs = D.sol[T.i], rs = D.r[T.i];
            xs.x = xs.x + alpha * p4.x;
            xs.y = xs.y + alpha * p4.y;
            xs.z = xs.z + alpha * p4.z;
            rs.x = rs.x - alpha * ap.x;
            rs.y = rs.y - alpha * ap.y;
            rs.z = rs.z - alpha * ap.z;
            D.sol[T.i] = xs;
            D.r[T.i] = rs;
            part = (double)dot3(f3(rs), f3(rs));
        }
    }
    block_finish<BLOCK>(D, T.sc, active, part, K_CG_B);
}

// compute_divergence (pressure_base.py:449-457): max(J v, 0) with v = d/dt.
template <int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_divergence(const Dev D) {
    const TileCtx T = tile_ctx<G>(D);
    const SceneParams& P = D.scenes[T.sc];
    const SceneCtl& C = D.ctl[T.sc];
    const float4* dc = (C.outer_it & 1) ? D.d1 : D.d0;
    const int cnt = T.valid ? D.nbr_cnt[T.row] : 0;
    const int2* nb = D.nbr + (size_t)T.row * D.stride;
    const float s = P.inv_dt;
    float3 xi = make_float3(0.f, 0.f, 0.f), vi = xi;
    if (T.valid) {
        xi = f3(D.xm[T.i]);
        vi = scale3(s, f3(dc[T.i]));
    }
    float acc = 0.0f;
    for (int k = T.lane; k < cnt; k += G) {
        const int2 e = nb[k];
        const float4 xj = D.xm[e.x];
        const float3 gw = scale3(__int_as_float(e.y), sub3(xi, f3(xj)));
        const float3 vj = scale3(s, f3(dc[e.x]));
        acc += xj.w * dot3(sub3(vi, vj), gw);
    }
    acc = group_sum<G>(acc);
    if (T.valid && T.lane == 0 && D.div_out) D.div_out[D.pid[T.i]] = acc > 0.0f ? acc : 0.0f;
}

__global__ void k_reset_counters(const Dev D) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= D.n_scenes) return;
    SceneCtl& C = D.ctl[s];
    C.acc_max_final_err = 0.0;
    C.acc_solves = C.acc_outer = C.acc_cg = C.acc_failed = C.acc_last_failure = 0;
}

// Neighbour lists of one scene in the reference layout, original indices.
__global__ void k_export(const Dev D, int scene, int* count, int* ids, int cache) {
    const SceneParams& P = D.scenes[scene];
    const int i = P.s_begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.s_dyn_end) return;
    const int row = P.row_base + (i - P.s_begin);
    const int p = D.pid[i] - P.p_begin;
    const int cnt = D.nbr_cnt[row];
    count[p] = cnt;
    for (int k = 0; k < cnt && k < cache; ++k) ids[(size_t)p * cache + k] = D.pid[D.nbr[(size_t)row * D.stride + k].x] - P.p_begin;
}

}  // namespace ivp
