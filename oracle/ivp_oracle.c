/*
 * ivp_oracle.c -- CPU restatement of the reference's implicit velocity
 * projection (IP) pressure step.  TEST INFRASTRUCTURE ONLY: it is the checker
 * for the CUDA engine and the timed CPU baseline, never part of the product.
 *
 * Parity status: the reference (medialab-ku/ImplicitVelocityProjection) is
 * Python + NVIDIA Warp kernels and ships no tests, fixtures or golden vectors.
 * Warp (`warp-lang>=1.11.1,<2`, requirements.txt:7) is not installable here,
 * so this restatement is pinned against golden vectors that were produced by
 * executing the reference's own kernel source (ip.py, pressure_base.py,
 * neighbour_search.py, sph_kernel.py, math_utils.py, framework.py,
 * boundary.py) on a NumPy FP32 stand-in for the Warp runtime
 * (tests/golden/make_golden.py), plus analytic known answers (rest-lattice
 * density, neighbour counts, gradient antisymmetry, CG vs dense solve).
 * Parity against real Warp execution is therefore unpinned.
 *
 * Layout follows the reference exactly: particle arrays in the caller's order,
 * neighbour cache rows of `cache_size` entries (`neighbor_ids[i*cache+k]`,
 * `neighbor_gradW[(i*cache+k)*3+c]`), FP32 arithmetic in the reference's
 * operation order.  Every function cites the reference lines it restates.
 *
 * Two reduction modes:
 *   REF  : FP32 dot products / averages accumulated in index order (what the
 *          reference computes with float atomics on a serial device) and the
 *          scatter form of J^T (ip.py:83-121), serial;
 *   FAST : FP64 reductions and the gather form of J^T (pressure_base.py:130-166,
 *          identical in exact arithmetic for symmetric lists), OpenMP over
 *          particles.  This is the policy of the CUDA engine and the mode the
 *          CPU baseline is timed in.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_NOT_SPD 1
#define ORC_NOT_CONVERGED 2
#define ORC_BAD_ARG 4

typedef struct {
    float h;              /* support radius (config_builder.py:51-52) */
    int cache_size;       /* neighborCacheSize (simulation_data.py:157) */
    float omega;          /* ip.py / pressure_base.py:317 */
    double tol_pcg;       /* ip.py:228 */
    double tol_opt;       /* densityErrorTol, pressure_base.py:316 */
    int max_outer;        /* maxOuterIters, pressure_base.py:314 */
    int max_pcg;          /* ip.py:229 */
    int fixed_iters;      /* fixedOuterIters, pressure_base.py:315 */
    int fast;             /* 0 = REF mode, 1 = FAST mode */
} orc_params;

typedef struct {
    int outer_iters;          /* stats_outer_iters */
    int n_err;                /* entries written to err_hist */
    double final_err;         /* stats_final_density_error */
    int status;
} orc_stats;

static inline float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline float len3(const float* a) { return sqrtf(dot3(a, a)); }

/* ---------------------------------------------------------------- kernels */

/* sph_kernel.py:8-25 */
float orc_cubic_kernel(float r, float h) {
    float res = 0.0f;
    float k = 8.0f / 3.14159265359f;
    k = k / (h * h * h);
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

/* sph_kernel.py:52-61 */
void orc_spiky_grad(const float* r, float h, float* out) {
    float k = 45.0f / (3.14159265359f * h * h * h * h * h * h);
    float rn = len3(r);
    if (rn < 1e-6f) rn = 1e-6f;
    float t = h - rn;
    float s = -k * (t * t);
    for (int c = 0; c < 3; ++c) out[c] = s * (r[c] / rn);
}

/* ------------------------------------------------------- neighbour cache */

static int cell_of(float v, float inv, int dim) {
    int c = (int)floorf(v * inv);
    return c < 0 ? 0 : (c >= dim ? dim - 1 : c);
}

/*
 * neighbour_search.py:10-51 (build_neighbor_cache) over a uniform grid of cell
 * size h anchored at the domain origin (neighbour_search.py:105-107: ceil(L/h)
 * cells per axis; cells of positions outside are clamped to the edge cells).
 * Candidate order is cell (z outermost, x innermost) then particle index, the
 * order in which Warp's hash grid query walks a scene whose domain starts at
 * the origin; it decides which hits a list keeps when a particle has more
 * than cache_size neighbours.  `domain` may be NULL (cells up to the largest
 * coordinate).  Lists are built for every particle when only_dynamic == 0 (as
 * the reference does) or for dynamic ones only.  Returns the number of
 * particles whose true count exceeded the cap.
 */
long orc_build_neighbor_cache(int n, const float* x, const int* is_dynamic, int only_dynamic,
                              float h, int cache, const float* domain, int* count, int* ids, float* gradW) {
    if (n <= 0) return 0;
    float hi[3] = {x[0], x[1], x[2]};
    for (int i = 1; i < n; ++i)
        for (int c = 0; c < 3; ++c)
            if (x[3 * i + c] > hi[c]) hi[c] = x[3 * i + c];
    int dim[3];
    float inv = 1.0f / h;
    for (int c = 0; c < 3; ++c) {
        if (domain) {
            dim[c] = (int)ceil((double)domain[c] / (double)h);
        } else {
            dim[c] = (int)floorf((hi[c] > 0.0f ? hi[c] : 0.0f) * inv) + 1;
        }
        if (dim[c] < 1) dim[c] = 1;
    }
    long ncell = (long)dim[0] * dim[1] * dim[2];
    int* cstart = (int*)calloc(ncell + 1, sizeof(int));
    int* cell = (int*)malloc(sizeof(int) * n);
    int* sorted = (int*)malloc(sizeof(int) * n);
    for (int i = 0; i < n; ++i) {
        int cx = cell_of(x[3 * i], inv, dim[0]);
        int cy = cell_of(x[3 * i + 1], inv, dim[1]);
        int cz = cell_of(x[3 * i + 2], inv, dim[2]);
        cell[i] = (int)(((long)cz * dim[1] + cy) * dim[0] + cx);
        cstart[cell[i] + 1]++;
    }
    for (long c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    int* fill = (int*)malloc(sizeof(int) * ncell);
    memcpy(fill, cstart, sizeof(int) * ncell);
    for (int i = 0; i < n; ++i) sorted[fill[cell[i]]++] = i;
    free(fill);

    long overflow = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : overflow)
    for (int i = 0; i < n; ++i) {
        if (only_dynamic && !is_dynamic[i]) { count[i] = 0; continue; }
        const float* xi = x + 3 * i;
        int ci = cell[i];
        int cx = ci % dim[0], cy = (ci / dim[0]) % dim[1], cz = ci / (dim[0] * dim[1]);
        int cnt = 0, found = 0;
        for (int dz = -1; dz <= 1; ++dz) {
            int z = cz + dz;
            if (z < 0 || z >= dim[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                int y = cy + dy;
                if (y < 0 || y >= dim[1]) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    int xx = cx + dx;
                    if (xx < 0 || xx >= dim[0]) continue;
                    long c = ((long)z * dim[1] + y) * dim[0] + xx;
                    for (int s = cstart[c]; s < cstart[c + 1]; ++s) {
                        int j = sorted[s];
                        if (j == i) continue;
                        float r[3] = {xi[0] - x[3 * j], xi[1] - x[3 * j + 1], xi[2] - x[3 * j + 2]};
                        float rn = len3(r);
                        if (rn < h) {
                            ++found;
                            if (cnt < cache) {
                                long b = (long)i * cache + cnt;
                                ids[b] = j;
                                orc_spiky_grad(r, h, gradW + 3 * b);
                                ++cnt;
                            }
                        }
                    }
                }
            }
        }
        count[i] = cnt;
        if (found > cache) ++overflow;
    }
    free(cstart);
    free(cell);
    free(sorted);
    return overflow;
}

static inline int clamp_cnt(int c, int cache) { return c > cache ? cache : c; }

/* Does any dynamic list hold cache entries?  Only then can a list have been
 * truncated, and only then may j in N(i) and i in N(j) disagree, so that the
 * gather form of J^T differs from the reference's scatter form. */
static int any_full_row(int n, const int* dyn, const int* count, int cache) {
    for (int i = 0; i < n; ++i)
        if (dyn[i] && count[i] >= cache) return 1;
    return 0;
}

/* pressure_base.py:12-46 */
void orc_compute_density(int n, const float* x, const float* m, const int* dyn, float h, int cache,
                         const int* count, const int* ids, float* density) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        if (!dyn[i]) continue;
        float rho = 0.0f;
        rho = rho + m[i] * orc_cubic_kernel(0.0f, h);
        int cnt = clamp_cnt(count[i], cache);
        for (int k = 0; k < cnt; ++k) {
            int j = ids[(long)i * cache + k];
            float r[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
            rho += m[j] * orc_cubic_kernel(len3(r), h);
        }
        density[i] = rho;
    }
}

/* pressure_base.py:49-87 */
void orc_compute_aii(int n, const float* m, const float* m_inv, const int* dyn, int cache,
                     const int* count, const int* ids, const float* gradW, float* kdiag) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        if (!dyn[i]) { kdiag[i] = 0.0f; continue; }
        float aii = 0.0f;
        float jii[3] = {0.0f, 0.0f, 0.0f};
        int cnt = clamp_cnt(count[i], cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * cache + k;
            int j = ids[b];
            float jij[3] = {m[j] * gradW[3 * b], m[j] * gradW[3 * b + 1], m[j] * gradW[3 * b + 2]};
            if (dyn[j]) aii += dot3(jij, jij) * m_inv[j];
            for (int c = 0; c < 3; ++c) jii[c] -= jij[c];
        }
        aii += dot3(jii, jii) * m_inv[i];
        kdiag[i] = 1.0f / (aii + 1e-3f);
    }
}

/* ip_pack_fused (ip.py:124-171) and compute_J_x_kernel (pressure_base.py:91-127):
 * out_i = sum_j m_j (val_i - [dyn j] val_j) . gradW_ij */
static void jx_plain(int n, const float* val, const float* m, const int* dyn, int cache, const int* count,
                     const int* ids, const float* gradW, float* out) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        if (!dyn[i]) { out[i] = 0.0f; continue; }
        const float* vi = val + 3 * i;
        float acc = 0.0f;
        int cnt = clamp_cnt(count[i], cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * cache + k;
            int j = ids[b];
            const float* g = gradW + 3 * b;
            if (dyn[j]) {
                float dv[3] = {vi[0] - val[3 * j], vi[1] - val[3 * j + 1], vi[2] - val[3 * j + 2]};
                acc += m[j] * dot3(dv, g);
            } else {
                acc += m[j] * dot3(vi, g);
            }
        }
        out[i] = acc;
    }
}

/* compute_Jx_pcg (ip.py:19-60): y_i = (sum_j (p_i - [dyn j] p_j) . (m_j gradW)) dfdt_i k_i */
static void jx_pcg(int n, const float* p, const float* m, const float* dfdt, const float* kd, const int* dyn,
                   int cache, const int* count, const int* ids, const float* gradW, float* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        y[i] = 0.0f;
        if (!dyn[i]) continue;
        if (dfdt[i] > 0.0f) {
            const float* pi = p + 3 * i;
            float acc = 0.0f;
            int cnt = clamp_cnt(count[i], cache);
            for (int k = 0; k < cnt; ++k) {
                long b = (long)i * cache + k;
                int j = ids[b];
                const float* g = gradW + 3 * b;
                float vij[3] = {m[j] * g[0], m[j] * g[1], m[j] * g[2]};
                if (dyn[j]) {
                    float dv[3] = {pi[0] - p[3 * j], pi[1] - p[3 * j + 1], pi[2] - p[3 * j + 2]};
                    acc += dot3(dv, vij);
                } else {
                    acc += dot3(pi, vij);
                }
            }
            y[i] = acc * dfdt[i] * kd[i];
        }
    }
}

/* compute_Ax_part1 + compute_Ax_part2 (ip.py:63-121), scatter form, serial */
static void ax_scatter(int n, const float* p, const float* y, const float* m, const float* dfdt, float omega,
                       const int* dyn, int cache, const int* count, const int* ids, const float* gradW,
                       float* ap) {
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) ap[3 * i + c] = dyn[i] ? m[i] * p[3 * i + c] : 0.0f;
    for (int i = 0; i < n; ++i) {
        if (!dyn[i] || dfdt[i] <= 0.0f) continue;
        float yi = y[i];
        int cnt = clamp_cnt(count[i], cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * cache + k;
            int j = ids[b];
            const float* g = gradW + 3 * b;
            float s = omega * yi;
            for (int c = 0; c < 3; ++c) {
                float contrib = s * (m[j] * g[c]);
                ap[3 * i + c] += contrib;
                if (dyn[j]) ap[3 * j + c] -= contrib;
            }
        }
    }
}

/* Ap = m p + omega J^T y, gather form (pressure_base.py:130-166 algebra) */
static void ax_gather(int n, const float* p, const float* y, const float* m, float omega, const int* dyn,
                      int cache, const int* count, const int* ids, const float* gradW, float* ap) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        if (!dyn[i]) { ap[3 * i] = ap[3 * i + 1] = ap[3 * i + 2] = 0.0f; continue; }
        float acc[3] = {0.0f, 0.0f, 0.0f};
        float yi = y[i], mi = m[i];
        int cnt = clamp_cnt(count[i], cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * cache + k;
            int j = ids[b];
            const float* g = gradW + 3 * b;
            float w = dyn[j] ? (m[j] * yi + mi * y[j]) : (m[j] * yi);
            for (int c = 0; c < 3; ++c) acc[c] += w * g[c];
        }
        for (int c = 0; c < 3; ++c) ap[3 * i + c] = mi * p[3 * i + c] + omega * acc[c];
    }
}

/* ip_rhs_fused (ip.py:174-215) */
static void rhs_fused(int n, const float* f, const float* kd, const float* m, float omega, const int* dyn,
                      int cache, const int* count, const int* ids, const float* gradW, float* rhs) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        if (!dyn[i]) { rhs[3 * i] = rhs[3 * i + 1] = rhs[3 * i + 2] = 0.0f; continue; }
        float fki = f[i] * kd[i], mi = m[i];
        float acc[3] = {0.0f, 0.0f, 0.0f};
        int cnt = clamp_cnt(count[i], cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * cache + k;
            int j = ids[b];
            const float* g = gradW + 3 * b;
            float w = dyn[j] ? (m[j] * fki + mi * (f[j] * kd[j])) : (m[j] * fki);
            for (int c = 0; c < 3; ++c) acc[c] += w * g[c];
        }
        for (int c = 0; c < 3; ++c) rhs[3 * i + c] = omega * acc[c];
    }
}

/* dot_vec3_tiled (math_utils.py:159-173) as summed by PressureBase.dot (pressure_base.py:425-436) */
static double dot_dyn(int n, const float* a, const float* b, const int* dyn, int fast) {
    if (fast) {
        double s = 0.0;
        for (int i = 0; i < n; ++i)
            if (dyn[i]) s += (double)dot3(a + 3 * i, b + 3 * i);
        return s;
    }
    float s = 0.0f;
    for (int i = 0; i < n; ++i)
        if (dyn[i]) s += dot3(a + 3 * i, b + 3 * i);
    return (double)s;
}

/* coef_wise_div + compute_avg_density_error (math_utils.py:77-91, pressure_base.py:187-203, 405-423):
 * avg over dynamic particles of max(t_i / max(rho0_i, 1e-6), 0) */
static double avg_density_error(int n, const float* t, const float* rho0, const int* dyn, int fast) {
    if (fast) {
        double s = 0.0;
        long cnt = 0;
        for (int i = 0; i < n; ++i) {
            if (!dyn[i]) continue;
            float den = rho0[i] < 1e-6f ? 1e-6f : rho0[i];
            float q = t[i] / den;
            s += (double)(q > 0.0f ? q : 0.0f);
            ++cnt;
        }
        return cnt > 0 ? s / (double)cnt : 0.0;
    }
    float s = 0.0f, cnt = 0.0f;
    for (int i = 0; i < n; ++i) {
        if (!dyn[i]) continue;
        float den = rho0[i] < 1e-6f ? 1e-6f : rho0[i];
        float q = t[i] / den;
        s += (q > 0.0f ? q : 0.0f);
        cnt += 1.0f;
    }
    return cnt > 0.0f ? (double)s / (double)cnt : 0.0;
}

/*
 * IP.PCG (ip.py:283-329): CG from x = 0 on A = M + omega J^T diag(dfdt k) J.
 * Returns the iteration count, or -1 on pAp < 0 (the reference raises).
 */
static int orc_pcg(int n, const orc_params* P, const float* m, const float* dfdt, const float* kd,
                   const int* dyn, const int* count, const int* ids, const float* gradW, float* x,
                   const float* b, float* r, float* p, float* ap, float* y) {
    int cache = P->cache_size;
    memcpy(r, b, sizeof(float) * 3 * (size_t)n);
    double rr_old = dot_dyn(n, r, r, dyn, P->fast);
    int it = 0;
    /* FAST mode gathers J^T y, which equals the scatter form only while every
     * pair is in both rows (no truncated list) */
    const int gather = P->fast && !any_full_row(n, dyn, count, cache);
    if (rr_old > 1e-30) {
        memcpy(p, r, sizeof(float) * 3 * (size_t)n);
        for (;;) {
            jx_pcg(n, p, m, dfdt, kd, dyn, cache, count, ids, gradW, y);
            if (gather)
                ax_gather(n, p, y, m, P->omega, dyn, cache, count, ids, gradW, ap);
            else
                ax_scatter(n, p, y, m, dfdt, P->omega, dyn, cache, count, ids, gradW, ap);
            double pap = dot_dyn(n, p, ap, dyn, P->fast);
            if (pap < 0.0) return -1;
            double alpha = rr_old / (pap > 1e-30 ? pap : 1e-30);
            float af = (float)alpha;
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i) {
                if (!dyn[i]) continue;
                for (int c = 0; c < 3; ++c) {
                    x[3 * i + c] = x[3 * i + c] + af * p[3 * i + c];
                    r[3 * i + c] = r[3 * i + c] - af * ap[3 * i + c];
                }
            }
            double rr_new = dot_dyn(n, r, r, dyn, P->fast);
            ++it;
            if ((rr_new < P->tol_pcg && it >= 2) || it >= P->max_pcg) break;
            double beta = rr_new / (rr_old > 1e-30 ? rr_old : 1e-30);
            float bf = (float)beta;
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i) {
                if (!dyn[i]) continue;
                for (int c = 0; c < 3; ++c) p[3 * i + c] = r[3 * i + c] + bf * p[3 * i + c];
            }
            rr_old = rr_new;
        }
    }
    return it;
}

/*
 * IP.solve(dt) (ip.py:331-404) with compute_constraint (pressure_base.py:169-184,
 * 394-403), check_converged (487-495) and final_density_error (438-447).
 * In: x-independent state (density, rho0, m, dyn, lists, kdiag), v.  Out: v
 * (overwritten with d/dt), err_hist[max_outer+1], pcg_hist[max_outer],
 * optional divergence (pressure_base.py:449-457; may be NULL) and stats.
 * Work buffers are allocated here (the oracle is not a hot path).
 */
int orc_ip_solve(int n, const orc_params* P, float dt, const float* density, const float* rho0,
                 const float* m, const int* dyn, const int* count, const int* ids, const float* gradW,
                 const float* kd, float* v, double* err_hist, int* pcg_hist, float* divergence,
                 float* d_out, orc_stats* st) {
    int cache = P->cache_size;
    size_t n3 = 3 * (size_t)n;
    float* c = (float*)calloc(n, sizeof(float));
    float* t = (float*)calloc(n, sizeof(float));
    float* f = (float*)calloc(n, sizeof(float));
    float* dfdt = (float*)calloc(n, sizeof(float));
    float* y = (float*)calloc(n, sizeof(float));
    float* d = (float*)calloc(n3, sizeof(float));
    float* rhs = (float*)calloc(n3, sizeof(float));
    float* sol = (float*)calloc(n3, sizeof(float));
    float* r = (float*)calloc(n3, sizeof(float));
    float* p = (float*)calloc(n3, sizeof(float));
    float* ap = (float*)calloc(n3, sizeof(float));

    for (int i = 0; i < n; ++i) c[i] = dyn[i] ? density[i] - rho0[i] : 0.0f;
    for (int i = 0; i < n; ++i)
        if (dyn[i])
            for (int q = 0; q < 3; ++q) d[3 * i + q] = dt * v[3 * i + q];

    int status = ORC_OK;
    int opt_iter = 0, n_err = 0;
    double err = 0.0;
    for (;;) {
        /* ip_pack_fused */
        jx_plain(n, d, m, dyn, cache, count, ids, gradW, t);
        for (int i = 0; i < n; ++i) {
            if (!dyn[i]) { t[i] = f[i] = dfdt[i] = 0.0f; continue; }
            float ti = t[i] + c[i];
            t[i] = ti;
            f[i] = ti > 0.0f ? ti : 0.0f;
            dfdt[i] = ti >= 1e-6f ? 1.0f : 0.0f;
        }
        err = avg_density_error(n, f, rho0, dyn, P->fast);
        if (err_hist && n_err < P->max_outer + 1) err_hist[n_err] = err;
        ++n_err;
        int converged = err < P->tol_opt && !P->fixed_iters;
        if ((converged && opt_iter >= 1) || opt_iter >= P->max_outer) break;
        rhs_fused(n, f, kd, m, P->omega, dyn, cache, count, ids, gradW, rhs);
        for (size_t q = 0; q < n3; ++q) sol[q] = 0.0f;
        int it = orc_pcg(n, P, m, dfdt, kd, dyn, count, ids, gradW, sol, rhs, r, p, ap, y);
        if (it < 0) { status = ORC_NOT_SPD; break; }
        if (pcg_hist && opt_iter < P->max_outer) pcg_hist[opt_iter] = it;
        for (int i = 0; i < n; ++i)
            if (dyn[i])
                for (int q = 0; q < 3; ++q) d[3 * i + q] = d[3 * i + q] + (-1.0f) * sol[3 * i + q];
        ++opt_iter;
    }
    if (status == ORC_OK && !P->fixed_iters && err >= P->tol_opt && opt_iter >= P->max_outer)
        status = ORC_NOT_CONVERGED;

    float inv_dt = (float)(1.0 / (double)dt);
    for (int i = 0; i < n; ++i)
        if (dyn[i])
            for (int q = 0; q < 3; ++q) v[3 * i + q] = inv_dt * d[3 * i + q];

    /* final_density_error: avg(max((c + J d) / rho0, 0)) */
    jx_plain(n, d, m, dyn, cache, count, ids, gradW, t);
    for (int i = 0; i < n; ++i)
        if (dyn[i]) t[i] = t[i] + 1.0f * c[i];
    double final_err = avg_density_error(n, t, rho0, dyn, P->fast);
    if (divergence) {
        jx_plain(n, v, m, dyn, cache, count, ids, gradW, t);
        for (int i = 0; i < n; ++i) divergence[i] = dyn[i] ? (t[i] > 0.0f ? t[i] : 0.0f) : 0.0f;
    }
    if (d_out) memcpy(d_out, d, sizeof(float) * n3);
    if (st) {
        st->outer_iters = opt_iter;
        st->n_err = n_err;
        st->final_err = final_err;
        st->status = status;
    }
    free(c); free(t); free(f); free(dfdt); free(y); free(d); free(rhs); free(sol); free(r); free(p); free(ap);
    return status;
}

/* apply_gravity (framework.py:26-41) */
void orc_apply_gravity(int n, float* v, const int* dyn, const float* g, float dt) {
    float gd[3] = {g[0] * dt, g[1] * dt, g[2] * dt};
    for (int i = 0; i < n; ++i)
        if (dyn[i])
            for (int c = 0; c < 3; ++c) v[3 * i + c] = v[3 * i + c] + gd[c];
}

/* advect_position (framework.py:117-136) then enforce_boundary (boundary.py:10-91) */
void orc_advect_and_clamp(int n, float* x, float* v, const int* dyn, float dt, const float* domain,
                          float padding) {
    for (int i = 0; i < n; ++i) {
        float* xi = x + 3 * i;
        float* vi = v + 3 * i;
        if (!dyn[i]) vi[0] = vi[1] = vi[2] = 0.0f;
        for (int c = 0; c < 3; ++c) xi[c] = xi[c] + dt * vi[c];
        if (!dyn[i]) continue;
        float nrm[3] = {0.0f, 0.0f, 0.0f};
        for (int c = 0; c < 3; ++c) {
            if (xi[c] > domain[c] - padding) { nrm[c] += 1.0f; xi[c] = domain[c] - padding; }
            if (xi[c] <= padding) { nrm[c] += -1.0f; xi[c] = padding; }
        }
        float nl = len3(nrm);
        if (nl > 1e-6f) {
            float u[3] = {nrm[0] / nl, nrm[1] / nl, nrm[2] / nl};
            float vn = dot3(vi, u);
            for (int c = 0; c < 3; ++c) vi[c] = vi[c] - (1.0f + 0.5f) * vn * u[c];
        }
    }
}

/* ------------------------------------------------- PRJ (projected Jacobi) */

/*
 * PRJ.solve (prj.py:296-340) with solve_PJ (prj.py:138-192): dt_v_0 = dt v,
 * cumulative dt^2 lambda from 0 (no warm start), then passes of
 *   head (pj_head_fused, prj.py:17-55): dt_v = dt_v_0 - dt^2 J^T lambda / max(m, 1e-6)
 *   tail (pj_tail_fused, prj.py:58-117): r = dt J dt_v + c,
 *        lambda = max(lambda + omega r D^-1, 0), err = avg max(r / rho0, 0)
 * stopping when (err < tol and pass >= 1) or pass >= max (the pass index is
 * the update count).  v = dt_v / dt unless it raises (check_converged).
 * `omega` is P->omega (PRJ uses 0.5, prj.py:127).
 */
int orc_prj_solve(int n, const orc_params* P, float dt, const float* density, const float* rho0, const float* m,
                  const int* dyn, const int* count, const int* ids, const float* gradW, const float* kd, float* v,
                  double* err_hist, orc_stats* st) {
    int cache = P->cache_size;
    size_t n3 = 3 * (size_t)n;
    float* c = (float*)calloc(n, sizeof(float));
    float* lam = (float*)calloc(n, sizeof(float));
    float* t = (float*)calloc(n, sizeof(float));
    float* v0 = (float*)calloc(n3, sizeof(float));
    float* dv = (float*)calloc(n3, sizeof(float));
    for (int i = 0; i < n; ++i) c[i] = dyn[i] ? density[i] - rho0[i] : 0.0f;
    for (int i = 0; i < n; ++i)
        if (dyn[i])
            for (int q = 0; q < 3; ++q) v0[3 * i + q] = dt * v[3 * i + q];
    memcpy(dv, v0, sizeof(float) * n3);
    double err = 0.0;
    int pass = 0, n_err = 0;
    for (pass = 0;; ++pass) {
        /* head */
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            if (!dyn[i]) continue;
            float acc[3] = {0.0f, 0.0f, 0.0f};
            int cnt = clamp_cnt(count[i], cache);
            for (int k = 0; k < cnt; ++k) {
                long b = (long)i * cache + k;
                int j = ids[b];
                const float* g = gradW + 3 * b;
                float s = dyn[j] ? (m[j] * lam[i] + m[i] * lam[j]) : (m[j] * lam[i]);
                for (int q = 0; q < 3; ++q) acc[q] = acc[q] + s * g[q];
            }
            float den = m[i] < 1e-6f ? 1e-6f : m[i];
            for (int q = 0; q < 3; ++q) dv[3 * i + q] = v0[3 * i + q] - acc[q] / den;
        }
        /* tail: r = J dt_v + c (the lambda update reads only its own lambda) */
        jx_plain(n, dv, m, dyn, cache, count, ids, gradW, t);
        for (int i = 0; i < n; ++i) {
            if (!dyn[i]) continue;
            t[i] = t[i] + c[i];
            float l = lam[i] + P->omega * t[i] * kd[i];
            lam[i] = l > 0.0f ? l : 0.0f;
        }
        err = avg_density_error(n, t, rho0, dyn, P->fast);
        if (err_hist) err_hist[n_err] = err;
        ++n_err;
        int converged = (err < P->tol_opt) && !P->fixed_iters;
        if ((converged && pass >= 1) || pass >= P->max_outer) break;
    }
    int status = ORC_OK;
    if (!P->fixed_iters && err >= P->tol_opt && pass >= P->max_outer) status = ORC_NOT_CONVERGED;
    if (status == ORC_OK) {
        float inv_dt = 1.0f / dt;
        for (int i = 0; i < n; ++i)
            if (dyn[i])
                for (int q = 0; q < 3; ++q) v[3 * i + q] = inv_dt * dv[3 * i + q];
    }
    st->outer_iters = pass;
    st->n_err = n_err;
    st->final_err = err;
    st->status = status;
    free(c); free(lam); free(t); free(v0); free(dv);
    return status;
}

/* ----------------------------------------------- Weiler 2018 viscosity */

/* wp.inverse of a 3x3 matrix: adjugate / determinant in FP32 */
static void inv33(const float* a, float* o) {
    float c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    float det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    float id = 1.0f / det;
    o[0] = c00 * id;
    o[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    o[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    o[3] = c01 * id;
    o[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    o[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    o[6] = c02 * id;
    o[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    o[8] = (a[0] * a[4] - a[1] * a[3]) * id;
}

typedef struct {
    float visc;        /* kinematic viscosity (viscosityCoeff) */
    float dt;
    float h;
    int cache;
    int max_iter;      /* weiler18.py:208 */
    double tol;        /* weiler18.py:209, absolute on r.r */
    int fast;          /* FP64 dots (1) or FP32 in index order (0) */
} orc_visc_params;

/* compute_precond_weiler18 (weiler18.py:21-85): inverse of the 3x3 diagonal
 * block of I - dt mu / rho L over fluid neighbours */
static void visc_precond(int n, const orc_visc_params* V, const float* x, const float* m, const float* density,
                         const float* rho0, const int* material, const int* dyn, const int* count, const int* ids,
                         const float* gradW, float* pinv) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        float* o = pinv + 9 * (size_t)i;
        if (!dyn[i] || material[i] != 1) {
            for (int q = 0; q < 9; ++q) o[q] = (q % 4 == 0) ? 1.0f : 0.0f;
            continue;
        }
        float eps2 = 0.01f * V->h * V->h;
        float d = 10.0f;
        float mu = V->visc * rho0[i];
        float factor = V->dt * mu / density[i];
        float L[9] = {0};
        int cnt = clamp_cnt(count[i], V->cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * V->cache + k;
            int j = ids[b];
            if (material[j] != 1) continue;
            float xij[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
            float rsq = dot3(xij, xij);
            const float* g = gradW + 3 * b;
            float c = d * (m[j] / density[j]) / (rsq + eps2);
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) L[3 * r + q] = L[3 * r + q] + c * (g[r] * xij[q]);
        }
        float M[9];
        for (int q = 0; q < 9; ++q) M[q] = ((q % 4 == 0) ? 1.0f : 0.0f) - factor * L[q];
        inv33(M, o);
    }
}

/* compute_Av_weiler18 (weiler18.py:103-172): (A v)_i = v_i - dt mu_i / rho_i L_i(v) */
static void visc_Av(int n, const orc_visc_params* V, const float* x, const float* vin, const float* m,
                    const float* density, const float* rho0, const int* material, const int* dyn, const int* count,
                    const int* ids, const float* gradW, float* av) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const float* vi = vin + 3 * i;
        if (!dyn[i] || material[i] != 1) {
            for (int c = 0; c < 3; ++c) av[3 * i + c] = vi[c];
            continue;
        }
        float eps2 = 0.01f * V->h * V->h;
        float d = 10.0f;
        float mu = V->visc * rho0[i];
        float factor = V->dt * mu / density[i];
        float lap[3] = {0.0f, 0.0f, 0.0f};
        int cnt = clamp_cnt(count[i], V->cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * V->cache + k;
            int j = ids[b];
            if (material[j] != 1) continue;
            float xij[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
            float vij[3] = {vi[0] - vin[3 * j], vi[1] - vin[3 * j + 1], vi[2] - vin[3 * j + 2]};
            float rsq = dot3(xij, xij);
            float vx = dot3(vij, xij);
            float s = d * (m[j] / density[j]) * (vx / (rsq + eps2));
            const float* g = gradW + 3 * b;
            for (int c = 0; c < 3; ++c) lap[c] += s * g[c];
        }
        for (int c = 0; c < 3; ++c) av[3 * i + c] = vi[c] - factor * lap[c];
    }
}

static void mat33_vec(const float* M, const float* v, float* o) {
    for (int r = 0; r < 3; ++r) o[r] = M[3 * r] * v[0] + M[3 * r + 1] * v[1] + M[3 * r + 2] * v[2];
}

/* Weiler18.solve (weiler18.py:371-401) with its block-Jacobi PCG
 * (weiler18.py:298-365): v += dv, A dv = v - A v, dv_0 = 0.  Returns the CG
 * iterations. */
int orc_weiler18_solve(int n, const orc_visc_params* V, const float* x, float* v, const float* m,
                       const float* density, const float* rho0, const int* material, const int* dyn,
                       const int* count, const int* ids, const float* gradW) {
    size_t n3 = 3 * (size_t)n;
    float* pinv = (float*)calloc(9 * (size_t)n, sizeof(float));
    float* dv = (float*)calloc(n3, sizeof(float));
    float* r = (float*)calloc(n3, sizeof(float));
    float* z = (float*)calloc(n3, sizeof(float));
    float* p = (float*)calloc(n3, sizeof(float));
    float* ap = (float*)calloc(n3, sizeof(float));
    float* rhs = (float*)calloc(n3, sizeof(float));
    visc_precond(n, V, x, m, density, rho0, material, dyn, count, ids, gradW, pinv);
    visc_Av(n, V, x, v, m, density, rho0, material, dyn, count, ids, gradW, ap);
    for (int i = 0; i < n; ++i)
        if (dyn[i])
            for (int c = 0; c < 3; ++c) rhs[3 * i + c] = v[3 * i + c] + (-1.0f) * ap[3 * i + c];
    memcpy(r, rhs, sizeof(float) * n3);
    for (int i = 0; i < n; ++i)
        if (dyn[i]) mat33_vec(pinv + 9 * (size_t)i, r + 3 * i, z + 3 * i);
    memcpy(p, z, sizeof(float) * n3);
    double rz_old = dot_dyn(n, r, z, dyn, V->fast);
    int it = 0;
    if (rz_old > 1e-12) {
        for (;;) {
            visc_Av(n, V, x, p, m, density, rho0, material, dyn, count, ids, gradW, ap);
            double pap = dot_dyn(n, p, ap, dyn, V->fast);
            if (pap <= 0.0) break;
            double alpha = rz_old / (pap > 1e-12 ? pap : 1e-12);
            float af = (float)alpha;
            for (int i = 0; i < n; ++i)
                if (dyn[i])
                    for (int c = 0; c < 3; ++c) dv[3 * i + c] = dv[3 * i + c] + af * p[3 * i + c];
            float naf = (float)(-alpha);
            for (int i = 0; i < n; ++i)
                if (dyn[i])
                    for (int c = 0; c < 3; ++c) r[3 * i + c] = r[3 * i + c] + naf * ap[3 * i + c];
            double rr = dot_dyn(n, r, r, dyn, V->fast);
            ++it;
            if ((rr < V->tol && it >= 2) || it >= V->max_iter) break;
            for (int i = 0; i < n; ++i)
                if (dyn[i]) mat33_vec(pinv + 9 * (size_t)i, r + 3 * i, z + 3 * i);
            double rz_new = dot_dyn(n, r, z, dyn, V->fast);
            double beta = rz_new / (rz_old > 1e-12 ? rz_old : 1e-12);
            float bf = (float)beta;
            for (int i = 0; i < n; ++i)
                if (dyn[i])
                    for (int c = 0; c < 3; ++c) p[3 * i + c] = z[3 * i + c] + bf * p[3 * i + c];
            rz_old = rz_new;
        }
    }
    for (int i = 0; i < n; ++i)
        if (dyn[i])
            for (int c = 0; c < 3; ++c) v[3 * i + c] = v[3 * i + c] + 1.0f * dv[3 * i + c];
    free(pinv); free(dv); free(r); free(z); free(p); free(ap); free(rhs);
    return it;
}

/* ----------------------------------------- Jeske 2023 surface tension */

typedef struct {
    float sigma;       /* surfaceTensionCoeff */
    float dt;
    float d;           /* particle diameter */
    float h_st;        /* jeske23.py:455: 2 d */
    int cache;
    int max_iter;      /* jeske23.py:470 */
    double tol;        /* jeske23.py:471, absolute on r.r */
    int fast;
} orc_st_params;

/* compute_Wst (jeske23.py:26-44): theta W_cubic(max(r, d); h_st), theta = 10/7 */
static float st_W(float r, float d, float h) {
    float theta = 10.0f / 7.0f;
    float rc = r > d ? r : d;
    float q = rc / h;
    float norm = 8.0f / (3.14159265358979f * h * h * h);
    float fq = 0.0f;
    if (q <= 0.5f) {
        fq = 1.0f - 6.0f * q * q + 6.0f * q * q * q;
    } else if (q <= 1.0f) {
        float t = 1.0f - q;
        fq = 2.0f * t * t * t;
    }
    return theta * norm * fq;
}

/* compute_grad_Wst (jeske23.py:47-67): zero for r <= d, else theta grad W_cubic */
static void st_gradW(const float* xij, float r, float d, float h, float* o) {
    o[0] = o[1] = o[2] = 0.0f;
    if (r <= d || r < 1.0e-12f) return;
    float q = r / h;
    if (q > 1.0f) return;
    float theta = 10.0f / 7.0f;
    float norm = 8.0f / (3.14159265358979f * h * h * h);
    float fpq;
    if (q <= 0.5f) {
        fpq = -12.0f * q + 18.0f * q * q;
    } else {
        float t = 1.0f - q;
        fpq = -6.0f * t * t;
    }
    float s = theta * norm * (1.0f / h) * fpq;
    for (int c = 0; c < 3; ++c) o[c] = s * (xij[c] / r);
}

/* compute_divergence_jeske23 (jeske23.py:74-115): m_j v_ij . gradW_ij over fluid j */
static void st_divergence(int n, const orc_st_params* S, const float* v, const float* m, const int* material,
                          const int* dyn, const int* count, const int* ids, const float* gradW, float* div) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        if (!dyn[i] || material[i] != 1) {
            div[i] = 0.0f;
            continue;
        }
        float acc = 0.0f;
        int cnt = clamp_cnt(count[i], S->cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * S->cache + k;
            int j = ids[b];
            if (material[j] != 1) continue;
            float vij[3] = {v[3 * i] - v[3 * j], v[3 * i + 1] - v[3 * j + 1], v[3 * i + 2] - v[3 * j + 2]};
            acc = acc + m[j] * dot3(vij, gradW + 3 * b);
        }
        div[i] = acc;
    }
}

/* compute_g_tilde_jeske23 (jeske23.py:118-188): per fluid pair
 * g~ = W / rho_bar + dt (gradW . v_ij / rho_bar - W / (2 rho_bar^2) (div_i + div_j)) */
static void st_g_tilde(int n, const orc_st_params* S, const float* x, const float* v, const float* density,
                       const int* material, const int* dyn, const int* count, const int* ids, const float* div,
                       float* gt) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        int cnt = clamp_cnt(count[i], S->cache);
        float* g = gt + (size_t)i * S->cache;
        if (!dyn[i] || material[i] != 1) {
            for (int k = 0; k < cnt; ++k) g[k] = 0.0f;
            continue;
        }
        for (int k = 0; k < cnt; ++k) {
            int j = ids[(size_t)i * S->cache + k];
            if (material[j] != 1) {
                g[k] = 0.0f;
                continue;
            }
            float xij[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
            float r = len3(xij);
            if (r >= S->h_st) {
                g[k] = 0.0f;
                continue;
            }
            float vij[3] = {v[3 * i] - v[3 * j], v[3 * i + 1] - v[3 * j + 1], v[3 * i + 2] - v[3 * j + 2]};
            float rho_bar = 0.5f * (density[i] + density[j]);
            float W = st_W(r, S->d, S->h_st);
            float gw[3];
            st_gradW(xij, r, S->d, S->h_st, gw);
            float gij = W / rho_bar;
            float term_kernel = dot3(gw, vij) / rho_bar;
            float term_density = W / (2.0f * rho_bar * rho_bar) * (div[i] + div[j]);
            g[k] = gij + S->dt * (term_kernel - term_density);
        }
    }
}

/* compute_rhs_jeske23 (jeske23.py:190-237): b_i = -dt sigma / m_i sum m_bar x_ij g~ */
static void st_rhs(int n, const orc_st_params* S, const float* x, const float* m, const int* material, const int* dyn,
                   const int* count, const int* ids, const float* gt, float* b) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        float* o = b + 3 * (size_t)i;
        if (!dyn[i] || material[i] != 1) {
            o[0] = o[1] = o[2] = 0.0f;
            continue;
        }
        float factor = -S->dt * S->sigma / m[i];
        float acc[3] = {0.0f, 0.0f, 0.0f};
        int cnt = clamp_cnt(count[i], S->cache);
        for (int k = 0; k < cnt; ++k) {
            long bb = (long)i * S->cache + k;
            int j = ids[bb];
            if (material[j] != 1) continue;
            float g = gt[bb];
            if (g == 0.0f) continue;
            float mbar = 0.5f * (m[i] + m[j]);
            for (int c = 0; c < 3; ++c) acc[c] = acc[c] + (mbar * (x[3 * i + c] - x[3 * j + c])) * g;
        }
        for (int c = 0; c < 3; ++c) o[c] = factor * acc[c];
    }
}

/* compute_Av_jeske23 (jeske23.py:240-292): (M v)_i = v_i + dt^2 sigma / m_i sum m_bar g~ v_ij */
static void st_Av(int n, const orc_st_params* S, const float* vin, const float* m, const int* material,
                  const int* dyn, const int* count, const int* ids, const float* gt, float* av) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const float* vi = vin + 3 * (size_t)i;
        if (!dyn[i] || material[i] != 1) {
            for (int c = 0; c < 3; ++c) av[3 * i + c] = vi[c];
            continue;
        }
        float dt2 = S->dt * S->dt;
        float factor = dt2 * S->sigma / m[i];
        float sum[3] = {0.0f, 0.0f, 0.0f};
        int cnt = clamp_cnt(count[i], S->cache);
        for (int k = 0; k < cnt; ++k) {
            long bb = (long)i * S->cache + k;
            int j = ids[bb];
            if (material[j] != 1) continue;
            float g = gt[bb];
            if (g == 0.0f) continue;
            float mbar = 0.5f * (m[i] + m[j]);
            float w = mbar * g;
            for (int c = 0; c < 3; ++c) sum[c] = sum[c] + w * (vi[c] - vin[3 * j + c]);
        }
        for (int c = 0; c < 3; ++c) av[3 * i + c] = vi[c] + factor * sum[c];
    }
}

/* compute_precond_jeske23 (jeske23.py:295-350): 1 / max(1 + dt^2 sigma / m_i sum m_bar g~, 1e-12) */
static void st_precond(int n, const orc_st_params* S, const float* m, const int* material, const int* dyn,
                       const int* count, const int* ids, const float* gt, float* inv) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        if (!dyn[i] || material[i] != 1) {
            inv[i] = 1.0f;
            continue;
        }
        float dt2 = S->dt * S->dt;
        float factor = dt2 * S->sigma / m[i];
        float ds = 0.0f;
        int cnt = clamp_cnt(count[i], S->cache);
        for (int k = 0; k < cnt; ++k) {
            long bb = (long)i * S->cache + k;
            int j = ids[bb];
            if (material[j] != 1) continue;
            float mbar = 0.5f * (m[i] + m[j]);
            ds = ds + mbar * gt[bb];
        }
        float dv = 1.0f + factor * ds;
        if (dv < 1.0e-12f) dv = 1.0e-12f;
        inv[i] = 1.0f / dv;
    }
}

/* Jeske23.solve (jeske23.py:585-655) with its PCG (jeske23.py:520-579):
 * v += dv, M dv = v - M v + b, dv_0 = 0, preconditioner diag(inv).  Returns
 * the CG iterations. */
int orc_jeske23_solve(int n, const orc_st_params* S, const float* x, float* v, const float* m, const float* density,
                      const int* material, const int* dyn, const int* count, const int* ids, const float* gradW,
                      float* div_out, float* b_out) {
    size_t n3 = 3 * (size_t)n;
    float* div = (float*)calloc((size_t)n, sizeof(float));
    float* gt = (float*)calloc((size_t)n * S->cache, sizeof(float));
    float* b = (float*)calloc(n3, sizeof(float));
    float* inv = (float*)calloc((size_t)n, sizeof(float));
    float* dv = (float*)calloc(n3, sizeof(float));
    float* r = (float*)calloc(n3, sizeof(float));
    float* z = (float*)calloc(n3, sizeof(float));
    float* p = (float*)calloc(n3, sizeof(float));
    float* ap = (float*)calloc(n3, sizeof(float));
    float* rhs = (float*)calloc(n3, sizeof(float));
    st_divergence(n, S, v, m, material, dyn, count, ids, gradW, div);
    st_g_tilde(n, S, x, v, density, material, dyn, count, ids, div, gt);
    st_rhs(n, S, x, m, material, dyn, count, ids, gt, b);
    st_precond(n, S, m, material, dyn, count, ids, gt, inv);
    st_Av(n, S, v, m, material, dyn, count, ids, gt, ap);
    for (int i = 0; i < n; ++i)
        if (dyn[i])
            for (int c = 0; c < 3; ++c) {
                rhs[3 * i + c] = v[3 * i + c] + (-1.0f) * ap[3 * i + c];
                rhs[3 * i + c] = rhs[3 * i + c] + 1.0f * b[3 * i + c];
            }
    memcpy(r, rhs, sizeof(float) * n3);
    /* z = (inv I3) r, as wp.mat33 * vec3 */
#define ST_PRECOND()                                                                   \
    for (int i = 0; i < n; ++i)                                                        \
        if (dyn[i]) {                                                                  \
            float M[9] = {inv[i], 0.0f, 0.0f, 0.0f, inv[i], 0.0f, 0.0f, 0.0f, inv[i]}; \
            mat33_vec(M, r + 3 * i, z + 3 * i);                                        \
        }
    ST_PRECOND();
    memcpy(p, z, sizeof(float) * n3);
    double rz_old = dot_dyn(n, r, z, dyn, S->fast);
    int it = 0;
    if (rz_old > 1e-12) {
        for (;;) {
            st_Av(n, S, p, m, material, dyn, count, ids, gt, ap);
            double pap = dot_dyn(n, p, ap, dyn, S->fast);
            if (pap <= 0.0) break;
            double alpha = rz_old / (pap > 1e-12 ? pap : 1e-12);
            float af = (float)alpha, naf = (float)(-alpha);
            for (int i = 0; i < n; ++i)
                if (dyn[i])
                    for (int c = 0; c < 3; ++c) dv[3 * i + c] = dv[3 * i + c] + af * p[3 * i + c];
            for (int i = 0; i < n; ++i)
                if (dyn[i])
                    for (int c = 0; c < 3; ++c) r[3 * i + c] = r[3 * i + c] + naf * ap[3 * i + c];
            double rr = dot_dyn(n, r, r, dyn, S->fast);
            ++it;
            if ((rr < S->tol && it >= 2) || it >= S->max_iter) break;
            ST_PRECOND();
            double rz_new = dot_dyn(n, r, z, dyn, S->fast);
            double beta = rz_new / (rz_old > 1e-12 ? rz_old : 1e-12);
            float bf = (float)beta;
            for (int i = 0; i < n; ++i)
                if (dyn[i])
                    for (int c = 0; c < 3; ++c) p[3 * i + c] = z[3 * i + c] + bf * p[3 * i + c];
            rz_old = rz_new;
        }
    }
#undef ST_PRECOND
    for (int i = 0; i < n; ++i)
        if (dyn[i])
            for (int c = 0; c < 3; ++c) v[3 * i + c] = v[3 * i + c] + 1.0f * dv[3 * i + c];
    if (div_out) memcpy(div_out, div, sizeof(float) * (size_t)n);
    if (b_out) memcpy(b_out, b, sizeof(float) * n3);
    free(div); free(gt); free(b); free(inv); free(dv); free(r); free(z); free(p); free(ap); free(rhs);
    return it;
}

/*
 * One Framework.forward() step with IP (framework.py:423-544): gravity,
 * Jeske23 implicit surface tension when `sigma` > 0, Weiler18 implicit
 * viscosity when `visc` > 0 (framework.py:400-421), IP.solve,
 * advect + clamp, neighbour rebuild, density, Aii.  `count/ids/gradW/density/kd` must hold the state of
 * the previous rebuild (Framework.initialize, framework.py:282-290).
 */
int orc_step(int n, const orc_params* P, float dt, const float* g, const float* domain, float* x, float* v,
             const float* rho0, const float* m, const float* m_inv, const int* dyn, int* count, int* ids,
             float* gradW, float* density, float* kd, double* err_hist, int* pcg_hist, orc_stats* st,
             long* overflow, const int* material, float visc, int* visc_iters, float sigma, int* st_iters,
             int prj) {
    orc_apply_gravity(n, v, dyn, g, dt);
    if (material && sigma > 0.0f) {
        /* Jeske23 implicit surface tension (framework.py:417-418) */
        orc_st_params S = {sigma, dt, 0.5f * P->h, P->h, P->cache_size, 100, 1e-5, P->fast};
        int it = orc_jeske23_solve(n, &S, x, v, m, density, material, dyn, count, ids, gradW, NULL, NULL);
        if (st_iters) *st_iters = it;
    }
    if (material && visc > 0.0f) {
        /* Weiler18 implicit viscosity (framework.py:400-421) */
        orc_visc_params V = {visc, dt, P->h, P->cache_size, 1000, 1e-5, P->fast};
        int it = orc_weiler18_solve(n, &V, x, v, m, density, rho0, material, dyn, count, ids, gradW);
        if (visc_iters) *visc_iters = it;
    }
    int status;
    if (prj) {
        /* PRJ (pressureMethod 0, framework.py:168-174) with its own omega (prj.py:127) */
        orc_params Q = *P;
        Q.omega = 0.5f;
        status = orc_prj_solve(n, &Q, dt, density, rho0, m, dyn, count, ids, gradW, kd, v, err_hist, st);
    } else {
        status = orc_ip_solve(n, P, dt, density, rho0, m, dyn, count, ids, gradW, kd, v, err_hist, pcg_hist,
                              NULL, NULL, st);
    }
    orc_advect_and_clamp(n, x, v, dyn, dt, domain, P->h);
    long ov = orc_build_neighbor_cache(n, x, dyn, 1, P->h, P->cache_size, domain, count, ids, gradW);
    if (overflow) *overflow = ov;
    orc_compute_density(n, x, m, dyn, P->h, P->cache_size, count, ids, density);
    orc_compute_aii(n, m, m_inv, dyn, P->cache_size, count, ids, gradW, kd);
    return status;
}

/*
 * FP64 CG on the same linear system as one IP outer iteration: given the
 * lists, mass, dfdt, k and rhs (all FP32 inputs), solve
 * (M + omega J^T diag(dfdt k) J) x = rhs in double precision until
 * ||r||^2 <= rel_tol^2 ||b||^2.  Returns iterations.  Used to state every
 * result's error against an FP64 solve.
 */
int orc_cg_f64(int n, float omega, int cache, const float* m, const float* dfdt, const float* kd,
               const int* dyn, const int* count, const int* ids, const float* gradW, const float* rhs,
               double rel_tol, int max_iter, double* x_out) {
    size_t n3 = 3 * (size_t)n;
    double* r = (double*)calloc(n3, sizeof(double));
    double* p = (double*)calloc(n3, sizeof(double));
    double* ap = (double*)calloc(n3, sizeof(double));
    double* y = (double*)calloc(n, sizeof(double));
    double bb = 0.0;
    for (int i = 0; i < n; ++i) {
        for (int c = 0; c < 3; ++c) {
            x_out[3 * i + c] = 0.0;
            r[3 * i + c] = dyn[i] ? (double)rhs[3 * i + c] : 0.0;
            p[3 * i + c] = r[3 * i + c];
            bb += r[3 * i + c] * r[3 * i + c];
        }
    }
    double rr = bb;
    int it = 0;
    const int gather = !any_full_row(n, dyn, count, cache);
    while (it < max_iter && rr > rel_tol * rel_tol * bb && rr > 0.0) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            y[i] = 0.0;
            if (!dyn[i] || dfdt[i] <= 0.0f) continue;
            double acc = 0.0;
            int cnt = clamp_cnt(count[i], cache);
            for (int k = 0; k < cnt; ++k) {
                long b = (long)i * cache + k;
                int j = ids[b];
                for (int c = 0; c < 3; ++c) {
                    double dv = p[3 * i + c] - (dyn[j] ? p[3 * j + c] : 0.0);
                    acc += (double)m[j] * dv * (double)gradW[3 * b + c];
                }
            }
            y[i] = acc * (double)dfdt[i] * (double)kd[i];
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            for (int c = 0; c < 3; ++c) ap[3 * i + c] = 0.0;
            if (!dyn[i]) continue;
            double acc[3] = {0.0, 0.0, 0.0};
            int cnt = clamp_cnt(count[i], cache);
            for (int k = 0; k < cnt; ++k) {
                long b = (long)i * cache + k;
                int j = ids[b];
                double w = (double)m[j] * y[i] + (dyn[j] ? (double)m[i] * y[j] : 0.0);
                for (int c = 0; c < 3; ++c) acc[c] += w * (double)gradW[3 * b + c];
            }
            for (int c = 0; c < 3; ++c) ap[3 * i + c] = (double)m[i] * p[3 * i + c] + (double)omega * acc[c];
        }
        if (!gather) {
            /* a truncated list: J^T y in the reference's scatter form */
            for (int i = 0; i < n; ++i)
                for (int c = 0; c < 3; ++c) ap[3 * i + c] = dyn[i] ? (double)m[i] * p[3 * i + c] : 0.0;
            for (int i = 0; i < n; ++i) {
                if (!dyn[i] || y[i] == 0.0) continue;
                int cnt = clamp_cnt(count[i], cache);
                for (int k = 0; k < cnt; ++k) {
                    long b = (long)i * cache + k;
                    int j = ids[b];
                    for (int c = 0; c < 3; ++c) {
                        double contrib = (double)omega * y[i] * (double)m[j] * (double)gradW[3 * b + c];
                        ap[3 * i + c] += contrib;
                        if (dyn[j]) ap[3 * j + c] -= contrib;
                    }
                }
            }
        }
        double pap = 0.0;
        for (size_t q = 0; q < n3; ++q) pap += p[q] * ap[q];
        if (pap <= 0.0) break;
        double alpha = rr / pap;
        double rr_new = 0.0;
        for (size_t q = 0; q < n3; ++q) {
            x_out[q] += alpha * p[q];
            r[q] -= alpha * ap[q];
            rr_new += r[q] * r[q];
        }
        double beta = rr_new / rr;
        for (size_t q = 0; q < n3; ++q) p[q] = r[q] + beta * p[q];
        rr = rr_new;
        ++it;
    }
    free(r); free(p); free(ap); free(y);
    return it;
}

/* One outer-iteration system at displacement d: returns t, f, dfdt and rhs as
 * ip_pack_fused + ip_rhs_fused compute them (ip.py:124-215). */
void orc_ip_system(int n, float omega, int cache, const float* d, const float* c, const float* m,
                   const int* dyn, const int* count, const int* ids, const float* gradW, const float* kd,
                   float* t, float* f, float* dfdt, float* rhs) {
    jx_plain(n, d, m, dyn, cache, count, ids, gradW, t);
    for (int i = 0; i < n; ++i) {
        if (!dyn[i]) { t[i] = f[i] = dfdt[i] = 0.0f; continue; }
        float ti = t[i] + c[i];
        t[i] = ti;
        f[i] = ti > 0.0f ? ti : 0.0f;
        dfdt[i] = ti >= 1e-6f ? 1.0f : 0.0f;
    }
    rhs_fused(n, f, kd, m, omega, dyn, cache, count, ids, gradW, rhs);
}

/* A p applied in FP64 (gather form) for symmetry / SPD checks on small cases. */
void orc_apply_A_f64(int n, float omega, int cache, const float* m, const float* dfdt, const float* kd,
                     const int* dyn, const int* count, const int* ids, const float* gradW, const double* p,
                     double* ap) {
    double* y = (double*)calloc(n, sizeof(double));
    for (int i = 0; i < n; ++i) {
        if (!dyn[i] || dfdt[i] <= 0.0f) continue;
        double acc = 0.0;
        int cnt = clamp_cnt(count[i], cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * cache + k;
            int j = ids[b];
            for (int c = 0; c < 3; ++c)
                acc += (double)m[j] * (p[3 * i + c] - (dyn[j] ? p[3 * j + c] : 0.0)) * (double)gradW[3 * b + c];
        }
        y[i] = acc * (double)dfdt[i] * (double)kd[i];
    }
    /* scatter form of J^T, exact transpose of J even for asymmetric lists */
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) ap[3 * i + c] = dyn[i] ? (double)m[i] * p[3 * i + c] : 0.0;
    for (int i = 0; i < n; ++i) {
        if (!dyn[i] || y[i] == 0.0) continue;
        int cnt = clamp_cnt(count[i], cache);
        for (int k = 0; k < cnt; ++k) {
            long b = (long)i * cache + k;
            int j = ids[b];
            for (int c = 0; c < 3; ++c) {
                double contrib = (double)omega * y[i] * (double)m[j] * (double)gradW[3 * b + c];
                ap[3 * i + c] += contrib;
                if (dyn[j]) ap[3 * j + c] -= contrib;
            }
        }
    }
    free(y);
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}
