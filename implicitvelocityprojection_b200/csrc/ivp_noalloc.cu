// ivp_noalloc.cu -- SPH density and k = 1/(Aii + eps) for one scene without
// any device allocation.
//
// Who needs this: callers that cannot allocate device memory themselves or let
// a library do it -- code that runs inside another runtime's memory arena
// (for example a host whose GPU memory is managed by Warp's or a renderer's
// fixed-budget allocator), code recorded into a CUDA stream capture in global
// capture mode, where cudaMalloc is illegal, and real-time loops that cannot
// afford the implicit device synchronisation of cudaMalloc/cudaFree.  The
// regular engine needs a caller-provided workspace sized by
// ivp_workspace_bytes; this entry point needs none.  Instead it works in one
// file-scope device array of fixed size (kScratchBytes below, about 6.3 MB),
// which every GPU that loads the library holds until the process exits.
//
// Limits: at most IVP_NOALLOC_MAX_PARTICLES particles and at most
// IVP_NOALLOC_MAX_CELLS grid cells (ceil(L/h) per axis multiplied).  Larger
// inputs are rejected with IVP_ERR_BAD_ARG before any device work.
//
// Sharing: every call, on every stream, uses the same array and leaves its
// contents behind.  The cell counters that must start at zero are cleared by
// each call; everything else is overwritten before it is read.  Two calls
// whose work overlaps on the GPU (different streams, or different host
// threads) race on the array and give wrong results: serialise them.
//
// Set-up: the device address of the array is looked up with
// cudaGetSymbolAddress the first time the entry point runs on a device (with
// that device current) and cached.  That first call must come before any
// stream capture that would record it.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/ivp.h"
#include "ivp_device.cuh"

namespace {

using ivp::cell_coord;
using ivp::cubic_W;
using ivp::dot3;
using ivp::f3;
using ivp::scale3;
using ivp::spiky_w;
using ivp::sub3;

constexpr int kMaxParticles = IVP_NOALLOC_MAX_PARTICLES;
constexpr int kMaxKeys = 2 * IVP_NOALLOC_MAX_CELLS;
constexpr int kMaxDevices = 64;

struct Scratch {
    int cell_count[kMaxKeys];
    int cell_start[kMaxKeys + 64];
    int key[kMaxParticles];
    int rank[kMaxParticles];
    int placed[kMaxParticles];
    int pid[kMaxParticles];
    float4 xm[kMaxParticles];
};
constexpr size_t kScratchBytes = sizeof(Scratch);

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_mutex;
Scratch* g_scratch_addr[kMaxDevices] = {};

struct Grid {
    int dims[3];
    int ncell;
    float cell_inv, h, cubic_k, spiky_k, W0;
    int cap;
};

__global__ void na_keys(const float* __restrict__ x, const int* __restrict__ dyn, int n, Grid g, Scratch* S) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int cx = cell_coord(x[3 * p], g.cell_inv, g.dims[0]);
    const int cy = cell_coord(x[3 * p + 1], g.cell_inv, g.dims[1]);
    const int cz = cell_coord(x[3 * p + 2], g.cell_inv, g.dims[2]);
    const int key = (dyn[p] ? 0 : g.ncell) + (cz * g.dims[1] + cy) * g.dims[0] + cx;
    S->key[p] = key;
    S->rank[p] = atomicAdd(&S->cell_count[key], 1);
}

// Exclusive scan of the cell counts in one CTA (the keys fit in the scratch
// limit, so one CTA walking 1024-wide chunks is enough for a utility path).
__global__ void __launch_bounds__(1024) na_scan(Scratch* S, int n_keys) {
    __shared__ int warp_tot[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < n_keys; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < n_keys ? S->cell_count[i] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_tot[w] = incl;
        __syncthreads();
        if (w == 0) {
            const int t = warp_tot[lane];
            int ti = t;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, ti, o);
                if (lane >= o) ti += u;
            }
            warp_tot[lane] = ti - t;
        }
        __syncthreads();
        const int off = carry + warp_tot[w];
        if (i < n_keys) S->cell_start[i] = off + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry = off + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) S->cell_start[n_keys] = carry;
}

__global__ void na_place(int n, Scratch* S) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    S->placed[S->cell_start[S->key[p]] + S->rank[p]] = p;
}

// Stable order by particle id inside each cell, and the slot-ordered copies.
__global__ void na_order(const float* __restrict__ x, const float* __restrict__ m, int n, Scratch* S) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = S->placed[s];
    const int key = S->key[p];
    const int b = S->cell_start[key], e = S->cell_start[key + 1];
    int before = 0;
    for (int q = b; q < e; ++q) before += (S->placed[q] < p);
    const int slot = b + before;
    S->pid[slot] = p;
    S->xm[slot] = make_float4(x[3 * p], x[3 * p + 1], x[3 * p + 2], m[p]);
}

// Density (pressure_base.py:12-46) and k (pressure_base.py:49-87) of every
// dynamic particle over its first `cap` neighbours |x_i - x_j| < h, j != i
// (neighbour_search.py:10-51), in the same candidate order as the engine's
// neighbour build, but without storing the lists.  Static particles get k = 0.
__global__ void na_density_aii(int n, Grid g, Scratch* S, float* __restrict__ density, float* __restrict__ kdiag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int n_dyn = S->cell_start[g.ncell];
    const int p = S->pid[i];
    if (i >= n_dyn) {
        kdiag[p] = 0.0f;
        return;
    }
    const float4 xi4 = S->xm[i];
    const float3 xi = f3(xi4);
    const float mi = xi4.w;
    const float h = g.h;
    const int cx = cell_coord(xi.x, g.cell_inv, g.dims[0]);
    const int cy = cell_coord(xi.y, g.cell_inv, g.dims[1]);
    const int cz = cell_coord(xi.z, g.cell_inv, g.dims[2]);
    float rho = 0.0f;
    rho = rho + mi * g.W0;
    float aii = 0.0f;
    float3 jii = make_float3(0.0f, 0.0f, 0.0f);
    int cnt = 0;
    const int x0 = cx > 0 ? cx - 1 : 0;
    const int x1 = cx < g.dims[0] - 1 ? cx + 1 : g.dims[0] - 1;
    for (int dz = -1; dz <= 1; ++dz) {
        const int z = cz + dz;
        if (z < 0 || z >= g.dims[2]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int yy = cy + dy;
            if (yy < 0 || yy >= g.dims[1]) continue;
            const int cb = (z * g.dims[1] + yy) * g.dims[0];
            for (int pass = 0; pass < 2; ++pass) {
                const int kb = (pass ? g.ncell : 0) + cb;
                const int jb = S->cell_start[kb + x0], je = S->cell_start[kb + x1 + 1];
                for (int j = jb; j < je; ++j) {
                    if (j == i) continue;
                    const float4 xj4 = S->xm[j];
                    const float3 r = sub3(xi, f3(xj4));
                    const float rn = sqrtf(dot3(r, r));
                    if (rn < h && cnt < g.cap) {
                        const float w = spiky_w(rn, h, g.spiky_k);
                        const float mj = xj4.w;
                        rho += mj * cubic_W(rn, h, g.cubic_k);
                        const float3 J = scale3(mj, scale3(w, r));
                        if (j < n_dyn) aii += dot3(J, J) * (1.0f / mj);
                        jii = sub3(jii, J);
                        ++cnt;
                    }
                }
            }
        }
    }
    aii += dot3(jii, jii) * (1.0f / mi);
    density[p] = rho;
    kdiag[p] = 1.0f / (aii + 1e-3f);
}

int fail(int code, const char*) { return code; }

}  // namespace

extern "C" int ivp_density_aii_noalloc(const float* x, const float* m, const int32_t* is_dynamic, int32_t n_particles,
                                       float particle_radius, const float* domain_size, int32_t cache_size,
                                       float* density, float* kdiag, void* stream) {
    if (n_particles < 0 || !domain_size || cache_size <= 0 || !(particle_radius > 0.0f))
        return fail(IVP_ERR_BAD_ARG, "ivp_density_aii_noalloc: bad argument");
    if (n_particles > kMaxParticles)
        return fail(IVP_ERR_BAD_ARG, "more particles than IVP_NOALLOC_MAX_PARTICLES");
    if (n_particles == 0) return IVP_OK;
    if (!x || !m || !is_dynamic || !density || !kdiag)
        return fail(IVP_ERR_BAD_ARG, "ivp_density_aii_noalloc: null array");
    Grid g;
    const float h = 4.0f * particle_radius;  // config_builder.py:51-52
    long ncell = 1;
    for (int a = 0; a < 3; ++a) {
        if (!(domain_size[a] > 0.0f)) return fail(IVP_ERR_BAD_ARG, "ivp_density_aii_noalloc: bad domain");
        double dd = std::ceil((double)domain_size[a] / (double)h);
        if (dd > 65536.0) return fail(IVP_ERR_BAD_ARG, "ivp_density_aii_noalloc: grid too large");
        g.dims[a] = dd < 1.0 ? 1 : (int)dd;
        ncell *= g.dims[a];
    }
    if (ncell > IVP_NOALLOC_MAX_CELLS)
        return fail(IVP_ERR_BAD_ARG, "more grid cells than IVP_NOALLOC_MAX_CELLS");
    g.ncell = (int)ncell;
    g.h = h;
    g.cell_inv = 1.0f / h;
    float k = 8.0f / 3.14159265359f;
    k = k / (h * h * h);
    g.cubic_k = k;
    g.W0 = k * (6.0f * 0.0f - 6.0f * 0.0f + 1.0f);
    g.spiky_k = 45.0f / (3.14159265359f * h * h * h * h * h * h);
    g.cap = cache_size;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(IVP_ERR_CUDA, "ivp_density_aii_noalloc: no current device");
    Scratch* S = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev]) {
            void* addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_scratch);
            if (e != cudaSuccess || !addr) return IVP_ERR_CUDA;
            g_scratch_addr[dev] = static_cast<Scratch*>(addr);
        }
        S = g_scratch_addr[dev];
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int n = n_particles, n_keys = 2 * g.ncell;
    const int B = 256, nb = (n + B - 1) / B;
    if (cudaMemsetAsync(S->cell_count, 0, sizeof(int) * (size_t)n_keys, s) != cudaSuccess)
        return fail(IVP_ERR_CUDA, "ivp_density_aii_noalloc: memset failed");
    na_keys<<<nb, B, 0, s>>>(x, is_dynamic, n, g, S);
    na_scan<<<1, 1024, 0, s>>>(S, n_keys);
    na_place<<<nb, B, 0, s>>>(n, S);
    na_order<<<nb, B, 0, s>>>(x, m, n, S);
    na_density_aii<<<nb, B, 0, s>>>(n, g, S, density, kdiag);
    if (cudaGetLastError() != cudaSuccess) return IVP_ERR_CUDA;
    return IVP_OK;
}
