// ivp_noalloc.cu -- SPH density and k = 1/(Aii + eps) for one scene without
// any device allocation.
//
// Who needs this: callers that cannot allocate device memory themselves or let
// a library do it -- code that runs inside another runtime's memory arena
// (for example a host whose GPU memory is managed by Warp's or a renderer's
// fixed-budget allocator), and real-time loops that cannot afford the
// implicit device synchronisation of cudaMalloc/cudaFree.  The
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
// that device current) and cached.  Make that first call on a device before
// any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include <string>

#include "../../include/ivp.h"
#include "ivp_device.cuh"
#include "ivp_scan.cuh"

namespace ivp {
// the engine's thread-local error text (ivp_last_error), set in ivp_engine.cu
void set_last_error(const std::string& msg);
}  // namespace ivp

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
    int block_sums[(kMaxKeys + ivp::SCAN_TILE - 1) / ivp::SCAN_TILE];
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

// Every failure leaves its reason where ivp_last_error() reads it.
int fail(int code, const char* msg) {
    ivp::set_last_error(msg);
    return code;
}

// One launch; its own status (cudaLaunchKernel reports this launch's error,
// not one left pending by earlier work of the caller).
int launch(const void* fn, int grid, int block, void** args, cudaStream_t s, const char* what) {
    const cudaError_t e = cudaLaunchKernel(fn, dim3(grid), dim3(block), args, 0, s);
    if (e != cudaSuccess) {
        cudaGetLastError();  // this launch's error is now the last error: clear it, it is reported here
        return fail(IVP_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
    }
    return IVP_OK;
}

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
            if (e != cudaSuccess || !addr) {
                if (e != cudaSuccess) cudaGetLastError();  // reported here
                return fail(IVP_ERR_CUDA, (std::string("ivp_density_aii_noalloc: cudaGetSymbolAddress: ") +
                                           cudaGetErrorString(e)).c_str());
            }
            g_scratch_addr[dev] = static_cast<Scratch*>(addr);
        }
        S = g_scratch_addr[dev];
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int n = n_particles, n_keys = 2 * g.ncell;
    const int B = 256, nb = (n + B - 1) / B;
    {
        const cudaError_t e = cudaMemsetAsync(S->cell_count, 0, sizeof(int) * (size_t)n_keys, s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(IVP_ERR_CUDA, (std::string("ivp_density_aii_noalloc: memset: ") + cudaGetErrorString(e)).c_str());
        }
    }
    int* counts = S->cell_count;
    int* starts = S->cell_start;
    int* bsums = S->block_sums;
    int nk = n_keys, nsb = (n_keys + ivp::SCAN_TILE - 1) / ivp::SCAN_TILE, nn = n;
    const float* px = x;
    const float* pm = m;
    const int* pd = is_dynamic;
    void* a_keys[] = {&px, &pd, &nn, &g, &S};
    void* a_scan1[] = {&counts, &starts, &bsums, &nk};
    void* a_scan2[] = {&starts, &bsums, &nk, &nsb};
    void* a_place[] = {&nn, &S};
    void* a_order[] = {&px, &pm, &nn, &S};
    void* a_dens[] = {&nn, &g, &S, &density, &kdiag};
    int st = launch((const void*)na_keys, nb, B, a_keys, s, "na_keys");
    if (st == IVP_OK) st = launch((const void*)ivp::k_scan_local, nsb, ivp::SCAN_BLOCK, a_scan1, s, "scan_local");
    if (st == IVP_OK) st = launch((const void*)ivp::k_scan_add, nsb, ivp::SCAN_BLOCK, a_scan2, s, "scan_add");
    if (st == IVP_OK) st = launch((const void*)na_place, nb, B, a_place, s, "na_place");
    if (st == IVP_OK) st = launch((const void*)na_order, nb, B, a_order, s, "na_order");
    if (st == IVP_OK) st = launch((const void*)na_density_aii, nb, B, a_dens, s, "na_density_aii");
    if (st != IVP_OK) return st;
    return IVP_OK;
}
