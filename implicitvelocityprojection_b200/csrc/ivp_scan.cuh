// ivp_scan.cuh -- two-pass exclusive scan of int counts (cell counts of the
// counting sort), shared by the engine and the allocation-free entry point.
// The kernels have internal linkage so each translation unit keeps its own.
#pragma once
#include <cuda_runtime.h>

namespace ivp {

// Exclusive scan, pass 1: per-block scan of 4 elements per thread.
constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

static __global__ void __launch_bounds__(SCAN_BLOCK) k_scan_local(const int* __restrict__ in, int* __restrict__ out,
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
static __global__ void __launch_bounds__(SCAN_BLOCK) k_scan_add(int* __restrict__ out, const int* __restrict__ block_sums,
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

}  // namespace ivp
