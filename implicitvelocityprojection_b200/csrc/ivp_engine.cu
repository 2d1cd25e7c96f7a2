// ivp_engine.cu -- host side of the IP pressure-step engine and its C ABI
// (include/ivp.h).  No device allocation after ivp_engine_create: every
// buffer is carved from the caller's workspace.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ivp.h"
#include "ivp_kernels.cuh"

using namespace ivp;

namespace {

thread_local std::string g_err;

#define CK(x)                                                                 \
    do {                                                                      \
        cudaError_t e_ = (x);                                                 \
        if (e_ != cudaSuccess) {                                              \
            g_err = std::string(#x) + ": " + cudaGetErrorString(e_);          \
            return IVP_ERR_CUDA;                                              \
        }                                                                     \
    } while (0)

#define CKS(x)                          \
    do {                                \
        int s_ = (x);                   \
        if (s_ != IVP_OK) return s_;    \
    } while (0)

inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

struct Layout {
    size_t total = 0;
    size_t add(size_t bytes) {
        size_t off = total;
        total = align256(total + bytes);
        return off;
    }
};

constexpr int ELEM_BLOCK = 256;

inline int blocks_for(int n, int b) { return (n + b - 1) / b; }

}  // namespace

namespace ivp {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace ivp

struct ivp_engine {
    std::vector<ivp_scene_desc> desc;
    std::vector<SceneParams> hp;
    std::vector<int4> tiles;
    ivp_options opt{};
    Dev D{};
    int G = 4, BLOCK = 128, T = 32;
    int n_total = 0, n_dyn_total = 0, n_keys = 0, n_tiles = 0, scan_blocks = 0, n_segs = 0;
    int fix_scan_blocks = 0;
    int* h_ovf = nullptr;        // pinned: truncated-list count read back by host-driven builds
    int* h_fix_scene = nullptr;  // pinned, n_scenes: corrections per scene
    int n_scenes = 0;
    bool bound = false;
    bool want_divergence = false;
    bool any_visc = false;
    bool any_st = false;
    bool any_ip = false, any_prj = false;
    // persistent solve
    bool persistent = false;
    int coop_grid = 0, coop_grid_visc = 0, coop_grid_st = 0, coop_grid_prj = 0;
    size_t coop_smem = 0;
    // graphs
    cudaGraph_t graph_step = nullptr, graph_solve = nullptr, graph_build = nullptr, graph_prj = nullptr;
    cudaGraphExec_t exec_step = nullptr, exec_solve = nullptr, exec_build = nullptr, exec_prj = nullptr;
    // steps with host input/output (ivp_step_io): the copies of the graph
    // below are baked in for the host pointers and range of `io_key`
    cudaGraph_t graph_step_io = nullptr;
    cudaGraphExec_t exec_step_io = nullptr;
    struct StepIO {
        const float* x_in = nullptr;
        const float* v_in = nullptr;
        float* x_out = nullptr;
        float* v_out = nullptr;
        int64_t first = 0, count = 0;
        bool operator==(const StepIO& o) const {
            return x_in == o.x_in && v_in == o.v_in && x_out == o.x_out && v_out == o.v_out && first == o.first &&
                   count == o.count;
        }
    } io, io_key;
    cudaStream_t io_side = nullptr;                              // stream-ordered steps: the copy stream
    cudaEvent_t io_ev_start = nullptr, io_ev_x = nullptr, io_ev_adv = nullptr, io_ev_out = nullptr;
    // host mirrors
    SceneCtl* h_ctl = nullptr;   // pinned
    Flags* h_flags = nullptr;    // pinned
    int* h_overflow = nullptr;   // pinned
    unsigned long long* h_pairs = nullptr;  // pinned
    double* h_err = nullptr;     // pinned, max_hist: one scene's density-error history
    int* h_pcg = nullptr;        // pinned, max_hist: one scene's CG counts per outer iteration
    unsigned char* h_stage = nullptr;  // pinned: one scene's statistics block (StatStage)
};

// ------------------------------------------------------------ launching

namespace {

typedef void (*DevKernel)(const Dev);

// Per-launch CUDA events of a profiled host-driven run.
struct Prof {
    std::vector<cudaEvent_t> ev;
    std::vector<int> ids;
    ~Prof() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
};

struct Launcher {
    // Either launches on a stream or appends a kernel node to a graph chain.
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphNode_t last = nullptr;
    bool has_last = false;
    Prof* prof = nullptr;
    // host copies of an ivp_step_io step (null otherwise), and a node the
    // next chained node must also wait for (graph mode)
    ivp_engine* io = nullptr;
    cudaGraphNode_t io_x = nullptr;  // the upload of x (graph mode)
    cudaGraphNode_t extra = nullptr;

    int deps(cudaGraphNode_t* d) {
        int n = 0;
        if (has_last) d[n++] = last;
        if (extra) d[n++] = extra;
        extra = nullptr;
        return n;
    }

    int launch_now(const void* fn, dim3 grid, dim3 block, void** args, size_t smem, bool coop) {
        if (coop) {
            CK(cudaLaunchCooperativeKernel(fn, grid, block, args, smem, stream));
        } else {
            CK(cudaLaunchKernel(fn, grid, block, args, smem, stream));
        }
        return IVP_OK;
    }
    int kernel(int id, const void* fn, dim3 grid, dim3 block, void** args, size_t smem = 0, bool coop = false) {
        if (grid.x == 0) return IVP_OK;
        if (!graph) {
            if (prof) {
                const size_t k = prof->ids.size();
                while (prof->ev.size() < 2 * (k + 1)) {
                    cudaEvent_t ev;
                    CK(cudaEventCreate(&ev));
                    prof->ev.push_back(ev);
                }
                CK(cudaEventRecord(prof->ev[2 * k], stream));
                CKS(launch_now(fn, grid, block, args, smem, coop));
                CK(cudaEventRecord(prof->ev[2 * k + 1], stream));
                prof->ids.push_back(id);
                return IVP_OK;
            }
            return launch_now(fn, grid, block, args, smem, coop);
        }
        cudaKernelNodeParams p;
        memset(&p, 0, sizeof(p));
        p.func = const_cast<void*>(fn);
        p.gridDim = grid;
        p.blockDim = block;
        p.sharedMemBytes = (unsigned)smem;
        p.kernelParams = args;
        p.extra = nullptr;
        cudaGraphNode_t n, d[2];
        const int nd = deps(d);
        CK(cudaGraphAddKernelNode(&n, graph, nd ? d : nullptr, nd, &p));
        if (coop) {
            cudaKernelNodeAttrValue v;
            memset(&v, 0, sizeof(v));
            v.cooperative = 1;
            CK(cudaGraphKernelNodeSetAttribute(n, cudaLaunchAttributeCooperative, &v));
        }
        last = n;
        has_last = true;
        return IVP_OK;
    }
    int dev(int id, DevKernel fn, int grid, int block, const Dev& D) {
        Dev copy = D;
        void* args[] = {&copy};
        return kernel(id, (const void*)fn, dim3(grid), dim3(block), args);
    }
    int memset0(void* ptr, size_t bytes) {
        if (bytes == 0) return IVP_OK;
        if (!graph) {
            CK(cudaMemsetAsync(ptr, 0, bytes, stream));
            return IVP_OK;
        }
        cudaMemsetParams mp;
        memset(&mp, 0, sizeof(mp));
        mp.dst = ptr;
        mp.value = 0;
        mp.elementSize = 1;
        mp.width = bytes;
        mp.height = 1;
        mp.pitch = 0;
        cudaGraphNode_t n, d[2];
        const int nd = deps(d);
        CK(cudaGraphAddMemsetNode(&n, graph, nd ? d : nullptr, nd, &mp));
        last = n;
        has_last = true;
        return IVP_OK;
    }
    // A host<->device copy: chained (after the last node, and the next node
    // waits for it) or, with `branch`, as a node after `after` (none: a root)
    // that nothing in the chain waits for unless it is handed to `extra`.
    int copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, bool branch = false,
             cudaGraphNode_t after = nullptr, cudaGraphNode_t* out = nullptr) {
        if (bytes == 0) return IVP_OK;
        cudaGraphNode_t n, d[2];
        int nd = 0;
        if (branch) {
            if (after) d[nd++] = after;
        } else {
            nd = deps(d);
        }
        CK(cudaGraphAddMemcpyNode1D(&n, graph, nd ? d : nullptr, nd, dst, src, bytes, kind));
        if (out) *out = n;
        if (!branch) {
            last = n;
            has_last = true;
        }
        return IVP_OK;
    }
};

template <int G, int BLOCK>
struct Kern {
    static DevKernel pack() { return k_pack<G, BLOCK>; }
    static DevKernel rhs() { return k_rhs<G, BLOCK>; }
    static DevKernel cg_a() { return k_cg_a<G, BLOCK>; }
    static DevKernel cg_b() { return k_cg_b<G, BLOCK>; }
    static DevKernel dens() { return k_density<G, BLOCK>; }
    static DevKernel aii() { return k_aii<G, BLOCK>; }
    static DevKernel div() { return k_divergence<G, BLOCK>; }
};

struct KernelSet {
    DevKernel pack, rhs, cg_a, cg_b, dens, aii, div, persist, v_setup, v_a, v_b, v_end, v_persist, st_div,
        st_persist, pj_head, pj_tail, prj_persist;
};

template <int G, int B>
KernelSet make_set() {
    return {Kern<G, B>::pack(), Kern<G, B>::rhs(), Kern<G, B>::cg_a(), Kern<G, B>::cg_b(),
            Kern<G, B>::dens(), Kern<G, B>::aii(), Kern<G, B>::div(), k_ip_persistent<G, B>,
            k_visc_setup<G, B>, k_visc_a<G, B>, k_visc_b<G, B>, k_visc_end<G, B>,
            k_force_persistent<G, B, FORCE_VISC>, k_st_div<G, B>, k_force_persistent<G, B, FORCE_ST>,
            k_pj_head<G, B>, k_pj_tail<G, B>, k_prj_persistent<G, B>};
}

// Instantiated launch shapes: G lanes per particle x {128, 256} threads.
bool kernel_set(int G, int B, KernelSet* out) {
    if (B == 128) {
        switch (G) {
            case 1: *out = make_set<1, 128>(); return true;
            case 2: *out = make_set<2, 128>(); return true;
            case 4: *out = make_set<4, 128>(); return true;
            case 8: *out = make_set<8, 128>(); return true;
            default: return false;
        }
    }
    if (B == 256) {
        switch (G) {
            case 2: *out = make_set<2, 256>(); return true;
            case 4: *out = make_set<4, 256>(); return true;
            case 8: *out = make_set<8, 256>(); return true;
            default: return false;
        }
    }
    return false;
}

int add_conditional(cudaGraph_t g, Launcher& L, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    cudaGraph_t* body);

// Rows of truncated lists in the reference's order, then the transpose
// corrections of CG phase B (k_ovf_* in ivp_kernels.cuh).  Runs only after a
// build that truncated a list.
int emit_overflow_fix(ivp_engine* e, Launcher& L) {
    const Dev& D = e->D;
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    CKS(L.dev(IVP_K_NBR_BUILD, k_ovf_rows, 2 * sms, 256, D));
    CKS(L.dev(IVP_K_NBR_BUILD, k_ovf_pairs, 4 * sms, 256, D));
    {
        int* in = D.fix_cnt;
        int* out = D.fix_off;
        int* bs = D.fix_bsums;
        int n = e->n_total;
        void* a1[] = {&in, &out, &bs, &n};
        CKS(L.kernel(IVP_K_NBR_BUILD, (const void*)k_scan_local, dim3(e->fix_scan_blocks), dim3(SCAN_BLOCK), a1));
        int nb = e->fix_scan_blocks;
        void* a2[] = {&out, &bs, &n, &nb};
        CKS(L.kernel(IVP_K_NBR_BUILD, (const void*)k_scan_add, dim3(e->fix_scan_blocks), dim3(SCAN_BLOCK), a2));
    }
    CKS(L.dev(IVP_K_NBR_BUILD, k_ovf_fill, 4 * sms, 256, D));
    return L.dev(IVP_K_NBR_BUILD, k_ovf_sort, blocks_for(e->n_total, ELEM_BLOCK), ELEM_BLOCK, D);
}

// with_advect: the step's advection runs fused with the key pass
int emit_build_impl(ivp_engine* e, Launcher& L, bool with_advect) {
    const Dev& D = e->D;
    // cell_count is all zero between builds (k_place clears what it used)
    if (with_advect) {
        // ivp_step_io: the advection is the step's first reader of x (and the
        // last writer of x and v), so the upload of x only has to land before
        // it and the downloads can start right after it
        const ivp_engine::StepIO* io = L.io ? &L.io->io : nullptr;
        if (io && io->x_in) {
            if (L.graph) L.extra = L.io_x;
            else CK(cudaStreamWaitEvent(L.stream, L.io->io_ev_x, 0));
        }
        CKS(L.dev(IVP_K_ADVECT, k_advect_keys, blocks_for(std::max(e->n_total, e->n_scenes), ELEM_BLOCK), ELEM_BLOCK,
                  D));
        if (io && (io->x_out || io->v_out)) {
            const size_t off = 3 * (size_t)io->first, bytes = 12 * (size_t)io->count;
            if (L.graph) {
                if (io->x_out) CKS(L.copy(io->x_out, D.x + off, bytes, cudaMemcpyDeviceToHost, true, L.last));
                if (io->v_out) CKS(L.copy(io->v_out, D.v + off, bytes, cudaMemcpyDeviceToHost, true, L.last));
            } else {
                CK(cudaEventRecord(L.io->io_ev_adv, L.stream));
                CK(cudaStreamWaitEvent(L.io->io_side, L.io->io_ev_adv, 0));
                if (io->x_out) CK(cudaMemcpyAsync(io->x_out, D.x + off, bytes, cudaMemcpyDeviceToHost, L.io->io_side));
                if (io->v_out) CK(cudaMemcpyAsync(io->v_out, D.v + off, bytes, cudaMemcpyDeviceToHost, L.io->io_side));
                CK(cudaEventRecord(L.io->io_ev_out, L.io->io_side));
            }
        }
    } else {
        CKS(L.memset0(D.overflow, sizeof(int) * (size_t)e->n_scenes));
        CKS(L.memset0(D.pairs, sizeof(unsigned long long) * (size_t)e->n_scenes));
        CKS(L.memset0(D.seg_ctr, sizeof(int)));
        CKS(L.memset0(D.ovf_ctr, 4 * sizeof(int)));
        CKS(L.memset0(D.fix_fail, sizeof(int) * (size_t)e->n_scenes));
        CKS(L.memset0(D.fix_scene, sizeof(int) * (size_t)e->n_scenes));
        CKS(L.dev(IVP_K_KEYS, k_keys, blocks_for(e->n_total, ELEM_BLOCK), ELEM_BLOCK, D));
    }
    {
        int* in = D.cell_count;
        int* out = D.cell_start;
        int* bs = D.block_sums;
        int n = e->n_keys;
        void* a1[] = {&in, &out, &bs, &n};
        CKS(L.kernel(IVP_K_SCAN_LOCAL, (const void*)k_scan_local, dim3(e->scan_blocks), dim3(SCAN_BLOCK), a1));
        int nb = e->scan_blocks;
        void* a2[] = {&out, &bs, &n, &nb};
        CKS(L.kernel(IVP_K_SCAN_ADD, (const void*)k_scan_add, dim3(e->scan_blocks), dim3(SCAN_BLOCK), a2));
    }
    CKS(L.dev(IVP_K_PLACE, k_place, blocks_for(std::max(e->n_total, e->n_segs), ELEM_BLOCK), ELEM_BLOCK, D));
    CKS(L.dev(IVP_K_ORDER, k_order, blocks_for(e->n_total, ELEM_BLOCK), ELEM_BLOCK, D));
    if (e->n_segs > 0 && e->n_tiles > 0) {
        Dev copy = D;
        cudaGraphConditionalHandle h_fix = 0;
        if (L.graph) {
            // the build sets it when a list was truncated; reset every launch
            CK(cudaGraphConditionalHandleCreate(&h_fix, L.graph, 0, cudaGraphCondAssignDefault));
            copy.h_fix = (unsigned long long)h_fix;
        }
        void* args[] = {&copy};
        if (e->opt.build_kernel == 2) {
            // cell-tiled build: one CTA per segment holding dynamic particles
            // (k_place listed them), one warp per cell
            CKS(L.kernel(IVP_K_NBR_BUILD, (const void*)k_nbr_build<kBuildPP>, dim3(e->n_segs), dim3(256), args,
                         sizeof(float4) * kStageCap));
        } else {
            // one thread per dynamic particle, one CTA per tile
            const int nt = std::max(e->T, 32);
            CKS(L.kernel(IVP_K_NBR_BUILD, (const void*)k_nbr_build_tpp, dim3(e->n_tiles), dim3(nt), args,
                         sizeof(unsigned short) * kTppHits * nt));
        }
        if (L.graph) {
            cudaGraph_t body;
            CKS(add_conditional(L.graph, L, h_fix, cudaGraphCondTypeIf, &body));
            Launcher Lb;
            Lb.graph = body;
            CKS(emit_overflow_fix(e, Lb));
        } else {
            CK(cudaMemcpyAsync(e->h_ovf, D.ovf_ctr, sizeof(int), cudaMemcpyDeviceToHost, L.stream));
            CK(cudaStreamSynchronize(L.stream));
            if (*e->h_ovf > 0) CKS(emit_overflow_fix(e, L));
        }
    }
    return IVP_OK;
}

int emit_build(ivp_engine* e, Launcher& L) { return emit_build_impl(e, L, false); }

int add_conditional(cudaGraph_t g, Launcher& L, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    cudaGraph_t* body) {
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaGraphNode_t n;
    CK(cudaGraphAddNode(&n, g, L.has_last ? &L.last : nullptr, L.has_last ? 1 : 0, &cp));
    *body = cp.conditional.phGraph_out[0];
    L.last = n;
    L.has_last = true;
    return IVP_OK;
}

// The IP outer loop and its CG, either as nested conditional graph nodes
// (device-side control) or driven from the host with flag read-backs.
int emit_solve_loop(ivp_engine* e, Launcher& L) {
    KernelSet K;
    if (!kernel_set(e->G, e->BLOCK, &K)) return IVP_ERR_BAD_ARG;
    const int nt = e->n_tiles, B = e->BLOCK;
    if (nt == 0) return IVP_OK;
    if (!L.graph) {
        // host-driven: one flag read-back after each decision launch
        for (int guard = 0; guard < 1000000; ++guard) {
            CKS(L.dev(IVP_K_PACK, K.pack, nt, B, e->D));
            CK(cudaMemcpyAsync(e->h_flags, e->D.flags, sizeof(Flags), cudaMemcpyDeviceToHost, L.stream));
            CK(cudaStreamSynchronize(L.stream));
            if (!e->h_flags->any_outer) break;
            if (!e->h_flags->any_solve) continue;
            CKS(L.dev(IVP_K_RHS, K.rhs, nt, B, e->D));
            CK(cudaMemcpyAsync(e->h_flags, e->D.flags, sizeof(Flags), cudaMemcpyDeviceToHost, L.stream));
            CK(cudaStreamSynchronize(L.stream));
            for (int cg_guard = 0; e->h_flags->any_cg && cg_guard < 1000000; ++cg_guard) {
                CKS(L.dev(IVP_K_CG_A, K.cg_a, nt, B, e->D));
                CKS(L.dev(IVP_K_CG_B, K.cg_b, nt, B, e->D));
                CK(cudaMemcpyAsync(e->h_flags, e->D.flags, sizeof(Flags), cudaMemcpyDeviceToHost, L.stream));
                CK(cudaStreamSynchronize(L.stream));
            }
        }
        return IVP_OK;
    }
    cudaGraphConditionalHandle h_outer, h_solve, h_cg;
    CK(cudaGraphConditionalHandleCreate(&h_outer, L.graph, 1, cudaGraphCondAssignDefault));
    cudaGraph_t body_outer, body_solve, body_cg;
    CKS(add_conditional(L.graph, L, h_outer, cudaGraphCondTypeWhile, &body_outer));
    CK(cudaGraphConditionalHandleCreate(&h_solve, body_outer, 0, 0));
    Launcher Lo;
    Lo.graph = body_outer;
    {
        Dev d = e->D;
        d.h_outer = (unsigned long long)h_outer;
        d.h_solve = (unsigned long long)h_solve;
        CKS(Lo.dev(IVP_K_PACK, K.pack, nt, B, d));
    }
    CKS(add_conditional(body_outer, Lo, h_solve, cudaGraphCondTypeIf, &body_solve));
    CK(cudaGraphConditionalHandleCreate(&h_cg, body_solve, 0, 0));
    Launcher Ls;
    Ls.graph = body_solve;
    {
        Dev d = e->D;
        d.h_cg = (unsigned long long)h_cg;
        CKS(Ls.dev(IVP_K_RHS, K.rhs, nt, B, d));
    }
    CKS(add_conditional(body_solve, Ls, h_cg, cudaGraphCondTypeWhile, &body_cg));
    Launcher Lc;
    Lc.graph = body_cg;
    {
        Dev d = e->D;
        d.h_cg = (unsigned long long)h_cg;
        CKS(Lc.dev(IVP_K_CG_A, K.cg_a, nt, B, d));
        CKS(Lc.dev(IVP_K_CG_B, K.cg_b, nt, B, d));
    }
    return IVP_OK;
}

bool force_any(const ivp_engine* e, int force) { return force == FORCE_ST ? e->any_st : e->any_visc; }

// PRJ.solve of every PRJ scene (prj.py:296-340): persistent, or one launch
// per pass half with the pass loop as a conditional WHILE node.
int emit_prj(ivp_engine* e, Launcher& L) {
    if (e->n_tiles == 0 || !e->any_prj) return IVP_OK;
    KernelSet K;
    if (!kernel_set(e->G, e->BLOCK, &K)) return IVP_ERR_BAD_ARG;
    const int nt = e->n_tiles, B = e->BLOCK;
    if (e->persistent) {
        CKS(L.memset0(e->D.bar_count, sizeof(unsigned)));
        Dev copy = e->D;
        void* args[] = {&copy};
        return L.kernel(IVP_K_PRJ, (const void*)K.prj_persist, dim3(e->coop_grid_prj), dim3(e->BLOCK), args,
                        e->coop_smem, true);
    }
    CKS(L.dev(IVP_K_PRJ, k_prj_begin, nt, e->T, e->D));
    if (!L.graph) {
        for (int guard = 0; guard < 1000000; ++guard) {
            CKS(L.dev(IVP_K_PRJ, K.pj_head, nt, B, e->D));
            CKS(L.dev(IVP_K_PRJ, K.pj_tail, nt, B, e->D));
            CK(cudaMemcpyAsync(e->h_flags, e->D.flags, sizeof(Flags), cudaMemcpyDeviceToHost, L.stream));
            CK(cudaStreamSynchronize(L.stream));
            if (!e->h_flags->any_outer) break;
        }
    } else {
        cudaGraphConditionalHandle h;
        CK(cudaGraphConditionalHandleCreate(&h, L.graph, 1, cudaGraphCondAssignDefault));
        cudaGraph_t body;
        CKS(add_conditional(L.graph, L, h, cudaGraphCondTypeWhile, &body));
        Launcher Lb;
        Lb.graph = body;
        Dev d = e->D;
        d.h_outer = (unsigned long long)h;
        CKS(Lb.dev(IVP_K_PRJ, K.pj_head, nt, B, d));
        CKS(Lb.dev(IVP_K_PRJ, K.pj_tail, nt, B, d));
    }
    CKS(L.dev(IVP_K_PRJ, k_prj_end, nt, e->T, e->D));
    if (e->want_divergence && e->D.div_out) CKS(L.dev(IVP_K_DIVERGENCE, K.div, nt, B, e->D));
    return IVP_OK;
}

// An implicit non-pressure solve, one launch per phase: Jeske 2023 surface
// tension (force 1, with its divergence pass) or Weiler 2018 viscosity
// (force 0).  The persistent kernel runs the same phases itself.
int emit_force(ivp_engine* e, Launcher& L, int force) {
    if (e->n_tiles == 0 || !force_any(e, force)) return IVP_OK;
    KernelSet K;
    if (!kernel_set(e->G, e->BLOCK, &K)) return IVP_ERR_BAD_ARG;
    const int nt = e->n_tiles, B = e->BLOCK;
    const int kid = force == FORCE_ST ? IVP_K_SURFACE_TENSION : IVP_K_VISC;
    Dev D0 = e->D;
    D0.force = force;
    // slot-ordered {v, 1/rho if fluid} for the setup's neighbour gathers
    CKS(L.dev(kid, k_slot_velocity, blocks_for(e->n_total, ELEM_BLOCK), ELEM_BLOCK, D0));
    CKS(L.dev(kid, k_visc_begin, nt, e->T, D0));
    if (force == FORCE_ST) CKS(L.dev(kid, K.st_div, nt, B, D0));
    if (!L.graph) {
        CKS(L.dev(kid, K.v_setup, nt, B, D0));
        CK(cudaMemcpyAsync(e->h_flags, e->D.flags, sizeof(Flags), cudaMemcpyDeviceToHost, L.stream));
        CK(cudaStreamSynchronize(L.stream));
        for (int guard = 0; e->h_flags->any_visc && guard < 1000000; ++guard) {
            CKS(L.dev(kid, K.v_a, nt, B, D0));
            CKS(L.dev(kid, K.v_b, nt, B, D0));
            CK(cudaMemcpyAsync(e->h_flags, e->D.flags, sizeof(Flags), cudaMemcpyDeviceToHost, L.stream));
            CK(cudaStreamSynchronize(L.stream));
        }
    } else {
        cudaGraphConditionalHandle h;
        CK(cudaGraphConditionalHandleCreate(&h, L.graph, 0, 0));
        Dev d = D0;
        d.h_visc = (unsigned long long)h;
        CKS(L.dev(kid, K.v_setup, nt, B, d));
        cudaGraph_t body;
        CKS(add_conditional(L.graph, L, h, cudaGraphCondTypeWhile, &body));
        Launcher Lb;
        Lb.graph = body;
        CKS(Lb.dev(kid, K.v_a, nt, B, d));
        CKS(Lb.dev(kid, K.v_b, nt, B, d));
    }
    return L.dev(kid, K.v_end, nt, B, D0);
}

int emit_solve(ivp_engine* e, Launcher& L, bool with_visc = false) {
    if (e->n_tiles == 0 || !e->any_ip) return IVP_OK;
    if (e->persistent) {
        KernelSet K;
        kernel_set(e->G, e->BLOCK, &K);
        CKS(L.memset0(e->D.bar_count, sizeof(unsigned)));
        Dev copy = e->D;
        copy.visc_enabled = with_visc ? 1 : 0;
        void* args[] = {&copy};
        return L.kernel(IVP_K_PERSISTENT, (const void*)K.persist, dim3(e->coop_grid), dim3(e->BLOCK), args,
                        e->coop_smem, true);
    }
    CKS(L.dev(IVP_K_SOLVE_BEGIN, k_solve_begin, e->n_tiles, e->T, e->D));
    CKS(emit_solve_loop(e, L));
    CKS(L.dev(IVP_K_SOLVE_END, k_solve_end, e->n_tiles, e->T, e->D));
    if (e->want_divergence && e->D.div_out) {
        KernelSet K;
        kernel_set(e->G, e->BLOCK, &K);
        CKS(L.dev(IVP_K_DIVERGENCE, K.div, e->n_tiles, e->BLOCK, e->D));
    }
    return IVP_OK;
}

int emit_advect(ivp_engine* e, Launcher& L) {
    return L.dev(IVP_K_ADVECT, k_advect, blocks_for(e->n_total, ELEM_BLOCK), ELEM_BLOCK, e->D);
}

int emit_force_persistent(ivp_engine* e, Launcher& L, int force, bool fold_gravity = false) {
    if (e->n_tiles == 0 || !force_any(e, force)) return IVP_OK;
    KernelSet K;
    kernel_set(e->G, e->BLOCK, &K);
    CKS(L.memset0(e->D.bar_count, sizeof(unsigned)));
    Dev copy = e->D;
    copy.force = force;
    copy.fold_gravity = fold_gravity && force == FORCE_VISC ? 1 : 0;
    if (force == FORCE_ST)
        CKS(L.dev(IVP_K_SURFACE_TENSION, k_slot_velocity, blocks_for(e->n_total, ELEM_BLOCK), ELEM_BLOCK, copy));
    void* args[] = {&copy};
    return L.kernel(force == FORCE_ST ? IVP_K_SURFACE_TENSION : IVP_K_VISC,
                    (const void*)(force == FORCE_ST ? K.st_persist : K.v_persist),
                    dim3(force == FORCE_ST ? e->coop_grid_st : e->coop_grid_visc), dim3(e->BLOCK), args, e->coop_smem,
                    true);
}

// Non-pressure forces in the reference's order (framework.py:400-421):
// surface tension, then viscosity.
int emit_forces(ivp_engine* e, Launcher& L) {
    for (int force : {FORCE_ST, FORCE_VISC}) {
        if (e->persistent) CKS(emit_force_persistent(e, L, force));
        else CKS(emit_force(e, L, force));
    }
    return IVP_OK;
}

int emit_step(ivp_engine* e, Launcher& L) {
    // with the viscosity as the step's first force (persistent, no surface
    // tension), its kernel applies gravity in its prologue, which visits every
    // slot before anything reads v
    const bool fold = e->persistent && e->n_tiles > 0 && e->any_visc && !e->any_st;
    if (fold) {
        CKS(emit_force_persistent(e, L, FORCE_VISC, true));
    } else {
        CKS(L.dev(IVP_K_GRAVITY, k_gravity, blocks_for(e->n_total, ELEM_BLOCK), ELEM_BLOCK, e->D));
        CKS(emit_forces(e, L));
    }
    CKS(emit_solve(e, L, true));
    CKS(emit_prj(e, L));
    CKS(emit_build_impl(e, L, true));  // advection (skipping scenes whose solve failed) + the next build
    return IVP_OK;
}

// A step with host input/output (ivp_step_io): v is uploaded before the
// step's first force reads it; x, first read by the advection, is uploaded
// beside the solves; x and v are downloaded beside the next step's build.
int emit_step_io(ivp_engine* e, Launcher& L) {
    const ivp_engine::StepIO& io = e->io;
    const size_t off = 3 * (size_t)io.first, bytes = 12 * (size_t)io.count;
    L.io = e;
    if (L.graph) {
        // x follows v over the bus: v, which the first kernel waits for, gets
        // the whole host-to-device bandwidth
        cudaGraphNode_t v_node = nullptr;
        if (io.v_in) CKS(L.copy(e->D.v + off, io.v_in, bytes, cudaMemcpyHostToDevice, false, nullptr, &v_node));
        if (io.x_in) CKS(L.copy(e->D.x + off, io.x_in, bytes, cudaMemcpyHostToDevice, true, v_node, &L.io_x));
    } else {
        if (io.v_in) CK(cudaMemcpyAsync(e->D.v + off, io.v_in, bytes, cudaMemcpyHostToDevice, L.stream));
        if (io.x_in) {
            CK(cudaEventRecord(e->io_ev_start, L.stream));
            CK(cudaStreamWaitEvent(e->io_side, e->io_ev_start, 0));
            CK(cudaMemcpyAsync(e->D.x + off, io.x_in, bytes, cudaMemcpyHostToDevice, e->io_side));
            CK(cudaEventRecord(e->io_ev_x, e->io_side));
        }
    }
    CKS(emit_step(e, L));
    // the step ends when its downloads have landed
    if (!L.graph && (io.x_out || io.v_out)) CK(cudaStreamWaitEvent(L.stream, e->io_ev_out, 0));
    return IVP_OK;
}

void destroy_graphs(ivp_engine* e) {
    if (e->exec_step_io) cudaGraphExecDestroy(e->exec_step_io);
    if (e->graph_step_io) cudaGraphDestroy(e->graph_step_io);
    e->exec_step_io = nullptr;
    e->graph_step_io = nullptr;
    if (e->exec_step) cudaGraphExecDestroy(e->exec_step);
    if (e->exec_solve) cudaGraphExecDestroy(e->exec_solve);
    if (e->exec_prj) cudaGraphExecDestroy(e->exec_prj);
    if (e->graph_prj) cudaGraphDestroy(e->graph_prj);
    e->exec_prj = nullptr;
    e->graph_prj = nullptr;
    if (e->exec_build) cudaGraphExecDestroy(e->exec_build);
    if (e->graph_step) cudaGraphDestroy(e->graph_step);
    if (e->graph_solve) cudaGraphDestroy(e->graph_solve);
    if (e->graph_build) cudaGraphDestroy(e->graph_build);
    e->exec_step = e->exec_solve = e->exec_build = nullptr;
    e->graph_step = e->graph_solve = e->graph_build = nullptr;
}

typedef int (*Emitter)(ivp_engine*, Launcher&);

int make_graph(ivp_engine* e, Emitter emit, cudaGraph_t* g, cudaGraphExec_t* x) {
    CK(cudaGraphCreate(g, 0));
    Launcher L;
    L.graph = *g;
    int st = emit(e, L);
    if (st != IVP_OK) return st;
    CK(cudaGraphInstantiate(x, *g, 0));
    return IVP_OK;
}

int run(ivp_engine* e, Emitter emit, cudaGraph_t* g, cudaGraphExec_t* x, cudaStream_t s) {
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    if (e->opt.use_graphs) {
        if (!*x) CKS(make_graph(e, emit, g, x));
        CK(cudaGraphLaunch(*x, s));
        return IVP_OK;
    }
    Launcher L;
    L.stream = s;
    return emit(e, L);
}

// Lane count 0: 4 lanes x 64 particles per tile while the dynamic particles
// fill at most kAutoTilesPerSM tiles of 64 per SM, else 2 lanes x 128.  With
// many tiles per CTA the persistent solves walk fewer, larger tiles per phase
// (one block reduction per tile); with few, 4 lanes split each row wider.
constexpr long kAutoTilesPerSM = 16;
// The thread-per-particle build lasts about one thread's walk of its 27-cell
// window, so it needs many particles per SM to hide its load latency; below
// this many dynamic particles per SM the warp-per-cell build (a warp tests a
// cell's candidates in parallel) is faster (8,192 particles: 0.08 against
// 0.03 ms; 102,400: 0.117 against 0.129 ms).
constexpr long kTppMinPerSM = 256;

int resolve_options(const ivp_scene_desc* sc, int n, const ivp_options* in, ivp_options* out) {
    if (!in || !out) return IVP_ERR_BAD_ARG;
    *out = *in;
    if (in->lanes_per_particle == 0 || in->build_kernel == 0) {
        if (n <= 0 || !sc) return IVP_ERR_BAD_ARG;
        long tiles = 0, dyn = 0;
        for (int s = 0; s < n; ++s)
            if (sc[s].n_dynamic > 0) {
                tiles += ((long)sc[s].n_dynamic + 63) / 64;
                dyn += sc[s].n_dynamic;
            }
        int dev = 0, sms = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
            cudaGetLastError();  // no device here: size for a B200
            sms = 148;
        }
        if (in->lanes_per_particle == 0) out->lanes_per_particle = tiles > kAutoTilesPerSM * sms ? 2 : 4;
        if (in->build_kernel == 0) out->build_kernel = dyn >= kTppMinPerSM * sms ? 1 : 2;
    }
    if (in->particles_per_block == 0 && out->lanes_per_particle > 0)
        out->particles_per_block = 256 / out->lanes_per_particle;
    return IVP_OK;
}

int validate(const ivp_scene_desc* sc, int n, const ivp_options* o) {
    if (n <= 0 || !sc || !o) return IVP_ERR_BAD_ARG;
    if (o->lanes_per_particle != 1 && o->lanes_per_particle != 2 && o->lanes_per_particle != 4 &&
        o->lanes_per_particle != 8)
        return IVP_ERR_BAD_ARG;
    {
        KernelSet K;
        if (o->particles_per_block <= 0 || !kernel_set(o->lanes_per_particle, o->particles_per_block * o->lanes_per_particle, &K))
            return IVP_ERR_BAD_ARG;
    }
    if (o->list_stride <= 0 || (o->list_stride & 1) || o->max_hist <= 0) return IVP_ERR_BAD_ARG;
    if (o->row_format < 0 || o->row_format > 3) return IVP_ERR_BAD_ARG;
    if (o->build_kernel < 0 || o->build_kernel > 2) return IVP_ERR_BAD_ARG;
    long expect = 0;
    for (int s = 0; s < n; ++s) {
        const ivp_scene_desc& d = sc[s];
        // scenes tile the particle arrays in order, without gaps
        if (d.particle_offset != expect) return IVP_ERR_BAD_ARG;
        expect += d.n_particles;
        if (expect > 0x7fffffffL) return IVP_ERR_BAD_ARG;
        if (d.n_particles < 0 || d.n_dynamic < 0 || d.n_dynamic > d.n_particles) return IVP_ERR_BAD_ARG;
        if (!(d.particle_radius > 0.0f) || !(d.dt > 0.0f)) return IVP_ERR_BAD_ARG;
        if (d.cache_size <= 0 || d.cache_size > o->list_stride) return IVP_ERR_BAD_ARG;
        for (int a = 0; a < 3; ++a)
            if (!(d.domain_size[a] > 0.0f)) return IVP_ERR_BAD_ARG;
        if (d.max_outer_iters < 0 || d.max_iteration_pcg < 0) return IVP_ERR_BAD_ARG;
    }
    return IVP_OK;
}

bool scene_st(const ivp_scene_desc& d) {
    return d.surface_tension_method == 1 && d.surface_tension_coeff > 0.0f && d.n_dynamic > 0;
}

struct Plan {
    std::vector<SceneParams> hp;
    std::vector<int4> tiles;
    std::vector<int4> segs;
    int n_total = 0, n_dyn = 0, n_keys = 0, scan_blocks = 0;
    int row_fmt = 0;       // ROW_FULL (16 B entries), ROW_COMPACT ({j, w}, 8 B), ROW_BF16 (4 B id + 6 B)
    bool any_st = false;   // some scene runs the implicit surface tension
    int drop_cap = 0;      // dropped-pair records of the overflow fix-up
    int fix_scan_blocks = 0;
    size_t off[73];
    Layout lay;
};

// Dropped-pair records: two per dynamic particle plus this floor.  A build
// that drops more pairs stops the affected scenes' IP solves with
// IVP_ERR_NBR_OVERFLOW rather than solve with an uncorrected operator.
constexpr int kDropFloor = 65536;

void plan(const ivp_scene_desc* sc, int n, const ivp_options* o, Plan& P) {
    const int T = o->particles_per_block;
    int s_begin = 0, row_base = 0, key_base = 0;
    P.hp.resize(n);
    for (int s = 0; s < n; ++s) {
        const ivp_scene_desc& d = sc[s];
        SceneParams& q = P.hp[s];
        memset(&q, 0, sizeof(q));
        q.p_begin = d.particle_offset;
        q.p_end = d.particle_offset + d.n_particles;
        q.s_begin = s_begin;
        q.s_dyn_end = s_begin + d.n_dynamic;
        q.s_end = s_begin + d.n_particles;
        q.n_dyn = d.n_dynamic;
        q.row_base = row_base;
        const float h = 4.0f * d.particle_radius;  // config_builder.py:51-52
        q.h = h;
        q.cell_inv = 1.0f / h;
        q.inv_h = 1.0f / h;
        {
            // largest float d2 with sqrtf(d2) < h (IEEE sqrt is monotone and
            // correctly rounded on host and device alike)
            float t = h * h;
            while (std::sqrt(t) >= h) t = std::nextafter(t, 0.0f);
            while (std::sqrt(std::nextafter(t, INFINITY)) < h) t = std::nextafter(t, INFINITY);
            q.r2_max = t;
        }
        long ncell = 1;
        for (int a = 0; a < 3; ++a) {
            // neighbour_search.py:105-107
            int dim = (int)std::ceil((double)d.domain_size[a] / (double)h);
            q.dims[a] = dim < 1 ? 1 : dim;
            ncell *= q.dims[a];
            q.domain[a] = d.domain_size[a];
            q.gravity[a] = d.gravity[a];
        }
        q.ncell = (int)ncell;
        q.key_base = key_base;
        q.dt = d.dt;
        q.inv_dt = (float)(1.0 / (double)d.dt);
        q.omega = d.omega;
        q.padding = h;
        float k = 8.0f / 3.14159265359f;
        k = k / (h * h * h);
        q.cubic_k = k;
        q.W0 = k * (6.0f * 0.0f - 6.0f * 0.0f + 1.0f);
        q.spiky_k = 45.0f / (3.14159265359f * h * h * h * h * h * h);
        q.visc_coeff = d.viscosity_coeff;
        q.visc_method = d.viscosity_method;
        q.st_coeff = d.surface_tension_coeff;
        q.st_method = d.surface_tension_method;
        q.st_d = 2.0f * d.particle_radius;  // jeske23.py:454-455
        q.st_h = 2.0f * q.st_d;
        q.solver = d.pressure_solver == IVP_SOLVER_PRJ ? SOLVER_PRJ : SOLVER_IP;
        q.max_outer = d.max_outer_iters;
        q.max_pcg = d.max_iteration_pcg;
        q.fixed_iters = d.fixed_outer_iters;
        q.cache = d.cache_size;
        q.tol_opt = d.density_error_tol;
        q.tol_pcg = d.tol_pcg;
        q.hist_base = s * o->max_hist;
        q.tile_begin = (int)P.tiles.size();
        for (int b = 0; b < d.n_dynamic; b += T) {
            int e = std::min(b + T, d.n_dynamic);
            P.tiles.push_back(make_int4(s, s_begin + b, s_begin + e, row_base + b));
        }
        q.tile_end = (int)P.tiles.size();
        if (d.n_dynamic > 0)
            for (int cz = 0; cz < q.dims[2]; ++cz)
                for (int cy = 0; cy < q.dims[1]; ++cy)
                    for (int x = 0; x < q.dims[0]; x += kSegW) P.segs.push_back(make_int4(s, cy, cz, x));
        s_begin += d.n_particles;
        row_base += d.n_dynamic;
        key_base += 2 * (int)ncell;
    }
    P.n_total = s_begin;
    P.n_dyn = row_base;
    // compact rows halve the list memory; they cost one more gather per
    // pair, which outweighs the halved list stream on B200, so the default
    // is full rows.  bf16 rows (10 B per entry) are the reduced-precision
    // variant of the gradient.
    P.row_fmt = o->row_format == 2 ? ROW_COMPACT : o->row_format == 3 ? ROW_BF16 : ROW_FULL;
    for (int s = 0; s < n; ++s)
        if (scene_st(sc[s])) P.any_st = true;
    P.n_keys = key_base;
    P.scan_blocks = std::max(1, (P.n_keys + SCAN_TILE - 1) / SCAN_TILE);
    const size_t N = (size_t)P.n_total, S = (size_t)n, NT = std::max<size_t>(P.tiles.size(), 1);
    Layout& L = P.lay;
    int i = 0;
    P.off[i++] = L.add(sizeof(SceneParams) * S);            // 0 scenes
    P.off[i++] = L.add(sizeof(SceneCtl) * S);               // 1 ctl
    P.off[i++] = L.add(sizeof(int4) * NT);                  // 2 tiles
    P.off[i++] = L.add(sizeof(int) * N);                    // 3 pscene
    P.off[i++] = L.add(sizeof(int) * N);                    // 4 key
    P.off[i++] = L.add(sizeof(int) * N);                    // 5 rank
    P.off[i++] = L.add(sizeof(int) * (size_t)P.n_keys);     // 6 cell_count
    P.off[i++] = L.add(sizeof(int) * ((size_t)P.n_keys + 1));  // 7 cell_start
    P.off[i++] = L.add(sizeof(int) * (size_t)P.scan_blocks);   // 8 block_sums
    P.off[i++] = L.add(sizeof(int) * N);                    // 9 placed
    P.off[i++] = L.add(sizeof(int) * N);                    // 10 pid
    P.off[i++] = L.add(sizeof(int) * N);                    // 11 inv
    P.off[i++] = L.add(sizeof(int) * S);                    // 12 overflow
    P.off[i++] = L.add(sizeof(float4) * N);                 // 13 xm
    P.off[i++] = L.add(sizeof(float) * N);                  // 14 rho0s
    P.off[i++] = L.add(sizeof(float) * N);                  // 15 dens
    P.off[i++] = L.add(sizeof(float) * N);                  // 16 kd
    P.off[i++] = L.add(sizeof(float) * N);                  // 17 c
    P.off[i++] = L.add(sizeof(float4) * N);                 // 18 d0
    P.off[i++] = L.add(sizeof(float4) * N);                 // 19 d1
    P.off[i++] = L.add(sizeof(float4) * N);                 // 20 sol
    P.off[i++] = L.add(sizeof(float4) * N);                 // 21 r
    P.off[i++] = L.add(2 * sizeof(float4) * N);             // 22 cg0
    P.off[i++] = L.add(2 * sizeof(float4) * N);             // 23 cg1
    P.off[i++] = L.add(sizeof(float) * N);                  // 24 y
    P.off[i++] = L.add(sizeof(float) * N);                  // 25 s
    P.off[i++] = L.add(sizeof(float) * N);                  // 26 fk
    const size_t entry_bytes = P.row_fmt == ROW_FULL ? sizeof(float4) : P.row_fmt == ROW_COMPACT ? sizeof(float2) : sizeof(int);
    P.off[i++] = L.add(entry_bytes * (size_t)P.n_dyn * (size_t)o->list_stride);  // 27 nbr (ids for bf16 rows)
    P.off[i++] = L.add(sizeof(int) * std::max<size_t>((size_t)P.n_dyn, 1));       // 28 nbr_cnt
    P.off[i++] = L.add(4 * sizeof(double) * NT);            // 29 partial (two per tile, two phase buffers)
    P.off[i++] = L.add(sizeof(int) * S);                    // 30 scene_counter
    P.off[i++] = L.add(sizeof(int));                        // 31 launch_counter
    P.off[i++] = L.add(sizeof(Flags));                      // 32 flags
    P.off[i++] = L.add(sizeof(double) * S * (size_t)o->max_hist);  // 33 err_hist
    P.off[i++] = L.add(sizeof(int) * S * (size_t)o->max_hist);     // 34 pcg_hist
    P.off[i++] = L.add(sizeof(unsigned long long) * S);            // 35 pairs
    P.off[i++] = L.add(2 * sizeof(unsigned));                        // 36 barrier words
    P.off[i++] = L.add(sizeof(float) * N);                           // 37 inv_m
    P.off[i++] = L.add(sizeof(float) * N);                           // 38 q
    P.off[i++] = L.add(sizeof(float) * N);                           // 39 z
    P.off[i++] = L.add(sizeof(float) * N);                           // 40 rflu
    P.off[i++] = L.add(sizeof(float4) * N);                          // 41 vs
    P.off[i++] = L.add(sizeof(float4) * N);                          // 42 vap
    P.off[i++] = L.add(3 * sizeof(float4) * N);                      // 43 pinv
    P.off[i++] = L.add(sizeof(int4) * std::max<size_t>(P.segs.size(), 1));  // 44 segs
    P.off[i++] = L.add(P.any_st ? sizeof(float2) * (size_t)P.n_dyn * (size_t)o->list_stride : 0);  // 45 st_w
    P.off[i++] = L.add(P.any_st ? 2 * sizeof(float4) * N : 0);       // 46 st_rec
    P.off[i++] = L.add(P.any_st ? sizeof(float) * N : 0);            // 47 st_inv
    P.off[i++] = L.add(P.row_fmt == ROW_BF16 ? 3 * sizeof(unsigned short) * (size_t)P.n_dyn * (size_t)o->list_stride
                                             : 0);                   // 48 bf16 gradients
    P.off[i++] = L.add(sizeof(int) * std::max<size_t>(P.segs.size(), 1));  // 49 live_segs
    P.off[i++] = L.add(sizeof(int));                                         // 50 seg_ctr (live segment count)
    P.off[i++] = L.add(sizeof(float4) * N);                                  // 51 e = d - sol
    // neighbour-cache overflow fix-up
    P.drop_cap = 2 * std::max(P.n_dyn, 1) + kDropFloor;
    P.fix_scan_blocks = std::max(1, (P.n_total + SCAN_TILE - 1) / SCAN_TILE);
    P.off[i++] = L.add(sizeof(int) * std::max<size_t>((size_t)P.n_dyn, 1));   // 52 ovf_list
    P.off[i++] = L.add(4 * sizeof(int));                                       // 53 ovf_ctr
    P.off[i++] = L.add(sizeof(int2) * (size_t)P.drop_cap);                     // 54 drop
    P.off[i++] = L.add(sizeof(float4) * (size_t)P.drop_cap);                   // 55 drop_w
    P.off[i++] = L.add(sizeof(int) * N);                                       // 56 fix_cnt
    P.off[i++] = L.add(sizeof(int) * (N + 1));                                 // 57 fix_off
    P.off[i++] = L.add(sizeof(int) * (size_t)P.fix_scan_blocks);               // 58 fix_bsums
    P.off[i++] = L.add(2 * sizeof(float4) * (size_t)P.drop_cap);               // 59 fix_w
    P.off[i++] = L.add(sizeof(int) * S);                                       // 60 fix_fail
    P.off[i++] = L.add(sizeof(int) * S);                                       // 61 fix_scene
    P.off[i++] = L.add(sizeof(float4) * N);                                    // 62 rip
    P.off[i++] = L.add(sizeof(float4) * N);                                    // 63 pip
    P.off[i++] = L.add(sizeof(float) * N);                                     // 64 jp
    P.off[i++] = L.add(sizeof(float4) * N);                                    // 65 vpp
    P.off[i++] = L.add(sizeof(float4) * N);                                    // 66 vlp
    P.off[i++] = L.add(P.any_st ? sizeof(float4) * N : 0);                     // 67 stz
    P.off[i++] = L.add(StatStage(o->max_hist).total);                          // 68 stage
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Reading a scene's solve statistics: the copies into the engine's pinned
// mirrors are enqueued on the caller's stream, the caller synchronises once,
// then the fill functions convert.
// One scene's statistics and histories (the whole history rows, max_hist
// entries each) in one device-to-host copy after a gather kernel, instead of
// one copy per array; unpack_stage places them in the host mirrors.
int enqueue_stage(ivp_engine* e, int scene, cudaStream_t s) {
    const int H = e->opt.max_hist;
    k_stage_stats<<<1, 256, 0, s>>>(e->D, scene, H);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(e->h_stage, e->D.stage, StatStage(H).total, cudaMemcpyDeviceToHost, s));
    return IVP_OK;
}

void unpack_stage(ivp_engine* e, int scene) {
    const int H = e->opt.max_hist;
    const StatStage L(H);
    const unsigned char* b = e->h_stage;
    memcpy(e->h_ctl + scene, b + L.ctl, sizeof(SceneCtl));
    memcpy(e->h_overflow + scene, b + L.ovf, sizeof(int));
    memcpy(e->h_flags, b + L.flags, sizeof(Flags));
    memcpy(e->h_pairs + scene, b + L.pairs, sizeof(unsigned long long));
    memcpy(e->h_fix_scene + scene, b + L.fix, sizeof(int));
    memcpy(e->h_err, b + L.err, sizeof(double) * (size_t)H);
    memcpy(e->h_pcg, b + L.pcg, sizeof(int) * (size_t)H);
}

int fill_stats(ivp_engine* e, int scene, ivp_solve_stats* out) {
    const SceneCtl& C = e->h_ctl[scene];
    memset(out, 0, sizeof(*out));
    out->status = C.status;
    out->outer_iters = C.outer_it;
    out->n_density_errors = C.n_err;
    out->overflow_particles = e->h_overflow[scene];
    out->final_density_error = C.final_err;
    out->last_density_error = C.err;
    out->total_pcg_iters = C.total_cg;
    out->solves = C.acc_solves;
    out->failed_solves = C.acc_failed;
    out->last_failure = C.acc_last_failure;
    out->sum_outer_iters = C.acc_outer;
    out->sum_pcg_iters = C.acc_cg;
    out->max_final_density_error = C.acc_max_final_err;
    out->neighbour_pairs = (int64_t)e->h_pairs[scene];
    out->sum_visc_iters = C.acc_visc;
    out->sum_st_iters = C.acc_st;
    out->last_pap = C.pap;
    out->last_cg_iter = C.cg_it;
    out->fixup_entries = e->h_fix_scene[scene];
    if (C.status == IVP_ERR_NBR_OVERFLOW)
        g_err = "truncated neighbour lists dropped more pairs than the engine's correction storage holds";
    if (e->h_flags->timeout) {
        g_err = "a solve exceeded its iteration budget or a grid barrier timed out";
        out->status = IVP_ERR_TIMEOUT;
    }
    if (e->h_flags->bad) {
        char buf[128];
        snprintf(buf, sizeof(buf), "device bounds check failed: index %d at site %d", e->h_flags->bad_index,
                 e->h_flags->bad_where);
        g_err = buf;
        return IVP_ERR_DEVICE_CHECK;
    }
    return IVP_OK;
}

// first n_err errors and outer_it CG counts of the control block in h_ctl
void fill_history(ivp_engine* e, int scene, double* errors, int32_t* pcg_iters, int cap, int32_t* n_errors,
                  int32_t* n_pcg) {
    const SceneCtl& C = e->h_ctl[scene];
    const int H = e->opt.max_hist;
    const int ne = std::min(std::min(C.n_err, H), cap);
    const int np = std::min(std::min(C.outer_it, H), cap);
    if (errors && ne > 0) memcpy(errors, e->h_err, sizeof(double) * ne);
    if (pcg_iters && np > 0) memcpy(pcg_iters, e->h_pcg, sizeof(int) * np);
    if (n_errors) *n_errors = ne;
    if (n_pcg) *n_pcg = np;
}

}  // namespace

// ================================================================ C ABI

extern "C" {

void ivp_default_options(ivp_options* o) {
    memset(o, 0, sizeof(*o));
    o->lanes_per_particle = 0;  // chosen from the scenes
    o->particles_per_block = 0;
    o->list_stride = 64;
    o->max_hist = kMaxHistDefault;
    o->use_graphs = 1;
}

int ivp_resolve_options(const ivp_scene_desc* scenes, int32_t n_scenes, const ivp_options* opt, ivp_options* out) {
    return resolve_options(scenes, n_scenes, opt, out);
}

int ivp_workspace_bytes(const ivp_scene_desc* scenes, int32_t n_scenes, const ivp_options* opt_in, size_t* bytes) {
    ivp_options ro;
    CKS(resolve_options(scenes, n_scenes, opt_in, &ro));
    const ivp_options* opt = &ro;
    CKS(validate(scenes, n_scenes, opt));
    if (!bytes) return IVP_ERR_BAD_ARG;
    Plan P;
    plan(scenes, n_scenes, opt, P);
    *bytes = P.lay.total;
    return IVP_OK;
}

int ivp_engine_create(const ivp_scene_desc* scenes, int32_t n_scenes, const ivp_options* opt_in, void* workspace,
                      size_t workspace_bytes, void* stream, ivp_engine** out) {
    if (!out || !workspace) return IVP_ERR_BAD_ARG;
    *out = nullptr;
    ivp_options ro;
    CKS(resolve_options(scenes, n_scenes, opt_in, &ro));
    const ivp_options* opt = &ro;
    CKS(validate(scenes, n_scenes, opt));
    if (reinterpret_cast<uintptr_t>(workspace) & 255) return IVP_ERR_BAD_ARG;
    Plan P;
    plan(scenes, n_scenes, opt, P);
    if (workspace_bytes < P.lay.total) return IVP_ERR_BAD_ARG;
    cudaStream_t s = as_stream(stream);
    ivp_engine* e = new ivp_engine();
    e->desc.assign(scenes, scenes + n_scenes);
    e->hp = P.hp;
    e->tiles = P.tiles;
    e->opt = *opt;
    e->G = opt->lanes_per_particle;
    e->T = opt->particles_per_block;
    e->BLOCK = e->G * e->T;
    e->n_total = P.n_total;
    e->n_dyn_total = P.n_dyn;
    e->n_keys = P.n_keys;
    e->n_tiles = (int)P.tiles.size();
    e->scan_blocks = P.scan_blocks;
    e->n_scenes = n_scenes;
    for (int sc = 0; sc < n_scenes; ++sc)
    {
        if (scenes[sc].viscosity_method == 1 && scenes[sc].viscosity_coeff > 0.0f && scenes[sc].n_dynamic > 0)
            e->any_visc = true;
        if (scene_st(scenes[sc])) e->any_st = true;
        if (scenes[sc].pressure_solver == IVP_SOLVER_PRJ) e->any_prj = true;
        else e->any_ip = true;
    }
    char* w = static_cast<char*>(workspace);
    Dev& D = e->D;
    int i = 0;
    D.scenes = reinterpret_cast<SceneParams*>(w + P.off[i++]);
    D.ctl = reinterpret_cast<SceneCtl*>(w + P.off[i++]);
    D.tiles = reinterpret_cast<int4*>(w + P.off[i++]);
    D.pscene = reinterpret_cast<int*>(w + P.off[i++]);
    D.key = reinterpret_cast<int*>(w + P.off[i++]);
    D.rank = reinterpret_cast<int*>(w + P.off[i++]);
    D.cell_count = reinterpret_cast<int*>(w + P.off[i++]);
    D.cell_start = reinterpret_cast<int*>(w + P.off[i++]);
    D.block_sums = reinterpret_cast<int*>(w + P.off[i++]);
    D.placed = reinterpret_cast<int*>(w + P.off[i++]);
    D.pid = reinterpret_cast<int*>(w + P.off[i++]);
    D.inv = reinterpret_cast<int*>(w + P.off[i++]);
    D.overflow = reinterpret_cast<int*>(w + P.off[i++]);
    D.xm = reinterpret_cast<float4*>(w + P.off[i++]);
    D.rho0s = reinterpret_cast<float*>(w + P.off[i++]);
    D.dens = reinterpret_cast<float*>(w + P.off[i++]);
    D.kd = reinterpret_cast<float*>(w + P.off[i++]);
    D.c = reinterpret_cast<float*>(w + P.off[i++]);
    D.d0 = reinterpret_cast<float4*>(w + P.off[i++]);
    D.d1 = reinterpret_cast<float4*>(w + P.off[i++]);
    D.sol = reinterpret_cast<float4*>(w + P.off[i++]);
    D.r = reinterpret_cast<float4*>(w + P.off[i++]);
    D.cg0 = reinterpret_cast<float4*>(w + P.off[i++]);
    D.cg1 = reinterpret_cast<float4*>(w + P.off[i++]);
    D.y = reinterpret_cast<float*>(w + P.off[i++]);
    D.s = reinterpret_cast<float*>(w + P.off[i++]);
    D.fk = reinterpret_cast<float*>(w + P.off[i++]);
    D.nbr = reinterpret_cast<float4*>(w + P.off[i++]);
    D.nbr_cnt = reinterpret_cast<int*>(w + P.off[i++]);
    D.partial = reinterpret_cast<double*>(w + P.off[i++]);
    D.scene_counter = reinterpret_cast<int*>(w + P.off[i++]);
    D.launch_counter = reinterpret_cast<int*>(w + P.off[i++]);
    D.flags = reinterpret_cast<Flags*>(w + P.off[i++]);
    D.err_hist = reinterpret_cast<double*>(w + P.off[i++]);
    D.pcg_hist = reinterpret_cast<int*>(w + P.off[i++]);
    D.pairs = reinterpret_cast<unsigned long long*>(w + P.off[i++]);
    D.bar_count = reinterpret_cast<unsigned*>(w + P.off[i]);
    D.bar_gen = reinterpret_cast<unsigned*>(w + P.off[i++]) + 1;
    D.inv_m = reinterpret_cast<float*>(w + P.off[i++]);
    D.q = reinterpret_cast<float*>(w + P.off[i++]);
    D.z = reinterpret_cast<float*>(w + P.off[i++]);
    D.rflu = reinterpret_cast<float*>(w + P.off[i++]);
    D.vs = reinterpret_cast<float4*>(w + P.off[i++]);
    D.vap = reinterpret_cast<float4*>(w + P.off[i++]);
    D.pinv = reinterpret_cast<float4*>(w + P.off[i++]);
    D.segs = reinterpret_cast<int4*>(w + P.off[i++]);
    D.st_w = reinterpret_cast<float2*>(w + P.off[i++]);
    D.st_rec = reinterpret_cast<float4*>(w + P.off[i++]);
    D.st_inv = reinterpret_cast<float*>(w + P.off[i++]);
    D.nbr_g = reinterpret_cast<unsigned short*>(w + P.off[i++]);
    D.live_segs = reinterpret_cast<int*>(w + P.off[i++]);
    D.seg_ctr = reinterpret_cast<int*>(w + P.off[i++]);
    D.e = reinterpret_cast<float4*>(w + P.off[i++]);
    D.ovf_list = reinterpret_cast<int*>(w + P.off[i++]);
    D.ovf_ctr = reinterpret_cast<int*>(w + P.off[i++]);
    D.drop = reinterpret_cast<int2*>(w + P.off[i++]);
    D.drop_w = reinterpret_cast<float4*>(w + P.off[i++]);
    D.fix_cnt = reinterpret_cast<int*>(w + P.off[i++]);
    D.fix_off = reinterpret_cast<int*>(w + P.off[i++]);
    D.fix_bsums = reinterpret_cast<int*>(w + P.off[i++]);
    D.fix_w = reinterpret_cast<float4*>(w + P.off[i++]);
    D.fix_fail = reinterpret_cast<int*>(w + P.off[i++]);
    D.fix_scene = reinterpret_cast<int*>(w + P.off[i++]);
    D.rip = reinterpret_cast<float4*>(w + P.off[i++]);
    D.pip = reinterpret_cast<float4*>(w + P.off[i++]);
    D.jp = reinterpret_cast<float*>(w + P.off[i++]);
    D.vpp = reinterpret_cast<float4*>(w + P.off[i++]);
    D.vlp = reinterpret_cast<float4*>(w + P.off[i++]);
    D.stz = reinterpret_cast<float4*>(w + P.off[i++]);
    D.stage = reinterpret_cast<unsigned char*>(w + P.off[i++]);
    D.drop_cap = P.drop_cap;
    e->fix_scan_blocks = P.fix_scan_blocks;
    D.n_segs = (int)P.segs.size();
    e->n_segs = D.n_segs;
    {
        long long lim = 64;
        for (int sc = 0; sc < n_scenes; ++sc)
            lim += (long long)(scenes[sc].max_outer_iters + 1) * (long long)(2 * scenes[sc].max_iteration_pcg + 3) +
                   2 * 1000 + 4;
        D.phase_limit = lim;
    }
    D.bar_limit_ns = kBarrierLimitNs;
    D.n_scenes = n_scenes;
    D.n_tiles = e->n_tiles;
    D.n_keys = e->n_keys;
    D.stride = opt->list_stride;
    D.row_fmt = P.row_fmt;
    {
        // rows hold about half their stride in use; beyond the L2 they
        // stream from DRAM in every pass of the solves
        int dev = 0, l2 = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) != cudaSuccess) {
            cudaGetLastError();
            l2 = 126 << 20;
        }
        const double row_bytes = (double)e->n_dyn_total * opt->list_stride / 2 * 16.0;
        D.row_stream = (P.row_fmt == ROW_FULL && row_bytes > (double)l2) ? 1 : 0;
    }
    // few partials: every CTA of the persistent solve sums them itself
    // (2 x 8 B x tiles read per CTA per phase) instead of waiting for the
    // last CTA's decisions to travel back
    D.bar_all_reduce = (n_scenes <= 2 && (int)P.tiles.size() <= 4096) ? 1 : 0;
    D.hist_len = opt->max_hist;
    D.n_total = e->n_total;

    auto fail = [&](int code) {
        ivp_engine_destroy(e);
        return code;
    };
    if (cudaMemsetAsync(workspace, 0, P.lay.total, s) != cudaSuccess) return fail(IVP_ERR_CUDA);
    std::vector<int> pscene(e->n_total);
    for (int sc = 0; sc < n_scenes; ++sc)
        for (int p = P.hp[sc].p_begin; p < P.hp[sc].p_end; ++p) {
            if (p < 0 || p >= e->n_total) return fail(IVP_ERR_BAD_ARG);
            pscene[p] = sc;
        }
    if (cudaHostAlloc((void**)&e->h_ctl, sizeof(SceneCtl) * n_scenes, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&e->h_flags, sizeof(Flags), cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&e->h_overflow, sizeof(int) * n_scenes, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&e->h_pairs, sizeof(unsigned long long) * n_scenes, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&e->h_err, sizeof(double) * opt->max_hist, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&e->h_pcg, sizeof(int) * opt->max_hist, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&e->h_ovf, sizeof(int), cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&e->h_fix_scene, sizeof(int) * n_scenes, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&e->h_stage, StatStage(opt->max_hist).total, cudaHostAllocDefault) != cudaSuccess)
        return fail(IVP_ERR_CUDA);
    if (cudaMemcpyAsync((void*)D.scenes, P.hp.data(), sizeof(SceneParams) * n_scenes, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        (e->n_tiles && cudaMemcpyAsync((void*)D.tiles, P.tiles.data(), sizeof(int4) * e->n_tiles,
                                       cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        (e->n_total && cudaMemcpyAsync((void*)D.pscene, pscene.data(), sizeof(int) * e->n_total,
                                       cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        (e->n_segs && cudaMemcpyAsync((void*)D.segs, P.segs.data(), sizeof(int4) * e->n_segs,
                                      cudaMemcpyHostToDevice, s) != cudaSuccess))
        return fail(IVP_ERR_CUDA);
    // the host vectors go out of scope: make the copies complete first
    if (cudaStreamSynchronize(s) != cudaSuccess) return fail(IVP_ERR_CUDA);
    // persistent solve: a co-resident grid of at most one CTA per tile
    e->persistent = false;
    if (opt->persistent && e->n_tiles > 0 && n_scenes <= 256) {
        int dev = 0, coop = 0, nsm = 0, per_sm = 0;
        KernelSet K;
        kernel_set(e->G, e->BLOCK, &K);
        e->coop_smem = (size_t)n_scenes * (2 * sizeof(double) + sizeof(SceneCtl) + 3 * sizeof(int)) + sizeof(int);
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && coop &&
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)K.persist, e->BLOCK, e->coop_smem) ==
                cudaSuccess &&
            per_sm > 0) {
            int per_sm_v = 0, per_sm_s = 0, per_sm_p = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_v, (const void*)K.v_persist, e->BLOCK,
                                                              e->coop_smem) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_s, (const void*)K.st_persist, e->BLOCK,
                                                              e->coop_smem) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_p, (const void*)K.prj_persist, e->BLOCK,
                                                              e->coop_smem) == cudaSuccess &&
                per_sm_v > 0 && per_sm_s > 0 && per_sm_p > 0) {
                e->coop_grid = std::min(e->n_tiles, per_sm * nsm);
                e->coop_grid_visc = std::min(e->n_tiles, per_sm_v * nsm);
                e->coop_grid_st = std::min(e->n_tiles, per_sm_s * nsm);
                e->coop_grid_prj = std::min(e->n_tiles, per_sm_p * nsm);
                e->persistent = true;
            }
        }
    }
    *out = e;
    return IVP_OK;
}

int ivp_engine_destroy(ivp_engine* e) {
    if (!e) return IVP_OK;
    destroy_graphs(e);
    if (e->io_side) {
        cudaStreamSynchronize(e->io_side);
        cudaStreamDestroy(e->io_side);
        cudaEventDestroy(e->io_ev_start);
        cudaEventDestroy(e->io_ev_x);
        cudaEventDestroy(e->io_ev_adv);
        cudaEventDestroy(e->io_ev_out);
    }
    if (e->h_ctl) cudaFreeHost(e->h_ctl);
    if (e->h_flags) cudaFreeHost(e->h_flags);
    if (e->h_overflow) cudaFreeHost(e->h_overflow);
    if (e->h_pairs) cudaFreeHost(e->h_pairs);
    if (e->h_err) cudaFreeHost(e->h_err);
    if (e->h_pcg) cudaFreeHost(e->h_pcg);
    if (e->h_ovf) cudaFreeHost(e->h_ovf);
    if (e->h_fix_scene) cudaFreeHost(e->h_fix_scene);
    if (e->h_stage) cudaFreeHost(e->h_stage);
    delete e;
    return IVP_OK;
}

int ivp_engine_bind(ivp_engine* e, const ivp_particles* p) {
    if (!e || !p) return IVP_ERR_BAD_ARG;
    if (p->n_total != e->n_total) return IVP_ERR_BAD_ARG;
    if (!p->x || !p->v || !p->m || !p->density0 || !p->is_dynamic || !p->density || !p->kdiag)
        return IVP_ERR_BAD_ARG;
    destroy_graphs(e);
    e->D.x = p->x;
    e->D.v = p->v;
    e->D.m = p->m;
    e->D.rho0 = p->density0;
    e->D.dyn = p->is_dynamic;
    e->D.material = p->material;
    e->D.density_out = p->density;
    e->D.k_out = p->kdiag;
    e->D.div_out = p->divergence;
    e->want_divergence = p->divergence != nullptr;
    e->bound = true;
    return IVP_OK;
}

int ivp_update_scene(ivp_engine* e, int32_t scene, const ivp_scene_desc* d, void* stream) {
    if (!e || !d || scene < 0 || scene >= e->n_scenes) return IVP_ERR_BAD_ARG;
    const ivp_scene_desc& o = e->desc[scene];
    if (d->particle_offset != o.particle_offset || d->n_particles != o.n_particles || d->n_dynamic != o.n_dynamic ||
        d->particle_radius != o.particle_radius || d->cache_size != o.cache_size ||
        d->domain_size[0] != o.domain_size[0] || d->domain_size[1] != o.domain_size[1] ||
        d->domain_size[2] != o.domain_size[2])
        return IVP_ERR_BAD_ARG;
    if (!(d->dt > 0.0f) || d->max_outer_iters < 0 || d->max_iteration_pcg < 0) return IVP_ERR_BAD_ARG;
    if (d->pressure_solver != e->desc[scene].pressure_solver) return IVP_ERR_BAD_ARG;  // planned at creation
    e->desc[scene] = *d;
    SceneParams& q = e->hp[scene];
    q.dt = d->dt;
    q.inv_dt = (float)(1.0 / (double)d->dt);
    q.omega = d->omega;
    for (int a = 0; a < 3; ++a) q.gravity[a] = d->gravity[a];
    q.max_outer = d->max_outer_iters;
    q.max_pcg = d->max_iteration_pcg;
    q.fixed_iters = d->fixed_outer_iters;
    q.tol_opt = d->density_error_tol;
    q.tol_pcg = d->tol_pcg;
    q.visc_coeff = d->viscosity_coeff;
    q.visc_method = d->viscosity_method;
    // a force may be switched off, not on: its buffers and launches were
    // planned at creation
    const bool st = d->surface_tension_method == 1 && d->surface_tension_coeff > 0.0f;
    const bool vi = d->viscosity_method == 1 && d->viscosity_coeff > 0.0f;
    if ((st && !e->any_st) || (vi && !e->any_visc)) return IVP_ERR_BAD_ARG;
    q.st_coeff = d->surface_tension_coeff;
    q.st_method = d->surface_tension_method;
    cudaStream_t s = as_stream(stream);
    CK(cudaMemcpyAsync((void*)(e->D.scenes + scene), &q, sizeof(SceneParams), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    return IVP_OK;
}

int ivp_neighbour_build(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    return run(e, emit_build, &e->graph_build, &e->exec_build, as_stream(stream));
}

int ivp_compute_density(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    KernelSet K;
    kernel_set(e->G, e->BLOCK, &K);
    Launcher L;
    L.stream = as_stream(stream);
    return L.dev(IVP_K_PACK, K.dens, e->n_tiles, e->BLOCK, e->D);
}

int ivp_compute_aii(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    KernelSet K;
    kernel_set(e->G, e->BLOCK, &K);
    Launcher L;
    L.stream = as_stream(stream);
    CKS(L.dev(IVP_K_PACK, K.aii, e->n_tiles, e->BLOCK, e->D));
    return L.dev(IVP_K_STATIC_OUT, k_static_outputs, blocks_for(e->n_total, ELEM_BLOCK), ELEM_BLOCK, e->D);
}

int emit_ip_only(ivp_engine* e, Launcher& L) { return emit_solve(e, L, false); }

int ivp_ip_solve(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    return run(e, emit_ip_only, &e->graph_solve, &e->exec_solve, as_stream(stream));
}

int ivp_prj_solve(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    return run(e, emit_prj, &e->graph_prj, &e->exec_prj, as_stream(stream));
}

int ivp_viscosity_solve(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    Launcher L;
    L.stream = as_stream(stream);
    return emit_force(e, L, FORCE_VISC);
}

int ivp_surface_tension_solve(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    Launcher L;
    L.stream = as_stream(stream);
    return emit_force(e, L, FORCE_ST);
}

int ivp_apply_gravity(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    Launcher L;
    L.stream = as_stream(stream);
    return L.dev(IVP_K_GRAVITY, k_gravity, blocks_for(e->n_total, ELEM_BLOCK), ELEM_BLOCK, e->D);
}

int ivp_advect(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    Launcher L;
    L.stream = as_stream(stream);
    return emit_advect(e, L);
}

int ivp_step(ivp_engine* e, int32_t n_steps, void* stream) {
    if (!e || n_steps < 0) return IVP_ERR_BAD_ARG;
    for (int k = 0; k < n_steps; ++k) CKS(run(e, emit_step, &e->graph_step, &e->exec_step, as_stream(stream)));
    return IVP_OK;
}

int ivp_step_io(ivp_engine* e, const float* x_in, const float* v_in, float* x_out, float* v_out, int64_t first,
                int64_t count, void* stream) {
    if (!e || first < 0 || count < 0 || first + count > e->n_total) return IVP_ERR_BAD_ARG;
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    // host buffers must be page-locked: the copies run inside the step
    const void* host[4] = {x_in, v_in, x_out, v_out};
    for (const void* h : host) {
        if (!h) continue;
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
            cudaGetLastError();
            return IVP_ERR_BAD_ARG;
        }
        if (a.type != cudaMemoryTypeHost) return IVP_ERR_BAD_ARG;
    }
    if (!e->io_side) {
        CK(cudaStreamCreateWithFlags(&e->io_side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&e->io_ev_start, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->io_ev_x, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->io_ev_adv, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->io_ev_out, cudaEventDisableTiming));
    }
    ivp_engine::StepIO io;
    io.x_in = x_in;
    io.v_in = v_in;
    io.x_out = x_out;
    io.v_out = v_out;
    io.first = first;
    io.count = count;
    e->io = io;
    cudaStream_t s = as_stream(stream);
    if (e->opt.use_graphs) {
        if (e->exec_step_io && !(io == e->io_key)) {
            cudaGraphExecDestroy(e->exec_step_io);
            cudaGraphDestroy(e->graph_step_io);
            e->exec_step_io = nullptr;
            e->graph_step_io = nullptr;
        }
        if (!e->exec_step_io) {
            CKS(make_graph(e, emit_step_io, &e->graph_step_io, &e->exec_step_io));
            e->io_key = io;
        }
        CK(cudaGraphLaunch(e->exec_step_io, s));
        return IVP_OK;
    }
    Launcher L;
    L.stream = s;
    return emit_step_io(e, L);
}

int ivp_read_stats(ivp_engine* e, int32_t scene, void* stream, ivp_solve_stats* out) {
    if (!e || !out || scene < 0 || scene >= e->n_scenes) return IVP_ERR_BAD_ARG;
    cudaStream_t s = as_stream(stream);
    CKS(enqueue_stage(e, scene, s));
    CK(cudaStreamSynchronize(s));
    unpack_stage(e, scene);
    return fill_stats(e, scene, out);
}

int ivp_prepare(ivp_engine* e) {
    if (!e) return IVP_ERR_BAD_ARG;
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    if (!e->opt.use_graphs) return IVP_OK;
    if (!e->exec_build) CKS(make_graph(e, emit_build, &e->graph_build, &e->exec_build));
    if (!e->exec_step) CKS(make_graph(e, emit_step, &e->graph_step, &e->exec_step));
    return IVP_OK;
}

int ivp_read_stats_all(ivp_engine* e, void* stream, ivp_solve_stats* out) {
    if (!e || !out) return IVP_ERR_BAD_ARG;
    cudaStream_t s = as_stream(stream);
    const int ns = e->n_scenes;
    CK(cudaMemcpyAsync(e->h_ctl, e->D.ctl, sizeof(SceneCtl) * ns, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(e->h_overflow, e->D.overflow, sizeof(int) * ns, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(e->h_flags, e->D.flags, sizeof(Flags), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(e->h_pairs, e->D.pairs, sizeof(unsigned long long) * ns, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(e->h_fix_scene, e->D.fix_scene, sizeof(int) * ns, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int k = 0; k < ns; ++k) CKS(fill_stats(e, k, out + k));
    return IVP_OK;
}

int ivp_read_history(ivp_engine* e, int32_t scene, void* stream, double* errors, int32_t* pcg_iters, int32_t cap,
                     int32_t* n_errors, int32_t* n_pcg) {
    if (!e || scene < 0 || scene >= e->n_scenes || cap < 0) return IVP_ERR_BAD_ARG;
    cudaStream_t s = as_stream(stream);
    CKS(enqueue_stage(e, scene, s));
    CK(cudaStreamSynchronize(s));
    unpack_stage(e, scene);
    fill_history(e, scene, errors, pcg_iters, cap, n_errors, n_pcg);
    return IVP_OK;
}

int ivp_read_solve(ivp_engine* e, int32_t scene, void* stream, ivp_solve_stats* out, double* errors,
                   int32_t* pcg_iters, int32_t cap, int32_t* n_errors, int32_t* n_pcg) {
    if (!e || !out || scene < 0 || scene >= e->n_scenes || cap < 0) return IVP_ERR_BAD_ARG;
    cudaStream_t s = as_stream(stream);
    CKS(enqueue_stage(e, scene, s));
    CK(cudaStreamSynchronize(s));
    unpack_stage(e, scene);
    fill_history(e, scene, errors, pcg_iters, cap, n_errors, n_pcg);
    return fill_stats(e, scene, out);
}

int ivp_export_neighbours(ivp_engine* e, int32_t scene, int32_t* count, int32_t* ids, int32_t cache, void* stream) {
    if (!e || scene < 0 || scene >= e->n_scenes || !count || !ids || cache <= 0) return IVP_ERR_BAD_ARG;
    cudaStream_t s = as_stream(stream);
    const int nd = e->hp[scene].n_dyn;
    if (nd == 0) return IVP_OK;
    k_export<<<blocks_for(nd, 128), 128, 0, s>>>(e->D, scene, count, ids, cache);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    return IVP_OK;
}

int ivp_set_wait_limit(ivp_engine* e, int64_t ns) {
    if (!e) return IVP_ERR_BAD_ARG;
    const unsigned long long v = ns > 0 ? (unsigned long long)ns : kBarrierLimitNs;
    if (v != e->D.bar_limit_ns) {
        destroy_graphs(e);  // the graphs hold the previous value in their kernel parameters
        e->D.bar_limit_ns = v;
    }
    return IVP_OK;
}

int ivp_reset_counters(ivp_engine* e, void* stream) {
    if (!e) return IVP_ERR_BAD_ARG;
    k_reset_counters<<<blocks_for(e->n_scenes, 128), 128, 0, as_stream(stream)>>>(e->D);
    CK(cudaGetLastError());
    return IVP_OK;
}

int ivp_profile_step(ivp_engine* e, int32_t n_steps, void* stream, double* ms, int32_t* launches) {
    if (!e || n_steps < 0 || !ms || !launches) return IVP_ERR_BAD_ARG;
    if (!e->bound) return IVP_ERR_NOT_BOUND;
    cudaStream_t s = as_stream(stream);
    Prof prof;
    Launcher L;
    L.stream = s;
    L.prof = &prof;
    for (int k = 0; k < n_steps; ++k) CKS(emit_step(e, L));
    CK(cudaStreamSynchronize(s));
    for (int k = 0; k < IVP_K_COUNT; ++k) {
        ms[k] = 0.0;
        launches[k] = 0;
    }
    for (size_t k = 0; k < prof.ids.size(); ++k) {
        float t = 0.0f;
        CK(cudaEventElapsedTime(&t, prof.ev[2 * k], prof.ev[2 * k + 1]));
        const int id = prof.ids[k];
        if (id >= 0 && id < IVP_K_COUNT) {
            ms[id] += t;
            launches[id] += 1;
        }
    }
    return IVP_OK;
}

const char* ivp_status_string(int32_t status) {
    switch (status) {
        case IVP_OK: return "ok";
        case IVP_ERR_NOT_SPD: return "non-positive definite matrix (pAp < 0)";
        case IVP_ERR_NOT_CONVERGED: return "outer iteration did not converge";
        case IVP_ERR_NBR_OVERFLOW: return "neighbour cache overflow: more dropped pairs than the correction storage holds";
        case IVP_ERR_BAD_ARG: return "bad argument";
        case IVP_ERR_CUDA: return "CUDA error";
        case IVP_ERR_TIMEOUT: return "timeout";
        case IVP_ERR_NOT_BOUND: return "particle arrays not bound";
        case IVP_ERR_DEVICE_CHECK: return "device-side bounds check failed";
        default: return "unknown status";
    }
}

const char* ivp_last_error(void) { return g_err.c_str(); }

}  // extern "C"
