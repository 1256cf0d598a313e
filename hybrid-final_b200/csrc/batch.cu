// batch.cu -- many independent cases advanced by one launch per phase.
//
// Every kernel already walks a list of case descriptors (kernels.cu), so a
// batch is the concatenation of the cases' work lists: item prefix arrays
// map a global warp or thread to (case, local item).  One step is captured
// once as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.hpp"

using namespace hp;
using hpi::cuda_fail;
using hpi::set_error;

#define CK(call)                                                                                                       \
    do {                                                                                                               \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);                                                           \
    } while (0)

struct hp_batch {
    std::vector<hp_case *> cases;
    hpi::BatchDev dev;
    LaunchCfg lc;
    int gas = 0;
    int device = 0;
    cudaStream_t own = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_kernels = 0;
};

namespace hpi {

hp_status batch_dev_build(hp_case *const *cases, int n, BatchDev &b) {
    std::vector<DevCase> hd(n);
    std::vector<int> part(n + 1, 0), cell(n + 1, 0), node(n + 1, 0), fl(2 * (n + 1), 0);
    b.fluid = FluidPlan();
    b.max_g = 0;
    b.any_eedf = false;
    b.max_smt = 0;
    b.surface = false;
    b.power = false;
    b.circuit = false;
    for (int i = 0; i < n; i++) {
        hd[i] = cases[i]->h;
        b.any_eedf |= cases[i]->h.eedf_every > 0;
        b.max_smt = std::max(b.max_smt, cases[i]->s.N_smt);
        b.surface = b.surface || cases[i]->s.diel_num > 0;
        b.power = b.power || cases[i]->s.power_driven() || cases[i]->s.external;
        b.circuit = b.circuit || cases[i]->s.external;
        const Setup &s = cases[i]->s;
        part[i + 1] = part[i] + s.nsp * s.Csize;
        cell[i + 1] = cell[i] + s.Csize;
        node[i + 1] = node[i] + s.Gsize;
        b.max_g = std::max(b.max_g, s.Gsize);
        const DevCase &h = cases[i]->h;
        const bool on = h.fluid_on != 0;
        fl[i + 1] = fl[i] + (on ? h.nfsp * h.nxl : 0);
        fl[n + 1 + i + 1] = fl[n + 1 + i] + (on ? h.nfsp * h.nyl : 0);
        if (on) {
            b.fluid.any = true;
            b.fluid.len_x = std::max(b.fluid.len_x, s.ncx);
            b.fluid.len_y = std::max(b.fluid.len_y, s.ncy);
        }
    }
    b.fluid.n_x = fl[n];
    b.fluid.n_y = fl[2 * n + 1];
    b.n = n;
    b.n_part = part[n];
    b.n_cell = cell[n];
    b.n_node = node[n];
    CK(cudaMalloc(&b.d_cases, sizeof(DevCase) * (size_t)n));
    CK(cudaMemcpy(b.d_cases, hd.data(), sizeof(DevCase) * (size_t)n, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&b.d_part, sizeof(int) * (size_t)(n + 1)));
    CK(cudaMalloc(&b.d_cell, sizeof(int) * (size_t)(n + 1)));
    CK(cudaMalloc(&b.d_node, sizeof(int) * (size_t)(n + 1)));
    CK(cudaMemcpy(b.d_part, part.data(), sizeof(int) * (size_t)(n + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.d_cell, cell.data(), sizeof(int) * (size_t)(n + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.d_node, node.data(), sizeof(int) * (size_t)(n + 1), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&b.d_fluid, sizeof(int) * fl.size()));
    CK(cudaMemcpy(b.d_fluid, fl.data(), sizeof(int) * fl.size(), cudaMemcpyHostToDevice));
    b.fluid.xl_items = b.d_fluid;
    b.fluid.yl_items = b.d_fluid + n + 1;
    if (b.fluid.n_x + b.fluid.n_y > 0) CK(fluid_fork_create(b.fluid_fork));
    std::vector<int> lists;
    for (int m = 0; m < 5; m++)
        for (int k = 0; k <= m; k++) {
            b.list_off[m][k] = (int)lists.size();
            for (int i = 0; i < n; i++) {
                if (cases[i]->h.field_mode == 2) continue; // separable inner solve, not PCG
                if (cases[i]->pcg_cluster > 16) continue;  // whole-GPU solve, launched on its own
                int cs = std::min(pcg_cluster_for_nodes(cases[i]->s.Gsize), 1 << m);
                if (cs == (1 << k)) lists.push_back(i);
            }
            b.list_n[m][k] = (int)lists.size() - b.list_off[m][k];
        }
    b.grid_cases.clear();
    for (int i = 0; i < n; i++)
        if (cases[i]->h.field_mode != 2 && cases[i]->pcg_cluster > 16) {
            b.grid_cases.push_back({(int)lists.size(), cases[i]->pcg_cluster});
            lists.push_back(i);
        }
    {
        std::vector<int> fidx;
        std::vector<hp_case *> fc;
        for (int i = 0; i < n; i++)
            if (cases[i]->h.field_mode == 2) {
                fidx.push_back(i);
                fc.push_back(cases[i]);
            }
        hp_status fs = fast_plan_build(fc.data(), fidx, b.fast);
        if (fs != HP_OK) return fs;
    }
    CK(cudaMalloc(&b.d_lists, sizeof(int) * std::max<size_t>(lists.size(), 1)));
    if (!lists.empty())
        CK(cudaMemcpy(b.d_lists, lists.data(), sizeof(int) * lists.size(), cudaMemcpyHostToDevice));
    return HP_OK;
}

std::vector<PcgGroup> BatchDev::groups(int cluster_max, int block) const {
    int m = 0;
    while ((1 << (m + 1)) <= cluster_max && m < 4) m++;
    std::vector<PcgGroup> g;
    for (int k = 0; k <= m; k++)
        if (list_n[m][k] > 0) g.push_back(PcgGroup{1 << k, block, d_lists + list_off[m][k], list_n[m][k]});
    for (const auto &gc : grid_cases) g.push_back(PcgGroup{gc.second, block, d_lists + gc.first, 1});
    return g;
}

void batch_dev_free(BatchDev &b) {
    cudaFree(b.d_cases);
    cudaFree(b.d_part);
    cudaFree(b.d_cell);
    cudaFree(b.d_node);
    cudaFree(b.d_lists);
    cudaFree(b.d_fluid);
    fast_plan_free(b.fast);
    fluid_fork_destroy(b.fluid_fork);
    b = BatchDev();
}

hp_status run_step(const BatchDev &b, const LaunchCfg &lc, int gas, cudaStream_t st) {
    CK(launch_advance(b.d_cases, b.n, st));
    if (b.fluid.any) CK(fluid_begin(b.d_cases, b.n, b.fluid, b.fluid_fork, st));
    const std::vector<PcgGroup> g = b.groups(lc.pcg_cluster_max, lc.pcg_block);
    CK(launch_field(b.d_cases, b.d_node, b.n, b.n_node, g.data(), (int)g.size(), &b.fast.plan, st, b.circuit));
    CK(launch_move(b.d_cases, b.d_part, b.n, b.n_part, lc, st));
    CK(launch_sort(b.d_cases, b.d_part, b.n, b.n_part, lc, st, b.surface));
    if (gas != GAS_AR) CK(launch_mcc_oxy(b.d_cases, b.d_cell, b.n, b.n_cell, gas, st));
    else CK(launch_mcc_ar(b.d_cases, b.d_cell, b.n, b.n_cell, lc, st));
    CK(launch_deposit(b.d_cases, b.d_part, b.d_node, b.n, b.n_part, b.n_node, lc, st, b.max_smt));
    if (b.fluid.any) CK(fluid_end(b.d_cases, b.d_node, b.n, b.n_node, b.fluid, b.fluid_fork, st));
    CK(launch_accumulate(b.d_cases, b.d_node, b.n, b.n_node, st));
    if (b.any_eedf) CK(launch_eedf(b.d_cases, b.d_cell, b.n, b.n_cell, st));
    if (b.power) CK(launch_power(b.d_cases, b.n, st));
    return HP_OK;
}

} // namespace hpi

namespace {

hp_status capture(hp_batch *b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal));
    hp_status s1 = hpi::run_step(b->dev, b->lc, b->gas, b->own);
    cudaError_t e = cudaStreamEndCapture(b->own, &g);
    if (s1 != HP_OK) return s1;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    b->graph_kernels = hpi::count_kernel_nodes(g);
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    return HP_OK;
}

} // namespace

extern "C" {

hp_status hp_batch_create(hp_case *const *cases, int n, hp_batch **out) {
    if (!cases || n <= 0 || !out) return set_error("empty batch"), HP_ERR_ARG;
    int dev = cases[0]->device, gas = cases[0]->s.main_gas;
    for (int i = 0; i < n; i++) {
        if (!cases[i]) return set_error("null case"), HP_ERR_ARG;
        if (cases[i]->batch) return set_error("case already in a batch"), HP_ERR_ARG;
        if (cases[i]->device != dev) return set_error("cases on different devices"), HP_ERR_ARG;
        if (cases[i]->s.main_gas != gas) return set_error("cases with different gases"), HP_ERR_ARG;
        for (int j = 0; j < i; j++)
            if (cases[j] == cases[i]) return set_error("case listed twice"), HP_ERR_ARG;
    }
    int passes = 0; // the separable solves of a batch run their refinement passes together
    for (int i = 0; i < n; i++) {
        if (cases[i]->h.field_mode != 2) continue;
        if (passes && cases[i]->h.fs_passes != passes)
            return set_error("field_mode 2 cases of a batch need the same fs_passes"), HP_ERR_ARG;
        passes = cases[i]->h.fs_passes;
    }
    CK(cudaSetDevice(dev));
    for (int i = 0; i < n; i++) CK(cudaStreamSynchronize(cases[i]->last_stream));
    hp_batch *b = new hp_batch();
    b->cases.assign(cases, cases + n);
    b->gas = gas;
    b->device = dev;
    hp_status st = hpi::batch_dev_build(cases, n, b->dev);
    if (st != HP_OK) {
        delete b;
        return st;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        hpi::batch_dev_free(b->dev);
        delete b;
        return cuda_fail(e, "cudaStreamCreate");
    }
    for (int i = 0; i < n; i++) cases[i]->batch = b;
    *out = b;
    return HP_OK;
}

hp_status hp_batch_destroy(hp_batch *b) {
    if (!b) return HP_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->own);
    cudaDeviceSynchronize();
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaStreamDestroy(b->own);
    hpi::batch_dev_free(b->dev);
    for (hp_case *c : b->cases) {
        c->batch = nullptr;
        c->last_stream = nullptr;
    }
    delete b;
    return HP_OK;
}

hp_status hp_batch_step(hp_batch *b, int nsteps, void *stream) {
    if (!b || nsteps < 0) return HP_ERR_ARG;
    CK(cudaSetDevice(b->device));
    cudaStream_t st = (cudaStream_t)stream;
    if (!b->graph) {
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CK(cudaEventRecord(ev, st));
        CK(cudaStreamWaitEvent(b->own, ev, 0));
        CK(cudaEventDestroy(ev));
        hp_status s1 = capture(b);
        if (s1 != HP_OK) return s1;
    }
    for (int k = 0; k < nsteps; k++) CK(cudaGraphLaunch(b->graph, st));
    for (hp_case *c : b->cases) c->last_stream = st;
    return HP_OK;
}

hp_status hp_batch_set_tune(hp_batch *b, const hp_tune *t) {
    if (!b || !t) return HP_ERR_ARG;
    if (!hpi::tune_valid(*t)) return set_error("hp_tune out of range"), HP_ERR_ARG;
    b->lc.warps_per_block = t->warps_per_block_particles;
    b->lc.pcg_block = t->pcg_block;
    b->lc.pcg_cluster_max = t->pcg_cluster_max;
    b->lc.move_unroll = t->move_unroll;
    b->lc.mcc_cells = t->mcc_cells_per_warp;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return HP_OK;
}

hp_status hp_batch_get_tune(hp_batch *b, hp_tune *t) {
    if (!b || !t) return HP_ERR_ARG;
    t->warps_per_block_particles = b->lc.warps_per_block;
    t->pcg_block = b->lc.pcg_block;
    t->pcg_cluster_max = b->lc.pcg_cluster_max;
    t->move_unroll = b->lc.move_unroll;
    t->mcc_cells_per_warp = b->lc.mcc_cells;
    return HP_OK;
}

// Times candidate launch shapes on the batch itself.  Every case's device
// state is copied aside first and restored after each trial, so the batch
// resumes exactly where it stood.
hp_status hp_batch_autotune(hp_batch *b, void *stream) {
    if (!b) return HP_ERR_ARG;
    CK(cudaSetDevice(b->device));
    cudaStream_t st = (cudaStream_t)stream;
    CK(cudaStreamSynchronize(st));
    size_t total = 0;
    for (hp_case *c : b->cases)
        for (size_t k = 0; k < c->allocs.size(); k++) total += c->alloc_bytes[k];
    char *save = nullptr;
    CK(cudaMalloc(&save, total));
    auto copy_all = [&](bool to_save) -> cudaError_t {
        size_t off = 0;
        for (hp_case *c : b->cases)
            for (size_t k = 0; k < c->allocs.size(); k++) {
                cudaError_t e = to_save ? cudaMemcpyAsync(save + off, c->allocs[k], c->alloc_bytes[k],
                                                          cudaMemcpyDeviceToDevice, st)
                                        : cudaMemcpyAsync(c->allocs[k], save + off, c->alloc_bytes[k],
                                                          cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) return e;
                off += c->alloc_bytes[k];
            }
        return cudaSuccess;
    };
    cudaError_t e = copy_all(true);
    if (e != cudaSuccess) { cudaFree(save); return cuda_fail(e, "autotune save"); }
    const LaunchCfg base = b->lc;
    LaunchCfg best = base;
    float best_ms = 1e30f;
    const int cl0 = pcg_cluster_for_nodes(b->dev.max_g);
    int warps[3] = {4, 8, 16};
    int blocks[3] = {128, 256, 512};
    int clus[3] = {std::max(1, cl0 / 4), std::max(1, cl0 / 2), cl0};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    hp_status result = HP_OK;
    // time 3 steps of one candidate (after a warm-up step), then restore the state
    auto trial = [&](const LaunchCfg &lc) {
        b->lc = lc;
        hp_status s = hpi::run_step(b->dev, b->lc, b->gas, st); // warm-up
        if (s != HP_OK) { result = s; return; }
        cudaEventRecord(e0, st);
        for (int k = 0; k < 3 && s == HP_OK; k++) s = hpi::run_step(b->dev, b->lc, b->gas, st);
        cudaEventRecord(e1, st);
        if (s != HP_OK) { result = s; return; }
        e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) { result = cuda_fail(e, "autotune trial"); return; }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best = lc; }
        e = copy_all(false);
        if (e != cudaSuccess) result = cuda_fail(e, "autotune restore");
    };
    const int unrolls[3] = {1, 2, 4};
    for (int pi = 0; pi < 3 && result == HP_OK; pi++)
        for (int wi = 0; wi < 3 && result == HP_OK; wi++)
            for (int bi = 0; bi < 3 && result == HP_OK; bi++)
                for (int ki = 0; ki < 3 && result == HP_OK; ki++) {
                    if (ki > 0 && clus[ki] == clus[ki - 1]) continue;
                    LaunchCfg lc = base;
                    lc.move_unroll = unrolls[pi];
                    lc.warps_per_block = warps[wi];
                    lc.pcg_block = blocks[bi];
                    lc.pcg_cluster_max = clus[ki];
                    trial(lc);
                }
    // then the MCC cell grouping around the best of those
    if (b->gas == GAS_AR) {
        const LaunchCfg around = best;
        const int groups[5] = {1, 2, 4, 8, 16};
        for (int gi = 0; gi < 5 && result == HP_OK; gi++) {
            if (groups[gi] == around.mcc_cells) continue;
            LaunchCfg lc = around;
            lc.mcc_cells = groups[gi];
            trial(lc);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    copy_all(false);
    cudaStreamSynchronize(st);
    cudaFree(save);
    b->lc = best;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return result;
}

} // extern "C"

extern "C" hp_status hp_batch_step_kernels(const hp_batch *b, int *n) {
    if (!b || !n) return HP_ERR_ARG;
    *n = b->graph_kernels;
    return HP_OK;
}
