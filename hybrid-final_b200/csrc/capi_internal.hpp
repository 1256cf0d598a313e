// capi_internal.hpp -- host-side objects behind the opaque C handles.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/hpic.h"
#include "dev.cuh"
#include "fastsolve.hpp"
#include "kernels.cuh"
#include "setup.hpp"

namespace hpi {
// Device lists for field_mode 2 over a set of cases (indices into the
// descriptor array the kernels see).
struct FastPlanDev {
    hp::FastPlan plan;
    int *d_list = nullptr, *d_items = nullptr;
    hp::GemmProb *d_probs = nullptr;
};
} // namespace hpi

struct hp_setup {
    hp::Setup s;
    hp_case_opts opts;
    bool fs_built = false;
    hp::FastSolver fs; // built on first request of its tables
};

struct hp_case {
    hp::Setup s;
    hp_case_opts opts;
    int device = 0;
    hp::DevCase h{};               // host image of the device descriptor
    hp::DevCase *d_case = nullptr; // device descriptor
    int *d_items = nullptr;        // item_start arrays: [0..1] particles, [2..3] cells, [4..5] nodes,
                                   // [6..7] fluid x lines, [8..9] fluid y lines
    std::vector<void *> allocs;
    std::vector<size_t> alloc_bytes;
    size_t bytes = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t last_stream = nullptr;
    hp::LaunchCfg lc;
    int pcg_cluster = 1;           // CTAs of this case's field-solve cluster
    int *d_list0 = nullptr;        // device {0}: the case's index in its own one-case list
    hp::FastSolver fs;             // field_mode 2: separable inverse (fs.ok false otherwise)
    int fs_passes = 3;
    hpi::FastPlanDev fplan;        // its device lists (one-case plan)
    cudaGraphExec_t graph = nullptr;
    int graph_kernels = 0; // kernel nodes in the captured step
    hp_batch *batch = nullptr;
    std::vector<float> prob; // [3*C] initial collision probabilities
    char *fl_state = nullptr;  // fluid averaging state (HP_GRID_FLUID_STATE), also holding h.prob
    size_t fl_state_bytes = 0;
    hp::FluidPlan fplan_fluid; // the case's own fluid launch lists (into d_items)
    hp::FluidFork fl_fork;     // side stream of the fluid sweeps (fluid cases)
    std::vector<uint32_t> mcc_base; // collision tallies at the last hp_reset_averages (empty: zeros)
};

extern "C" hp_status hpi_grid_ptr(hp_case *c, hp_grid_field f, void **p, size_t *nb);

namespace hpi {
hp_status fast_plan_build(hp_case *const *cases, const std::vector<int> &idx, FastPlanDev &out);
void fast_plan_free(FastPlanDev &f);
void set_error(const std::string &m);
// kernel nodes of a captured graph
int count_kernel_nodes(cudaGraph_t g);
// launch shapes the kernels accept
bool tune_valid(const hp_tune &t);
hp_status cuda_fail(cudaError_t e, const char *what);
// Build the per-case prefix arrays and device descriptor array of a batch.
struct BatchDev {
    hp::DevCase *d_cases = nullptr;
    int *d_part = nullptr, *d_cell = nullptr, *d_node = nullptr;
    int n = 0, n_part = 0, n_cell = 0, n_node = 0;
    int max_g = 0;
    bool any_eedf = false;
    int max_smt = 0; // most density smoothing passes of any case
    bool surface = false; // some case has dielectric blocks
    bool power = false;   // some case has power-driven sources or an external circuit
    bool circuit = false; // some case has an external circuit
    int *d_fluid = nullptr; // fluid line prefixes: x lines [n+1], then y lines [n+1]
    hp::FluidPlan fluid;
    hp::FluidFork fluid_fork; // side stream of the fluid sweeps (batches with fluid cases)
    // PCG groups for every cluster cap 1,2,4,8,16: lists of case indices per
    // cluster size, concatenated in d_lists
    int *d_lists = nullptr;
    int list_off[5][5] = {}, list_n[5][5] = {};
    std::vector<std::pair<int, int>> grid_cases; // whole-GPU PCG cases: (offset in the lists, CTAs)
    std::vector<hp::PcgGroup> groups(int cluster_max, int block) const;
    FastPlanDev fast;
};
hp_status batch_dev_build(hp_case *const *cases, int n, BatchDev &b);
void batch_dev_free(BatchDev &b);
hp_status run_step(const BatchDev &b, const hp::LaunchCfg &lc, int gas, cudaStream_t st);
// a case that takes over a set-up (its host particle load is released once uploaded)
hp_status case_from_setup_owned(hp::Setup &&s, const hp_case_opts &o, hp_case **out);
hp_status device_load(hp_case *c, int isp); // the initial particles of a deferred load (load.cu)
// an upper estimate of a case's device footprint before it is created
size_t estimate_device_bytes(const hp::Setup &s, const hp_case_opts &o);
} // namespace hpi
