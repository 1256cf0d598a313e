// kernels.cuh -- launch wrappers for the per-step kernels (kernels.cu).
//
// Every kernel takes the whole batch: an array of device case descriptors
// and, for the warp-per-cell kernels, a prefix array item_start[ncases+1]
// that maps a global work item to its case.  A single case is a batch of one.
#pragma once
#include <cuda_runtime.h>
#include "dev.cuh"

namespace hp {

struct LaunchCfg {
    int warps_per_block = 4;   // particle kernels: one warp per (species, cell)
    int pcg_block = 512;       // PCG: threads per CTA
    int pcg_cluster_max = 16;  // PCG: upper bound on CTAs per case
    int move_unroll = 1;       // Move: chunks of 32 loaded per iteration (1: k_move, one-chunk prefetch)
    int mcc_cells = 16;        // MCC (Ar): consecutive cells per warp, sharing collision batches (1, 2, 4, 8, 16)
};

// Move: gather + push + single-cell exit test (src/cuda_Move.cu:181-270)
cudaError_t launch_move(const DevCase *cases, const int *item_start, int ncases, int items, const LaunchCfg &lc,
                        cudaStream_t st);
// SortBoundary: boundary handling + deterministic re-bin (src/cuda_Sortboundary.cu:41-258)
// the power controller of power-driven cases, after Deposit (cases without
// one return at once)
cudaError_t launch_power(DevCase *cases, int ncases, cudaStream_t st);
// surface: some case has dielectric blocks (apply the crossings Move queued)
cudaError_t launch_sort(const DevCase *cases, const int *item_start, int ncases, int items, const LaunchCfg &lc,
                        cudaStream_t st, bool surface);
// MCC, Ar set (src/cuda_mcc.cu:97-106, src/cuda_mccAr.cu:41-232)
// MCC of the Ar/O2 (gas 2) reaction set, one warp per cell (mcc_oxy.cu)
cudaError_t launch_mcc_oxy(const DevCase *cases, const int *item_start, int ncases, int items, int gas,
                           cudaStream_t st);
cudaError_t launch_mcc_ar(const DevCase *cases, const int *item_start, int ncases, int items, const LaunchCfg &lc,
                          cudaStream_t st);
// Deposit: per-cell CIC sums, then node gather + boundary scale + rho/eps0 + RHS
// (src/cuda_Deposit.cu:3-20,30-104,277-325)
// max_smt: the most 1-2-1 smoothing passes any of the cases asks for (0: none)
cudaError_t launch_deposit(const DevCase *cases, const int *cell_items, const int *node_items, int ncases,
                           int n_cell_items, int n_node_items, const LaunchCfg &lc, cudaStream_t st, int max_smt);
// Field: PCG (src/cuda_Field.cu:133-181,942-1072), potential assembly and
// E at nodes (src/cuda_Field.cu:2-42,500-558,698-846).  The PCG runs one
// cluster per case; cases are grouped by cluster size (a launch has one
// cluster shape), and each case's cluster size depends only on its own grid,
// so a case gets the same reduction order alone and inside any batch.
struct PcgGroup {
    int cluster;      // CTAs per case (above 16: one cooperative launch per case over the grid)
    int block;        // threads per CTA
    const int *list;  // device array of case indices
    int n;
};
// field_mode 2 (fastsolve.cu): refinement passes with the separable inverse
struct GemmProb {
    int M, N, K;
    const float *A, *B;
    float *C;
    const float *S;  // epi 1: elementwise scale of the product
    double *x64;     // epi 2: x64[(i0 + n) * ngy + (j0 + m)] += product
    int ngy, i0, j0, epi;
    int tiles_n, tile_start;
};
struct FastPlan {
    const int *list = nullptr;       // device: case indices
    const int *item_start = nullptr; // device: prefix of rectangle sizes [n+1]
    int n = 0, items = 0;
    const GemmProb *probs[4] = {nullptr, nullptr, nullptr, nullptr}; // device, one list per product
    int ntiles[4] = {0, 0, 0, 0};
    int passes = 3;
    int final_chunks = 0; // max over the cases of ceil(G / FS_CHUNK)
};
// nodes per CTA of the final residual pass; a case's fs_res holds
// 2 + 2 * ceil(G / FS_CHUNK) doubles
constexpr int FS_CHUNK = 1024;
constexpr int FS_TILE = 32; // GEMM output tile edge
cudaError_t launch_fast_field(const DevCase *cases, const FastPlan &fp, cudaStream_t st);
cudaError_t launch_field(const DevCase *cases, const int *node_items, int ncases, int n_node_items,
                         const PcgGroup *groups, int ngroups, const FastPlan *fast, cudaStream_t st,
                         bool circuit = false);
// CTAs per case for a grid of G nodes
int pcg_cluster_for_nodes(int G);
// CTAs of the whole-GPU cooperative PCG for a case of G nodes (0: a cluster suffices)
int pcg_grid_ctas(int G, int block);
// CSR particles (5 arrays of start[C] floats back to back: x, y, vx, vy, vz)
// into the cell-blocked slots of one species; sets cnt and clears nmov
cudaError_t launch_scatter(const DevSpecies &sp, int C, const int *start, const float *src, cudaStream_t st);
// tstep += 1 for every case (device-side step counter, graph friendly)
cudaError_t launch_advance(const DevCase *cases, int ncases, cudaStream_t st);
// running sums of den and phi (N_ave accumulation, src/cuda_Diagnostic.cu:505-547)
// electron energy histogram of the cases whose eedf_every divides the step
cudaError_t launch_eedf(const DevCase *cases, const int *cell_items, int ncases, int n_cell_items, cudaStream_t st);
cudaError_t launch_accumulate(const DevCase *cases, const int *node_items, int ncases, int n_node_items,
                              cudaStream_t st);
// fluid species (fluid.cu): the continuity sweeps, one warp per line, and the
// averaging cycle, one thread per node
struct FluidPlan {
    const int *xl_items = nullptr; // device prefix [n+1] of nfsp x lines per case (0 where held fixed)
    const int *yl_items = nullptr; // the same for the y lines
    int n_x = 0, n_y = 0;          // total line items
    int len_x = 0, len_y = 0;      // longest line in cells (ncx, ncy of the widest case)
    bool any = false;              // some case runs the fluid cycle
};
constexpr size_t FLUID_SMEM_MAX = 200 * 1024;
// warps per CTA of the sweep for lines of up to L cells (0: L too long)
int fluid_sweep_warps(int L);
cudaError_t launch_fluid(const DevCase *cases, const int *node_items, int ncases, int n_node_items,
                         const FluidPlan &fp, cudaStream_t st);
// The same split around the step's particle phases: the sweeps read only the
// fluid arrays (densities, fluxes, the sources of the last averaging cycle)
// and the step counter, and nothing between k_advance and the averaging cycle
// touches those arrays, so fluid_begin (right after k_advance) runs the
// sweeps on a side stream forked from st, concurrently with Field ... Deposit,
// and fluid_end (before the accumulation) joins it back and runs the
// averaging cycle.  Without a side stream, or while a per-kernel profile is
// recorded, fluid_begin does nothing and fluid_end runs launch_fluid.
struct FluidFork {
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
cudaError_t fluid_fork_create(FluidFork &f);
void fluid_fork_destroy(FluidFork &f);
cudaError_t fluid_begin(const DevCase *cases, int ncases, const FluidPlan &fp, const FluidFork &f, cudaStream_t st);
cudaError_t fluid_end(const DevCase *cases, const int *node_items, int ncases, int n_node_items, const FluidPlan &fp,
                      const FluidFork &f, cudaStream_t st);

} // namespace hp
