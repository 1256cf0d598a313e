// fluid.cu -- the fluid species (Ar*, the O2 metastables and O atoms): the
// continuity solve and the averaging cycle that feeds it.
//
// Per step, after Deposit, in the reference's order (src/cuda_main.cu:84-91):
//   1. from the step after the first average on, the continuity solve
//      (Solve_Continuity_eqn, src/cuda_Fluid.cu:34-167): per species an
//      implicit sweep along every x line of plasma cells (a tridiagonal system
//      per line, Thomas algorithm) and the x-face fluxes, then the same along
//      the y lines;
//   2. the diagnostic cycle (Diagnostic_Basic, src/cuda_Diagnostic.cu:268-330):
//      N_ave steps sum the electron density, the next one averages it and the
//      collision tallies into rates and sources (Average_*_MCC_rate,
//      *_Update_Source, src/cuda_Diagnostic.cu:548-743); from that step on
//      the cell densities are copied to the nodes each step
//      (Sync_Fluid_GFCtoGFG_forDen, src/cuda_Fluid.cu:321-339), where the
//      collisions read them, and for Ar the electron collision probability of
//      each cell follows (src/cuda_mccAr.cu:57-58).
//
// The sweep is sequential along a line, so a warp owns a line: its lanes
// build the system's four diagonals in shared memory (coalesced loads of the
// Gummel coefficients, densities and fluxes), one lane runs the elimination
// and back substitution, and the lanes write the densities and fluxes.  The
// float operations are those of the reference, in its order, so the result is
// bit-identical to a sequential CPU sweep.  The diagnostic is one thread per
// node: a node's source, its density copy and its cell's probability read and
// write only that node and that cell.
#include <cstdint>

#include "devutil.cuh"
#include "hp_fluid.h"
#include "hp_math.h"
#include "kernels.cuh"
#include "prof.cuh"

namespace hp {
namespace {

using dv::find_case;
using dv::FULL;

__device__ __forceinline__ bool fluid_running(const DevCase &d) { return d.fluid_on && d.nfsp > 0; }

// One warp per (case, species, line); DIR 0 an x line, 1 a y line.  Shared
// memory: 4 x L floats per warp (sub-, main and super-diagonal, right-hand
// side), the super-diagonal then holding gam and the right-hand side x.
template <int DIR>
__global__ void __launch_bounds__(128) k_fluid_sweep(const DevCase *__restrict__ cases,
                                                     const int *__restrict__ item_start, int ncases, int items,
                                                     int L) {
    extern __shared__ float sm[];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = (int)(blockIdx.x * (blockDim.x >> 5)) + wib;
    if (w >= items) return;
    const int ci = find_case(item_start, ncases, w);
    const DevCase &d = cases[ci];
    if (!fluid_running(d) || *d.tstep < (int64_t)d.n_ave + 2) return;
    const int nl = DIR ? d.nyl : d.nxl;
    const int n = w - item_start[ci];
    const int f = n / nl, k = n - f * nl;
    const int ngx = d.ngx, ngy = d.ngy, ncx = d.ncx, ncy = d.ncy, C = d.C;
    const int *Ln = (DIR ? d.fl_yl : d.fl_xl) + 3 * k;
    // x line: x1, x2, y; y line: x, y1, y2
    const int first = DIR ? Ln[1] : Ln[0], last = DIR ? Ln[2] : Ln[1], fixed = DIR ? Ln[0] : Ln[2];
    const int num = last - first + 1;
    const size_t fo = DIR ? (size_t)f * ncx * ngy : (size_t)f * ngx * ncy;
    const float *ga = (DIR ? d.gay : d.gax) + fo, *gb = (DIR ? d.gby : d.gbx) + fo;
    float *flux = (DIR ? d.ffly : d.fflx) + fo;
    const float *other = DIR ? d.fflx + (size_t)f * ngx * ncy : d.ffly + (size_t)f * ncx * ngy;
    float *den = d.fden + (size_t)f * C;
    const float *src = d.fsrc + (size_t)f * C;
    const float dtc = d.dtc, del_f = dtc / (DIR ? d.dy : d.dx), dother = DIR ? d.dx : d.dy;
    // faces and cells along the line, and the other direction's two faces of a cell
    auto face = [&](int q) { return DIR ? fixed * ngy + q : q * ncy + fixed; };
    auto cell = [&](int q) { return DIR ? fixed * ncy + q : q * ncy + fixed; };
    auto olo = [&](int q) { return DIR ? fixed * ncy + q : q * ngy + fixed; };
    auto ohi = [&](int q) { return DIR ? (fixed + 1) * ncy + q : q * ngy + fixed + 1; };
    float *A = sm + (size_t)wib * 4 * L, *B = A + L, *Cc = B + L, *D = Cc + L;
    for (int i = lane; i < num; i += 32) {
        const int q = i + first;
        A[i] = -ga[face(q)] * del_f;
        B[i] = 1 + (ga[face(q + 1)] + gb[face(q)]) * del_f;
        Cc[i] = -gb[face(q + 1)] * del_f;
        D[i] = den[cell(q)] + src[cell(q)] * dtc - (other[ohi(q)] - other[olo(q)]) * dtc / dother;
    }
    __syncwarp();
    int ok = 1;
    if (lane == 0) { // tridiag, src/cuda_Fluid.cu:168-184
        // The recurrences carry their last values in registers and the next
        // cell's coefficients are loaded one cell ahead, so the loop's chain
        // is the arithmetic alone (a shared-memory load per step otherwise:
        // the compiler cannot tell the four diagonals apart).  The float
        // operations and their order are the reference's.
        float bet = B[0];
        float dprev = D[0] / bet;
        D[0] = dprev;
        float c1 = Cc[0], a = 0.f, b = 0.f, dj = 0.f, cn = 0.f;
        if (num > 1) {
            a = A[1];
            b = B[1];
            dj = D[1];
            cn = Cc[1];
        }
        for (int j = 1; j < num; j++) {
            float an = 0.f, bn = 0.f, dn = 0.f, cnn = 0.f;
            if (j + 1 < num) {
                an = A[j + 1];
                bn = B[j + 1];
                dn = D[j + 1];
                cnn = Cc[j + 1];
            }
            const float gam = c1 / bet;
            const float nb = b - a * c1 / bet;
            dprev = (dj - a * dprev) / nb;
            D[j] = dprev;
            Cc[j - 1] = gam;
            bet = nb;
            if (bet == 0) {
                ok = 0;
                break;
            }
            c1 = cn;
            a = an;
            b = bn;
            dj = dn;
            cn = cnn;
        }
        if (ok && num > 1) {
            float xn = dprev, dk = D[num - 2], ck = Cc[num - 2];
            for (int j = num - 2; j >= 0; j--) {
                float dk1 = 0.f, ck1 = 0.f;
                if (j > 0) {
                    dk1 = D[j - 1];
                    ck1 = Cc[j - 1];
                }
                xn = dk - ck * xn;
                D[j] = xn;
                dk = dk1;
                ck = ck1;
            }
        }
    }
    ok = __shfl_sync(FULL, ok, 0);
    __syncwarp();
    if (!ok) return; // a vanishing pivot: the line keeps its state
    for (int i = lane; i < num; i += 32) {
        const int q = i + first;
        const float x = D[i];
        const float v = (d.plasma[cell(q)] == 1 && x > 1e9f) ? x : 0.0f;
        den[cell(q)] = v;
        B[i] = v;
    }
    __syncwarp();
    // Calculate_Flux_x / _y (src/cuda_Fluid.cu:54-95)
    const float *fg = DIR ? d.fl_yfg : d.fl_xfg;
    for (int i = lane; i <= num; i += 32) {
        const int q = i + first;
        if (i == 0) flux[face(first)] = -fg[(size_t)f * nl + k] * gb[face(first)] * B[0];
        else if (i == num) flux[face(last + 1)] = fg[(size_t)d.nfsp * nl + (size_t)f * nl + k] * ga[face(last + 1)] * B[num - 1];
        else flux[face(q)] = ga[face(q)] * B[i - 1] - gb[face(q)] * B[i];
    }
}

// The diagnostic cycle of one node (see the file comment).
__global__ void __launch_bounds__(256) k_fluid_diag(const DevCase *__restrict__ cases,
                                                    const int *__restrict__ item_start, int ncases, int items) {
    const int t = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (t >= items) return;
    const int ci = find_case(item_start, ncases, t);
    const DevCase &d = cases[ci];
    if (!fluid_running(d)) return;
    const int g = t - item_start[ci];
    const int N = d.n_ave;
    const int64_t per = (int64_t)N + 1, ts = *d.tstep;
    const int ph = (int)((ts - 1) % per);
    const int ngy = d.ngy, ncx = d.ncx, ncy = d.ncy, C = d.C, G = d.G, F = d.nfsp;
    const int i = g / ngy, j = g - i * ngy;
    const bool has_cell = i < ncx && j < ncy;
    const int cell = i * ncy + j;
    if (ph < N) {
        d.fl_sum[g] += d.den[g];
    } else {
        // Average_Particle_Density of the electrons, 0.25 x as the sources read it
        const float temp = d.denscale0 / (float)N;
        const float ave = temp * (float)(d.fl_sum[g] + d.den[g]);
        d.fl_sum[g] = 0.0;
        const float eden = (float)(0.25 * (double)ave);
        float R[96], S[5], nn[5];
        for (int ch = 0; ch < 96; ch++) R[ch] = 0.0f;
        if (has_cell) {
            const int st = d.mcc_stride;
            for (int ch = 0; ch < st && ch < d.tnrct; ch++) {
                const size_t q = (size_t)cell * st + ch;
                const unsigned now = d.mcc_count[q];
                R[ch] = d.rate_f[ch] * (float)(now - d.fl_base[q]);
                d.fl_base[q] = now;
            }
        }
        for (int f = 0; f < 5; f++) nn[f] = f < F ? d.fluid_den[(size_t)f * G + g] : 0.0f;
        const float bd1 = d.back_den1 ? d.back_den1[g] : 0.0f, bd2 = d.back_den2 ? d.back_den2[g] : 0.0f;
        hp_fluid_sources(d.gas, R, nn, bd1, bd2, eden, d.rr, S);
        if (has_cell)
            for (int f = 0; f < F; f++) d.fsrc[(size_t)f * C + cell] = S[f];
    }
    if (ts < per) return;
    // the node's density from its cell: (i, j) itself, or for the last row and
    // column of nodes the cell below-left; nodes (0, ncy) and (ncx, 0) have none
    int from = -1;
    if (has_cell) from = cell;
    else if (i == ncx && j >= 1) from = (ncx - 1) * ncy + (j - 1);
    else if (j == ncy && i >= 1) from = (i - 1) * ncy + (ncy - 1);
    if (from < 0) return;
    for (int f = 0; f < F; f++) d.fluid_den[(size_t)f * G + g] = d.fden[(size_t)f * C + from];
    if (d.gas == 0 && has_cell) {
        const float e = hp_expf(-1 * d.dt_mcc * d.sigv[1] * d.fluid_den[g]);
        d.prob[(size_t)C + cell] = d.prob[cell] + 1.0f - e;
    }
}

int blocks_for(int n, int per) { return (n + per - 1) / per; }

} // namespace

int fluid_sweep_warps(int L) {
    const size_t per_warp = (size_t)16 * (size_t)(L > 0 ? L : 1);
    int w = 4;
    while (w > 1 && per_warp * (size_t)w > FLUID_SMEM_MAX) w >>= 1;
    return per_warp > FLUID_SMEM_MAX ? 0 : w;
}

namespace {
cudaError_t launch_fluid_sweeps(const DevCase *cases, int ncases, const FluidPlan &fp, cudaStream_t st) {
    for (int dir = 0; dir < 2; dir++) {
        const int items = dir ? fp.n_y : fp.n_x, L = dir ? fp.len_y : fp.len_x;
        if (items <= 0) continue;
        const int w = fluid_sweep_warps(L);
        if (w == 0) return cudaErrorInvalidValue;
        const size_t smem = (size_t)w * 16 * (size_t)L;
        if (dir == 0) {
            if (smem > 48 * 1024) cudaFuncSetAttribute(k_fluid_sweep<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            prof::mark(st, "k_fluid_sweep_x");
            k_fluid_sweep<0><<<blocks_for(items, w), 32 * w, smem, st>>>(cases, fp.xl_items, ncases, items, L);
        } else {
            if (smem > 48 * 1024) cudaFuncSetAttribute(k_fluid_sweep<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            prof::mark(st, "k_fluid_sweep_y");
            k_fluid_sweep<1><<<blocks_for(items, w), 32 * w, smem, st>>>(cases, fp.yl_items, ncases, items, L);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_fluid_diag(const DevCase *cases, const int *node_items, int ncases, int n_node_items,
                              const FluidPlan &fp, cudaStream_t st) {
    if (fp.n_x > 0 || fp.n_y > 0 || fp.any) {
        prof::mark(st, "k_fluid_diag");
        k_fluid_diag<<<blocks_for(n_node_items, 256), 256, 0, st>>>(cases, node_items, ncases, n_node_items);
        return cudaGetLastError();
    }
    return cudaSuccess;
}

bool forked(const FluidPlan &fp, const FluidFork &f) { return f.side && !prof::g_on && (fp.n_x > 0 || fp.n_y > 0); }
} // namespace

cudaError_t launch_fluid(const DevCase *cases, const int *node_items, int ncases, int n_node_items,
                         const FluidPlan &fp, cudaStream_t st) {
    cudaError_t e = launch_fluid_sweeps(cases, ncases, fp, st);
    if (e != cudaSuccess) return e;
    return launch_fluid_diag(cases, node_items, ncases, n_node_items, fp, st);
}

cudaError_t fluid_fork_create(FluidFork &f) {
    cudaError_t e = cudaStreamCreateWithFlags(&f.side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f.join, cudaEventDisableTiming);
    if (e != cudaSuccess) fluid_fork_destroy(f);
    return e;
}

void fluid_fork_destroy(FluidFork &f) {
    if (f.side) {
        cudaStreamSynchronize(f.side);
        cudaStreamDestroy(f.side);
    }
    if (f.fork) cudaEventDestroy(f.fork);
    if (f.join) cudaEventDestroy(f.join);
    f = FluidFork();
}

cudaError_t fluid_begin(const DevCase *cases, int ncases, const FluidPlan &fp, const FluidFork &f, cudaStream_t st) {
    if (!forked(fp, f)) return cudaSuccess;
    cudaError_t e = cudaEventRecord(f.fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(f.side, f.fork, 0);
    if (e == cudaSuccess) e = launch_fluid_sweeps(cases, ncases, fp, f.side);
    if (e == cudaSuccess) e = cudaEventRecord(f.join, f.side);
    return e;
}

cudaError_t fluid_end(const DevCase *cases, const int *node_items, int ncases, int n_node_items, const FluidPlan &fp,
                      const FluidFork &f, cudaStream_t st) {
    if (!forked(fp, f)) return launch_fluid(cases, node_items, ncases, n_node_items, fp, st);
    cudaError_t e = cudaStreamWaitEvent(st, f.join, 0);
    if (e != cudaSuccess) return e;
    return launch_fluid_diag(cases, node_items, ncases, n_node_items, fp, st);
}

} // namespace hp
