// noalloc.cu -- the charge deposit with no device allocation in the call.
//
// hp_Deposit keeps its per-cell CIC corner sums in a buffer that the case
// allocated at creation.  Some callers cannot let a library allocate device
// memory at all: a host that owns every byte of the GPU through its own pool
// or budget (a serving process that admits work by memory footprint), or
// code that must not trigger cudaMalloc's implicit device synchronisation in
// a timed loop.  hp_Deposit_noalloc gives them the same densities with the
// corner sums in one fixed array compiled into the library (HP_NOALLOC_CELLS
// entries of 32 bytes, 16 MiB, resident on every GPU that loads the library
// until the process exits), and writes the result into the caller's buffer.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "capi_internal.hpp"

#define HP_NOALLOC_CELLS (1 << 19) /* species x cells the scratch array holds */

namespace {

// the shared scratch: one double4 (WS, WN, ES, EN) per (species, cell)
static __device__ __align__(256) double4 g_corner_scratch[HP_NOALLOC_CELLS];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double4 *g_scratch_ptr[kMaxDevices] = {nullptr};

__device__ __forceinline__ double warp_sum_na(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// per-cell corner sums, as k_deposit_cells: FP32 lane sums, FP64 warp tree
__global__ void __launch_bounds__(256) k_na_cells(const hp::DevCase *__restrict__ dc, double4 *__restrict__ scratch) {
    const hp::DevCase &d = *dc;
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= d.nsp * d.C) return;
    const int s = warp / d.C, c = warp - s * d.C;
    const hp::DevSpecies &sp = d.sp[s];
    const int n = sp.cnt[c];
    const size_t base = (size_t)c * sp.cap;
    float WS = 0.f, WN = 0.f, ES = 0.f, EN = 0.f;
    for (int k = lane; k < n; k += 32) {
        const float lx = sp.x[base + k], ly = sp.y[base + k];
        WS += (1 - lx) * (1 - ly);
        WN += (1 - lx) * ly;
        ES += lx * (1 - ly);
        EN += lx * ly;
    }
    const double a = warp_sum_na(WS), b = warp_sum_na(WN), e = warp_sum_na(ES), f = warp_sum_na(EN);
    if (lane == 0) scratch[warp] = make_double4(a, b, e, f);
}

// node gather and DepositBoundary scaling into the caller's den[nsp*Gsize]
__global__ void __launch_bounds__(256) k_na_nodes(const hp::DevCase *__restrict__ dc,
                                                  const double4 *__restrict__ scratch, double *__restrict__ den) {
    const hp::DevCase &d = *dc;
    const int n = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (n >= d.G) return;
    const int i = n / d.ngy, j = n - i * d.ngy, ncy = d.ncy;
    for (int s = 0; s < d.nsp; s++) {
        const double4 *cw = scratch + (size_t)s * d.C;
        double v = 0.0;
        if (i < d.ncx && j < ncy) v += cw[i * ncy + j].x;
        if (i < d.ncx && j > 0) v += cw[i * ncy + j - 1].y;
        if (i > 0 && j < ncy) v += cw[(i - 1) * ncy + j].z;
        if (i > 0 && j > 0) v += cw[(i - 1) * ncy + j - 1].w;
        den[(size_t)s * d.G + n] = v * (double)d.dep_factor[n];
    }
}

// Makes the case's device current for the call and puts the caller's back.
struct DeviceGuard {
    int prev = -1;
    cudaError_t set(int dev) {
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) {
            prev = -1;
            return e;
        }
        return prev == dev ? cudaSuccess : cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

} // namespace

extern "C" hp_status hp_Deposit_noalloc(hp_case *c, double *den_out, void *stream) {
    if (!c || !den_out) return hpi::set_error("null argument"), HP_ERR_ARG;
    // a batched case is stepped on the batch's stream; reading its pools here
    // would not be ordered after that step
    if (c->batch) return hpi::set_error("case belongs to a batch"), HP_ERR_ARG;
    if (c->s.N_smt > 0)
        return hpi::set_error("hp_Deposit_noalloc: the deck smooths its densities (DensitySmoothing); use hp_Deposit"),
               HP_ERR_UNSUPPORTED;
    const long long need = (long long)c->s.nsp * c->s.Csize;
    if (need > HP_NOALLOC_CELLS) {
        hpi::set_error("hp_Deposit_noalloc: the case has " + std::to_string(need) +
                       " species x cells; the fixed scratch holds " + std::to_string(HP_NOALLOC_CELLS));
        return HP_ERR_CAPACITY;
    }
    if (c->device < 0 || c->device >= kMaxDevices) return hpi::set_error("device ordinal too large"), HP_ERR_ARG;
    DeviceGuard guard;
    cudaError_t e = guard.set(c->device);
    if (e != cudaSuccess) return hpi::cuda_fail(e, "cudaSetDevice");
    cudaStream_t st = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return hpi::cuda_fail(e, "cudaStreamIsCapturing");
    double4 *scratch;
    {
        // The device address of the scratch array (its host-side name is not
        // a device address), looked up with the case's device current.  It is
        // looked up again on every call outside stream capture, so a context
        // that was torn down and recreated (cudaDeviceReset) is followed; a
        // call under capture uses the address of the last call outside it.
        std::lock_guard<std::mutex> lk(g_mu);
        if (cap == cudaStreamCaptureStatusNone) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_corner_scratch);
            if (e != cudaSuccess) return hpi::cuda_fail(e, "cudaGetSymbolAddress (deposit scratch)");
            g_scratch_ptr[c->device] = (double4 *)p;
        } else if (!g_scratch_ptr[c->device]) {
            return hpi::set_error("hp_Deposit_noalloc: the first call on a device must come before any stream capture"),
                   HP_ERR_ARG;
        }
        scratch = g_scratch_ptr[c->device];
    }
    const long long threads = need * 32;
    k_na_cells<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(c->d_case, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return hpi::cuda_fail(e, "hp_Deposit_noalloc cells");
    k_na_nodes<<<(unsigned)((c->s.Gsize + 255) / 256), 256, 0, st>>>(c->d_case, scratch, den_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return hpi::cuda_fail(e, "hp_Deposit_noalloc nodes");
    c->last_stream = st;
    return HP_OK;
}
