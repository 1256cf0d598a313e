// load.cu -- the initial particle load on the device (hp_case_opts.gpu_load).
//
// The same load as the host's (SetParticleLoad/Copy_HCPtoGCP,
// src/Particle.c:3-226, src/cuda_Particle.cu:28-58): loading cells in the
// reference's order, n particles per loading cell, five Park-Miller draws
// per particle (speed index, azimuth, polar cosine, x, y), the cell from the
// integer part of the position.  Particle k of a species starts at draw 5k,
// reached by jump-ahead (16807^5k mod 2^31-1), so every thread generates its
// own run of particles.  A draw of exactly 1.0f (seeds within 64 of 2^31-2)
// puts a particle on the next cell's edge: such "edge" particles are listed,
// the list is ordered on the host, and each particle's slot follows from it:
//   own particle of cell L: edges into L first, then L's own particles in
//     load order less those that left;
//   edge particle into D: after the edges into D with smaller k.
// These are the places the host's stable counting sort gives.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "capi_internal.hpp"

using namespace hp;

namespace {

constexpr uint32_t PM_M = 2147483647u;
constexpr int LOAD_RUN = 16;       // particles per thread (one jump-ahead each)
constexpr int EDGE_CAP = 4096;     // edge particles listed per species
constexpr int EDGE_SCAN_MAX = 256; // above this the host places the species

// a * b mod 2^31 - 1 for a, b < 2^31
__device__ __forceinline__ uint32_t pm_mul(uint32_t a, uint32_t b) {
    const uint64_t p = (uint64_t)a * b;
    uint64_t r = (p & PM_M) + (p >> 31);
    r = (r & PM_M) + (r >> 31);
    return (uint32_t)(r >= PM_M ? r - PM_M : r);
}

__device__ __forceinline__ uint32_t pm_skip_dev(uint32_t seed, uint64_t k) {
    uint32_t a = 16807u, r = 1u;
    while (k) {
        if (k & 1) r = pm_mul(r, a);
        a = pm_mul(a, a);
        k >>= 1;
    }
    return pm_mul(r, seed);
}

// ParkMiller::next: the next state, returned as (float)(seed / 2147483646.0)
__device__ __forceinline__ float pm_next(uint32_t &seed) {
    seed = pm_mul(16807u, seed);
    return (float)((double)seed / 2147483646.0);
}

struct LoadArgs {
    const int *lc;     // loading cells
    int npc;           // particles per loading cell
    long long np;
    uint32_t seed0;
    float vti;
    const float *vsave;
    int nvel, ncx, ncy;
    float *tmp;        // [5][np] in load order: offsets x, y, then vx, vy, vz
    int *dest;         // [np] cell of each particle
    int *edge_n;       // edge particles found
    long long *edge_k; // [EDGE_CAP]
};

constexpr double MPI_D = 3.14159265358979323846;

__global__ void k_load_gen(LoadArgs a) {
    const long long k0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * LOAD_RUN;
    if (k0 >= a.np) return;
    uint32_t q = pm_skip_dev(a.seed0, 5ull * (unsigned long long)k0);
    const long long k1 = k0 + LOAD_RUN < a.np ? k0 + LOAD_RUN : a.np;
    for (long long k = k0; k < k1; k++) {
        const int L = a.lc[k / a.npc];
        const int i = L / a.ncy, j = L - i * a.ncy;
        // maxwellv (src/Particle.c:203-209), in the host's arithmetic
        const int n = (int)((a.nvel - 1) * pm_next(q));
        const float aphi = (float)(2 * MPI_D * (double)pm_next(q));
        const float costheta = 1 - 2 * pm_next(q);
        const float sintheta = (float)sqrt((double)(1 - costheta * costheta));
        const float vs = a.vti * a.vsave[n];
        const float vx = (float)((double)(vs * sintheta) * cos((double)aphi));
        const float vy = (float)((double)(vs * sintheta) * sin((double)aphi));
        const float vz = (float)(vs * costheta);
        const float hx = (float)i + pm_next(q);
        const float hy = (float)j + pm_next(q);
        int XID = (int)hx, YID = (int)hy;
        float ox = hx - XID, oy = hy - YID;
        if (XID >= a.ncx) { XID = a.ncx - 1; ox = 0.99999994f; }
        if (YID >= a.ncy) { YID = a.ncy - 1; oy = 0.99999994f; }
        const int D = XID * a.ncy + YID;
        a.tmp[k] = ox;
        a.tmp[a.np + k] = oy;
        a.tmp[2 * a.np + k] = vx;
        a.tmp[3 * a.np + k] = vy;
        a.tmp[4 * a.np + k] = vz;
        a.dest[k] = D;
        if (D != L) {
            const int e = atomicAdd(a.edge_n, 1);
            if (e < EDGE_CAP) a.edge_k[e] = k;
        }
    }
}

struct PlaceArgs {
    const int *lc;
    int npc;
    long long np;
    const float *tmp;
    const int *dest;
    const long long *ek; // edge particles, ascending k
    const int *esrc, *edst;
    int ne;
    DevSpecies sp;
};

__global__ void k_load_place(PlaceArgs a) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.np) return;
    const int L = a.lc[k / a.npc];
    const int D = a.dest[k];
    int slot;
    if (D == L) {
        int in = 0, out_before = 0;
        for (int e = 0; e < a.ne; e++) {
            in += a.edst[e] == L;
            out_before += a.esrc[e] == L && a.ek[e] < k;
        }
        slot = in + (int)(k % a.npc) - out_before;
    } else {
        int before = 0;
        for (int e = 0; e < a.ne; e++) before += a.edst[e] == D && a.ek[e] < k;
        slot = before;
    }
    const size_t q = (size_t)D * a.sp.cap + (size_t)slot;
    a.sp.x[q] = a.tmp[k];
    a.sp.y[q] = a.tmp[a.np + k];
    a.sp.vx[q] = a.tmp[2 * a.np + k];
    a.sp.vy[q] = a.tmp[3 * a.np + k];
    a.sp.vz[q] = a.tmp[4 * a.np + k];
}

template <class T> struct DevBuf {
    T *p = nullptr;
    ~DevBuf() { cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc((void **)&p, sizeof(T) * std::max<size_t>(n, 1)); }
};

} // namespace

namespace hpi {

// Generates species isp of a case whose set-up deferred its load, straight
// into the slot pool, and sets the cell counts.
hp_status device_load(hp_case *c, int isp) {
    const Setup &s = c->s;
    const DevSpecies &sp = c->h.sp[isp];
    const std::vector<int> &lc = s.load_cells[isp];
    const int npc = s.load_npc[isp];
    const long long np = (long long)lc.size() * npc;
    std::vector<int> cnt((size_t)s.Csize, 0);
    if (np == 0) {
        if (cudaMemcpy(sp.cnt, cnt.data(), cnt.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
            return cuda_fail(cudaGetLastError(), "device load");
        return HP_OK;
    }
    DevBuf<int> d_lc, d_dest, d_en, d_esrc, d_edst;
    DevBuf<float> d_tmp;
    DevBuf<long long> d_ek;
    cudaError_t e;
    if ((e = d_lc.alloc(lc.size())) != cudaSuccess || (e = d_dest.alloc((size_t)np)) != cudaSuccess ||
        (e = d_en.alloc(1)) != cudaSuccess || (e = d_tmp.alloc(5 * (size_t)np)) != cudaSuccess ||
        (e = d_ek.alloc(EDGE_CAP)) != cudaSuccess || (e = d_esrc.alloc(EDGE_SCAN_MAX)) != cudaSuccess ||
        (e = d_edst.alloc(EDGE_SCAN_MAX)) != cudaSuccess)
        return cuda_fail(e, "device load buffers");
    if ((e = cudaMemcpy(d_lc.p, lc.data(), lc.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(d_en.p, 0, 4)) != cudaSuccess)
        return cuda_fail(e, "device load");
    LoadArgs a;
    a.lc = d_lc.p;
    a.npc = npc;
    a.np = np;
    a.seed0 = (uint32_t)s.load_seed[isp];
    a.vti = s.sp[isp].vti;
    a.vsave = c->h.vsave;
    a.nvel = s.nvel;
    a.ncx = s.ncx;
    a.ncy = s.ncy;
    a.tmp = d_tmp.p;
    a.dest = d_dest.p;
    a.edge_n = d_en.p;
    a.edge_k = d_ek.p;
    const long long runs = (np + LOAD_RUN - 1) / LOAD_RUN;
    k_load_gen<<<(unsigned)((runs + 255) / 256), 256>>>(a);
    int ne = 0;
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaMemcpy(&ne, d_en.p, 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "device load (generate)");
    // edge particles, ascending k, with their source and destination cells
    std::vector<long long> ek((size_t)std::min(ne, EDGE_CAP));
    std::vector<int> esrc(ek.size()), edst(ek.size());
    if (!ek.empty() && (e = cudaMemcpy(ek.data(), d_ek.p, ek.size() * 8, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "device load (edges)");
    std::sort(ek.begin(), ek.end());
    for (size_t q = 0; q < ek.size(); q++) {
        esrc[q] = lc[(size_t)(ek[q] / npc)];
        if ((e = cudaMemcpy(&edst[q], d_dest.p + ek[q], 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cuda_fail(e, "device load (edges)");
    }
    if (ne > EDGE_SCAN_MAX) {
        set_error("device load: " + std::to_string(ne) + " particles on cell edges; load this deck on the host");
        return HP_ERR_UNSUPPORTED;
    }
    for (int L : lc) cnt[(size_t)L] = npc;
    for (size_t q = 0; q < ek.size(); q++) {
        cnt[(size_t)esrc[q]]--;
        cnt[(size_t)edst[q]]++;
    }
    for (int cell = 0; cell < s.Csize; cell++)
        if (2 * cnt[(size_t)cell] > sp.cap) {
            set_error("cell " + std::to_string(cell) + " holds " + std::to_string(cnt[(size_t)cell]) +
                      " particles; the slot pool takes at most " + std::to_string(sp.cap / 2));
            return HP_ERR_CAPACITY;
        }
    DevBuf<long long> d_eks;
    if ((e = d_eks.alloc(ek.size())) != cudaSuccess) return cuda_fail(e, "device load buffers");
    if (!ek.empty() &&
        ((e = cudaMemcpy(d_eks.p, ek.data(), ek.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
         (e = cudaMemcpy(d_esrc.p, esrc.data(), esrc.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
         (e = cudaMemcpy(d_edst.p, edst.data(), edst.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess))
        return cuda_fail(e, "device load (edges)");
    PlaceArgs b;
    b.lc = d_lc.p;
    b.npc = npc;
    b.np = np;
    b.tmp = d_tmp.p;
    b.dest = d_dest.p;
    b.ek = d_eks.p;
    b.esrc = d_esrc.p;
    b.edst = d_edst.p;
    b.ne = (int)ek.size();
    b.sp = sp;
    k_load_place<<<(unsigned)((np + 255) / 256), 256>>>(b);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpy(sp.cnt, cnt.data(), cnt.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaDeviceSynchronize()) != cudaSuccess)
        return cuda_fail(e, "device load (place)");
    return HP_OK;
}

} // namespace hpi
