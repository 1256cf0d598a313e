// load.cu -- the initial particle load on the device (hp_case_opts.gpu_load).
//
// The same load as the host's (SetParticleLoad/Copy_HCPtoGCP,
// src/Particle.c:3-226, src/cuda_Particle.cu:28-58): loading cells in the
// reference's order with their particle counts, five Park-Miller draws
// per particle (speed index, azimuth, polar cosine, x, y), the cell from the
// integer part of the position.  Particle k of a species starts at draw 5k,
// reached by jump-ahead (16807^5k mod 2^31-1), so every thread generates its
// own run of particles.  A position whose float sum i + r rounds up to i + 1
// (r within half an ulp of 1 at that magnitude, or a draw of exactly 1.0f)
// puts the particle in the next cell: such "edge" particles (about one in
// 10^5 on a 512-column grid) are listed, the list is ordered on the host, and
// every particle's slot follows from it:
//   own particle of cell L: edges into L first (they come from cells loaded
//     earlier), then L's own particles in load order less those that left;
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
constexpr int EDGE_CAP = 1 << 20;  // edge particles listed per species

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
    const long long *ls; // [cells + 1] first particle of each loading cell
    int nlc;
    long long np;
    uint32_t seed0;
    float vti;
    const float *vsave;
    int nvel, ncx, ncy;
    float *tmp;        // [5][np] in load order: offsets x, y, then vx, vy, vz
    int *dest;         // [np] cell of each particle
    int *edge_n;       // edge particles found
    long long *edge_k; // [EDGE_CAP]
    int *edge_d;       // [EDGE_CAP] their cells
};

constexpr double MPI_D = 3.14159265358979323846;

// the loading cell q with ls[q] <= k < ls[q + 1]
__device__ __forceinline__ int loading_cell(const long long *ls, int n, long long k) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (ls[mid] <= k) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_load_gen(LoadArgs a) {
    const long long k0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * LOAD_RUN;
    if (k0 >= a.np) return;
    uint32_t q = pm_skip_dev(a.seed0, 5ull * (unsigned long long)k0);
    const long long k1 = k0 + LOAD_RUN < a.np ? k0 + LOAD_RUN : a.np;
    int li = loading_cell(a.ls, a.nlc, k0);
    for (long long k = k0; k < k1; k++) {
        while (k >= a.ls[li + 1]) li++;
        const int L = a.lc[li];
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
            if (e < EDGE_CAP) {
                a.edge_k[e] = k;
                a.edge_d[e] = D;
            }
        }
    }
}

struct PlaceArgs {
    const int *lc;
    const long long *ls;
    int nlc;
    long long np;
    const float *tmp;
    const int *dest;
    const long long *ek; // edge particles, ascending k
    const int *eslot;    // the slot of each in its cell
    int ne;
    const int *in_n;     // [C] edges into the cell
    const int *out_first, *out_n; // [C] the cell's own edges: first index in ek, count
    DevSpecies sp;
};

__global__ void k_load_place(PlaceArgs a) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.np) return;
    const int li = loading_cell(a.ls, a.nlc, k);
    const int L = a.lc[li];
    const int D = a.dest[k];
    int slot;
    if (D == L) {
        int ob = 0; // own edges that left before k
        for (int e = a.out_first[L], e1 = e + a.out_n[L]; e < e1; e++) ob += a.ek[e] < k;
        slot = a.in_n[L] + (int)(k - a.ls[li]) - ob;
    } else {
        int lo = 0, hi = a.ne; // k is in ek: find it
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (a.ek[mid] <= k) lo = mid;
            else hi = mid;
        }
        slot = a.eslot[lo];
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
    const std::vector<long long> &ls = s.load_start[isp];
    const long long np = ls.empty() ? 0 : ls.back();
    std::vector<int> cnt((size_t)s.Csize, 0);
    if (np == 0) {
        if (cudaMemcpy(sp.cnt, cnt.data(), cnt.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
            return cuda_fail(cudaGetLastError(), "device load");
        return HP_OK;
    }
    DevBuf<int> d_lc, d_dest, d_en, d_ed;
    DevBuf<float> d_tmp;
    DevBuf<long long> d_ek, d_ls;
    cudaError_t e;
    if ((e = d_lc.alloc(lc.size())) != cudaSuccess || (e = d_ls.alloc(ls.size())) != cudaSuccess || (e = d_dest.alloc((size_t)np)) != cudaSuccess ||
        (e = d_en.alloc(1)) != cudaSuccess || (e = d_tmp.alloc(5 * (size_t)np)) != cudaSuccess ||
        (e = d_ek.alloc(EDGE_CAP)) != cudaSuccess || (e = d_ed.alloc(EDGE_CAP)) != cudaSuccess)
        return cuda_fail(e, "device load buffers");
    if ((e = cudaMemcpy(d_lc.p, lc.data(), lc.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d_ls.p, ls.data(), ls.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(d_en.p, 0, 4)) != cudaSuccess)
        return cuda_fail(e, "device load");
    LoadArgs a;
    a.lc = d_lc.p;
    a.ls = d_ls.p;
    a.nlc = (int)lc.size();
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
    a.edge_d = d_ed.p;
    const long long runs = (np + LOAD_RUN - 1) / LOAD_RUN;
    k_load_gen<<<(unsigned)((runs + 255) / 256), 256>>>(a);
    int ne = 0;
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaMemcpy(&ne, d_en.p, 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "device load (generate)");
    if (ne > EDGE_CAP) {
        set_error("device load: " + std::to_string(ne) + " particles on cell edges; load this deck on the host");
        return HP_ERR_UNSUPPORTED;
    }
    // edge particles in ascending k, their cells and their slots there
    std::vector<long long> ek((size_t)ne);
    std::vector<int> ed((size_t)ne);
    if (ne && ((e = cudaMemcpy(ek.data(), d_ek.p, ek.size() * 8, cudaMemcpyDeviceToHost)) != cudaSuccess ||
               (e = cudaMemcpy(ed.data(), d_ed.p, ed.size() * 4, cudaMemcpyDeviceToHost)) != cudaSuccess))
        return cuda_fail(e, "device load (edges)");
    std::vector<size_t> ord((size_t)ne);
    for (size_t q = 0; q < ord.size(); q++) ord[q] = q;
    std::sort(ord.begin(), ord.end(), [&](size_t u, size_t v) { return ek[u] < ek[v]; });
    std::vector<long long> eks((size_t)ne);
    std::vector<int> eslot((size_t)ne), in_n((size_t)s.Csize, 0), out_first((size_t)s.Csize, 0),
        out_n((size_t)s.Csize, 0);
    for (size_t q = 0; q < ord.size(); q++) {
        eks[q] = ek[ord[q]];
        const size_t li = (size_t)(std::upper_bound(ls.begin(), ls.end(), eks[q]) - ls.begin()) - 1;
        const int D = ed[ord[q]], L = lc[li];
        eslot[q] = in_n[(size_t)D]++;
        if (out_n[(size_t)L]++ == 0) out_first[(size_t)L] = (int)q;
    }
    for (size_t q = 0; q < lc.size(); q++) cnt[(size_t)lc[q]] = (int)(ls[q + 1] - ls[q]);
    for (int cell = 0; cell < s.Csize; cell++) {
        cnt[(size_t)cell] += in_n[(size_t)cell] - out_n[(size_t)cell];
        if (2 * cnt[(size_t)cell] > sp.cap) {
            set_error("cell " + std::to_string(cell) + " holds " + std::to_string(cnt[(size_t)cell]) +
                      " particles; the slot pool takes at most " + std::to_string(sp.cap / 2));
            return HP_ERR_CAPACITY;
        }
    }
    DevBuf<long long> d_eks;
    DevBuf<int> d_eslot, d_in, d_of, d_on;
    if ((e = d_eks.alloc(eks.size())) != cudaSuccess || (e = d_eslot.alloc(eslot.size())) != cudaSuccess ||
        (e = d_in.alloc(in_n.size())) != cudaSuccess || (e = d_of.alloc(out_first.size())) != cudaSuccess ||
        (e = d_on.alloc(out_n.size())) != cudaSuccess)
        return cuda_fail(e, "device load buffers");
    if ((ne && ((e = cudaMemcpy(d_eks.p, eks.data(), eks.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
                (e = cudaMemcpy(d_eslot.p, eslot.data(), eslot.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess)) ||
        (e = cudaMemcpy(d_in.p, in_n.data(), in_n.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d_of.p, out_first.data(), out_first.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d_on.p, out_n.data(), out_n.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "device load (edges)");
    PlaceArgs b;
    b.lc = d_lc.p;
    b.ls = d_ls.p;
    b.nlc = (int)lc.size();
    b.np = np;
    b.tmp = d_tmp.p;
    b.dest = d_dest.p;
    b.ek = d_eks.p;
    b.eslot = d_eslot.p;
    b.ne = ne;
    b.in_n = d_in.p;
    b.out_first = d_of.p;
    b.out_n = d_on.p;
    b.sp = sp;
    k_load_place<<<(unsigned)((np + 255) / 256), 256>>>(b);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpy(sp.cnt, cnt.data(), cnt.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaDeviceSynchronize()) != cudaSuccess)
        return cuda_fail(e, "device load (place)");
    return HP_OK;
}

} // namespace hpi
