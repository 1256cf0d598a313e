// fastsolve.cu -- field_mode 2: FP64 iterative refinement whose inner solve
// applies the separable inverse of the symmetrised operator (fastsolve.cpp)
// as four dense products per pass, run as grouped FP32 GEMMs over all cases.
//
// One refinement pass for every case in the plan:
//   k_fs_resid   X = D^-1 (b - A x64) on the rectangle of unknowns (FP64 residual, FP32 out)
//   k_gemm x4    A1 = X V;  Y = (W^T A1) .* inv_eig;  A2 = Y V^T;  x64 += W A2
// and after the last pass k_fs_final + k_fs_norm write phi_Pois and the final
// relative residual.  Each output element of a product is accumulated in k order from
// zero with separate multiply and add roundings (the file is built with
// --fmad=false), so a CPU loop reproduces it exactly.
#include <cstdint>

#include "kernels.cuh"
#include "prof.cuh"

namespace hp {
namespace {

constexpr uint32_t ST_NOCONV = 0x4u, ST_NONFINITE = 0x2u;

__device__ __forceinline__ int find_le(const int *start, int n, int w) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (start[mid] <= w) lo = mid;
        else hi = mid;
    }
    return lo;
}

// residual of the symmetrised system on the rectangle, one thread per unknown
__global__ void __launch_bounds__(256) k_fs_resid(const DevCase *__restrict__ cases, const int *__restrict__ list,
                                                  const int *__restrict__ item_start, int n, int items) {
    const int t = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (t >= items) return;
    const int li = find_le(item_start, n, t);
    const DevCase &d = cases[list[li]];
    const int u = t - item_start[li];
    const int j = u / d.fs_nx, i = u - j * d.fs_nx;
    const int node = (d.fs_i0 + i) * d.ngy + (d.fs_j0 + j);
    const int G = d.G, ngy = d.ngy;
    const float *st = d.st;
    const double *v = d.x64;
    double ax = 0.0;
    const float cw = st[node], cs = st[G + node], cc = st[2 * G + node], cn = st[3 * G + node], ce = st[4 * G + node];
    if (cw != 0.0f) ax += (double)cw * v[node - ngy];
    if (cs != 0.0f) ax += (double)cs * v[node - 1];
    ax += (double)cc * v[node];
    if (cn != 0.0f) ax += (double)cn * v[node + 1];
    if (ce != 0.0f) ax += (double)ce * v[node + ngy];
    const double r64 = d.b64[node] - ax;
    d.fs_x[u] = (float)(r64 * (double)d.row_scale[node]);
}

// Grouped C = A B (row-major, contiguous) over a list of problems.  32x32
// output tile per CTA of 256 threads (2x2 outputs per thread: eight warps a
// tile, so that a single 511 x 255 case keeps ~1000 warps busy); 32-deep K
// slices staged in shared memory, the next slice fetched into registers while
// the current one is multiplied.  Each output is accumulated in k order from
// zero, whatever the tiling.
constexpr int GT = FS_TILE, GK = 32, GTHREADS = 256;
static_assert(GT == 32, "the thread layout assumes 32x32 tiles");

__global__ void __launch_bounds__(GTHREADS) k_gemm(const GemmProb *__restrict__ probs, int nprob) {
    int lo = 0, hi = nprob;
    const int t = (int)blockIdx.x;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (probs[mid].tile_start <= t) lo = mid;
        else hi = mid;
    }
    const GemmProb &P = probs[lo];
    const int lt = t - P.tile_start;
    const int tm = lt / P.tiles_n, tn = lt - tm * P.tiles_n;
    const int m0 = tm * GT, n0 = tn * GT;
    const int M = P.M, N = P.N, K = P.K;
    const float *__restrict__ A = P.A;
    const float *__restrict__ B = P.B;
    // As[k][m] (row stride 34 keeps float2 reads aligned, 2-way store conflicts)
    __shared__ __align__(16) float As[GK][GT + 2];
    __shared__ __align__(16) float Bs[GK][GT];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    // this thread's loads: rows tid/32 + 8q, column lane = tid & 31
    const int lr = tid >> 5, lc = tid & 31;
    float ra[4], rb[4];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int r = lr + 8 * q;
            const int gm = m0 + r, gk = k0 + lc;
            ra[q] = (gm < M && gk < K) ? A[(size_t)gm * K + gk] : 0.0f;
            const int gkb = k0 + r, gn = n0 + lc;
            rb[q] = (gkb < K && gn < N) ? B[(size_t)gkb * N + gn] : 0.0f;
        }
    };
    auto stage = [&]() {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int r = lr + 8 * q;
            As[lc][r] = ra[q];
            Bs[r][lc] = rb[q];
        }
    };
    float c00 = 0.0f, c01 = 0.0f, c10 = 0.0f, c11 = 0.0f;
    auto mac = [&](int kk) {
        const float2 av = *reinterpret_cast<const float2 *>(&As[kk][ty * 2]);
        const float2 bv = *reinterpret_cast<const float2 *>(&Bs[kk][tx * 2]);
        c00 = c00 + av.x * bv.x;
        c01 = c01 + av.x * bv.y;
        c10 = c10 + av.y * bv.x;
        c11 = c11 + av.y * bv.y;
    };
    fetch(0);
    stage();
    __syncthreads();
    for (int k0 = 0; k0 < K; k0 += GK) {
        const bool more = k0 + GK < K;
        if (more) fetch(k0 + GK);
        if (more) {
#pragma unroll
            for (int kk = 0; kk < GK; kk++) mac(kk);
        } else { // the last slice: exactly K - k0 terms, no padded ones
            const int kmax = K - k0;
            for (int kk = 0; kk < kmax; kk++) mac(kk);
        }
        __syncthreads();
        if (more) {
            stage();
            __syncthreads();
        }
    }
    const float cv[2][2] = {{c00, c01}, {c10, c11}};
#pragma unroll
    for (int a = 0; a < 2; a++) {
        const int gm = m0 + ty * 2 + a;
        if (gm >= M) continue;
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const int gn = n0 + tx * 2 + b;
            if (gn >= N) continue;
            const size_t o = (size_t)gm * N + gn;
            if (P.epi == 0) P.C[o] = cv[a][b];
            else if (P.epi == 1) P.C[o] = cv[a][b] * P.S[o];
            else P.x64[(size_t)(P.i0 + gn) * P.ngy + (P.j0 + gm)] += (double)cv[a][b];
        }
    }
}

// After the passes: phi_Pois on every node of the case and the relative
// residual ||b - A x64|| / ||b||.  k_fs_final: FS_CHUNK nodes per CTA, CTA
// partial sums (warp trees, warps in order) into fs_res[2 + 2*chunk];
// k_fs_norm: one warp per case adds the partials in a fixed order.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(256) k_fs_final(const DevCase *__restrict__ cases, const int *__restrict__ list) {
    const DevCase &d = cases[list[blockIdx.y]];
    const int G = d.G, ngy = d.ngy;
    const int n0 = (int)blockIdx.x * FS_CHUNK;
    if (n0 >= G) return;
    const int n1 = min(G, n0 + FS_CHUNK);
    const float *st = d.st;
    const double *v = d.x64;
    double rr = 0.0, bb = 0.0;
    for (int node = n0 + (int)threadIdx.x; node < n1; node += blockDim.x) {
        const float cc = st[2 * G + node];
        if (cc == 0.0f) {
            d.phi_p[node] = 0.0f;
            continue;
        }
        d.phi_p[node] = (float)v[node];
        double ax = 0.0;
        const float cw = st[node], cs = st[G + node], cn = st[3 * G + node], ce = st[4 * G + node];
        if (cw != 0.0f) ax += (double)cw * v[node - ngy];
        if (cs != 0.0f) ax += (double)cs * v[node - 1];
        ax += (double)cc * v[node];
        if (cn != 0.0f) ax += (double)cn * v[node + 1];
        if (ce != 0.0f) ax += (double)ce * v[node + ngy];
        const double r = d.b64[node] - ax;
        rr += r * r;
        bb += d.b64[node] * d.b64[node];
    }
    __shared__ double s_r[8], s_b[8];
    rr = warp_sum(rr);
    bb = warp_sum(bb);
    if ((threadIdx.x & 31) == 0) {
        s_r[threadIdx.x >> 5] = rr;
        s_b[threadIdx.x >> 5] = bb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { a += s_r[w]; b += s_b[w]; }
        d.fs_res[2 + 2 * blockIdx.x] = a;
        d.fs_res[3 + 2 * blockIdx.x] = b;
    }
}

__global__ void __launch_bounds__(32) k_fs_norm(const DevCase *__restrict__ cases, const int *__restrict__ list) {
    const DevCase &d = cases[list[blockIdx.x]];
    const int nch = (d.G + FS_CHUNK - 1) / FS_CHUNK;
    double a = 0.0, b = 0.0;
    for (int k = (int)threadIdx.x; k < nch; k += 32) {
        a += d.fs_res[2 + 2 * k];
        b += d.fs_res[3 + 2 * k];
    }
    a = warp_sum(a);
    b = warp_sum(b);
    if (threadIdx.x == 0) {
        d.fs_res[0] = sqrt(a);
        d.fs_res[1] = sqrt(b);
        d.pcg_iters[0] = d.fs_passes;
        d.pcg_iters[1] = d.fs_passes;
        if (!(a == a) || isinf(a)) atomicOr(d.status, ST_NONFINITE);
        else if (b > 0.0 && sqrt(a) > 10.0 * d.pcg_rtol * sqrt(b)) atomicOr(d.status, ST_NOCONV);
    }
}

inline unsigned nblocks(long long threads, int per) { return (unsigned)((threads + per - 1) / per); }

} // namespace

cudaError_t launch_fast_field(const DevCase *cases, const FastPlan &fp, cudaStream_t st) {
    if (fp.n <= 0) return cudaSuccess;
    for (int pass = 0; pass < fp.passes; pass++) {
        prof::mark(st, "k_fs_resid");
        k_fs_resid<<<nblocks(fp.items, 256), 256, 0, st>>>(cases, fp.list, fp.item_start, fp.n, fp.items);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        for (int s = 0; s < 4; s++) {
            prof::mark(st, "k_gemm");
            k_gemm<<<(unsigned)fp.ntiles[s], GTHREADS, 0, st>>>(fp.probs[s], fp.n);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    prof::mark(st, "k_fs_final");
    k_fs_final<<<dim3((unsigned)fp.final_chunks, (unsigned)fp.n), 256, 0, st>>>(cases, fp.list);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    prof::mark(st, "k_fs_norm");
    k_fs_norm<<<(unsigned)fp.n, 32, 0, st>>>(cases, fp.list);
    return cudaGetLastError();
}

} // namespace hp
