// kernels.cu -- sm_100a kernels of one PIC/MCC step, batched over cases.
//
// Work mapping: the particle kernels give one warp to one (case, species,
// cell); the slots of a cell are contiguous, so each warp access is one or
// more full 128-byte lines.  The grid kernels give one thread to one node.
// The Poisson solve runs one thread-block cluster per case and keeps the
// whole CG iteration inside one launch, with cluster barriers between the
// phases and cluster-wide (DSMEM) reductions of the dot products.
//
// Floating-point contract: this file is compiled with --fmad=false so that
// every a*b+c is two roundings, exactly as the CPU checker evaluates it; the
// elementary functions come from hp_math.h, identical on host and device.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdint>

#include "devutil.cuh"
#include "hp_math.h"
#include "hp_rng.h"
#include "kernels.cuh"
#include "prof.cuh"

namespace cg = cooperative_groups;

namespace hp {
namespace {

using namespace dv;

struct MoverFate {
    int fi, fj;
    bool absorbed, flipx, flipy;
    int cond; // conductor index, -2 - (di+1)*3 - (dj+1) on a dielectric, else -1
};

// The geometry a crossing needs, held in registers by the caller: the
// particle stores of Move could alias the case descriptor as far as the
// compiler knows, so fields read through it would be re-loaded after every
// store.
struct Geo {
    const int *__restrict__ sidx;
    int ncx, ncy, move_mode;
};
__device__ __forceinline__ Geo geo_of(const DevCase &d) { return Geo{d.sidx, d.ncx, d.ncy, d.move_mode}; }

__device__ __forceinline__ MoverFate mover_fate(const Geo d, int si, int sj, int di, int dj) {
    MoverFate f;
    f.fi = si + di;
    f.fj = sj + dj;
    f.absorbed = false;
    f.flipx = f.flipy = false;
    f.cond = -1;
    const int S = d.sidx[(si + 1 + di) * (d.ncy + 2) + (sj + 1 + dj)];
    switch (S) {
    case 0: break;
    case -2: f.fi += 1; f.flipx = true; break;
    case -6: f.fi -= 1; f.flipx = true; break;
    case -4: f.fj += 1; f.flipy = true; break;
    case -8: f.fj -= 1; f.flipy = true; break;
    case -12: f.fi += 1; f.fj += 1; f.flipx = f.flipy = true; break;
    case -16: f.fi -= 1; f.fj += 1; f.flipx = f.flipy = true; break;
    case -20: f.fi += 1; f.fj -= 1; f.flipx = f.flipy = true; break;
    case -24: f.fi -= 1; f.fj -= 1; f.flipx = f.flipy = true; break;
    default:
        f.absorbed = true;
        if (S >= 100) f.cond = S - 101;
        else if (S >= 1) f.cond = -2 - ((di + 1) * 3 + (dj + 1));
        break;
    }
    if (!f.absorbed && (f.fi < 0 || f.fi >= d.ncx || f.fj < 0 || f.fj >= d.ncy)) f.absorbed = true;
    return f;
}

// One share of a particle's weight on a dielectric surface node, in fixed
// point.  A share that is not finite or not below 2^20 in magnitude (a
// crossing with a vanishing velocity component) is dropped, as is a node
// outside the grid (the reference's index would reach another species' or
// no array there).
__device__ __forceinline__ void surface_add(long long *sig, int G, int s, int node, float w) {
    if (node < 0 || node >= G || !(fabsf(w) < 1048576.0f)) return;
    const long long q = __float2ll_rn(w * (float)(1 << HP_SIGMA_FRAC_BITS));
    atomicAdd((unsigned long long *)&sig[(size_t)s * G + node], (unsigned long long)q);
}

// A particle that entered a dielectric cell: Move queues the crossing and
// the Sort phase applies it (surface_split), as the reference's Move leaves
// the mover for SortBoundary.  The queue keeps Move's register budget: two
// stores on this rare path instead of the split's arithmetic.
__device__ __noinline__ void surface_enqueue(const DevCase &d, int s, int i, int j, int dir, float x, float y,
                                             float vx, float vy) {
    const int q = atomicAdd(d.dq_n, 1);
    if (q >= d.dq_cap) {
        atomicOr(d.status, ST_SURFACE);
        return;
    }
    d.dq_k[q] = ((i * d.ncy + j) << 7) | (s << 4) | dir;
    d.dq_v[q] = make_float4(x, y, vx, vy);
}

// SortBoundary's dielectric branch (src/cuda_Sortboundary.cu:93-207): a
// particle that entered a dielectric cell from cell (i, j) in direction dir
// = (di+1)*3 + (dj+1) leaves its weight on the two nodes of the face it
// crossed, split linearly by where it crossed.  (x, y) is its offset after
// the wrap, in the frame of the cell entered; for a diagonal crossing the
// cell passed first decides the face when it is not plasma.  The node
// arithmetic is the reference's, on the flat node index, including its
// choice of node for the lower-left diagonal (CID where the face's node is
// CID+1).
__device__ __forceinline__ void surface_split(const DevCase &d, int s, int i, int j, int dir, float x, float y, float vx,
                                           float vy) {
    const int ngy = d.ngy, SY = d.ncy + 2;
    const int di = dir / 3 - 1, dj = dir % 3 - 1;
    const int T = i * ngy + j, C = T + di * ngy + dj;
    const int g = (i + 1 + di) * SY + (j + 1 + dj);
    const int *SI = d.sidx;
    int pa = 0, pb = 0;
    float a = 0.0f, b = 0.0f, delta;
    switch (dir) {
    case 5: delta = x - vx / vy * y; pa = C; a = 1 - delta; pb = C + ngy; b = delta; break;
    case 3: delta = x + vx / vy * (1 - y); pa = T; a = 1 - delta; pb = T + ngy; b = delta; break;
    case 7: delta = y - vy / vx * x; pa = C; a = 1 - delta; pb = C + 1; b = delta; break;
    case 1: delta = y + vy / vx * (1 - x); pa = T; a = 1 - delta; pb = T + 1; b = delta; break;
    case 8:
        delta = x - vx / vy * y;
        if (delta >= 0) {
            if (SI[g - 1]) { delta = y - vy / vx * x; pa = C - 1; a = -delta; pb = C; b = 1 + delta; }
            else { pa = C; a = 1 - delta; pb = C + ngy; b = delta; }
        } else {
            if (SI[g - SY]) { pa = T + 1; a = -delta; pb = C; b = 1 + delta; }
            else { delta = y - vy / vx * x; pa = C; a = 1 - delta; pb = C + 1; b = delta; }
        }
        break;
    case 6:
        delta = x + vx / vy * (1 - y);
        if (delta >= 0) {
            if (SI[g + 1]) { delta = y - vy / vx * x; pa = C + 1; a = 2 - delta; pb = C + 2; b = delta - 1; }
            else { pa = C + 1; a = 1 - delta; pb = C + 1 + ngy; b = delta; }
        } else {
            if (SI[g - SY]) { pa = T; a = -delta; pb = C + 1; b = 1 + delta; }
            else { delta = y - vy / vx * x; pa = C; a = 1 - delta; pb = C + 1; b = delta; }
        }
        break;
    case 2:
        delta = x - vx / vy * y;
        if (delta < 1) {
            if (SI[g - 1]) { delta = y + vy / vx * (1 - x); pa = C + ngy - 1; a = -delta; pb = C + ngy; b = 1 + delta; }
            else { pa = C; a = 1 - delta; pb = C + ngy; b = delta; }
        } else {
            if (SI[g + SY]) { pa = T + 1; a = 2 - delta; pb = T + 1 + ngy; b = delta - 1; }
            else { delta = y + vy / vx * (1 - x); pa = T + 1; a = 1 - delta; pb = T + 2; b = delta; }
        }
        break;
    case 0:
        delta = x + vx / vy * (1 - y);
        if (delta < 1) {
            if (SI[g + 1]) { delta = y + vy / vx * (1 - x); pa = T; a = 2 - delta; pb = T + 1; b = delta - 1; }
            else { pa = C; a = 1 - delta; pb = T; b = delta; }
        } else {
            if (SI[g + SY]) { pa = T; a = 2 - delta; pb = T + ngy; b = delta - 1; }
            else { delta = y + vy / vx * (1 - x); pa = T - 1; a = 1 - delta; pb = T; b = delta; }
        }
        break;
    default: return;
    }
    surface_add(d.sig, d.G, s, pa, a);
    surface_add(d.sig, d.G, s, pb, b);
}

constexpr int CODE_FAR = 14, CODE_ABSORBED = 15;
// far movers a destination cell accepts per step (per species)
constexpr int FAR_B = HP_FAR_BUCKET;
constexpr int FAR_W = FAR_B / 32; // bucket keys per lane when a warp sorts a bucket
constexpr int FAR_LANE = 8;       // buckets up to this size are finished by one lane
static_assert(FAR_B % 32 == 0, "far buckets hold whole warps of keys");

// Where a particle that left cell (i, j) ends.  Each crossing wraps the
// offset by one cell (src/cuda_Move.cu:227-255) and applies the rule of the
// ghost code of the cell entered (mover_fate), flipping the offset and the
// velocity on a Neumann wall.  move_mode 0 stops after the first crossing as
// the reference does (its multi-cell loop, src/cuda_Move.cu:247-253, is
// commented out, so a particle faster than one cell per step keeps an offset
// outside [0,1)); move_mode 1 crosses until the offset is back in [0,1).
// Returns 0 when the particle stays in the domain, 1 when absorbed, 2 when the
// crossing bound was hit (absorbed and flagged).
__device__ __forceinline__ int walk(const Geo d, int &i, int &j, float &lx, float &ly, float &vx, float &vy,
                                    int &cond) {
    const int maxs = d.move_mode ? 2 * (d.ncx + d.ncy) + 4 : 1;
    for (int s = 0; s < maxs; s++) {
        // the reference computes these in double and rounds back to float;
        // for float operands a -+ 1 is exact in double, so the single
        // float operation rounds the same exact value to the same result
        int di = 0, dj = 0;
        if (ly >= 1) { dj = 1; ly = ly - 1.0f; }
        else if (ly < 0) { dj = -1; ly = ly + 1.0f; }
        if (lx >= 1) { di = 1; lx = lx - 1.0f; }
        else if (lx < 0) { di = -1; lx = lx + 1.0f; }
        const MoverFate f = mover_fate(d, i, j, di, dj);
        if (f.absorbed) {
            cond = f.cond;
            return 1;
        }
        if (f.flipx) { lx = 1 - lx; vx = -1 * vx; }
        if (f.flipy) { ly = 1 - ly; vy = -1 * vy; }
        // a particle that reaches a wall exactly (offset 0 after the wrap) flips
        // to offset 1, the wall itself, which no cell holds: keep it just inside
        // (move_mode 0 keeps offset 1, as the reference does)
        if (d.move_mode) {
            if (f.flipx && lx == 1) lx = 0x1.fffffep-1f;
            if (f.flipy && ly == 1) ly = 0x1.fffffep-1f;
        }
        i = f.fi;
        j = f.fj;
        if (!(ly >= 1 || ly < 0 || lx >= 1 || lx < 0)) return 0;
    }
    if (d.move_mode) {
        cond = -1;
        return 2;
    }
    return 0;
}

// asynchronous global -> shared copies (LDGSTS): 4 bytes per lane, committed
// per chunk; a lane waits for its own groups and reads only what it copied
__device__ __forceinline__ void cp_async4(float *smem, const float *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(float *smem, const float *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ------------------------------------------------------------------ Move
// MoveE_Basic (src/cuda_Move.cu:181-270): bilinear gather of the node field,
// v += Ascale E, x += v dt/dx in cell units (the reference's sums of
// products, built with contraction, evaluated here as bilinear weights and
// explicit fused multiply-adds).  A particle that leaves its
// cell is resolved here (walk), including the boundary rules the reference
// applies in SortBoundary.  Stayers are compacted in place (order kept);
// movers are parked at the top of the cell's slots, r-th mover at slot
// cap-1-r, with a code: the destination (di+1)*3 + (dj+1) when it lies in the
// 3x3 neighbourhood, CODE_FAR beyond it (also listed in the destination's
// bucket as source<<18 | r), CODE_ABSORBED when it left
// the domain.
// The particle loads are asynchronous copies into a ring of R chunk slots per
// warp in shared memory, so that R - 1 chunks of every warp are in flight
// without holding registers.  vz is copied with the other arrays and written
// back only where the slot changes: a per-particle load of it where needed
// measured 4 % slower on the 257x129 case (148 vs 142 us) than the extra
// 4 bytes per particle.
constexpr int MOVE_RING = 4;

template <int R>
__global__ void __launch_bounds__(512) k_move(const DevCase *__restrict__ cases,
                                                   const int *__restrict__ item_start, int ncases, int items) {
    extern __shared__ float move_ring_s[];
    __shared__ int dc_s[16][12]; // at most 16 warps per block (512 threads)
    float *ring = move_ring_s + (threadIdx.x >> 5) * (R * 5 * 32);
    int *dc = dc_s[threadIdx.x >> 5];
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= items) return;
    const int ci = find_case(item_start, ncases, warp);
    const DevCase &d = cases[ci];
    const int w = warp - item_start[ci];
    const int s = w / d.C, c = w - s * d.C;
    const DevSpecies &sp = d.sp[s];
    const int cap = sp.cap;
    const size_t base = (size_t)c * cap;
    const int i = c / d.ncy, j = c - i * d.ncy;
    const int node = i * d.ngy + j;
    // the count, the cell's field corners and the first chunk are independent
    // loads: issue them together (slots 0..31 of a cell are always inside the
    // pool, cap >= 32; lanes past the count are ignored)
    const int n = sp.cnt[c];
    const float ex_ws = d.Ex[node], ex_wn = d.Ex[node + 1], ex_es = d.Ex[node + d.ngy], ex_en = d.Ex[node + d.ngy + 1];
    const float ey_ws = d.Ey[node], ey_wn = d.Ey[node + 1], ey_es = d.Ey[node + d.ngy], ey_en = d.Ey[node + d.ngy + 1];
    // chunk q of the cell (all 32 slots: k0 + 32 <= cap, as cap is a multiple
    // of 32 and k0 < n <= cap) goes to ring slot q % R as 16-byte copies: lanes
    // 0-7 x, 8-15 y, 16-23 vx, 24-31 vy, then lanes 0-7 vz; one commit group
    // per chunk (possibly empty)
    const float *arr4 = lane < 8 ? sp.x : lane < 16 ? sp.y : lane < 24 ? sp.vx : sp.vy;
    auto issue = [&](int k0, int lim) {
        float *sl = ring + ((k0 >> 5) % R) * 160;
        if (k0 < lim) {
            cp_async16(sl + 4 * lane, arr4 + base + k0 + 4 * (lane & 7));
            if (lane < 8) cp_async16(sl + 128 + 4 * lane, sp.vz + base + k0 + 4 * lane);
        }
        cp_async_commit();
    };
    issue(0, 32); // slots 0..31 of a cell are always inside the pool (cap >= 32)
    // an interior cell whose 3x3 neighbourhood is all plasma (ghost code 0):
    // a particle that ends in a neighbour after one wrap needs no walk
    const int g3 = lane < 9 ? d.sidx[(i + lane / 3) * (d.ncy + 2) + (j + lane % 3)] : 0;
    const bool open3 = __ballot_sync(FULL, g3 != 0) == 0u && i >= 1 && i + 1 < d.ncx && j >= 1 && j + 1 < d.ncy;
    if (n == 0) {
        cp_async_wait_all();
        if (lane == 0) sp.nmov[c] = 0;
        if (lane < 9) sp.dcount[(size_t)c * 9 + lane] = 0;
        return;
    }
    if (lane == 0) atomicAdd(&d.pushes[warp & 31], (unsigned long long)n);
    if (2 * n > cap) { // the reference's ReArg condition (src/cuda_Sortboundary.cu:63-65)
        if (lane == 0) {
            sp.nmov[c] = 0;
            atomicOr(d.status, ST_OVERFLOW);
        }
        if (lane < 9) sp.dcount[(size_t)c * 9 + lane] = 0;
        cp_async_wait_all();
        return;
    }
#pragma unroll
    for (int q = 1; q < R - 1; q++) issue(q * 32, n);
    const float As = sp.Ascale, dtdx = d.dt_dx, dtdy = d.dt_dy;
    const unsigned lt = lanemask_lt();
    int m = 0, shifted = 0;
    // movers per destination code, counted in shared memory
    if (lane < 9) dc[lane] = 0;
    __syncwarp();
    // R - 1 chunks in flight while one is pushed (stores only go to slots at
    // or below the current chunk, or to the top region at or above
    // cap - n >= n, so no slot still to be copied is touched)
    for (int k0 = 0; k0 < n; k0 += 32) {
        const int k = k0 + lane;
        const bool act = k < n;
        issue(k0 + (R - 1) * 32, n);
        cp_async_wait<R - 1>();
        __syncwarp(); // the chunk was copied by eight lanes per array
        const float *sl = ring + ((k0 >> 5) % R) * 160;
        float lx = sl[lane], ly = sl[32 + lane], vx = sl[64 + lane], vy = sl[96 + lane];
        const float vz = sl[128 + lane];
        // bilinear weights once, then fused multiply-adds (one rounding each)
        const float wx = 1 - lx, wy = 1 - ly;
        const float w00 = wx * wy, w01 = wx * ly, w10 = lx * wy, w11 = lx * ly;
        const float del_vx = __fmaf_rn(ex_en, w11, __fmaf_rn(ex_es, w10, __fmaf_rn(ex_wn, w01, ex_ws * w00)));
        const float del_vy = __fmaf_rn(ey_en, w11, __fmaf_rn(ey_es, w10, __fmaf_rn(ey_wn, w01, ey_ws * w00)));
        float mvX = __fmaf_rn(del_vx, As, vx);
        float mvY = __fmaf_rn(del_vy, As, vy);
        lx = __fmaf_rn(mvX, dtdx, lx);
        ly = __fmaf_rn(mvY, dtdy, ly);
        const bool out = act && (ly >= 1 || ly < 0 || lx >= 1 || lx < 0);
        int code = 4, fi = i, fj = j;
        bool near = false;
        if (out && open3) { // the walk's first crossing with ghost code 0: a wrap, no flip
            // (lx - (float)di is lx - 1, lx + 1 or lx, exactly the walk's wrap)
            const int dj = (int)(ly >= 1) - (int)(ly < 0), di = (int)(lx >= 1) - (int)(lx < 0);
            const float wy = ly - (float)dj, wx = lx - (float)di;
            if (!(wy >= 1 || wy < 0 || wx >= 1 || wx < 0)) {
                lx = wx;
                ly = wy;
                code = 3 * di + dj + 4;
                near = true;
            }
        }
        if (out && !near) {
            int cond = -1;
            const int r = walk(geo_of(d), fi, fj, lx, ly, mvX, mvY, cond);
            if (r) {
                code = CODE_ABSORBED;
                if (cond >= 0 && cond < d.cond_numr) {
                    atomicAdd(&d.cond_charge[s * d.cond_numr + cond], 1.0f);
                    if (d.cond_step) atomicAdd(&d.cond_step[s * d.cond_numr + cond], 1u);
                } else if (cond <= -2 && d.sig) {
                    surface_enqueue(d, s, fi, fj, -2 - cond, lx, ly, mvX, mvY);
                }
                if (r == 2) atomicOr(d.status, ST_WALK);
            } else {
                const int ddi = fi - i, ddj = fj - j;
                code = (ddi >= -1 && ddi <= 1 && ddj >= -1 && ddj <= 1) ? (ddi + 1) * 3 + (ddj + 1) : CODE_FAR;
            }
        }
        if (out && code < 9) atomicAdd(&dc[code], 1);
        const unsigned bout = __ballot_sync(FULL, out);
        const int before = m + __popc(bout & lt);
        const bool moved = act && (out || before != 0); // its slot changes
        shifted += __popc(__ballot_sync(FULL, moved));
        __syncwarp(); // every lane's loads of this chunk precede the in-place stores
        if (act) {
            const size_t dst = out ? base + (size_t)(cap - 1 - before) : base + (size_t)(k - before);
            sp.x[dst] = lx;
            sp.y[dst] = ly;
            sp.vx[dst] = mvX;
            sp.vy[dst] = mvY;
            if (moved) sp.vz[dst] = vz;
            if (out) sp.code[dst] = (int8_t)code;
            if (code == CODE_FAR) {
                const size_t b = (size_t)s * d.C + (size_t)(fi * d.ncy + fj);
                const int q = atomicAdd(&d.far_in[b], 1);
                if (q < FAR_B)
                    d.far_key[b * FAR_B + q] = ((unsigned long long)c << 18) | (unsigned long long)before;
                else
                    atomicOr(d.status, ST_OVERFLOW);
            }
        }
        m += __popc(bout);
    }
    cp_async_wait_all();
    if (lane == 0) {
        sp.cnt[c] = n - m;
        sp.nmov[c] = m;
        atomicAdd(&d.pushes[32 + (warp & 31)], (unsigned long long)shifted);
    }
    __syncwarp();
    if (lane < 9) sp.dcount[(size_t)c * 9 + lane] = dc[lane];
}

// The same push with U chunks of 32 particles loaded per iteration before
// any of them is pushed (5*U independent loads in flight per lane instead of
// a one-chunk prefetch).  In-place stores of a chunk only reach slots at or
// below it, and all U chunks are loaded before the first store of the
// iteration, so no unread slot is overwritten.  Results, slot order, codes
// and counts are identical to k_move's.
template <int U>
__global__ void __launch_bounds__(512) k_move_u(const DevCase *__restrict__ cases, const int *__restrict__ item_start,
                                                int ncases, int items) {
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= items) return;
    const int ci = find_case(item_start, ncases, warp);
    const DevCase &d = cases[ci];
    const int w = warp - item_start[ci];
    const int s = w / d.C, c = w - s * d.C;
    const DevSpecies &sp = d.sp[s];
    const int n = sp.cnt[c];
    if (n == 0) {
        if (lane == 0) sp.nmov[c] = 0;
        if (lane < 9) sp.dcount[(size_t)c * 9 + lane] = 0;
        return;
    }
    if (lane == 0) atomicAdd(&d.pushes[warp & 31], (unsigned long long)n);
    const int cap = sp.cap;
    if (2 * n > cap) { // the reference's ReArg condition (src/cuda_Sortboundary.cu:63-65)
        if (lane == 0) {
            sp.nmov[c] = 0;
            atomicOr(d.status, ST_OVERFLOW);
        }
        if (lane < 9) sp.dcount[(size_t)c * 9 + lane] = 0;
        return;
    }
    const int i = c / d.ncy, j = c - i * d.ncy;
    const int node = i * d.ngy + j;
    const float ex_ws = d.Ex[node], ex_wn = d.Ex[node + 1], ex_es = d.Ex[node + d.ngy], ex_en = d.Ex[node + d.ngy + 1];
    const float ey_ws = d.Ey[node], ey_wn = d.Ey[node + 1], ey_es = d.Ey[node + d.ngy], ey_en = d.Ey[node + d.ngy + 1];
    const float As = sp.Ascale, dtdx = d.dt_dx, dtdy = d.dt_dy;
    const size_t base = (size_t)c * cap;
    float *__restrict__ px = sp.x + base;
    float *__restrict__ py = sp.y + base;
    float *__restrict__ pvx = sp.vx + base;
    float *__restrict__ pvy = sp.vy + base;
    float *__restrict__ pvz = sp.vz + base;
    const unsigned lt = lanemask_lt();
    int m = 0, shifted = 0;
    unsigned long long pk0 = 0, pk1 = 0, pk2 = 0;
    for (int k0 = 0; k0 < n; k0 += 32 * U) {
        float lx[U], ly[U], mvx[U], mvy[U], vz[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = k0 + 32 * u + lane;
            lx[u] = ly[u] = mvx[u] = mvy[u] = vz[u] = 0.f;
            if (k < n) {
                lx[u] = px[k];
                ly[u] = py[k];
                mvx[u] = pvx[k];
                mvy[u] = pvy[k];
                vz[u] = pvz[k];
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = k0 + 32 * u + lane;
            const bool act = k < n;
            const float x0 = lx[u], y0 = ly[u];
            const float wx = 1 - x0, wy = 1 - y0;
            const float w00 = wx * wy, w01 = wx * y0, w10 = x0 * wy, w11 = x0 * y0;
            const float del_vx = __fmaf_rn(ex_en, w11, __fmaf_rn(ex_es, w10, __fmaf_rn(ex_wn, w01, ex_ws * w00)));
            const float del_vy = __fmaf_rn(ey_en, w11, __fmaf_rn(ey_es, w10, __fmaf_rn(ey_wn, w01, ey_ws * w00)));
            float vX = __fmaf_rn(del_vx, As, mvx[u]);
            float vY = __fmaf_rn(del_vy, As, mvy[u]);
            float X = __fmaf_rn(vX, dtdx, x0);
            float Y = __fmaf_rn(vY, dtdy, y0);
            const bool out = act && (Y >= 1 || Y < 0 || X >= 1 || X < 0);
            int code = 4, fi = i, fj = j;
            if (out) {
                int cond = -1;
                const int r = walk(geo_of(d), fi, fj, X, Y, vX, vY, cond);
                if (r) {
                    code = CODE_ABSORBED;
                    if (cond >= 0 && cond < d.cond_numr) {
                        atomicAdd(&d.cond_charge[s * d.cond_numr + cond], 1.0f);
                        if (d.cond_step) atomicAdd(&d.cond_step[s * d.cond_numr + cond], 1u);
                    } else if (cond <= -2 && d.sig) {
                        surface_enqueue(d, s, fi, fj, -2 - cond, X, Y, vX, vY);
                    }
                    if (r == 2) atomicOr(d.status, ST_WALK);
                } else {
                    const int ddi = fi - i, ddj = fj - j;
                    code = (ddi >= -1 && ddi <= 1 && ddj >= -1 && ddj <= 1) ? (ddi + 1) * 3 + (ddj + 1) : CODE_FAR;
                }
                if (code < 9) {
                    const int q3 = code / 3;
                    const unsigned long long one = 1ull << (21 * (code - 3 * q3));
                    if (q3 == 0) pk0 += one;
                    else if (q3 == 1) pk1 += one;
                    else pk2 += one;
                }
            }
            const unsigned bout = __ballot_sync(FULL, out);
            const int before = m + __popc(bout & lt);
            shifted += __popc(__ballot_sync(FULL, act && (out || before != 0)));
            __syncwarp(); // every lane's loads of this iteration precede the in-place stores
            if (act) {
                const int dst = out ? cap - 1 - before : k - before;
                px[dst] = X;
                py[dst] = Y;
                pvx[dst] = vX;
                pvy[dst] = vY;
                pvz[dst] = vz[u];
                if (out) sp.code[base + dst] = (int8_t)code;
                if (code == CODE_FAR) {
                    const size_t b = (size_t)s * d.C + (size_t)(fi * d.ncy + fj);
                    const int q = atomicAdd(&d.far_in[b], 1);
                    if (q < FAR_B)
                        d.far_key[b * FAR_B + q] = ((unsigned long long)c << 18) | (unsigned long long)before;
                    else
                        atomicOr(d.status, ST_OVERFLOW);
                }
            }
            m += __popc(bout);
        }
    }
    if (lane == 0) {
        sp.cnt[c] = n - m;
        sp.nmov[c] = m;
        atomicAdd(&d.pushes[32 + (warp & 31)], (unsigned long long)shifted);
    }
    int mine = 0;
#pragma unroll
    for (int D = 0; D < 9; D++) {
        const unsigned long long wv = D < 3 ? pk0 : D < 6 ? pk1 : pk2;
        const unsigned tt = __reduce_add_sync(FULL, (unsigned)((wv >> (21 * (D % 3))) & 0x1FFFFFull));
        if (lane == D) mine = (int)tt;
    }
    if (lane < 9) sp.dcount[(size_t)c * 9 + lane] = mine;
}

// ------------------------------------------------------------------ Sort
// SortBoundary_Basic re-bins movers by destination with an atomicAdd on the
// destination count, so the order inside a cell depends on arrival order.
// Here the order is fixed: a destination cell keeps its stayers, then the
// movers addressed to it from its 3x3 neighbourhood, sources in increasing
// cell index and each source's movers in list order, then the movers that
// travelled further (its bucket) in (source cell, r) order.  The boundary
// rules were applied by Move, which also counted each cell's movers per
// destination (dcount).  From those counts every source knows where its
// movers go, so the re-binning is a push with no loop-carried dependency:
//   k_sort_push  (warp per source cell) slot of each near mover = stayers of
//                the destination + movers sent to it by lower-index sources
//                + rank among this source's movers to it;
//   k_sort_count (lane per destination cell) new count, then the far movers.
constexpr int SORT_MAXW = 16; // warps per block, at most

// Memory-level parallelism: a source warp's movers arrive through a ring of
// SORT_PRE chunk slots in shared memory, filled by asynchronous 16-byte copies
// of the cell's top slots (no registers held while they are in flight); the
// first chunk is requested before the mover count is known (the top 32 slots
// exist in every cell), the next ones with the destinations' counts, so a
// warp waits for about one round trip after its count.
#ifndef SORT_PRE
#define SORT_PRE 4
#endif
constexpr int SORT_SLOT = 5 * 32 + 8; // floats per ring slot: x, y, vx, vy, vz, then 32 code bytes
#ifndef SORT_MINB
#define SORT_MINB 2 // resident blocks per SM the register budget is set for
#endif

// One warp per (species, source cell): its movers (the r-th at slot cap-1-r)
// go to their destinations' free slots in (source, rank) order.
__global__ void __launch_bounds__(SORT_MAXW * 32, SORT_MINB) k_sort_push(const DevCase *__restrict__ cases,
                                                           const int *__restrict__ item_start, int ncases, int items) {
    extern __shared__ float sort_ring_s[];
    __shared__ int s_off[SORT_MAXW][9], s_lim[SORT_MAXW][9];
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    if (warp >= items) return;
    float *ring = sort_ring_s + wl * (SORT_PRE * SORT_SLOT);
    const int ci = find_case(item_start, ncases, warp);
    const DevCase &d = cases[ci];
    const int w = warp - item_start[ci];
    const int s = w / d.C, c = w - s * d.C;
    const DevSpecies &sp = d.sp[s];
    const int cap = sp.cap, ncy = d.ncy;
    const size_t base = (size_t)c * cap;
    // chunk h (movers 32h .. 32h+31) is the 32 slots cap-32-32h .. cap-1-32h,
    // all inside the cell as m <= cap/2 and cap is a multiple of 32; mover
    // 32h + l is element 31 - l of each array in ring slot h % SORT_PRE.
    // Lanes 0-7 copy x, 8-15 y, 16-23 vx, 24-31 vy, then lanes 0-7 vz and
    // lanes 8-9 the codes; one commit group per chunk (possibly empty).  Slots
    // of the chunk below the movers belong to the cell's free region, which
    // other warps may be filling: those values are copied but never used
    const float *arr4 = lane < 8 ? sp.x : lane < 16 ? sp.y : lane < 24 ? sp.vx : sp.vy;
    auto issue = [&](int h, bool any) {
        if (any) {
            float *sl = ring + (h % SORT_PRE) * SORT_SLOT;
            const size_t o = base + (size_t)(cap - 32 - 32 * h);
            cp_async16(sl + 4 * lane, arr4 + o + 4 * (lane & 7));
            if (lane < 8) cp_async16(sl + 128 + 4 * lane, sp.vz + o + 4 * lane);
            else if (lane < 10) cp_async16(sl + 160 + 4 * (lane - 8), (const float *)(sp.code + o) + 4 * (lane - 8));
        }
        cp_async_commit();
    };
    issue(0, true);
    const int m = sp.nmov[c];
    if (m == 0) {
        cp_async_wait_all();
        return;
    }
#pragma unroll
    for (int h = 1; h < SORT_PRE; h++) issue(h, 32 * h < m);
    const int i = c / ncy, j = c - i * ncy;
    // destination D = code (di+1)*3 + (dj+1): its stayers and slot limit ...
    int off9 = 0, lim9 = 0;
    if (lane < 9) {
        const int Di = i + lane / 3 - 1, Dj = j + lane % 3 - 1;
        if (Di >= 0 && Di < d.ncx && Dj >= 0 && Dj < ncy) {
            const int D = Di * ncy + Dj;
            off9 = sp.cnt[D];
            lim9 = cap - sp.nmov[D];
        }
    }
    // ... and the movers sent to D by its other neighbours S < c; (D, S) pair
    // p = 9*Dd + Ss, S = D + (Ss/3 - 1, Ss%3 - 1), and S's code for D is 8 - Ss
    int pv[3];
#pragma unroll
    for (int t = 0; t < 3; t++) {
        const int p = lane + 32 * t;
        pv[t] = 0;
        if (p < 81) {
            const int Dd = p / 9, Ss = p - 9 * Dd;
            const int Di = i + Dd / 3 - 1, Dj = j + Dd % 3 - 1;
            const int Si = Di + Ss / 3 - 1, Sj = Dj + Ss % 3 - 1;
            const int S = Si * ncy + Sj;
            if (Di >= 0 && Di < d.ncx && Dj >= 0 && Dj < ncy && Si >= 0 && Si < d.ncx && Sj >= 0 && Sj < ncy && S < c)
                pv[t] = sp.dcount[(size_t)S * 9 + (8 - Ss)];
        }
    }
    int *so = s_off[wl], *sm = s_lim[wl];
    if (lane < 9) {
        so[lane] = off9;
        sm[lane] = lim9;
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < 3; t++)
        if (pv[t]) atomicAdd(&so[(lane + 32 * t) / 9], pv[t]);
    __syncwarp();
    const unsigned lt = lanemask_lt();
    bool overflow = false;
    for (int h = 0; 32 * h < m; h++) {
        cp_async_wait<SORT_PRE - 1>();
        __syncwarp(); // the chunk was copied by other lanes
        const float *sl = ring + (h % SORT_PRE) * SORT_SLOT;
        const int code = 32 * h + lane < m ? (int)((const int8_t *)(sl + 160))[31 - lane] : -1;
        const float x = sl[31 - lane], y = sl[63 - lane], vx = sl[95 - lane], vy = sl[127 - lane],
                    vz = sl[159 - lane];
        __syncwarp(); // every lane has read the slot before it is refilled
        issue(h + SORT_PRE, 32 * (h + SORT_PRE) < m);
        // rank among this chunk's movers to the same destination (the lanes
        // holding the same code); so[D] then advances by their number, added
        // by the group's highest lane
        const unsigned grp = __match_any_sync(FULL, code);
        const int rank = __popc(grp & lt);
        const bool near = code >= 0 && code < 9;
        const int slot = near ? so[code] + rank : 0;
        __syncwarp();
        if (near && (grp >> lane) == 1u) so[code] += __popc(grp);
        __syncwarp();
        if (code >= 0 && code < 9) {
            if (slot < sm[code]) {
                const size_t dst = (size_t)(c + (code / 3 - 1) * ncy + (code % 3 - 1)) * cap + (size_t)slot;
                sp.x[dst] = x;
                sp.y[dst] = y;
                sp.vx[dst] = vx;
                sp.vy[dst] = vy;
                sp.vz[dst] = vz;
            } else {
                overflow = true;
            }
        }
    }
    cp_async_wait_all();
    if (__any_sync(FULL, overflow) && lane == 0) atomicOr(d.status, ST_OVERFLOW);
}

// One lane per destination cell (32 cells per warp): the new count is its
// stayers plus the near movers addressed to it (nine dcount entries, all
// loads independent); the cells with a far bucket are then finished one at a
// time by the whole warp (bucket ordered by (source cell, r), then copied).
__global__ void __launch_bounds__(SORT_MAXW * 32) k_sort_count(const DevCase *__restrict__ cases,
                                                         const int *__restrict__ item_start, int ncases, int items) {
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp * 32 >= items) return;
    const int item = warp * 32 + lane;
    int ci = 0, s = 0, c = 0, out = 0, limit = 0, nf = 0;
    if (item < items) {
        ci = find_case(item_start, ncases, item);
        const DevCase &d = cases[ci];
        const int w = item - item_start[ci];
        s = w / d.C;
        c = w - s * d.C;
        const DevSpecies &sp = d.sp[s];
        const int ncy = d.ncy, i = c / ncy, j = c - i * ncy;
        // near movers in: source S = c + (q/3 - 1, q%3 - 1) sends code 8 - q
        int in = 0;
#pragma unroll
        for (int q = 0; q < 9; q++) {
            const int Si = i + q / 3 - 1, Sj = j + q % 3 - 1;
            if (Si >= 0 && Si < d.ncx && Sj >= 0 && Sj < ncy) in += sp.dcount[(size_t)(Si * ncy + Sj) * 9 + (8 - q)];
        }
        limit = sp.cap - sp.nmov[c];
        out = sp.cnt[c] + in;
        nf = d.far_in[(size_t)s * d.C + c];
    }
    bool overflow = false;
    // a bucket of at most FAR_LANE keys is finished by its own lane: keys
    // sorted in registers by a fixed 19-comparator network (padding keys ~0
    // sort last), then its movers copied in that order; the lanes' buckets
    // proceed together instead of one after the other
    if (nf > 0 && nf <= FAR_LANE) {
        const DevCase &d = cases[ci];
        const DevSpecies &sp = d.sp[s];
        const int cap = sp.cap;
        const size_t b = (size_t)s * d.C + c;
        unsigned long long k8[FAR_LANE];
#pragma unroll
        for (int t = 0; t < FAR_LANE; t++) k8[t] = t < nf ? d.far_key[b * FAR_B + t] : ~0ull;
        d.far_in[b] = 0;
        constexpr int NET[19][2] = {{0, 2}, {1, 3}, {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}, {0, 1}, {2, 3},
                                    {4, 5}, {6, 7}, {2, 4}, {3, 5}, {1, 4}, {3, 6}, {1, 2}, {3, 4}, {5, 6}};
#pragma unroll
        for (int e = 0; e < 19; e++) {
            const unsigned long long lo = k8[NET[e][0]], hi = k8[NET[e][1]];
            k8[NET[e][0]] = lo < hi ? lo : hi;
            k8[NET[e][1]] = lo < hi ? hi : lo;
        }
#pragma unroll
        for (int t = 0; t < FAR_LANE; t++) {
            if (t >= nf) break;
            const int slot = out + t;
            if (slot < limit) {
                const int sc = (int)(k8[t] >> 18), r = (int)(k8[t] & 0x3FFFF);
                const size_t q = (size_t)sc * cap + (size_t)(cap - 1 - r);
                const size_t dst = (size_t)c * cap + (size_t)slot;
                sp.x[dst] = sp.x[q];
                sp.y[dst] = sp.y[q];
                sp.vx[dst] = sp.vx[q];
                sp.vy[dst] = sp.vy[q];
                sp.vz[dst] = sp.vz[q];
            } else {
                overflow = true;
            }
        }
        out += nf;
    }
    for (unsigned fm = __ballot_sync(FULL, nf > FAR_LANE); fm; fm &= fm - 1) {
        const int src = __ffs(fm) - 1;
        const int fci = __shfl_sync(FULL, ci, src), fs = __shfl_sync(FULL, s, src), fc = __shfl_sync(FULL, c, src);
        const int fout = __shfl_sync(FULL, out, src), flimit = __shfl_sync(FULL, limit, src);
        const int fnf = min(__shfl_sync(FULL, nf, src), FAR_B); // Move flagged an overflow
        const DevCase &d = cases[fci];
        const DevSpecies &sp = d.sp[fs];
        const int cap = sp.cap;
        const size_t b = (size_t)fs * d.C + fc;
        // key w*32 + lane of the bucket in key[w]; its place in (source
        // cell, r) order in pos[w] (the keys are distinct)
        unsigned long long key[FAR_W];
        int pos[FAR_W];
#pragma unroll
        for (int w = 0; w < FAR_W; w++) {
            key[w] = w * 32 + lane < fnf ? d.far_key[b * FAR_B + w * 32 + lane] : ~0ull;
            pos[w] = w * 32 + lane;
        }
        __syncwarp();
        if (lane == 0) d.far_in[b] = 0;
        if (fnf <= 32) {
            // bitonic network across the lanes
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
                for (int jj = k >> 1; jj > 0; jj >>= 1) {
                    const unsigned long long o = __shfl_xor_sync(FULL, key[0], jj);
                    const bool keep_min = ((lane & jj) == 0) == ((lane & k) == 0);
                    key[0] = keep_min ? (o < key[0] ? o : key[0]) : (o > key[0] ? o : key[0]);
                }
        } else {
            // a rare full bucket: rank every key against all the others
#pragma unroll
            for (int w = 0; w < FAR_W; w++) pos[w] = 0;
            for (int w2 = 0; w2 * 32 < fnf; w2++) {
                unsigned long long kw = key[0];
#pragma unroll
                for (int w = 1; w < FAR_W; w++)
                    if (w == w2) kw = key[w];
                for (int l = 0; l < 32; l++) {
                    const unsigned long long o = __shfl_sync(FULL, kw, l);
#pragma unroll
                    for (int w = 0; w < FAR_W; w++) pos[w] += o < key[w] ? 1 : 0;
                }
            }
        }
        bool ov = false;
#pragma unroll
        for (int w = 0; w < FAR_W; w++) {
            if (w * 32 + lane >= fnf) continue;
            const int slot = fout + pos[w];
            if (slot < flimit) {
                const int sc = (int)(key[w] >> 18), r = (int)(key[w] & 0x3FFFF);
                const size_t q = (size_t)sc * cap + (size_t)(cap - 1 - r);
                const size_t dst = (size_t)fc * cap + (size_t)slot;
                sp.x[dst] = sp.x[q];
                sp.y[dst] = sp.y[q];
                sp.vx[dst] = sp.vx[q];
                sp.vy[dst] = sp.vy[q];
                sp.vz[dst] = sp.vz[q];
            } else {
                ov = true;
            }
        }
        const bool any_ov = __any_sync(FULL, ov);
        if (lane == src) {
            out += fnf;
            overflow |= any_ov;
        }
    }
    if (item < items) {
        const DevCase &d = cases[ci];
        if (overflow) atomicOr(d.status, ST_OVERFLOW);
        d.sp[s].cnt[c] = out < limit ? out : limit;
    }
}

// ------------------------------------------------------------------ MCC (Ar)
// MCC_Ar_Basic (src/cuda_mcc.cu:97-106): in every cell the ions collide first
// (Direct_Argon_ArIon, src/cuda_mccAr.cu:175-232), then the electrons
// (Direct_Argon_Electron, src/cuda_mccAr.cu:41-174).  Each particle draws from
// its own Philox stream (slot, cell, step, species) in the same order as the
// reference draws from its per-cell curand state; where the reference passes
// two curand_uniform() calls as arguments, the left one is drawn first.
// Channel tallies go to the cell's own counters (the reference's MCCR).
//
// Most particles do not collide in a step (a few per cent), and a colliding
// lane runs a long path (cross sections, scattering angles, the ionisation
// energy split) while the rest of its warp would idle.  So each warp first
// runs the cheap null-collision test over its cell, four slots per lane and
// one Philox block per lane (hp_test_block), and queues the colliders in
// particle order in a shared-memory ring; every 32 queued colliders are then
// processed by the whole warp, one per lane, each from its own stream.  Every
// particle's arithmetic and draws are exactly those of a lane-per-particle
// loop, and new particles are still appended in particle order.
constexpr int MCC_TPB = 256;
constexpr int MCC_RING = 256; // >= 128 new entries per pass + 31 pending

// one ion that passed the null-collision test; returns the channel tallied
// (5 charge exchange, 6 scattering) or -1 for a null collision
__device__ __forceinline__ int mcc_ion_collide(const DevCase &d, const DevSpecies &ion, size_t q, hp_stream &rs,
                                               float bvel) {
    const int nn = (int)((d.nvel - 1) * hp_stream_next(&rs));
    float vnx, vny, vnz;
    {
        const float a = hp_stream_next(&rs);
        const float b = hp_stream_next(&rs);
        maxwellv_dev(vnx, vny, vnz, d.vsave[nn], bvel, a, b);
    }
    const float vx = ion.vx[q], vy = ion.vy[q], vz = ion.vz[q];
    float VX = vx - vnx, VY = vy - vnz, VZ = vz - vny; // y/z of the neutral swapped as in src/cuda_mccAr.cu:200-202
    const float dum = VX * VX + VY * VY + VZ * VZ;
    const float engy = ion.Escale * dum;
    const float vel = sqrtf(dum);
    const float R1 = hp_stream_next(&rs) * d.sigv[2] / vel;
    const XsecPos xp = xsec_pos(d, engy);
    float SumSigma = xsec_at(xp, 5);
    float ox, oy, oz;
    int ch = -1;
    if (R1 <= SumSigma) {
        ox = vnx; oy = vny; oz = vnz;
        ch = 5;
    } else if (R1 <= (SumSigma += xsec_at(xp, 6))) {
        const float a = hp_stream_next(&rs);
        const float b = hp_stream_next(&rs);
        newvel_ionsc_dev(VX, VY, VZ, vel, a, b);
        ox = VX + vnx; oy = VY + vny; oz = VZ + vnz;
        ch = 6;
    } else {
        return -1; // velocity unchanged
    }
    ion.vx[q] = ox;
    ion.vy[q] = oy;
    ion.vz[q] = oz;
    return ch;
}

struct NewPair {
    float x, y, evx, evy, evz, ivx, ivy, ivz;
};

// one electron that passed the null-collision test with draw R1; returns the
// channel tallied (0-4; 3 and 4 ionise, the new electron/ion pair in np) or
// -1 for a null collision
__device__ __forceinline__ int mcc_el_collide(const DevCase &d, const DevSpecies &el, size_t q, hp_stream &rs,
                                              float R1, float P1, float bvel, NewPair &np) {
    int colltype = 1, ch = -1;
    const int target = (R1 <= P1) ? 0 : 1;
    float VX = el.vx[q], VY = el.vy[q], VZ = el.vz[q];
    const float dum = VX * VX + VY * VY + VZ * VZ;
    float vel = sqrtf(dum);
    VX /= vel; VY /= vel; VZ /= vel;
    float engy = el.Escale * dum;
    float rengy = 0.f, vel2 = 0.f;
    const XsecPos xp = xsec_pos(d, engy);
    if (target == 0) {
        const float R2 = hp_stream_next(&rs) * d.sigv[0] / vel;
        float SumSigma = xsec_at(xp, 0);
        if (R2 <= SumSigma) {
            colltype = 0;
            ch = 0;
        } else if (engy > d.th[1] && R2 <= (SumSigma += xsec_at(xp, 1))) {
            colltype = 0;
            engy -= d.th[1];
            vel = sqrtf(fabsf(engy) / el.Escale);
            ch = 1;
        } else if (engy > d.th[2] && R2 <= (SumSigma += xsec_at(xp, 2))) {
            colltype = 0;
            engy -= d.th[2];
            vel = sqrtf(fabsf(engy) / el.Escale);
            ch = 2;
        } else if (engy > d.th[3] && R2 <= (SumSigma += xsec_at(xp, 3))) {
            colltype = 2;
            ch = 3;
        }
    } else {
        const float R2 = hp_stream_next(&rs) * d.sigv[1] / vel;
        if (engy > d.th[4] && R2 <= xsec_at(xp, 4)) {
            colltype = 2;
            ch = 4;
        }
    }
    if (colltype == 1) return -1; // null collision: velocity unchanged
    if (colltype == 2) {          // ionisation: energy split (src/cuda_mccAr.cu:120-170)
        engy -= d.th[ch];
        const float u = hp_stream_next(&rs);
        rengy = (float)(10.0 * (double)hp_tanf_q1(u * hp_atanf((float)(engy / 20.0))));
        engy -= rengy;
        vel = sqrtf(fabsf(rengy) / el.Escale);
        vel2 = sqrtf(fabsf(engy) / el.Escale);
        np.x = el.x[q];
        np.y = el.y[q];
        np.evx = VX; np.evy = VY; np.evz = VZ;
        {
            const float a = hp_stream_next(&rs);
            const float b = hp_stream_next(&rs);
            anewvel_dev(rengy, vel, np.evx, np.evy, np.evz, a, b);
        }
        np.ivx = VX; np.ivy = VY; np.ivz = VZ;
        {
            const int nn = (int)((d.nvel - 1) * hp_stream_next(&rs));
            const float a = hp_stream_next(&rs);
            const float b = hp_stream_next(&rs);
            maxwellv_dev(np.ivx, np.ivy, np.ivz, d.vsave[nn], bvel, a, b);
        }
        vel = vel2; // the primary scatters with the energy left
    }
    const float a = hp_stream_next(&rs);
    const float b = hp_stream_next(&rs);
    anewvel_dev(engy, vel, VX, VY, VZ, a, b);
    el.vx[q] = VX;
    el.vy[q] = VY;
    el.vz[q] = VZ;
    return ch;
}

// The cells one warp works on, with what its lanes need while colliding.
struct MccCell {
    int c, ne, ni, add; // cell, electrons and ions before the step, births so far
    float P1, P2, Pion, bvel;
};

#ifndef MCC_MINB
#define MCC_MINB 3 // 80 registers: three 256-thread blocks per SM
#endif

// Ions of up to G consecutive cells of one case, then their electrons.  Each
// queue entry is (slot | cell-in-group << 24, test draw); the queue is
// drained 32 colliders at a time, so the cells of a group share collision
// batches.  A cell's new pairs are appended behind its own particles in
// queue order, which is the cell's particle order.
template <int G>
__device__ __forceinline__ void mcc_ar_cells(const DevCase &d, int c0, int n, int2 *ring, MccCell *cs,
                                             unsigned *tally, int lane, unsigned lt, bool &overflow) {
    const uint32_t step = (uint32_t)(*d.tstep);
    const DevSpecies &el = d.sp[0];
    const DevSpecies &ion = d.sp[1];
    if (lane < n) {
        const int c = c0 + lane;
        const int i = c / d.ncy, j = c - i * d.ncy;
        MccCell m;
        m.c = c;
        m.ne = el.cnt[c];
        m.ni = ion.cnt[c];
        m.add = 0;
        m.P1 = d.prob[c];
        m.P2 = d.prob[d.C + c];
        m.Pion = d.prob[2 * d.C + c];
        m.bvel = d.back_vel1[i * d.ngy + j];
        cs[lane] = m;
    }
    for (int k = lane; k < G * 8; k += 32) tally[k] = 0u;
    __syncwarp();
    int head = 0, tail = 0;
    // queue the slots of `hits` (four per lane, slot k + t) behind the tail
    auto enqueue = [&](unsigned hits, int k, int cl, const float *R) {
        int total;
        int pos = tail + lower_lane_hits(hits, lt, total);
#pragma unroll
        for (int t = 0; t < 4; t++)
            if ((hits >> t) & 1u) ring[(pos++) & (MCC_RING - 1)] = make_int2((k + t) | (cl << 24), __float_as_int(R[t]));
        tail += total;
        __syncwarp();
    };
    // ---- ions: test four slots per lane from one Philox block, queue, collide
    auto ion_batch = [&]() {
        const int e = head + lane;
        if (e < tail) {
            const int2 ent = ring[e & (MCC_RING - 1)];
            const int k = ent.x & 0xFFFFFF, q = ent.x >> 24;
            const int c = cs[q].c;
            hp_stream rs;
            hp_stream_init(&rs, d.seed, (uint32_t)k, (uint32_t)c, step, 1u);
            const int ch = mcc_ion_collide(d, ion, (size_t)c * ion.cap + k, rs, cs[q].bvel);
            if (ch >= 0) atomicAdd(&tally[q * 8 + ch], 1u);
        }
        head = min(head + 32, tail);
        __syncwarp();
    };
    for (int cl = 0; cl < n; cl++) {
        const int c = cs[cl].c, ni = cs[cl].ni;
        const float Pion = cs[cl].Pion;
        for (int k0 = 0; k0 < ni; k0 += 128) {
            const int k = k0 + 4 * lane;
            unsigned hits = 0;
            float R[4] = {0.f, 0.f, 0.f, 0.f};
            if (k < ni) {
                const hp_u4 u = hp_test_block(d.seed, (uint32_t)(k >> 2), (uint32_t)c, step, 1u, 0u);
#pragma unroll
                for (int t = 0; t < 4; t++)
                    if (k + t < ni && hp_u01(hp_word(u, (uint32_t)t)) <= Pion) hits |= 1u << t;
            }
            enqueue(hits, k, cl, R);
            while (tail - head >= 32) ion_batch();
        }
    }
    while (tail > head) ion_batch();
    // ---- electrons: up to mcc_n test blocks (sub-cycles) per four slots
    auto el_batch = [&]() {
        const int e = head + lane;
        int q = -1, ch = -1;
        NewPair np;
        if (e < tail) {
            const int2 ent = ring[e & (MCC_RING - 1)];
            const int k = ent.x & 0xFFFFFF;
            q = ent.x >> 24;
            const int c = cs[q].c;
            hp_stream rs;
            hp_stream_init(&rs, d.seed, (uint32_t)k, (uint32_t)c, step, 0u);
            ch = mcc_el_collide(d, el, (size_t)c * el.cap + k, rs, __int_as_float(ent.y), cs[q].P1, cs[q].bvel, np);
            if (ch >= 0) atomicAdd(&tally[q * 8 + ch], 1u);
        }
        const bool create = ch >= 3;
        const unsigned bc = __ballot_sync(FULL, create);
        if (bc) {
            const unsigned same = __match_any_sync(FULL, q); // lanes of the same cell (contiguous)
            if (create) {
                const MccCell m = cs[q];
                const int off = m.add + __popc(bc & same & lt);
                const int se = m.ne + off, sn = m.ni + off;
                if (se < el.cap && sn < ion.cap) {
                    const size_t qe = (size_t)m.c * el.cap + se, qi = (size_t)m.c * ion.cap + sn;
                    el.x[qe] = np.x; el.y[qe] = np.y;
                    el.vx[qe] = np.evx; el.vy[qe] = np.evy; el.vz[qe] = np.evz;
                    ion.x[qi] = np.x; ion.y[qi] = np.y;
                    ion.vx[qi] = np.ivx; ion.vy[qi] = np.ivy; ion.vz[qi] = np.ivz;
                } else {
                    overflow = true;
                }
            }
            __syncwarp();
            if (q >= 0 && (same & lt) == 0) cs[q].add += __popc(bc & same);
        }
        head = min(head + 32, tail);
        __syncwarp();
    };
    for (int cl = 0; cl < n; cl++) {
        const int c = cs[cl].c, ne = cs[cl].ne;
        const float P2 = cs[cl].P2;
        for (int k0 = 0; k0 < ne; k0 += 128) {
            const int k = k0 + 4 * lane;
            unsigned hits = 0;
            float R[4] = {0.f, 0.f, 0.f, 0.f};
            if (k < ne) {
                const unsigned live = k + 4 <= ne ? 0xFu : (1u << (ne - k)) - 1u;
                for (int jj = 0; jj < d.mcc_n && (hits != live); jj++) {
                    const hp_u4 u = hp_test_block(d.seed, (uint32_t)(k >> 2), (uint32_t)c, step, 0u, (uint32_t)jj);
#pragma unroll
                    for (int t = 0; t < 4; t++) {
                        const float r = hp_u01(hp_word(u, (uint32_t)t));
                        if (((live & ~hits) >> t) & 1u && r < P2) {
                            hits |= 1u << t;
                            R[t] = r;
                        }
                    }
                }
            }
            enqueue(hits, k, cl, R);
            while (tail - head >= 32) el_batch();
        }
    }
    while (tail > head) el_batch();
    __syncwarp();
    // counts with this step's pairs (clamped to the room left when a cell overflowed)
    if (lane < n) {
        const MccCell m = cs[lane];
        const int add = min(m.add, min(el.cap - m.ne, ion.cap - m.ni));
        el.cnt[m.c] = m.ne + add;
        ion.cnt[m.c] = m.ni + add;
    }
    // per-cell channel tallies (the reference's MCCR per node)
    for (int k = lane; k < n * 8; k += 32)
        if (tally[k]) d.mcc_count[(size_t)cs[k >> 3].c * 8 + (k & 7)] += tally[k];
    __syncwarp();
}

template <int G>
__global__ void __launch_bounds__(MCC_TPB, MCC_MINB) k_mcc_ar(const DevCase *__restrict__ cases,
                                                              const int *__restrict__ item_start, int ncases,
                                                              int items) {
    __shared__ int2 ring_s[MCC_TPB / 32][MCC_RING];
    __shared__ MccCell cell_s[MCC_TPB / 32][G];
    __shared__ unsigned tally_s[MCC_TPB / 32][G * 8];
    const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int first = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5) * G;
    if (first >= items) return;
    const unsigned lt = lanemask_lt();
    const int end = min(first + G, items);
    bool overflow = false;
    // a group that straddles two cases of a batch runs as two groups
    for (int g0 = first; g0 < end;) {
        const int ci = find_case(item_start, ncases, g0);
        const int g1 = min(end, item_start[ci + 1]);
        const DevCase &d = cases[ci];
        overflow = false;
        mcc_ar_cells<G>(d, g0 - item_start[ci], g1 - g0, ring_s[wl], cell_s[wl], tally_s[wl], lane, lt, overflow);
        if (__any_sync(FULL, overflow) && lane == 0) atomicOr(d.status, ST_OVERFLOW);
        g0 = g1;
    }
}

// ------------------------------------------------------------------ Deposit
// DepositAtom (src/cuda_Deposit.cu:289-317): per-cell sums of the four CIC
// weights; lanes accumulate in FP32, the warp reduces in FP64 and writes one
// double4 per cell, which the node pass gathers in a fixed order.
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// DEP_G consecutive (species, cell) items per warp: lanes 0..G-1 resolve
// their item's case, count and array bases together, every lane then loads
// its first slot of all G cells at once, and the cells are summed one after
// the other (each lane adds its slots lane, lane + 32, ... of a cell in that
// order, the warp tree reduces in FP64), so the sums are those of one cell
// per warp.
#ifndef DEP_G
#define DEP_G 2
#endif
__global__ void __launch_bounds__(512) k_deposit_cells(const DevCase *__restrict__ cases,
                                                       const int *__restrict__ item_start, int ncases, int items) {
    constexpr int G = DEP_G;
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp * G >= items) return;
    int my_n = 0;
    const float *my_x = nullptr, *my_y = nullptr;
    double4 *my_cw = nullptr;
    if (lane < G && warp * G + lane < items) {
        const int item = warp * G + lane;
        const int ci = find_case(item_start, ncases, item);
        const DevCase &d = cases[ci];
        const int w = item - item_start[ci];
        const int s = w / d.C, c = w - s * d.C;
        const DevSpecies &sp = d.sp[s];
        const size_t base = (size_t)c * sp.cap;
        my_n = sp.cnt[c];
        my_x = sp.x + base;
        my_y = sp.y + base;
        my_cw = d.cw[s] + c;
    }
    int n[G];
    const float *px[G], *py[G];
    float x0[G], y0[G];
#pragma unroll
    for (int g = 0; g < G; g++) {
        n[g] = __shfl_sync(FULL, my_n, g);
        px[g] = (const float *)__shfl_sync(FULL, (unsigned long long)my_x, g);
        py[g] = (const float *)__shfl_sync(FULL, (unsigned long long)my_y, g);
    }
    // the first chunk of every cell: slots 0..31 are inside the pool (cap >= 32)
#pragma unroll
    for (int g = 0; g < G; g++) {
        x0[g] = px[g] ? px[g][lane] : 0.f;
        y0[g] = py[g] ? py[g][lane] : 0.f;
    }
#pragma unroll
    for (int g = 0; g < G; g++) {
        if (!px[g]) continue; // past the last item (warp-uniform)
        const int ng = n[g];
        if (ng == 0) { // warp-uniform: the sums of an empty cell are +0, as the tree would give
            double4 *cw = (double4 *)__shfl_sync(FULL, (unsigned long long)my_cw, g);
            if (lane == 0) *cw = make_double4(0.0, 0.0, 0.0, 0.0);
            continue;
        }
        float WS = 0.f, WN = 0.f, ES = 0.f, EN = 0.f;
        auto add = [&](float lx, float ly) {
            WS += (1 - lx) * (1 - ly);
            WN += (1 - lx) * ly;
            ES += lx * (1 - ly);
            EN += lx * ly;
        };
        if (lane < ng) add(x0[g], y0[g]);
        for (int k0 = 32; k0 < ng; k0 += 128) {
            float xs[4], ys[4];
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const int k = k0 + 32 * h + lane;
                xs[h] = k < ng ? px[g][k] : 0.f;
                ys[h] = k < ng ? py[g][k] : 0.f;
            }
#pragma unroll
            for (int h = 0; h < 4; h++)
                if (k0 + 32 * h + lane < ng) add(xs[h], ys[h]);
        }
        const double a = warp_sum_d(WS), b = warp_sum_d(WN), e = warp_sum_d(ES), f = warp_sum_d(EN);
        double4 *cw = (double4 *)__shfl_sync(FULL, (unsigned long long)my_cw, g);
        if (lane == 0) *cw = make_double4(a, b, e, f);
    }
}

// The Sort phase's pass over the dielectric crossings Move queued: one block
// per case, then the queue is emptied for the next step.  The fixed-point
// sums make the result independent of the order of the entries.
__global__ void __launch_bounds__(256) k_surface(const DevCase *__restrict__ cases, int ncases) {
    const DevCase &d = cases[blockIdx.x];
    if (!d.sig) return;
    const int n = min(*d.dq_n, d.dq_cap);
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const int k = d.dq_k[q];
        const float4 v = d.dq_v[q];
        const int cell = k >> 7, i = cell / d.ncy, j = cell - i * d.ncy;
        surface_split(d, (k >> 4) & 7, i, j, k & 15, v.x, v.y, v.z, v.w);
    }
    __syncthreads();
    if (threadIdx.x == 0) *d.dq_n = 0;
    (void)ncases;
}

// SumSource's surface-charge term (src/cuda_Deposit.cu:40-97): at a node of
// dielectric class the species' surface weights times q*np2c, which also
// sets Sigma (that charge over the node Area, doubled on a domain edge); a
// node of conductor class clears its surface weights.
__device__ __forceinline__ double surface_charge(const DevCase &d, int n) {
    const int m = d.sig_mode[n];
    if (m == 0) return 0.0;
    if (m == 3) {
        for (int s = 0; s < d.nsp; s++) d.sig[(size_t)s * d.G + n] = 0;
        return 0.0;
    }
    double q = 0.0;
    for (int s = 0; s < d.nsp; s++)
        q += (double)d.sig[(size_t)s * d.G + n] * (1.0 / (double)(1ll << HP_SIGMA_FRAC_BITS)) * (double)d.sp[s].q_density;
    d.sigma[n] = (m == 2 ? 2.0 : 1.0) * q / (double)d.area[n];
    return q;
}

// DepositBoundary + SumSource + PCG_Set (src/cuda_Deposit.cu:277-288,35-104,30-34)
__global__ void __launch_bounds__(256) k_deposit_nodes(const DevCase *__restrict__ cases,
                                                       const int *__restrict__ item_start, int ncases, int items) {
    const int t = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (t >= items) return;
    const int ci = find_case(item_start, ncases, t);
    const DevCase &d = cases[ci];
    const int n = t - item_start[ci];
    const int i = n / d.ngy, j = n - i * d.ngy;
    const int ncy = d.ncy;
    double sum = 0.0;
    for (int s = 0; s < d.nsp; s++) {
        const double4 *cw = d.cw[s];
        double den = 0.0;
        if (i < d.ncx && j < ncy) den += cw[i * ncy + j].x;
        if (i < d.ncx && j > 0) den += cw[i * ncy + j - 1].y;
        if (i > 0 && j < ncy) den += cw[(i - 1) * ncy + j].z;
        if (i > 0 && j > 0) den += cw[(i - 1) * ncy + j - 1].w;
        den *= (double)d.dep_factor[n];
        d.den[(size_t)s * d.G + n] = den;
        sum += den * (double)d.sp[s].q_density;
    }
    if (d.sig) sum += surface_charge(d, n);
    const double source = sum / 8.8542e-12;
    d.source[n] = source;
    d.b64[n] = d.st[2 * d.G + n] != 0.0f ? source : 0.0;
}

// Smooth_121_x / Smooth_121_y (src/cuda_Deposit.cu:105-170): one pass of the
// 1-2-1 filter along x (den -> smt), then along y (smt -> den), with the
// reference's weights at the edges of the density region (a doubled
// neighbour at a wall, 8/4 on an isolated node).  A neighbour whose weight is
// 0 is not read (the densities are non-negative, so 0 * it adds nothing).
__device__ __forceinline__ double smooth_121(const int *dr, const double *v, int id, int at, int last, int step) {
    int a1 = 0, a2 = 1, a3 = 0;
    if (dr[id]) {
        if (at == 0) a3 = 2;
        else if (at == last) a1 = 2;
        else if (dr[id - step] == 0 && dr[id + step] != 0) a3 = 2;
        else if (dr[id - step] != 0 && dr[id + step] == 0) a1 = 2;
        else if (dr[id - step] == 0 && dr[id + step] == 0) a2 = 4;
        else { a1 = 1; a3 = 1; }
    } else {
        a2 = 0;
    }
    const double l = a1 ? (double)a1 * v[id - step] : 0.0;
    const double r = a3 ? (double)a3 * v[id + step] : 0.0;
    return 0.25 * (l + (double)(2 * a2) * v[id] + r);
}

__global__ void __launch_bounds__(256) k_smooth(const DevCase *__restrict__ cases, const int *__restrict__ item_start,
                                                int ncases, int items, int pass, int along_y) {
    const int t = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (t >= items) return;
    const int ci = find_case(item_start, ncases, t);
    const DevCase &d = cases[ci];
    if (pass >= d.n_smt) return;
    const int n = t - item_start[ci];
    const int x = n / d.ngy, y = n - x * d.ngy;
    for (int s = 0; s < d.nsp; s++) {
        const size_t o = (size_t)s * d.G;
        if (!along_y) d.smt[o + n] = smooth_121(d.dens_region, d.den + o, n, x, d.ngx - 1, d.ngy);
        else d.den[o + n] = smooth_121(d.dens_region, d.smt + o, n, y, d.ngy - 1, 1);
    }
}

// SumSource + PCG_Set after the smoothing: rho/eps0 and the right-hand side
__global__ void __launch_bounds__(256) k_source(const DevCase *__restrict__ cases, const int *__restrict__ item_start,
                                                int ncases, int items) {
    const int t = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (t >= items) return;
    const int ci = find_case(item_start, ncases, t);
    const DevCase &d = cases[ci];
    if (d.n_smt <= 0) return;
    const int n = t - item_start[ci];
    double sum = 0.0;
    for (int s = 0; s < d.nsp; s++) sum += d.den[(size_t)s * d.G + n] * (double)d.sp[s].q_density;
    if (d.sig) sum += surface_charge(d, n);
    const double source = sum / 8.8542e-12;
    d.source[n] = source;
    d.b64[n] = d.st[2 * d.G + n] != 0.0f ? source : 0.0;
}

// ------------------------------------------------------------------ Field
__device__ __forceinline__ float spmv_f(const float *__restrict__ st, int G, int ngy, int n, int i, int j, int ngx,
                                        const float *__restrict__ v) {
    // CSR order of the reference rows: W, S, C, N, E (src/load.c:170-240)
    float out = 0.0f;
    const float cw = st[n], cs = st[G + n], cc = st[2 * G + n], cn = st[3 * G + n], ce = st[4 * G + n];
    if (cw != 0.0f) out += cw * v[n - ngy];
    if (cs != 0.0f) out += cs * v[n - 1];
    out += cc * v[n];
    if (cn != 0.0f) out += cn * v[n + 1];
    if (ce != 0.0f) out += ce * v[n + ngy];
    (void)i; (void)j; (void)ngx;
    return out;
}

__device__ __forceinline__ double spmv_d(const float *__restrict__ st, int G, int ngy, int n,
                                         const double *__restrict__ v) {
    double out = 0.0;
    const float cw = st[n], cs = st[G + n], cc = st[2 * G + n], cn = st[3 * G + n], ce = st[4 * G + n];
    if (cw != 0.0f) out += (double)cw * v[n - ngy];
    if (cs != 0.0f) out += (double)cs * v[n - 1];
    out += (double)cc * v[n];
    if (cn != 0.0f) out += (double)cn * v[n + 1];
    if (ce != 0.0f) out += (double)ce * v[n + ngy];
    return out;
}

// CTAs of the whole-GPU solve, at most
constexpr int PCG_GRID_MAX = 512;

struct ClusterRed {
    double *warp_part; // [32] in shared memory
    double *slot;      // [4]  in shared memory, read by the whole cluster
    double *bcast;     // [4]
    double *grid_part; // [2 * PCG_GRID_MAX] in shared memory (whole-GPU solve)
};

// Sum of v over the cluster.  Deterministic for a fixed launch shape: warp
// shuffle tree, warps in order, CTAs in rank order.  One cluster barrier.
__device__ double cluster_sum2(cg::cluster_group &cl, double v0, double v1, const ClusterRed &sh, int parity,
                               double *out1) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v0 = warp_sum_d(v0);
    v1 = warp_sum_d(v1);
    if (lane == 0) {
        sh.warp_part[wid] = v0;
        sh.warp_part[16 + wid] = v1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < nw; k++) { a += sh.warp_part[k]; b += sh.warp_part[16 + k]; }
        sh.slot[2 * parity] = a;
        sh.slot[2 * parity + 1] = b;
    }
    cl.sync();
    // the CTA totals are read in parallel (lane r reads rank r) and added in
    // rank order by one thread, so the remote reads do not queue one behind
    // another
    const unsigned ncta = cl.num_blocks();
    if (threadIdx.x < ncta) {
        const double *rem = cl.map_shared_rank(sh.slot, threadIdx.x);
        sh.warp_part[threadIdx.x] = rem[2 * parity];
        sh.warp_part[16 + threadIdx.x] = rem[2 * parity + 1];
    }
    __syncwarp();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (unsigned r = 0; r < ncta; r++) {
            a += sh.warp_part[r];
            b += sh.warp_part[16 + r];
        }
        sh.bcast[0] = a;
        sh.bcast[1] = b;
    }
    __syncthreads();
    if (out1) *out1 = sh.bcast[1];
    const double r = sh.bcast[0];
    __syncthreads();
    return r;
}

// The same sum over all CTAs of a cooperative grid: the CTA totals go to
// global memory (two buffers by parity, as the cluster slots), a grid
// barrier, and every CTA adds them in rank order -- the same tree as
// cluster_sum2 for the same number of CTAs.
__device__ double grid_sum2(cg::grid_group &gr, double v0, double v1, const ClusterRed &sh, int parity,
                            double *out1, double *part, int ncta, int rank) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v0 = warp_sum_d(v0);
    v1 = warp_sum_d(v1);
    if (lane == 0) {
        sh.warp_part[wid] = v0;
        sh.warp_part[16 + wid] = v1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < nw; k++) { a += sh.warp_part[k]; b += sh.warp_part[16 + k]; }
        part[2 * ((size_t)parity * ncta + rank)] = a;
        part[2 * ((size_t)parity * ncta + rank) + 1] = b;
    }
    gr.sync();
    // the CTA totals are loaded in parallel into shared memory, then added in
    // rank order by one thread
    for (int r = threadIdx.x; r < ncta; r += blockDim.x) {
        sh.grid_part[r] = __ldcg(&part[2 * ((size_t)parity * ncta + r)]);
        sh.grid_part[PCG_GRID_MAX + r] = __ldcg(&part[2 * ((size_t)parity * ncta + r) + 1]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int r = 0; r < ncta; r++) {
            a += sh.grid_part[r];
            b += sh.grid_part[PCG_GRID_MAX + r];
        }
        sh.bcast[0] = a;
        sh.bcast[1] = b;
    }
    __syncthreads();
    if (out1) *out1 = sh.bcast[1];
    const double r = sh.bcast[0];
    __syncthreads();
    return r;
}

// PCG_float (src/cuda_Field.cu:942-1072) as one launch per case cluster, or
// (GRID) as one cooperative launch over the whole GPU for a case too large for
// a 16-CTA cluster: the same algorithm, node partition and reduction tree
// for its number of CTAs, with grid barriers for cluster barriers.  Every
// CTA takes the same branches (the sums are identical on all of them), so
// every CTA reaches every barrier.
// field_mode 0 keeps the reference's rule: FP32 Jacobi-PCG on the assembled
// operator from the previous solution, until r'z <= PCGtol^2 (absolute).
// field_mode 1: FP64 residual b - A x on the FP64 solution, an FP32 PCG
// inner solve of the symmetrised system D^-1 A e = D^-1 r (D = 2 on each
// Neumann edge the reference doubles), x += e, until ||r|| <= rtol ||b||.
// Dot products are accumulated in FP64 in both modes.
template <bool GRID>
__global__ void __launch_bounds__(512) k_pcg(const DevCase *__restrict__ cases, const int *__restrict__ list,
                                             int nlist) {
    cg::cluster_group cl = cg::this_cluster();
    const int CS = GRID ? (int)gridDim.x : (int)cl.num_blocks();
    const int rank = GRID ? (int)blockIdx.x : (int)cl.block_rank();
    const int li = GRID ? 0 : (int)blockIdx.x / CS;
    if (li >= nlist) return;
    const DevCase &d = cases[list[li]];
    const int G = d.G, ngy = d.ngy, ngx = d.ngx;
    const int per = (G + CS - 1) / CS;
    const int lo = rank * per, hi = min(G, lo + per);
    const int T = blockDim.x;
    __shared__ double s_warp[32];
    __shared__ double s_slot[4];
    __shared__ double s_bcast[4];
    __shared__ double s_grid[GRID ? 2 * PCG_GRID_MAX : 1];
    const ClusterRed sh{s_warp, s_slot, s_bcast, s_grid};
    cg::grid_group gr = cg::this_grid();
    // one barrier and one sum over the case's CTAs, in the launch's scope
    auto bar = [&]() {
        if (GRID) gr.sync();
        else cl.sync();
    };
    auto sum2 = [&](double v0, double v1, int par, double *out1) {
        return GRID ? grid_sum2(gr, v0, v1, sh, par, out1, d.pcg_part, CS, rank)
                    : cluster_sum2(cl, v0, v1, sh, par, out1);
    };
    int parity = 0;
    float *__restrict__ x = d.pf_x;
    float *__restrict__ r = d.pf_r;
    float *__restrict__ ap = d.pf_ap;
    // The search direction p alternates between two buffers, and each CTA
    // keeps its own copy of the p values of the other CTAs' unknowns its
    // product reads (the nodes [lo - ngy, lo) and [hi, hi + ngy): its halo),
    // computed from the same operands as their owners compute them.  An
    // iteration then needs no barrier after the direction update: the two
    // sums' barriers are the only ones.
    float *const pbuf0 = d.pf_p, *const pbuf1 = d.pf_p2;
    auto pbuf = [&](int k) { return k ? pbuf1 : pbuf0; };
    float *__restrict__ halo = d.pcg_halo + (size_t)rank * 2 * ngy;
    auto hnode = [&](int q) { return q < ngy ? lo - ngy + q : hi + (q - ngy); };
    auto owned = [&](int m) { return m >= lo && m < hi; };
    // p at node m of the current direction: own nodes from the buffer, the others from the halo
    auto pv = [&](const float *pc, int m) { return owned(m) ? pc[m] : halo[m < lo ? m - (lo - ngy) : ngy + (m - hi)]; };
    // the 5-point product at own node n on the current direction (CSR order W, S, C, N, E)
    auto spmv_h = [&](const float *__restrict__ stc, const float *pc, int n) {
        float out = 0.0f;
        const float cw = stc[n], cs = stc[G + n], cc = stc[2 * G + n], cn = stc[3 * G + n], ce = stc[4 * G + n];
        if (cw != 0.0f) out += cw * pv(pc, n - ngy);
        if (cs != 0.0f) out += cs * pv(pc, n - 1);
        out += cc * pc[n];
        if (cn != 0.0f) out += cn * pv(pc, n + 1);
        if (ce != 0.0f) out += ce * pv(pc, n + ngy);
        return out;
    };
    // the halo of p_0 = D^-1 r_0 (the owners' residuals are visible after the sum's barrier)
    auto halo_first = [&](const float *__restrict__ stc) {
        for (int q = threadIdx.x; q < 2 * ngy; q += T) {
            const int h = hnode(q);
            float v = 0.0f;
            if (h >= 0 && h < G) {
                const float cc = stc[2 * G + h];
                if (cc != 0.0f) v = (1 / cc) * r[h];
            }
            halo[q] = v;
        }
        __syncthreads();
    };
    // own p_{k+1} = beta p_k + D^-1 r_{k+1} into the other buffer, and the halo likewise
    auto next_dir = [&](const float *__restrict__ stc, const float *pc, float *pn, float beta) {
        for (int n = lo + threadIdx.x; n < hi; n += T) {
            const float cc = stc[2 * G + n];
            if (cc == 0.0f) continue;
            pn[n] = beta * pc[n] + (1 / cc) * r[n];
        }
        for (int q = threadIdx.x; q < 2 * ngy; q += T) {
            const int h = hnode(q);
            float v = 0.0f;
            if (h >= 0 && h < G) {
                const float cc = stc[2 * G + h];
                if (cc != 0.0f) v = beta * pc[h] + (1 / cc) * r[h];
            }
            halo[q] = v;
        }
        __syncthreads();
    };
    const int maxit = d.pcg_max_iter;
    int iters = 0, outer = 0;
    bool bad = false;
    if (d.field_mode == 0) {
        const float *__restrict__ st = d.st;
        float *p0 = pbuf(0);
        double part = 0.0;
        for (int n = lo + threadIdx.x; n < hi; n += T) {
            const float cc = st[2 * G + n];
            if (cc == 0.0f) continue;
            const float ax = spmv_f(st, G, ngy, n, 0, 0, ngx, x);
            const float rr = -1.0f * ax + (float)d.b64[n];
            r[n] = rr;
            const float z = (1 / cc) * rr;
            p0[n] = z;
            part += (double)(rr * z);
        }
        double rz = sum2(part, 0.0, parity, nullptr);
        parity ^= 1;
        halo_first(st);
        // a non-finite right-hand side or warm start: the reference's loop
        // test (r'z > tol^2) is false for NaN and leaves x as it was
        if (!(rz == rz) || isinf(rz)) bad = true;
        int iter = 1, pb = 0;
        while (rz > (double)d.pcg_tol2 && iter <= maxit) {
            const float *pc = pbuf(pb);
            part = 0.0;
            for (int n = lo + threadIdx.x; n < hi; n += T) {
                const float cc = st[2 * G + n];
                if (cc == 0.0f) continue;
                const float a = spmv_h(st, pc, n);
                ap[n] = a;
                part += (double)(pc[n] * a);
            }
            const double pap = sum2(part, 0.0, parity, nullptr);
            parity ^= 1;
            const float alpha = (pap != 0.0) ? (float)rz / (float)pap : 0.0f;
            part = 0.0;
            for (int n = lo + threadIdx.x; n < hi; n += T) {
                const float cc = st[2 * G + n];
                if (cc == 0.0f) continue;
                x[n] = alpha * pc[n] + x[n];
                const float rr = -alpha * ap[n] + r[n];
                r[n] = rr;
                part += (double)(rr * ((1 / cc) * rr));
            }
            const double rznew = sum2(part, 0.0, parity, nullptr);
            parity ^= 1;
            if (!(rznew == rznew) || isinf(rznew)) { bad = true; break; }
            const float beta = (rz != 0.0) ? (float)rznew / (float)rz : 0.0f;
            next_dir(st, pc, pbuf(pb ^ 1), beta);
            pb ^= 1;
            rz = rznew;
            iter++;
        }
        iters = iter;
        for (int n = lo + threadIdx.x; n < hi; n += T) d.phi_p[n] = d.st[2 * G + n] != 0.0f ? x[n] : 0.0f;
        if (iter > maxit && rank == 0 && threadIdx.x == 0) atomicOr(d.status, ST_NOCONV);
    } else {
        const float *__restrict__ st = d.st;
        const float *__restrict__ ss = d.st_sym;
        double *__restrict__ x64 = d.x64;
        const double *__restrict__ b64 = d.b64;
        double bb = 0.0;
        for (int n = lo + threadIdx.x; n < hi; n += T) bb += b64[n] * b64[n];
        bb = sum2(bb, 0.0, parity, nullptr);
        parity ^= 1;
        const double target = d.pcg_rtol * d.pcg_rtol * bb;
        const double inner_rel2 = 1e-10; // inner solve: 1e-5 reduction of the preconditioned residual norm
        for (outer = 0; outer < 12; outer++) {
            float *p0 = pbuf(0);
            double rr = 0.0, rz = 0.0;
            for (int n = lo + threadIdx.x; n < hi; n += T) {
                const float cc = st[2 * G + n];
                if (cc == 0.0f) continue;
                const double r64 = b64[n] - spmv_d(st, G, ngy, n, x64);
                rr += r64 * r64;
                const float rs = (float)(r64 * (double)d.row_scale[n]);
                r[n] = rs;
                x[n] = 0.0f;
                const float z = (1 / ss[2 * G + n]) * rs;
                p0[n] = z;
                rz += (double)(rs * z);
            }
            rr = sum2(rr, rz, parity, &rz);
            parity ^= 1;
            if (!(rr == rr) || isinf(rr)) { bad = true; break; }
            if (rr <= target || bb == 0.0) break;
            halo_first(ss);
            const double rz0 = rz;
            int iter = 0, pb = 0;
            while (rz > inner_rel2 * rz0 && iter < maxit) {
                const float *pc = pbuf(pb);
                double part = 0.0;
                for (int n = lo + threadIdx.x; n < hi; n += T) {
                    const float cc = ss[2 * G + n];
                    if (cc == 0.0f) continue;
                    const float a = spmv_h(ss, pc, n);
                    ap[n] = a;
                    part += (double)(pc[n] * a);
                }
                const double pap = sum2(part, 0.0, parity, nullptr);
                parity ^= 1;
                const float alpha = (pap != 0.0) ? (float)(rz / pap) : 0.0f;
                part = 0.0;
                for (int n = lo + threadIdx.x; n < hi; n += T) {
                    const float cc = ss[2 * G + n];
                    if (cc == 0.0f) continue;
                    x[n] = alpha * pc[n] + x[n];
                    const float rs = -alpha * ap[n] + r[n];
                    r[n] = rs;
                    part += (double)(rs * ((1 / cc) * rs));
                }
                const double rznew = sum2(part, 0.0, parity, nullptr);
                parity ^= 1;
                if (!(rznew == rznew) || isinf(rznew)) { bad = true; break; }
                const float beta = (rz != 0.0) ? (float)(rznew / rz) : 0.0f;
                next_dir(ss, pc, pbuf(pb ^ 1), beta);
                pb ^= 1;
                rz = rznew;
                iter++;
            }
            iters += iter;
            if (bad) break;
            for (int n = lo + threadIdx.x; n < hi; n += T)
                if (st[2 * G + n] != 0.0f) x64[n] += (double)x[n];
            bar();
        }
        if (outer >= 12 && rank == 0 && threadIdx.x == 0) atomicOr(d.status, ST_NOCONV);
        for (int n = lo + threadIdx.x; n < hi; n += T) d.phi_p[n] = st[2 * G + n] != 0.0f ? (float)x64[n] : 0.0f;
    }
    if (rank == 0 && threadIdx.x == 0) {
        d.pcg_iters[0] = iters;
        d.pcg_iters[1] = outer;
        if (bad) atomicOr(d.status, ST_NONFINITE);
    }
    // no CTA may leave while another can still read its shared memory
    bar();
}

// Efield_cuda_Basic potential assembly (src/cuda_Field.cu:9-34):
// V_k(t) of conductor k (src/cuda_Field.cu:10-20): its sources' DC + AC
// sin(2 pi f t + phase), summed in the reference's precision; the AC
// amplitudes are the ones in use (a power controller revises them)
__device__ __forceinline__ float cond_voltage(const DevCase &d, int k, double time) {
    float vk = 0.0f;
    if (d.efield_flag[k]) {
        for (int q = 0; q < d.src_num; q++)
            if (d.src_mid[q] == k + 1)
                vk = (float)((double)vk + ((double)d.src_dc[q] +
                                           (double)d.src_amp[q] * sin((double)d.src_2pif[q] * time + (double)d.src_rphase[q])));
    }
    return vk;
}

// TotPotential = sum_k V_k(t) * phi_Lap,k + phi_Pois, in the reference's
// order and precision (float accumulation, V_k(t) from a double sine).
__global__ void __launch_bounds__(256) k_potential(const DevCase *__restrict__ cases, const int *__restrict__ item_start,
                                                   int ncases, int items) {
    const int t = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (t >= items) return;
    const int ci = find_case(item_start, ncases, t);
    const DevCase &d = cases[ci];
    const int n = t - item_start[ci];
    const double time = (double)(*d.tstep) * (double)d.dt;
    float tot = 0.0f;
    // with an external circuit the conductors sit at the circuit's potentials
    for (int k = 0; k < d.cond_numr; k++)
        tot += (d.cs ? d.cs->phi[k] : cond_voltage(d, k, time)) * d.lap[(size_t)k * d.G + n];
    tot += 1 * d.phi_p[n];
    d.phi[n] = tot;
}

// Cond_Sigma at one face node (src/cuda_Field.cu:500-558), on the Poisson part
__device__ float cond_sigma(const DevCase &d, int n, int x, int y, int eT, int eL, int eD, int eX, int pL, int pR,
                            int pD, int pU) {
    const int b = d.boundary[n], f = d.face[n];
    // a Neumann node keeps the Sigma that SumSource left there (0 unless its
    // inward neighbour is dielectric)
    if (b == 2) return d.sigma ? (float)d.sigma[n] : 0.0f;
    if (!((b == 3 || b == 1) && f != 8)) return 0.0f;
    float SumSig = 0.0f;
    for (int s = 0; s < d.nsp; s++) SumSig += (float)d.den[(size_t)s * d.G + n] * d.sp[s].q_density;
    const float *P = d.phi_p;
    const float *E = d.eps;
    const float hdx = d.hdx, hdy = d.hdy, idxy = d.idxy;
    switch (f) {
    case 2: return hdy * (E[eT] + E[eL]) * (P[n] - P[pU]) - hdx * SumSig;
    case 3: return hdy * (E[eD] + E[eX]) * (P[n] - P[pD]) - hdx * SumSig;
    case 0: return hdx * (E[eL] + E[eX]) * (P[n] - P[pL]) - hdy * SumSig;
    case 1: return hdx * (E[eT] + E[eD]) * (P[n] - P[pR]) - hdy * SumSig;
    case 4: return hdy * (E[eT] + E[eL]) * (P[n] - P[pU]) + hdx * (E[eL] + E[eX]) * (P[n] - P[pL]) - idxy * SumSig;
    case 5: return hdy * (E[eT] + E[eL]) * (P[n] - P[pU]) + hdx * (E[eT] + E[eD]) * (P[n] - P[pR]) - idxy * SumSig;
    case 6: return hdy * (E[eD] + E[eX]) * (P[n] - P[pD]) + hdx * (E[eL] + E[eX]) * (P[n] - P[pL]) - idxy * SumSig;
    case 7: return hdy * (E[eD] + E[eX]) * (P[n] - P[pD]) + hdx * (E[eT] + E[eD]) * (P[n] - P[pR]) - idxy * SumSig;
    default: return 0.0f;
    }
    (void)x; (void)y;
}

// Cond_Sigma at node n, with the index arithmetic of VtoEfield
__device__ float cond_sigma_at(const DevCase &d, int n) {
    const int ngx = d.ngx, ngy = d.ngy;
    const int x = n / ngy, y = n - x * ngy;
    const int pL = x ? n - ngy : n, pR = (x == ngx - 1) ? n : n + ngy;
    const int pD = y ? n - 1 : n, pU = (y == ngy - 1) ? n : n + 1;
    int eT = x * (ngy - 1) + y;
    int eL = x ? eT - ngy + 1 : eT;
    int eD = y ? eT - 1 : eT;
    const int eX = eL + eD - eT;
    const int xo = (x == ngx - 1) ? ngy - 1 : 0, yo = (y == ngy - 1) ? 1 : 0;
    eT -= (xo + yo);
    eL -= yo;
    eD -= xo;
    return cond_sigma(d, n, x, y, eT, eL, eD, eX, pL, pR, pD, pU);
}

// VtoEfield (src/cuda_Field.cu:698-846): E = -grad phi at nodes with the
// reference's face, corner and boundary special cases.
__global__ void __launch_bounds__(256) k_efield(const DevCase *__restrict__ cases, const int *__restrict__ item_start,
                                                int ncases, int items) {
    const int t = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (t >= items) return;
    const int ci = find_case(item_start, ncases, t);
    const DevCase &d = cases[ci];
    const int n = t - item_start[ci];
    const int ngx = d.ngx, ngy = d.ngy;
    const int x = n / ngy, y = n - x * ngy;
    const int pL = x ? n - ngy : n, pR = (x == ngx - 1) ? n : n + ngy;
    const int pD = y ? n - 1 : n, pU = (y == ngy - 1) ? n : n + 1;
    int eT = x * (ngy - 1) + y;
    int eL = x ? eT - ngy + 1 : eT;
    int eD = y ? eT - 1 : eT;
    const int eX = eL + eD - eT;
    const int xo = (x == ngx - 1) ? ngy - 1 : 0, yo = (y == ngy - 1) ? 1 : 0;
    eT -= (xo + yo);
    eL -= yo;
    eD -= xo;
    const float *P = d.phi;
    const float *E = d.eps;
    const int f = d.face[n], b = d.boundary[n];
    const float idx = d.idx, idy = d.idy, hdx = d.hdx, hdy = d.hdy, dx = d.dx, dy = d.dy;
    float Ex, Ey;
    bool write = true;
    // Cond_Sigma's Sigma at conductor and Dirichlet face nodes, kept for the
    // power controller's surface charge
    if (d.sigma && (b == 3 || b == 1) && f != 8)
        d.sigma[n] = (double)cond_sigma(d, n, x, y, eT, eL, eD, eX, pL, pR, pD, pU);
    if (f == 0) { // LEFT
        if (b == 3 || b == 2 || b == 1) {
            Ex = -2.0f * cond_sigma(d, n, x, y, eT, eL, eD, eX, pL, pR, pD, pU) / (E[eL] + E[eX]);
            Ey = 0.0f;
        } else if (b == 4 || b >= 100) {
            Ex = idx * (P[pL] - P[n]);
            Ey = hdy * (P[pD] - P[pU]);
        } else {
            Ex = 0.5f * (E[eT] + E[eD]) * (P[pR] - P[n]) * idx;
            Ex -= (0.5f * dx / dy) * E[eT] * (P[n] - P[pU]) * idy;
            Ex -= (0.5f * dx / dy) * E[eD] * (P[n] - P[pD]) * idy;
            Ex /= -0.5f * (E[eL] + E[eX]);
            Ey = hdy * (P[pD] - P[pU]);
        }
    } else if (f == 1) { // RIGHT
        if (b == 3 || b == 2 || b == 1) {
            Ex = 2.0f * cond_sigma(d, n, x, y, eT, eL, eD, eX, pL, pR, pD, pU) / (E[eT] + E[eD]);
            Ey = 0.0f;
        } else if (b == 4 || b >= 100) {
            Ex = idx * (P[n] - P[pR]);
            Ey = hdy * (P[pD] - P[pU]);
        } else {
            Ex = 0.5f * (E[eL] + E[eX]) * (P[pL] - P[n]) * idx;
            Ex -= (0.5f * dx / dy) * E[eL] * (P[n] - P[pU]) * idy;
            Ex -= (0.5f * dx / dy) * E[eX] * (P[n] - P[pD]) * idy;
            Ex /= 0.5f * (E[eT] + E[eD]);
            Ey = hdy * (P[pD] - P[pU]);
        }
    } else if (f == 2) { // UP
        if (b == 3 || b == 2 || b == 1) {
            Ex = 0.0f;
            Ey = 2.0f * cond_sigma(d, n, x, y, eT, eL, eD, eX, pL, pR, pD, pU) / (E[eT] + E[eL]);
        } else if (b == 4 || b >= 100) {
            Ex = hdx * (P[pL] - P[pR]);
            Ey = idy * (P[n] - P[pU]);
        } else {
            Ex = hdx * (P[pL] - P[pR]);
            Ey = 0.5f * (E[eD] + E[eX]) * (P[pD] - P[n]) * idy;
            Ey -= (0.5f * dy / dx) * E[eD] * (P[n] - P[pR]) * idx;
            Ey -= (0.5f * dy / dx) * E[eX] * (P[n] - P[pL]) * idx;
            Ey /= 0.5f * (E[eT] + E[eL]);
        }
    } else if (f == 3) { // DOWN
        if (b == 3 || b == 2 || b == 1) {
            Ex = 0.0f;
            Ey = -2.0f * cond_sigma(d, n, x, y, eT, eL, eD, eX, pL, pR, pD, pU) / (E[eD] + E[eX]);
        } else if (b == 4 || b >= 100) {
            Ex = hdx * (P[pL] - P[pR]);
            Ey = idy * (P[pD] - P[n]);
        } else {
            Ex = hdx * (P[pL] - P[pR]);
            Ey = 0.5f * (E[eT] + E[eL]) * (P[pU] - P[n]) * idy;
            Ey -= (0.5f * dy / dx) * E[eT] * (P[n] - P[pR]) * idx;
            Ey -= (0.5f * dy / dx) * E[eL] * (P[n] - P[pL]) * idx;
            Ey /= -0.5f * (E[eD] + E[eX]);
        }
    } else if (f >= 4 && f <= 7) { // corners
        const bool solid = (b == 3 || b == 1 || b == 4);
        if (!solid) {
            Ex = hdx * (P[pL] - P[pR]);
            Ey = hdy * (P[pD] - P[pU]);
        } else if (f == 4) { // UL
            Ex = idx * (P[pL] - P[n]);
            Ey = idy * (P[n] - P[pU]);
        } else if (f == 5) { // UR
            Ex = idx * (P[n] - P[pR]);
            Ey = idy * (P[n] - P[pU]);
        } else if (f == 6) { // LL
            Ex = idx * (P[pL] - P[n]);
            Ey = idy * (P[pD] - P[n]);
        } else { // LR
            Ex = idx * (P[n] - P[pR]);
            Ey = idy * (P[pD] - P[n]);
        }
    } else if (b == 2) { // Neumann node without a face
        if (x == 0 || x == ngx - 1) {
            Ex = 0.0f;
            Ey = hdy * (P[pD] - P[pU]);
        } else if (y == 0 || y == ngy - 1) {
            Ex = hdx * (P[pL] - P[pR]);
            Ey = 0.0f;
        } else {
            write = false; // the reference leaves E unchanged here
            Ex = Ey = 0.0f;
        }
    } else {
        Ex = hdx * (P[pL] - P[pR]);
        Ey = hdy * (P[pD] - P[pU]);
    }
    if (write) {
        d.Ex[n] = Ex;
        d.Ey[n] = Ey;
    }
}

// The reference's power controller (Diagnostic, src/cuda_Diagnostic.cu:
// 365-420), once per step after Deposit, one block per case: the conductor
// surface charges sum Sigma * Area over the nodes with a CondID (FP64; each
// thread a strided share of the node list, then a fixed tree), the
// conduction current of this step's absorbed particles, the displacement
// current from the last three surface charges, and every pd_intv steps the
// revision of the first power-driven source's amplitude: (target / mean
// power)^0.2 times the amplitude, or at most 5 % up when that would exceed
// (1 + VoltageUpDownRatio) times it; the first revision only arms the
// controller.  hp_powf stands for the reference's double pow.
constexpr int PW_T = 256;
__global__ void __launch_bounds__(PW_T) k_power(DevCase *cases, int ncases) {
    const DevCase &d = cases[blockIdx.x];
    if (!d.pw) return;
    __shared__ double part[PW_T][DMAXCOND];
    const int t = threadIdx.x, nc = d.cond_numr;
    double acc[DMAXCOND];
#pragma unroll
    for (int k = 0; k < DMAXCOND; k++) acc[k] = 0.0;
    for (int q = t; q < d.n_cond_nodes; q += PW_T) {
        const int v = d.cond_nodes[q], n = v & 0xFFFFFF, k = v >> 24;
        const double a = d.sigma[n] * (double)d.area[n];
#pragma unroll
        for (int kk = 0; kk < DMAXCOND; kk++)
            if (kk == k) acc[kk] += a;
    }
#pragma unroll
    for (int k = 0; k < DMAXCOND; k++) part[t][k] = acc[k];
    __syncthreads();
    for (int h = PW_T / 2; h > 0; h >>= 1) {
        if (t < h)
            for (int k = 0; k < nc; k++) part[t][k] += part[t + h][k];
        __syncthreads();
    }
    if (t != 0) return;
    PowerState &P = *d.pw;
    const double time = (double)(*d.tstep) * (double)d.dt;
    for (int i = 0; i < nc; i++) {
        P.old2[i] = P.old[i];
        P.old[i] = P.surf[i];
        P.surf[i] = part[0][i];
        float cond_current = 0.0f, q_conv = 0.0f;
        for (int s = 0; s < d.nsp; s++) {
            unsigned int &cnt = d.cond_step[s * nc + i];
            cond_current += d.sp[s].q_density * (float)cnt / d.dt;
            q_conv -= d.sp[s].q_density * (float)cnt; // the circuit's convective charge (src/cuda_Field.cu:61-64)
            cnt = 0;
        }
        if (d.cs) d.cs->qconv[i] = q_conv;
        const float dis_current = (float)(0.5 * (3.0 * P.surf[i] - 4.0 * P.old[i] + P.old2[i]) / (double)d.dt);
        const float current = dis_current - cond_current;
        if (d.cond_src_num[i] != 1) continue; // voltage driven, or the reference's (empty) dual-power branch
        float phi_now = cond_voltage(d, i, time);
        P.power[i] += phi_now * current;
        P.count[i]++;
        if (P.count[i] != d.pd_intv) continue;
        P.power[i] /= (float)P.count[i];
        P.count[i] = 0;
        const int q = d.cond_power_id[i];
        if (P.power[i] > 0) phi_now = d.src_amp[q] * hp_powf(fabsf(d.src_power[q] / P.power[i]), 0.2f);
        if (P.power_init) {
            if (phi_now > (1.0f + d.pd_ratio) * d.src_amp[q]) d.src_amp[q] = (float)((double)d.src_amp[q] * 1.05);
            else d.src_amp[q] = phi_now;
        }
        P.power[i] = 0.0f;
        P.power_init++;
    }
    (void)ncases;
}

// Efield_cuda's circuit (src/cuda_Field.cu:43-81), once per step after the
// Poisson solve, one block per case (cases without a circuit return): the
// surface charge of this step's Poisson part, Sigma (Cond_Sigma on phi_p,
// den of the last Deposit) x Area over the conductor nodes, summed as
// k_power sums the surface charge (FP64, a strided share per thread, then a
// fixed tree; rounded to float, where the reference adds floats with
// atomics), then the circuit solve of hp_circuit.h on one thread with the
// last step's surface charge and absorbed charge.  k_potential then puts the
// conductors at the circuit's potentials.
__global__ void __launch_bounds__(PW_T) k_circuit(DevCase *cases, int ncases) {
    const DevCase &d = cases[blockIdx.x];
    if (!d.cs) return;
    __shared__ double part[PW_T][HP_CIRCUIT_MAX];
    const int t = threadIdx.x, nc = d.cond_numr;
    double acc[HP_CIRCUIT_MAX];
#pragma unroll
    for (int k = 0; k < HP_CIRCUIT_MAX; k++) acc[k] = 0.0;
    for (int q = t; q < d.n_cond_nodes; q += PW_T) {
        const int v = d.cond_nodes[q], n = v & 0xFFFFFF, k = v >> 24;
        const int b = d.boundary[n], f = d.face[n];
        const double sg = ((b == 3 || b == 1) && f != 8) ? (double)cond_sigma_at(d, n) : 0.0;
        const double a = sg * (double)d.area[n];
#pragma unroll
        for (int kk = 0; kk < HP_CIRCUIT_MAX; kk++)
            if (kk == k) acc[kk] += a;
    }
#pragma unroll
    for (int k = 0; k < HP_CIRCUIT_MAX; k++) part[t][k] = acc[k];
    __syncthreads();
    for (int h = PW_T / 2; h > 0; h >>= 1) {
        if (t < h)
            for (int k = 0; k < nc; k++) part[t][k] += part[t + h][k];
        __syncthreads();
    }
    if (t != 0) return;
    CircuitState &C = *d.cs;
    const double time = (double)(*d.tstep) * (double)d.dt;
    float vt[HP_CIRCUIT_MAX], surf[HP_CIRCUIT_MAX], pois[HP_CIRCUIT_MAX];
    for (int i = 0; i < nc; i++) {
        vt[i] = cond_voltage(d, i, time);
        surf[i] = (float)d.pw->surf[i];
        pois[i] = (float)part[0][i];
    }
    hp_circuit_step(nc, d.cc_a, d.lap_sig, vt, C.qconv, surf, pois, C.q, C.phi, C.pois, d.circuit_mode);
    (void)ncases;
}

__global__ void k_advance(const DevCase *__restrict__ cases, int ncases) {
    const int t = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (t < ncases) *cases[t].tstep += 1;
}

__global__ void __launch_bounds__(256) k_accumulate(const DevCase *__restrict__ cases,
                                                    const int *__restrict__ item_start, int ncases, int items) {
    const int t = (int)(blockIdx.x * (unsigned)blockDim.x + threadIdx.x);
    if (t >= items) return;
    const int ci = find_case(item_start, ncases, t);
    const DevCase &d = cases[ci];
    const int n = t - item_start[ci];
    for (int s = 0; s < d.nsp; s++) d.ave_den[(size_t)s * d.G + n] += d.den[(size_t)s * d.G + n];
    d.ave_phi[n] += (double)d.phi[n];
    d.ave_src[n] += d.source[n];
    d.ave_ex[n] += (double)d.Ex[n];
    d.ave_ey[n] += (double)d.Ey[n];
    if (n == 0) *d.ave_count += 1;
}

// Electron energy distribution: every eedf_every steps, a histogram of
// E = Escale |v|^2 (eV) over all electrons, HP_EEDF_BINS bins of
// HP_EEDF_DE eV and one overflow bin (the reference has no EEDF; its deck
// keys for one are commented out, src/start.c:935-968).  One warp per cell,
// counts gathered per block in shared memory and added to the case's
// 64-bit histogram: integer counts, so the result does not depend on order.
__global__ void __launch_bounds__(256) k_eedf(const DevCase *__restrict__ cases, const int *__restrict__ item_start,
                                              int ncases, int items) {
    __shared__ unsigned int h[HP_EEDF_BINS + 1];
    __shared__ int case_of_block;
    for (int b = threadIdx.x; b <= HP_EEDF_BINS; b += blockDim.x) h[b] = 0;
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int first_warp = (int)(blockIdx.x * (blockDim.x >> 5));
    if (threadIdx.x == 0) case_of_block = first_warp < items ? find_case(item_start, ncases, first_warp) : -1;
    __syncthreads();
    if (warp < items) {
        const int ci = find_case(item_start, ncases, warp);
        const DevCase &d = cases[ci];
        const int c = warp - item_start[ci];
        if (d.eedf_every > 0 && (*d.tstep % d.eedf_every) == 0) {
            const DevSpecies &el = d.sp[0];
            const int n = el.cnt[c];
            const size_t base = (size_t)c * el.cap;
            for (int k = lane; k < n; k += 32) {
                const float vx = el.vx[base + k], vy = el.vy[base + k], vz = el.vz[base + k];
                const float e = el.Escale * (vx * vx + vy * vy + vz * vz);
                const int b = e < HP_EEDF_BINS * HP_EEDF_DE ? (int)(e * (1.0f / HP_EEDF_DE)) : HP_EEDF_BINS;
                if (ci == case_of_block) atomicAdd(&h[b], 1u);
                else atomicAdd(&d.eedf[b], 1ull); // a block that straddles two cases
            }
        }
    }
    __syncthreads();
    if (case_of_block >= 0) {
        const DevCase &d = cases[case_of_block];
        for (int b = threadIdx.x; b <= HP_EEDF_BINS; b += blockDim.x)
            if (h[b]) atomicAdd(&d.eedf[b], (unsigned long long)h[b]);
    }
}

// CSR particle arrays (cell order, start[c] = first particle of cell c) into
// the cell-blocked slot pool of one species; one warp per cell.
__global__ void __launch_bounds__(256) k_scatter(DevSpecies sp, int C, const int *__restrict__ start,
                                                 const float *__restrict__ src) {
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= C) return;
    const int b = start[warp], n = start[warp + 1] - b;
    const size_t total = (size_t)start[C];
    const size_t base = (size_t)warp * sp.cap;
    for (int k = lane; k < n; k += 32) {
        sp.x[base + k] = src[b + k];
        sp.y[base + k] = src[total + b + k];
        sp.vx[base + k] = src[2 * total + b + k];
        sp.vy[base + k] = src[3 * total + b + k];
        sp.vz[base + k] = src[4 * total + b + k];
    }
    if (lane == 0) {
        sp.cnt[warp] = n;
        sp.nmov[warp] = 0;
    }
}

inline unsigned blocks_for(long long threads, int per_block) { return (unsigned)((threads + per_block - 1) / per_block); }

} // namespace

cudaError_t launch_move(const DevCase *cases, const int *item_start, int ncases, int items, const LaunchCfg &lc,
                        cudaStream_t st) {
    if (items <= 0) return cudaSuccess;
    const int tpb = 32 * std::min(std::max(lc.warps_per_block, 1), 16);
    const unsigned nb = blocks_for((long long)items * 32, tpb);
    prof::mark(st, "k_move");
    if (lc.move_unroll == 2) k_move_u<2><<<nb, tpb, 0, st>>>(cases, item_start, ncases, items);
    else if (lc.move_unroll == 4) k_move_u<4><<<nb, tpb, 0, st>>>(cases, item_start, ncases, items);
    else
        k_move<MOVE_RING><<<nb, tpb, (size_t)(tpb / 32) * MOVE_RING * 5 * 32 * sizeof(float), st>>>(
            cases, item_start, ncases, items);
    return cudaGetLastError();
}

cudaError_t launch_power(DevCase *cases, int ncases, cudaStream_t st) {
    if (ncases <= 0) return cudaSuccess;
    prof::mark(st, "k_power");
    k_power<<<ncases, PW_T, 0, st>>>(cases, ncases);
    return cudaGetLastError();
}

cudaError_t launch_sort(const DevCase *cases, const int *item_start, int ncases, int items, const LaunchCfg &lc,
                        cudaStream_t st, bool surface) {
    if (items <= 0) return cudaSuccess;
    if (surface) {
        prof::mark(st, "k_surface");
        k_surface<<<ncases, 256, 0, st>>>(cases, ncases);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    // at least 8 warps per block: the push gains from them even where Move
    // and Deposit prefer smaller blocks
    const int tpb = 32 * std::min(std::max(lc.warps_per_block, 8), SORT_MAXW);
    prof::mark(st, "k_sort_push");
    k_sort_push<<<blocks_for((long long)items * 32, tpb), tpb, (size_t)(tpb / 32) * SORT_PRE * SORT_SLOT * sizeof(float),
                  st>>>(cases, item_start, ncases, items);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    prof::mark(st, "k_sort_count");
    k_sort_count<<<blocks_for((long long)(items + 31) / 32 * 32, tpb), tpb, 0, st>>>(cases, item_start, ncases,
                                                                                     items);
    return cudaGetLastError();
}

cudaError_t launch_mcc_ar(const DevCase *cases, const int *item_start, int ncases, int items, const LaunchCfg &lc,
                          cudaStream_t st) {
    if (items <= 0) return cudaSuccess;
    const int g = lc.mcc_cells;
    const long long threads = (long long)((items + g - 1) / g) * 32;
    prof::mark(st, "k_mcc_ar");
    if (g == 1) k_mcc_ar<1><<<blocks_for(threads, MCC_TPB), MCC_TPB, 0, st>>>(cases, item_start, ncases, items);
    else if (g == 2) k_mcc_ar<2><<<blocks_for(threads, MCC_TPB), MCC_TPB, 0, st>>>(cases, item_start, ncases, items);
    else if (g == 8) k_mcc_ar<8><<<blocks_for(threads, MCC_TPB), MCC_TPB, 0, st>>>(cases, item_start, ncases, items);
    else if (g == 16) k_mcc_ar<16><<<blocks_for(threads, MCC_TPB), MCC_TPB, 0, st>>>(cases, item_start, ncases, items);
    else k_mcc_ar<4><<<blocks_for(threads, MCC_TPB), MCC_TPB, 0, st>>>(cases, item_start, ncases, items);
    return cudaGetLastError();
}

cudaError_t launch_deposit(const DevCase *cases, const int *cell_items, const int *node_items, int ncases,
                           int n_cell_items, int n_node_items, const LaunchCfg &lc, cudaStream_t st, int max_smt) {
    const int tpb = 32 * std::min(std::max(lc.warps_per_block, 1), 16);
    if (n_cell_items > 0) {
        prof::mark(st, "k_deposit_cells");
        k_deposit_cells<<<blocks_for((long long)(n_cell_items + DEP_G - 1) / DEP_G * 32, tpb), tpb, 0, st>>>(cases, cell_items, ncases,
                                                                                        n_cell_items);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (n_node_items > 0) {
        prof::mark(st, "k_deposit_nodes");
        k_deposit_nodes<<<blocks_for(n_node_items, 256), 256, 0, st>>>(cases, node_items, ncases, n_node_items);
    }
    if (max_smt > 0 && n_node_items > 0) {
        for (int p = 0; p < max_smt; p++)
            for (int yy = 0; yy < 2; yy++) {
                prof::mark(st, "k_smooth");
                k_smooth<<<blocks_for(n_node_items, 256), 256, 0, st>>>(cases, node_items, ncases, n_node_items, p, yy);
            }
        prof::mark(st, "k_source");
        k_source<<<blocks_for(n_node_items, 256), 256, 0, st>>>(cases, node_items, ncases, n_node_items);
    }
    return cudaGetLastError();
}

// CTAs of the cooperative grid solve for a case of G nodes: about 1024 nodes
// (two per thread) per CTA, at most what the device keeps resident at once;
// 0 where a cluster of at most 16 CTAs covers the case at 8 nodes per thread
int pcg_grid_ctas(int G, int block) {
    if ((long long)G <= 16LL * 512 * 8) return 0;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg<true>, block, 0) != cudaSuccess)
        return 0;
    const int want = (G + 1023) / 1024;
    const int most = std::min(sms * per_sm, PCG_GRID_MAX);
    return most > 16 ? std::min(want, most) : 0;
}

int pcg_cluster_for_nodes(int G) {
    // about 8 nodes per thread at 512 threads per CTA, up to a 16-CTA cluster
    int cs = 1;
    while (cs < 16 && (long long)G > (long long)cs * 512 * 8) cs *= 2;
    return cs;
}

cudaError_t launch_field(const DevCase *cases, const int *node_items, int ncases, int n_node_items,
                         const PcgGroup *groups, int ngroups, const FastPlan *fast, cudaStream_t st, bool circuit) {
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_pcg<false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        attr_set = true;
    }
    for (int g = 0; g < ngroups; g++) {
        const PcgGroup &pg = groups[g];
        if (pg.n <= 0) continue;
        if (pg.cluster > 16) { // one cooperative launch per case over pg.cluster CTAs
            for (int k = 0; k < pg.n; k++) {
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)pg.cluster, 1, 1);
                cfg.blockDim = dim3((unsigned)pg.block, 1, 1);
                cfg.dynamicSmemBytes = 0;
                cfg.stream = st;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeCooperative;
                attr[0].val.cooperative = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                prof::mark(st, "k_pcg_grid");
                cudaError_t e = cudaLaunchKernelEx(&cfg, k_pcg<true>, cases, pg.list + k, 1);
                if (e != cudaSuccess) return e;
            }
            continue;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(pg.n * pg.cluster), 1, 1);
        cfg.blockDim = dim3((unsigned)pg.block, 1, 1);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)pg.cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        prof::mark(st, "k_pcg");
        cudaError_t e = cudaLaunchKernelEx(&cfg, k_pcg<false>, cases, pg.list, pg.n);
        if (e != cudaSuccess) return e;
    }
    if (fast && fast->n > 0) {
        cudaError_t ef = launch_fast_field(cases, *fast, st);
        if (ef != cudaSuccess) return ef;
    }
    if (circuit) {
        prof::mark(st, "k_circuit");
        k_circuit<<<ncases, PW_T, 0, st>>>(const_cast<DevCase *>(cases), ncases);
        cudaError_t ec = cudaGetLastError();
        if (ec != cudaSuccess) return ec;
    }
    prof::mark(st, "k_potential");
    k_potential<<<blocks_for(n_node_items, 256), 256, 0, st>>>(cases, node_items, ncases, n_node_items);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    prof::mark(st, "k_efield");
    k_efield<<<blocks_for(n_node_items, 256), 256, 0, st>>>(cases, node_items, ncases, n_node_items);
    return cudaGetLastError();
}

cudaError_t launch_scatter(const DevSpecies &sp, int C, const int *start, const float *src, cudaStream_t st) {
    k_scatter<<<blocks_for((long long)C * 32, 256), 256, 0, st>>>(sp, C, start, src);
    return cudaGetLastError();
}

cudaError_t launch_advance(const DevCase *cases, int ncases, cudaStream_t st) {
    prof::mark(st, "k_advance");
    k_advance<<<blocks_for(ncases, 128), 128, 0, st>>>(cases, ncases);
    return cudaGetLastError();
}

cudaError_t launch_eedf(const DevCase *cases, const int *cell_items, int ncases, int n_cell_items, cudaStream_t st) {
    if (n_cell_items <= 0) return cudaSuccess;
    prof::mark(st, "k_eedf");
    k_eedf<<<blocks_for((long long)n_cell_items * 32, 256), 256, 0, st>>>(cases, cell_items, ncases, n_cell_items);
    return cudaGetLastError();
}

cudaError_t launch_accumulate(const DevCase *cases, const int *node_items, int ncases, int n_node_items,
                              cudaStream_t st) {
    if (n_node_items <= 0) return cudaSuccess;
    prof::mark(st, "k_accumulate");
    k_accumulate<<<blocks_for(n_node_items, 256), 256, 0, st>>>(cases, node_items, ncases, n_node_items);
    return cudaGetLastError();
}

} // namespace hp
