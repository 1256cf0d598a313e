// devutil.cuh -- device helpers shared by the step kernels (kernels.cu) and
// the oxygen-chemistry collision kernel (mcc_oxy.cu): warp bookkeeping, the
// cross-section lookup and the scattering kinematics of the reference's MCC
// (src/cuda_mcc.cu:139-201), in the arithmetic the CPU checker repeats.
#pragma once
#include <cstdint>

#include "dev.cuh"
#include "hp_math.h"
#include "hp_rng.h"

namespace hp {
namespace dv {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t ST_OVERFLOW = 0x1u, ST_NONFINITE = 0x2u, ST_NOCONV = 0x4u, ST_WALK = 0x10u, ST_SURFACE = 0x20u;

__device__ __forceinline__ int find_case(const int *start, int n, int w) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (start[mid] <= w) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ------------------------------------------------------------------ mover fate
// Outcome of one cell crossing, from the ghost-grid code of the cell entered
// (src/cuda_Sortboundary.cu:70-256): 0 plasma; >=100 conductor (absorbed and
// counted); -1 Dirichlet (absorbed); -2/-6 Neumann x walls, -4/-8 Neumann y
// walls and -12/-16/-20/-24 Neumann corners (specular reflection back into
// the domain).  The reference leaves any other code undefined (its
// uninitialised Sum_CID/Flag_* are used); here such a mover is absorbed.
// exclusive count of set bits of `mask4` (4 slots per lane) in lower lanes
__device__ __forceinline__ int lower_lane_hits(unsigned mask4, unsigned lt, int &total) {
    int pre = 0;
    total = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const unsigned b = __ballot_sync(FULL, (mask4 >> t) & 1u);
        pre += __popc(b & lt);
        total += __popc(b);
    }
    return pre;
}

// ------------------------------------------------------------------ MCC helpers
// Argon_CrossSection (src/cuda_mccAr.cu:707-776): linear interpolation on the
// 81-point log10 grid, constant below it, 0.1*exp decay above it.  The
// reference reads one row past the table when log10(E) equals the last grid
// point exactly; the index is clamped here.
// (the same for every reaction set: one column per channel)
// Where an energy falls on that grid.  A collider evaluates it once and reads
// every channel of its ladder from it; each channel value is computed with
// the same operations as a lookup of that channel alone.
struct XsecPos {
    const float *row; // table row of the lower grid point (or the clamped end)
    float a1, a2;     // interpolation weights (mode 3)
    float tail;       // exp(-(log10 E - last grid point)) (mode 2)
    int mode;         // 0: E == 0; 1: below the grid; 2: above it; 3: inside
    int W;            // row width
};

__device__ __forceinline__ XsecPos xsec_pos(const DevCase &d, float engy) {
    XsecPos p;
    p.W = d.xw;
    p.row = d.xsec;
    p.a1 = p.a2 = p.tail = 0.f;
    if (engy == 0) {
        p.mode = 0;
        return p;
    }
    const float lengy = hp_log10f(engy);
    const float *t = d.xsec;
    const float xe0 = t[0], xeN = t[(d.n_logx - 1) * p.W];
    if (lengy < xe0) {
        p.mode = 1;
        return p;
    }
    if (lengy > xeN) {
        p.mode = 2;
        p.row = t + (d.n_logx - 1) * p.W;
        p.tail = hp_expf(-1 * (lengy - xeN));
        return p;
    }
    const float ee1 = d.idlogx * (lengy - xe0);
    int ee2 = (int)ee1;
    if (ee2 > d.n_logx - 2) ee2 = d.n_logx - 2;
    if (ee2 < 0) ee2 = 0; // NaN energy: keep the read inside the table
    p.a1 = ee1 - ee2;
    p.a2 = 1 - p.a1;
    p.row = t + ee2 * p.W;
    p.mode = 3;
    return p;
}

__device__ __forceinline__ float xsec_at(const XsecPos &p, int ch) {
    if (p.mode == 3) return p.a2 * p.row[2 + ch] + p.a1 * p.row[p.W + 2 + ch];
    if (p.mode == 2) return p.row[2 + ch] * 0.1f * p.tail;
    return p.mode == 1 ? p.row[2 + ch] : 0.0f;
}

__device__ __forceinline__ float xsec_lookup(const DevCase &d, int ch, float engy) {
    return xsec_at(xsec_pos(d, engy), ch);
}

// dev_maxwellv (src/cuda_mcc.cu:139-147); cos/sin of 2*pi*Rphi in turns
__device__ __forceinline__ void maxwellv_dev(float &vx, float &vy, float &vz, float vsaven, float vti, float Rphi,
                                             float Rthe) {
    float sn, cs;
    hp_sincos_turns(Rphi, &sn, &cs);
    const float costheta = 1 - 2 * Rthe;
    const float sintheta = sqrtf(1 - costheta * costheta);
    vx = vti * vsaven * sintheta * cs;
    vy = vti * vsaven * sintheta * sn;
    vz = vti * vsaven * costheta;
}

// dev_anewvel (src/cuda_mcc.cu:148-173): electron scattering with the
// Surendra angle; massrate term only when e_flag (never set on this path)
__device__ __forceinline__ void anewvel_dev(float energy, float vel, float &nvx, float &nvy, float &nvz, float rand1,
                                            float rand2) {
    float coschi;
    if (energy < 1e-30f) coschi = 1;
    else coschi = (float)(((double)energy + 2.0 - 2.0 * (double)hp_powf((float)(energy + 1.0), rand1)) / energy);
    const float sinchi = (float)sqrt(fabs(1.0 - (double)(coschi * coschi)));
    float sinphi, cosphi;
    hp_sincos_turns(rand2, &sinphi, &cosphi);
    const float r13 = nvx, r23 = nvy, r33 = nvz;
    float up1, up2, up3;
    if (r33 == 1.0f || r33 == -1.0f) { up1 = 0; up2 = 1; up3 = 0; }
    else { up1 = 0; up2 = 0; up3 = 1; }
    float r12 = r23 * up3 - r33 * up2;
    float r22 = r33 * up1 - r13 * up3;
    float r32 = r13 * up2 - r23 * up1;
    const float mag = sqrtf(r12 * r12 + r22 * r22 + r32 * r32);
    r12 /= mag; r22 /= mag; r32 /= mag;
    const float r11 = r22 * r33 - r32 * r23;
    const float r21 = r32 * r13 - r12 * r33;
    const float r31 = r12 * r23 - r22 * r13;
    nvx = vel * (r11 * sinchi * cosphi + r12 * sinchi * sinphi + r13 * coschi);
    nvy = vel * (r21 * sinchi * cosphi + r22 * sinchi * sinphi + r23 * coschi);
    nvz = vel * (r31 * sinchi * cosphi + r32 * sinchi * sinphi + r33 * coschi);
}

// dev_newvel_IONSC (src/cuda_mcc.cu:174-201): isotropic ion scattering in the CM frame
__device__ __forceinline__ void newvel_ionsc_dev(float &vxs, float &vys, float &vzs, float vel, float rand1,
                                                 float rand2) {
    const float coschi = sqrtf(rand1);
    const float sinchi = (float)sqrt(fabs(1.0 - (double)(coschi * coschi)));
    float sinphi, cosphi;
    hp_sincos_turns(rand2, &sinphi, &cosphi);
    const float r13 = vxs / vel, r23 = vys / vel, r33 = vzs / vel;
    float up1, up2, up3;
    if (r33 == 1.0f || r33 == -1.0f) { up1 = 0; up2 = 1; up3 = 0; }
    else { up1 = 0; up2 = 0; up3 = 1; }
    float r12 = r23 * up3 - r33 * up2;
    float r22 = r33 * up1 - r13 * up3;
    float r32 = r13 * up2 - r23 * up1;
    const float mag = sqrtf(r12 * r12 + r22 * r22 + r32 * r32);
    r12 /= mag; r22 /= mag; r32 /= mag;
    const float r11 = r22 * r33 - r32 * r23;
    const float r21 = r32 * r13 - r12 * r33;
    const float r31 = r12 * r23 - r22 * r13;
    vxs = vel * coschi * (r11 * sinchi * cosphi + r12 * sinchi * sinphi + r13 * coschi);
    vys = vel * coschi * (r21 * sinchi * cosphi + r22 * sinchi * sinphi + r23 * coschi);
    vzs = vel * coschi * (r31 * sinchi * cosphi + r32 * sinchi * sinphi + r33 * coschi);
}

} // namespace dv
} // namespace hp
