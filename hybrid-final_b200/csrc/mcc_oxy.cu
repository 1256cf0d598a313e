// mcc_oxy.cu -- null-collision MCC of the Ar/O2 reaction set (5 species:
// e, Ar+, O2+, O+, O-) and of the O2 set (4 species: e, O2+, O+, O-), one
// warp per cell (MCC_ArO2_Basic and MCC_O2_Basic, src/cuda_mcc.cu:21-96;
// the collision checks and species handlers of src/cuda_mccArO2.cu:51-1265
// and src/cuda_mccO2.cu:2-977).
//
// The reference runs one thread per (species, node) with the species
// handlers concurrently: a handler that creates or deletes particles of
// another species races with that species' own thread.  Here one warp owns
// the cell and the order is fixed:
//   * every species' collision test uses the counts at the start of the call
//     (particles created during the call are not tested this step);
//   * the species are handled in order e, Ar+, O2+, O+, O-; within a species
//     the colliders in slot order, 32 at a time (one per lane);
//   * a collider that leaves its species (attachment, recombination, charge
//     transfer to another ion, detachment) leaves a hole; particles created
//     are appended to their species in collider order;
//   * the O- that an electron detachment (e + O- -> 2e + O) removes is drawn
//     uniformly among the O- present at the start of the call and still
//     there (the reference copies the slot one past its count into the
//     victim, a stale particle); a removed O- is not processed by the O-
//     handler afterwards;
//   * at the end every species' holes are filled with its last particles.
// Draws: the collision test from the shared test blocks (hp_test_block), all
// later draws of a collider from its own stream, in the reference's order.
// Reference behaviour kept as is: the first channel of a ladder whose
// threshold fails leaves the running cross-section sum at 0 (uninitialised in
// the reference); ion ladders compare each channel alone where the reference
// does; O2+ always takes its neutral velocity from the Ar temperature and O+
// from the O2 one; an O- scatters with the reference's renormalised
// direction and a detached electron takes the O-'s unit direction as its
// velocity; recombination removes only the projectile; channel 16 loses the
// threshold of channel 11.
#include <cstdint>

#include "devutil.cuh"
#include "kernels.cuh"
#include "prof.cuh"

namespace hp {
namespace {

using namespace dv;

constexpr int OXY_TPB = 128;
constexpr int OXY_RING = 256;
constexpr int HOLE_CAP = 64;
constexpr int NSP_ARO2 = 5;

enum : int { A_ELASTIC, A_LOSS, A_GAIN, A_ATTACH, A_IONIZE, A_RECOMB, A_DETACH };

struct Rung {
    int8_t ch, act, a1, a2; // a1: threshold index (loss) or first new species (ionisation); a2: second
    float gain;
};

// electron ladders per target (src/cuda_mccArO2.cu:91-435)
__constant__ Rung c_erung[] = {
    // 0: e + Ar
    {0, A_ELASTIC, 0, 0, 0}, {1, A_LOSS, 1, 0, 0}, {2, A_LOSS, 2, 0, 0}, {3, A_IONIZE, 0, 1, 0},
    // 1: e + Ar*
    {4, A_IONIZE, 0, 1, 0},
    // 2: e + O2
    {5, A_ELASTIC, 0, 0, 0}, {6, A_LOSS, 6, 0, 0}, {7, A_LOSS, 7, 0, 0}, {8, A_LOSS, 8, 0, 0},
    {9, A_LOSS, 9, 0, 0}, {10, A_LOSS, 10, 0, 0}, {11, A_ATTACH, 0, 0, 0}, {12, A_LOSS, 12, 0, 0},
    {13, A_LOSS, 13, 0, 0}, {14, A_LOSS, 14, 0, 0}, {15, A_IONIZE, 0, 2, 0}, {16, A_LOSS, 11, 0, 0},
    {17, A_IONIZE, 3, 4, 0}, {18, A_IONIZE, 0, 3, 0},
    // 3: e + O2(a)
    {19, A_IONIZE, 0, 2, 0}, {20, A_ATTACH, 0, 0, 0}, {21, A_GAIN, 0, 0, 0.977f}, {22, A_GAIN, 0, 0, 0.977f},
    {23, A_LOSS, 23, 0, 0}, {24, A_LOSS, 24, 0, 0}, {25, A_LOSS, 25, 0, 0}, {26, A_IONIZE, 0, 3, 0},
    // 4: e + O2(b)
    {27, A_IONIZE, 0, 2, 0}, {28, A_ATTACH, 0, 0, 0}, {29, A_GAIN, 0, 0, 1.627f}, {30, A_GAIN, 0, 0, 1.627f},
    {31, A_LOSS, 31, 0, 0}, {32, A_LOSS, 32, 0, 0}, {33, A_LOSS, 33, 0, 0}, {34, A_IONIZE, 0, 3, 0},
    // 5: e + O-
    {35, A_DETACH, 0, 0, 0},
    // 6: e + O2+
    {36, A_RECOMB, 0, 0, 0},
    // 7: e + O(3P)
    {37, A_LOSS, 37, 0, 0}, {38, A_LOSS, 38, 0, 0}, {39, A_LOSS, 39, 0, 0}, {40, A_LOSS, 40, 0, 0},
    {41, A_LOSS, 41, 0, 0}, {42, A_IONIZE, 0, 3, 0}, {43, A_LOSS, 43, 0, 0},
    // 8: e + O(1D)
    {44, A_IONIZE, 0, 3, 0}, {45, A_GAIN, 0, 0, 1.96f},
};
__constant__ int c_erung_start[10] = {0, 4, 5, 19, 27, 35, 36, 37, 44, 46};

// the O2 set's electron ladders (src/cuda_mccO2.cu:2-429)
__constant__ Rung c_orung[] = {
    // 0: e + O2
    {0, A_ELASTIC, 0, 0, 0}, {1, A_LOSS, 1, 0, 0}, {2, A_LOSS, 2, 0, 0}, {3, A_LOSS, 3, 0, 0},
    {4, A_LOSS, 4, 0, 0}, {5, A_LOSS, 5, 0, 0}, {6, A_ATTACH, 0, 0, 0}, {7, A_LOSS, 7, 0, 0},
    {8, A_LOSS, 8, 0, 0}, {9, A_LOSS, 9, 0, 0}, {10, A_IONIZE, 0, 1, 0}, {11, A_LOSS, 11, 0, 0},
    {12, A_IONIZE, 2, 3, 0}, {13, A_IONIZE, 0, 2, 0},
    // 1: e + O2(a)
    {14, A_IONIZE, 0, 1, 0}, {15, A_ATTACH, 0, 0, 0}, {16, A_GAIN, 0, 0, 0.977f}, {17, A_GAIN, 0, 0, 0.977f},
    {18, A_LOSS, 18, 0, 0}, {19, A_LOSS, 19, 0, 0}, {20, A_LOSS, 20, 0, 0}, {21, A_IONIZE, 0, 2, 0},
    // 2: e + O2(b)
    {22, A_IONIZE, 0, 1, 0}, {23, A_ATTACH, 0, 0, 0}, {24, A_GAIN, 0, 0, 1.627f}, {25, A_GAIN, 0, 0, 1.627f},
    {26, A_LOSS, 26, 0, 0}, {27, A_LOSS, 27, 0, 0}, {28, A_LOSS, 28, 0, 0}, {29, A_IONIZE, 0, 2, 0},
    // 3: e + O-
    {30, A_DETACH, 0, 0, 0},
    // 4: e + O2+
    {31, A_RECOMB, 0, 0, 0},
    // 5: e + O(3P)
    {32, A_LOSS, 32, 0, 0}, {33, A_LOSS, 33, 0, 0}, {34, A_LOSS, 34, 0, 0}, {35, A_LOSS, 35, 0, 0},
    {36, A_LOSS, 36, 0, 0}, {37, A_IONIZE, 0, 2, 0}, {38, A_LOSS, 38, 0, 0},
    // 6: e + O(1D)
    {39, A_IONIZE, 0, 2, 0}, {40, A_GAIN, 0, 0, 1.96f},
};
__constant__ int c_orung_start[8] = {0, 14, 22, 30, 31, 32, 39, 41};

// collision probabilities of one cell (cumulative over the targets) from the
// node's background, fluid and charged densities (ArO2_Collision_Check,
// src/cuda_mccArO2.cu:1130-1190).  The electron sums run in float with 1.0f,
// the ion sums in double as the reference's 1.0 literal makes them.
struct CellProb {
    float p[5][9];
    int n[5];
};

__device__ __forceinline__ float xe(float a, float b, float c) { return hp_expf(-1 * a * b * c); }

__device__ __forceinline__ float ion_acc(float prev, bool first, float e) {
    return first ? (float)(1.0 - (double)e) : (float)((double)prev + 1.0 - (double)e);
}

// One survival factor exp(-dt sigma_v n) of the check: time step (1: the
// electron sub-step dt_mcc, 0: dt), sigma-v maximum, and the density it
// multiplies (0 Ar background, 1 O2 background, 2-6 fluid species 0-4,
// 8 + s charged species s from the last deposit).
struct Term {
    unsigned char sub, sv, src;
};
// ArO2_Collision_Check (src/cuda_mccArO2.cu:1130-1190), per species in target
// order: e (O2-scaled targets Ar, Ar*, O2, O2A, O2B, O-, O2+, OP, OD),
// Ar+ (Ar, O2), O2+ (OP, O2, O2A, O2B, Ar), O+ (O2, OP, O2A, O2B),
// O- (O2, OP, O2+, O+, O2A)
__constant__ Term c_terms_aro2[25] = {
    {1, 0, 0}, {1, 1, 2}, {1, 2, 1}, {1, 3, 3}, {1, 4, 4}, {1, 5, 12}, {1, 6, 10}, {1, 7, 5}, {1, 8, 6},
    {0, 23, 0}, {0, 24, 1},
    {0, 14, 5}, {0, 15, 1}, {0, 16, 3}, {0, 17, 4}, {0, 18, 0},
    {0, 19, 1}, {0, 20, 5}, {0, 21, 3}, {0, 22, 4},
    {0, 9, 1}, {0, 10, 5}, {0, 11, 10}, {0, 12, 11}, {0, 13, 3}};
__constant__ int c_first_aro2[6] = {0, 9, 11, 16, 20, 25};
// O2Collision_Check (src/cuda_mccO2.cu:867-911): e (O2, O2A, O2B, O-, O2+,
// OP, OD), O2+ on the electron sub-step (OP, O2, O2A, O2B), O+ (O2, OP, O2A,
// O2B), O- (O2, OP, O2+, O+, O2A)
__constant__ Term c_terms_o2[20] = {
    {1, 0, 0}, {1, 1, 2}, {1, 2, 3}, {1, 3, 11}, {1, 4, 9}, {1, 5, 4}, {1, 6, 5},
    {1, 12, 4}, {1, 13, 0}, {1, 14, 2}, {1, 15, 3},
    {0, 16, 0}, {0, 17, 4}, {0, 18, 2}, {0, 19, 3},
    {0, 7, 0}, {0, 8, 4}, {0, 9, 9}, {0, 10, 10}, {0, 11, 2}};
__constant__ int c_first_o2[5] = {0, 7, 11, 15, 20};

// The collision probabilities of one cell, cumulative over the targets (the
// electron sums run in float with 1.0f, the ion sums in double as the
// reference's 1.0 literal makes them).  Lane l evaluates factor l; lane 0
// accumulates them in the reference's order into shared memory.
template <int GAS>
__device__ void cell_prob(const DevCase &d, int node, CellProb &P, int lane) {
    constexpr int NT = GAS == 2 ? 25 : 20;
    constexpr int NSPC = GAS == 2 ? 5 : 4;
    const Term *terms = GAS == 2 ? c_terms_aro2 : c_terms_o2;
    const int *first = GAS == 2 ? c_first_aro2 : c_first_o2;
    float x = 0.f;
    if (lane < NT) {
        const Term T = terms[lane];
        const float dtx = T.sub ? d.dt_mcc : d.dt;
        const float sig = d.sigv[T.sv];
        if (T.src >= 8) { // charged density: den * np2c * idx * idy, in this order
            const int sp = T.src - 8;
            float t = -1 * dtx;
            t = t * sig;
            t = t * (float)d.den[(size_t)sp * d.G + node];
            t = t * d.sp[sp].np2c;
            t = t * d.idx;
            t = t * d.idy;
            x = hp_expf(t);
        } else {
            const float dens = T.src == 0 ? d.back_den1[node]
                             : T.src == 1 ? d.back_den2[node]
                                          : d.fluid_den[(size_t)(T.src - 2) * d.G + node];
            x = xe(dtx, sig, dens);
        }
    }
    float acc = 0.f;
    int s = 0;
#pragma unroll
    for (int k = 0; k < NT; k++) {
        const float xk = __shfl_sync(FULL, x, k);
        while (k >= first[s + 1]) s++;
        const bool head = k == first[s];
        if (s == 0) acc = head ? 1.0f - xk : acc + 1.0f - xk;
        else acc = ion_acc(acc, head, xk);
        if (lane == 0) P.p[s][k - first[s]] = acc;
    }
    if (lane < 5) P.n[lane] = lane < NSPC ? first[lane + 1] - first[lane] : 1;
    __syncwarp();
}

// target of a hit: the first cumulative probability R1 does not exceed
__device__ __forceinline__ int target_of(const CellProb &P, int s, float R1) {
    const int n = P.n[s];
    for (int t = 0; t < n - 1; t++)
        if (R1 <= P.p[s][t]) return t;
    return n - 1;
}

// a particle created by a collision
struct Born {
    int sp; // -1: none
    float vx, vy, vz;
};

// outcome of one collider
struct Outcome {
    bool keep;           // stays in its species (velocity updated in place)
    float vx, vy, vz;    // its new velocity when kept
    Born b[2];
    bool kill_partner;   // electron detachment: remove one O-
    float r2;            // the draw that picks it
    int ch;              // channel counted (-1: null)
};

__device__ __forceinline__ void no_birth(Outcome &o) {
    o.b[0].sp = o.b[1].sp = -1;
    o.kill_partner = false;
    o.r2 = 0.f;
    o.ch = -1;
}

// ArO2_Electron (src/cuda_mccArO2.cu:51-560) and O2_Electron
// (src/cuda_mccO2.cu:2-429), one collider with target t.  The two differ in
// how R1 is scaled (R1 *= sigma_v/v vs R1 = U sigma_v / v) and in ionisation:
// the Ar/O2 set splits the energy with 10 tan(U atan(E/20)) and scatters the
// new electron, the O2 set gives the new electron the primary's unit
// direction as its velocity.
template <int GAS>
__device__ void electron_collide(const DevCase &d, float vx, float vy, float vz, int t, float bv1, hp_stream &rs,
                                 Outcome &o) {
    constexpr int OMINUS = GAS == 2 ? 4 : 3;
    no_birth(o);
    const float Esc = d.sp[0].Escale;
    float VX = vx, VY = vy, VZ = vz;
    const float dum = VX * VX + VY * VY + VZ * VZ;
    float vel = sqrtf(dum);
    VX /= vel; VY /= vel; VZ /= vel;
    float engy = Esc * dum;
    int colltype = 1, i1 = 0, i2 = 0;
    float rengy = 0.f, vel2 = 0.f;
    float R1;
    if (GAS == 2) {
        R1 = hp_stream_next(&rs);
        R1 *= d.sigv[t] / vel;
    } else {
        R1 = hp_stream_next(&rs) * d.sigv[t] / vel;
    }
    const Rung *rung = GAS == 2 ? c_erung : c_orung;
    const int k0 = GAS == 2 ? c_erung_start[t] : c_orung_start[t];
    const int k1 = GAS == 2 ? c_erung_start[t + 1] : c_orung_start[t + 1];
    float sum = 0.f;
    bool hit = false;
    const XsecPos xp = xsec_pos(d, engy); // engy is fixed until the hit
    for (int k = k0; k < k1; k++) {
        const Rung r = rung[k];
        if (!(engy > d.th[r.ch])) continue;
        sum = sum + xsec_at(xp, r.ch);
        if (!(R1 <= sum)) continue;
        hit = true;
        o.ch = r.ch;
        switch (r.act) {
        case A_ELASTIC: break;
        case A_LOSS:
            engy -= d.th[r.a1];
            vel = sqrtf(fabsf(engy) / Esc);
            break;
        case A_GAIN:
            engy += r.gain;
            vel = sqrtf(fabsf(engy) / Esc);
            break;
        case A_ATTACH: colltype = 2; break;
        case A_RECOMB: colltype = 4; break;
        case A_DETACH:
            colltype = 5;
            engy -= d.th[r.ch];
            vel = sqrtf(fabsf(engy) / Esc);
            break;
        default: { // A_IONIZE
            colltype = 3;
            engy -= d.th[r.ch];
            if (GAS == 2) {
                const float u = hp_stream_next(&rs);
                rengy = (float)(10.0 * (double)hp_tanf_q1(u * hp_atanf((float)(engy / 20.0))));
                engy -= rengy;
                vel = sqrtf(fabsf(rengy) / Esc);
                vel2 = sqrtf(fabsf(engy) / Esc);
            } else {
                vel = sqrtf(fabsf(engy) / Esc);
            }
            i1 = r.a1;
            i2 = r.a2;
            break;
        }
        }
        break;
    }
    if (!hit) colltype = 0;
    o.keep = true;
    o.vx = vx; o.vy = vy; o.vz = vz;
    switch (colltype) {
    case 0: break;
    case 1: {
        const float a = hp_stream_next(&rs), b = hp_stream_next(&rs);
        anewvel_dev(engy, vel, VX, VY, VZ, a, b);
        o.vx = VX; o.vy = VY; o.vz = VZ;
        break;
    }
    case 2: { // attachment: the electron becomes an O- with a neutral's thermal velocity
        o.keep = false;
        const int n = (int)((d.nvel - 1) * hp_stream_next(&rs));
        const float a = hp_stream_next(&rs), b = hp_stream_next(&rs);
        o.b[0].sp = OMINUS;
        maxwellv_dev(o.b[0].vx, o.b[0].vy, o.b[0].vz, d.vsave[n], bv1, a, b);
        break;
    }
    case 3: { // ionisation: two new charged particles, then the primary loses energy
        const int isp[2] = {i1, i2};
        for (int q = 0; q < 2; q++) {
            Born &b = o.b[q];
            b.sp = isp[q];
            if (isp[q] == 0) {
                b.vx = VX; b.vy = VY; b.vz = VZ;
                if (GAS == 2) {
                    const float a = hp_stream_next(&rs), c = hp_stream_next(&rs);
                    anewvel_dev(rengy, vel, b.vx, b.vy, b.vz, a, c);
                }
            } else {
                const int n = (int)((d.nvel - 1) * hp_stream_next(&rs));
                const float a = hp_stream_next(&rs), c = hp_stream_next(&rs);
                maxwellv_dev(b.vx, b.vy, b.vz, d.vsave[n], bv1, a, c);
            }
        }
        const float a = hp_stream_next(&rs), b = hp_stream_next(&rs);
        anewvel_dev(engy, GAS == 2 ? vel2 : vel, VX, VY, VZ, a, b);
        o.vx = VX; o.vy = VY; o.vz = VZ;
        break;
    }
    case 4: o.keep = false; break; // recombination: only the electron goes
    default: {                      // 5: detachment e + O- -> 2e + O
        o.b[0].sp = 0;
        o.b[0].vx = VX; o.b[0].vy = VY; o.b[0].vz = VZ; // the unit direction, as the reference
        const float a = hp_stream_next(&rs), b = hp_stream_next(&rs);
        anewvel_dev(engy, vel, VX, VY, VZ, a, b);
        o.vx = VX; o.vy = VY; o.vz = VZ;
        o.kill_partner = true;
        o.r2 = hp_stream_next(&rs);
        break;
    }
    }
}

// ArO2_Ar_ion / _O2_ion / _O_ion / _O_negative (src/cuda_mccArO2.cu:561-1129)
// and O2_O2_ion / _O_ion / _O_negative (src/cuda_mccO2.cu:430-866)
enum : int { I_NULL, I_SCAT, I_CX, I_TO_OP, I_TO_ARP, I_TO_O2P, I_DETACH, I_RECOMB };

template <int GAS>
__device__ void ion_collide(const DevCase &d, int s, float vx, float vy, float vz, int t, float bv1, float bv2,
                            hp_stream &rs, Outcome &o) {
    constexpr int OMINUS = GAS == 2 ? 4 : 3, O2P = GAS == 2 ? 2 : 1, OP = GAS == 2 ? 3 : 2;
    no_birth(o);
    o.keep = true;
    o.vx = vx; o.vy = vy; o.vz = vz;
    const float Esc = d.sp[s].Escale;
    float vnx = 0.f, vny = 0.f, vnz = 0.f;
    float VX, VY, VZ, vel, engy;
    if (s == OMINUS) { // O-: no neutral velocity; the direction is normalised
        VX = vx; VY = vy; VZ = vz;
        const float dum = VX * VX + VY * VY + VZ * VZ;
        vel = sqrtf(dum);
        VX /= vel; VY /= vel; VZ /= vel;
        engy = Esc * dum;
    } else {
        float vneut;
        if (GAS == 2) vneut = s == 1 ? (t == 0 ? bv1 : bv2) : (s == 2 ? bv1 : bv2);
        else vneut = bv1;
        const int n = (int)((d.nvel - 1) * hp_stream_next(&rs));
        const float a = hp_stream_next(&rs), b = hp_stream_next(&rs);
        maxwellv_dev(vnx, vny, vnz, d.vsave[n], vneut, a, b);
        VX = vx - vnx; VY = vy - vny; VZ = vz - vnz;
        const float dum = VX * VX + VY * VY + VZ * VZ;
        vel = sqrtf(dum);
        engy = Esc * dum;
        if (GAS == 2 && s == 1) (void)hp_stream_next(&rs); // the reference draws R1 and overwrites it
    }
    // (sigma-v index, channels, actions, cumulative second rung)
    int sv = 0, nr = 0, ch[3] = {0, 0, 0}, act[3] = {0, 0, 0};
    bool cum = false;
    if (GAS == 2) {
        switch (s) {
        case 1:
            sv = 23 + t;
            if (t == 0) { nr = 2; ch[0] = 65; act[0] = I_CX; ch[1] = 66; act[1] = I_SCAT; }
            else { nr = 1; ch[0] = 67; act[0] = I_SCAT; }
            break;
        case 2:
            sv = 14 + t;
            if (t == 0) { nr = 1; ch[0] = 52; act[0] = I_TO_OP; }
            else if (t == 1) { nr = 3; ch[0] = 53; act[0] = I_CX; ch[1] = 54; act[1] = I_SCAT; ch[2] = 55; act[2] = I_TO_OP; }
            else if (t == 2) { nr = 1; ch[0] = 56; act[0] = I_CX; }
            else if (t == 3) { nr = 1; ch[0] = 57; act[0] = I_CX; }
            else { nr = 2; ch[0] = 58; act[0] = I_TO_ARP; ch[1] = 59; act[1] = I_CX; }
            break;
        case 3:
            sv = 19 + t;
            if (t == 0) { nr = 2; ch[0] = 60; act[0] = I_TO_O2P; ch[1] = 61; act[1] = I_SCAT; }
            else if (t == 1) { nr = 1; ch[0] = 62; act[0] = I_CX; }
            else { nr = 1; ch[0] = 61 + t; act[0] = I_TO_O2P; }
            break;
        default: // O-
            sv = 9 + t;
            if (t == 0) { nr = 2; ch[0] = 46; act[0] = I_SCAT; ch[1] = 47; act[1] = I_DETACH; cum = true; }
            else if (t == 1) { nr = 1; ch[0] = 48; act[0] = I_DETACH; }
            else if (t == 2) { nr = 1; ch[0] = 49; act[0] = I_RECOMB; }
            else if (t == 3) { nr = 1; ch[0] = 50; act[0] = I_RECOMB; }
            else { nr = 1; ch[0] = 51; act[0] = I_DETACH; }
            break;
        }
    } else {
        switch (s) {
        case 1: // O2+
            sv = 12 + t;
            if (t == 0) { nr = 1; ch[0] = 47; act[0] = I_TO_OP; }
            else if (t == 1) { nr = 3; ch[0] = 48; act[0] = I_CX; ch[1] = 49; act[1] = I_SCAT; ch[2] = 50; act[2] = I_TO_OP; }
            else { nr = 1; ch[0] = 49 + t; act[0] = I_CX; }
            break;
        case 2: // O+
            sv = 16 + t;
            if (t == 0) { nr = 2; ch[0] = 53; act[0] = I_TO_O2P; ch[1] = 54; act[1] = I_SCAT; }
            else if (t == 1) { nr = 1; ch[0] = 55; act[0] = I_CX; }
            else { nr = 1; ch[0] = 54 + t; act[0] = I_TO_O2P; }
            break;
        default: // O-: the handler scales R1 by sigma_v 9..13 (the check used 7..11)
            sv = 9 + t;
            if (t == 0) { nr = 2; ch[0] = 41; act[0] = I_SCAT; ch[1] = 42; act[1] = I_DETACH; cum = true; }
            else if (t == 1) { nr = 1; ch[0] = 43; act[0] = I_DETACH; }
            else if (t == 2) { nr = 1; ch[0] = 44; act[0] = I_RECOMB; }
            else if (t == 3) { nr = 1; ch[0] = 45; act[0] = I_RECOMB; }
            else { nr = 1; ch[0] = 46; act[0] = I_DETACH; }
            break;
        }
    }
    const float R1 = hp_stream_next(&rs) * d.sigv[sv] / vel;
    int what = I_NULL;
    float sum = 0.f;
    const XsecPos xp = xsec_pos(d, engy);
    for (int k = 0; k < nr; k++) {
        if (!(engy > d.th[ch[k]])) continue;
        const float xs = xsec_at(xp, ch[k]);
        sum = (k > 0 && cum) ? sum + xs : xs;
        if (R1 <= sum) {
            what = act[k];
            o.ch = ch[k];
            break;
        }
    }
    switch (what) {
    case I_NULL: break;
    case I_SCAT: {
        const float a = hp_stream_next(&rs), b = hp_stream_next(&rs);
        newvel_ionsc_dev(VX, VY, VZ, vel, a, b);
        if (s == OMINUS) { o.vx = VX; o.vy = VY; o.vz = VZ; }
        else { o.vx = VX + vnx; o.vy = VY + vny; o.vz = VZ + vnz; }
        break;
    }
    case I_CX: o.vx = vnx; o.vy = vny; o.vz = vnz; break;
    case I_TO_OP: o.keep = false; o.b[0] = Born{OP, vnx, vny, vnz}; break;
    case I_TO_ARP: o.keep = false; o.b[0] = Born{1, vnx, vny, vnz}; break;
    case I_TO_O2P: o.keep = false; o.b[0] = Born{O2P, vnx, vny, vnz}; break;
    case I_DETACH: o.keep = false; o.b[0] = Born{0, VX, VY, VZ}; break;
    default: o.keep = false; break; // I_RECOMB
    }
}

__device__ __forceinline__ bool is_hole(float x) { return x != x; }

#ifndef OXY_MINB
#define OXY_MINB 5 // 96 registers: five 128-thread blocks per SM
#endif
#ifndef OXY_G
#define OXY_G 4
#endif

// The per-cell state a warp keeps for each cell of its group.
struct OxyCell {
    int c, n0[NSP_ARO2], cnt[NSP_ARO2], nh[NSP_ARO2];
    float bv1, bv2;
    bool hole_over[NSP_ARO2];
};

// Up to G consecutive cells of one case per warp.  Species by species (e,
// Ar+, O2+, O+, O- in every cell), the colliders of the group's cells are
// queued together as (slot | target << 20 | cell-in-group << 24) and
// collided 32 at a time, so sparse species share batches.  Within a cell
// everything keeps the order of one cell per warp: colliders in slot order,
// births appended per species in collider order, holes recorded in collider
// order, detachment victims drawn in collider order.
template <int GAS, int G>
__device__ __forceinline__ void mcc_oxy_cells(const DevCase &d, int c0, int ncell, int *ring,
                                              int (*holes)[NSP_ARO2][HOLE_CAP], CellProb *P, OxyCell *cs,
                                              int lane, unsigned lt, bool &overflow) {
    constexpr int NSP = GAS == 2 ? 5 : 4;
    constexpr int OMINUS = GAS == 2 ? 4 : 3;
    const uint32_t step = (uint32_t)(*d.tstep);
    for (int cl = 0; cl < ncell; cl++) {
        const int c = c0 + cl;
        const int i = c / d.ncy, j = c - i * d.ncy;
        const int node = i * d.ngy + j;
        cell_prob<GAS>(d, node, P[cl], lane);
        if (lane < NSP) {
            const int n = d.sp[lane].cnt[c];
            cs[cl].n0[lane] = n;
            cs[cl].cnt[lane] = n;
            cs[cl].nh[lane] = 0;
            cs[cl].hole_over[lane] = false;
        }
        if (lane == 0) {
            cs[cl].c = c;
            cs[cl].bv1 = d.back_vel1[node];
            cs[cl].bv2 = d.back_vel2[node];
        }
    }
    __syncwarp();
    // lane-uniform call: one hole of species s in cell cl
    auto add_hole = [&](int cl, int s, int slot) {
        const int h = cs[cl].nh[s];
        if (lane == 0) {
            if (h < HOLE_CAP) holes[cl][s][h] = slot;
            else cs[cl].hole_over[s] = true;
            cs[cl].nh[s] = h + 1;
        }
        __syncwarp();
    };
    // the reference's O2 launch covers Gsize threads, so only its electrons
    // collide (src/cuda_mcc.cu:76-77); mcc_all_species extends it to every species
    const int nactive = (GAS == 2 || d.mcc_all_species) ? NSP : 1;
#pragma unroll 1
    for (int s = 0; s < nactive; s++) {
        const DevSpecies &sp = d.sp[s];
        const int nsub = (s == 0 || (GAS == 1 && s == 1)) ? d.mcc_n : 1; // O2: O2+ sub-cycles too
        int head = 0, tail = 0;
        // one batch: up to 32 queued colliders, one per lane
        auto batch = [&]() {
            const int e = head + lane;
            Outcome o;
            no_birth(o);
            o.keep = true;
            bool active = false;
            int k = 0, q = -1;
            float px = 0.f, py = 0.f;
            if (e < tail) {
                const int ent = ring[e & (OXY_RING - 1)];
                k = ent & 0xFFFFF;
                const int t = (ent >> 20) & 0xF;
                q = ent >> 24;
                const int c = cs[q].c;
                const size_t base = (size_t)c * sp.cap;
                px = sp.x[base + k];
                if (!is_hole(px)) { // an O- removed earlier this call is gone
                    active = true;
                    py = sp.y[base + k];
                    const float vx = sp.vx[base + k], vy = sp.vy[base + k], vz = sp.vz[base + k];
                    hp_stream rs;
                    hp_stream_init(&rs, d.seed, (uint32_t)k, (uint32_t)c, step, (uint32_t)s);
                    if (s == 0) electron_collide<GAS>(d, vx, vy, vz, t, cs[q].bv1, rs, o);
                    else ion_collide<GAS>(d, s, vx, vy, vz, t, cs[q].bv1, cs[q].bv2, rs, o);
                    if (o.ch >= 0) atomicAdd(&d.mcc_count[(size_t)c * d.mcc_stride + o.ch], 1u);
                    if (o.keep) {
                        sp.vx[base + k] = o.vx;
                        sp.vy[base + k] = o.vy;
                        sp.vz[base + k] = o.vz;
                    } else {
                        sp.x[base + k] = __int_as_float(0x7fc00000); // hole
                    }
                }
            }
            // holes left by the colliders, in slot order
            const unsigned bgone = __ballot_sync(FULL, active && !o.keep);
            for (unsigned m = bgone; m; m &= m - 1) {
                const int src = __ffs(m) - 1;
                add_hole(__shfl_sync(FULL, q, src), s, __shfl_sync(FULL, k, src));
            }
            // births, per species in lane (= collider) order and per cell; a
            // collider's two births, if any, go to two different species
            const unsigned same = __match_any_sync(FULL, q); // lanes of one cell (contiguous)
#pragma unroll 1
            for (int t = 0; t < NSP; t++) {
                const int b = (active && o.b[0].sp == t) ? 0 : (active && o.b[1].sp == t) ? 1 : -1;
                const unsigned bm = __ballot_sync(FULL, b >= 0);
                if (!bm) continue;
                const DevSpecies &tp = d.sp[t];
                if (b >= 0) {
                    const int slot = cs[q].cnt[t] + __popc(bm & same & lt);
                    if (slot < tp.cap) {
                        const size_t q2 = (size_t)cs[q].c * tp.cap + slot;
                        tp.x[q2] = px;
                        tp.y[q2] = py;
                        tp.vx[q2] = o.b[b].vx;
                        tp.vy[q2] = o.b[b].vy;
                        tp.vz[q2] = o.b[b].vz;
                    } else {
                        overflow = true;
                    }
                }
                __syncwarp();
                if (q >= 0 && (same & lt) == 0 && (bm & same))
                    cs[q].cnt[t] = min(cs[q].cnt[t] + __popc(bm & same), tp.cap);
                __syncwarp();
            }
            // O- removed by detachments, in lane order, among the O- of the
            // collider's cell present at the start of the call that are still there
            const unsigned bk = __ballot_sync(FULL, active && o.kill_partner);
            for (unsigned m = bk; m; m &= m - 1) {
                const int src = __ffs(m) - 1;
                const float r2 = __shfl_sync(FULL, o.r2, src);
                const int qc = __shfl_sync(FULL, q, src);
                const DevSpecies &om = d.sp[OMINUS];
                const size_t ob = (size_t)cs[qc].c * om.cap;
                const int nom = cs[qc].n0[OMINUS];
                int victim = -1;
                if (lane == 0) {
                    int nlive = 0;
                    for (int a = 0; a < nom; a++) nlive += is_hole(om.x[ob + a]) ? 0 : 1;
                    if (nlive > 0) {
                        int pick = 0;
                        if (nlive > 1) {
                            pick = (int)((float)nlive * r2);
                            if (pick > nlive - 1) pick = nlive - 1;
                        }
                        for (int a = 0; a < nom; a++) {
                            if (is_hole(om.x[ob + a])) continue;
                            if (pick-- == 0) { victim = a; break; }
                        }
                        om.x[ob + victim] = __int_as_float(0x7fc00000);
                    }
                }
                victim = __shfl_sync(FULL, victim, 0);
                __syncwarp();
                if (victim >= 0) add_hole(qc, OMINUS, victim);
            }
            head = min(head + 32, tail);
            __syncwarp();
        };
        for (int cl = 0; cl < ncell; cl++) {
            const int c = cs[cl].c, n = cs[cl].n0[s];
            const CellProb &Pc = P[cl];
            const float Tprob = Pc.p[s][Pc.n[s] - 1];
            for (int k0 = 0; k0 < n; k0 += 128) {
                // the test: four slots per lane from one Philox block per sub-cycle
                const int k = k0 + 4 * lane;
                unsigned hits = 0;
                int ent[4] = {0, 0, 0, 0};
                if (k < n) {
                    const unsigned live = k + 4 <= n ? 0xFu : (1u << (n - k)) - 1u;
                    for (int jj = 0; jj < nsub && hits != live; jj++) {
                        const hp_u4 u = hp_test_block(d.seed, (uint32_t)(k >> 2), (uint32_t)c, step, (uint32_t)s,
                                                      (uint32_t)jj);
#pragma unroll
                        for (int t = 0; t < 4; t++) {
                            const float R1 = hp_u01(hp_word(u, (uint32_t)t));
                            if (((live & ~hits) >> t) & 1u && R1 < Tprob) {
                                hits |= 1u << t;
                                ent[t] = (k + t) | (target_of(Pc, s, R1) << 20) | (cl << 24);
                            }
                        }
                    }
                }
                int total;
                int pos = tail + lower_lane_hits(hits, lt, total);
#pragma unroll
                for (int t = 0; t < 4; t++)
                    if ((hits >> t) & 1u) ring[(pos++) & (OXY_RING - 1)] = ent[t];
                tail += total;
                __syncwarp();
                while (tail - head >= 32) batch();
            }
        }
        while (tail > head) batch();
    }
    // fill every species' holes with its last particles, cell by cell
    for (int cl = 0; cl < ncell; cl++) {
        const int c = cs[cl].c;
#pragma unroll 1
        for (int s = 0; s < NSP; s++) {
            const DevSpecies &sp = d.sp[s];
            const size_t base = (size_t)c * sp.cap;
            int n = cs[cl].cnt[s];
            const int nh = cs[cl].nh[s];
            if (nh == 0) {
                if (lane == 0) sp.cnt[c] = n;
                continue;
            }
            if (!cs[cl].hole_over[s]) {
                if (lane == 0) {
                    int *h = holes[cl][s];
                    for (int a = 1; a < nh; a++) { // insertion sort: the list is short
                        const int v = h[a];
                        int b = a - 1;
                        while (b >= 0 && h[b] > v) { h[b + 1] = h[b]; b--; }
                        h[b + 1] = v;
                    }
                    for (int a = 0; a < nh; a++) {
                        while (n > 0 && is_hole(sp.x[base + n - 1])) n--;
                        const int hpos = h[a];
                        if (hpos >= n) continue;
                        const size_t from = base + n - 1, to = base + hpos;
                        sp.x[to] = sp.x[from]; sp.y[to] = sp.y[from];
                        sp.vx[to] = sp.vx[from]; sp.vy[to] = sp.vy[from]; sp.vz[to] = sp.vz[from];
                        n--;
                    }
                    while (n > 0 && is_hole(sp.x[base + n - 1])) n--;
                    sp.cnt[c] = n;
                }
            } else {
                // more holes than the list holds: stable compaction of the whole species
                int out = 0;
                for (int k0 = 0; k0 < n; k0 += 32) {
                    const int k = k0 + lane;
                    float x = 0.f, y = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
                    const bool in = k < n;
                    if (in) { x = sp.x[base + k]; y = sp.y[base + k]; vx = sp.vx[base + k]; vy = sp.vy[base + k]; vz = sp.vz[base + k]; }
                    const bool live = in && !is_hole(x);
                    const unsigned bl = __ballot_sync(FULL, live);
                    __syncwarp();
                    if (live) {
                        const size_t to = base + out + __popc(bl & lt);
                        sp.x[to] = x; sp.y[to] = y; sp.vx[to] = vx; sp.vy[to] = vy; sp.vz[to] = vz;
                    }
                    out += __popc(bl);
                    __syncwarp();
                }
                if (lane == 0) sp.cnt[c] = out;
            }
            __syncwarp();
        }
    }
}

template <int GAS, int G>
__global__ void __launch_bounds__(OXY_TPB, OXY_MINB) k_mcc_oxy(const DevCase *__restrict__ cases,
                                                     const int *__restrict__ item_start, int ncases, int items) {
    __shared__ int ring_s[OXY_TPB / 32][OXY_RING];
    __shared__ int holes_s[OXY_TPB / 32][G][NSP_ARO2][HOLE_CAP];
    __shared__ CellProb prob_s[OXY_TPB / 32][G];
    __shared__ OxyCell cell_s[OXY_TPB / 32][G];
    const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int first = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5) * G;
    if (first >= items) return;
    const unsigned lt = lanemask_lt();
    const int end = min(first + G, items);
    // a group that straddles two cases of a batch runs as two groups
    for (int g0 = first; g0 < end;) {
        const int ci = find_case(item_start, ncases, g0);
        const int g1 = min(end, item_start[ci + 1]);
        const DevCase &d = cases[ci];
        bool overflow = false;
        mcc_oxy_cells<GAS, G>(d, g0 - item_start[ci], g1 - g0, ring_s[wl], holes_s[wl], prob_s[wl], cell_s[wl],
                              lane, lt, overflow);
        if (__any_sync(FULL, overflow) && lane == 0) atomicOr(d.status, ST_OVERFLOW);
        g0 = g1;
    }
}

} // namespace

cudaError_t launch_mcc_oxy(const DevCase *cases, const int *item_start, int ncases, int items, int gas,
                           cudaStream_t st) {
    if (items <= 0) return cudaSuccess;
    constexpr int G = OXY_G;
    const unsigned nb = (unsigned)(((items + G - 1) / G * 32LL + OXY_TPB - 1) / OXY_TPB);
    prof::mark(st, "k_mcc_oxy");
    if (gas == 2) k_mcc_oxy<2, G><<<nb, OXY_TPB, 0, st>>>(cases, item_start, ncases, items);
    else if (gas == 1) k_mcc_oxy<1, G><<<nb, OXY_TPB, 0, st>>>(cases, item_start, ncases, items);
    else return cudaErrorNotSupported;
    return cudaGetLastError();
}

} // namespace hp
