// dev.cuh -- device-side case descriptors shared by the kernels and the host API.
//
// HBM layout of one case (all arrays owned by the library):
//   particles, per species s, structure of arrays over a cell-blocked slot pool:
//     x[s][c*cap + k], y, vx, vy, vz    float   (x, y = offset inside cell c in [0,1))
//     code[s][c*cap + k]                int8    (mover destination after Move)
//     cnt[s][c]                         int32   particles resident in cell c
//     nmov[s][c]                        int32   movers parked at the top of cell c
//     dcount[s][c*9 + code]             int32   of those, movers to each of the 3x3 cells
//   cell c = i*ncy + j for the cell whose lower-left node is (i, j); the
//   reference indexes the same cell by its node i*ngy + j and strides its
//   slots by Gsize (src/cuda_Particle.cu:44-52).  Slots of one cell are
//   contiguous here, so a warp that owns a cell reads 32 consecutive floats
//   per access.
//   grid: Ex, Ey, phi (float, node layout), den (double, nsp*Gsize),
//   source (double), PCG vectors in node layout (Gsize entries, non-unknown
//   nodes held at zero).
#pragma once
#include <cstdint>

// far movers (beyond the 3x3 neighbourhood) one destination cell accepts per
// step and species; more sets the overflow status.  Strongly driven small
// cases (65x33 nodes at 260-290 V) send up to ~45 into one cell in a step.
#define HP_FAR_BUCKET 128

#include "hpic.h" // HP_EEDF_BINS, HP_EEDF_DE
#include "hp_circuit.h"

namespace hp {

constexpr int DMAXSP = 5;
constexpr int DMAXCOND = 8;
constexpr int DMAXSRC = 8;

struct DevSpecies {
    float *x, *y, *vx, *vy, *vz;
    int8_t *code;
    int *cnt;
    int *nmov;
    int *dcount; // [C*9] movers per cell and destination code 0..8 (after Move)
    int cap;
    float Ascale, q_density, Escale, np2c;
};

// The power controller of the reference's Diagnostic (src/cuda_Diagnostic.cu:
// 365-420) per case: conductor surface charges of the last three steps,
// power accumulated since the last revision and the revision count.
struct PowerState {
    double surf[DMAXCOND], old[DMAXCOND], old2[DMAXCOND];
    float power[DMAXCOND];
    int count[DMAXCOND];
    int power_init;
    int pad;
};
static_assert(sizeof(PowerState) == 8 * DMAXCOND * 3 + 4 * DMAXCOND * 2 + 8, "PowerState layout (the Python binding sizes it)");

// The external circuit (src/cuda_Field.cu:43-103) per case: the circuit
// charge history, the absorbed charge of the last step, and the conductor
// potentials and Poisson-part surface charges of the last solve.
struct CircuitState {
    float q[4 * HP_CIRCUIT_MAX]; // q(t-1), q(t-2), q(t-3), q(t-4) per conductor
    float qconv[HP_CIRCUIT_MAX]; // -sum_s q_density_s x particles absorbed in the last step
    float phi[HP_CIRCUIT_MAX];   // conductor potentials (phi_cond)
    float pois[HP_CIRCUIT_MAX];  // Pois_SIG_Sol
};

struct DevCase {
    // geometry
    int ngx, ngy, ncx, ncy, G, C, nsp, gas, cond_numr, n_unknowns;
    float dt_dx, dt_dy, dt;
    float dx, dy, idx, idy, hdx, hdy, idxy;
    const int *sidx;        // StructureIndex [(ncx+2)*(ncy+2)]
    const int *boundary, *face, *cond_id; // [G]
    const float *eps;       // [C] EPS0 * eps_r
    const float *dep_factor;// [G]
    int n_smt;                      // 1-2-1 smoothing passes per Deposit (DensitySmoothing)
    const int *dens_region;         // [G] nodes the smoothing treats as inside
    double *smt;                    // [nsp*G] smoothing scratch (n_smt > 0)
    // dielectric surface charge (null without dielectric blocks): per
    // (species, node) particle weight in fixed point, HP_SIGMA_FRAC_BITS
    // fraction bits, added by Move's surface split and summed by SumSource
    long long *sig;                 // [nsp*G]
    const int *sig_mode;            // [G] SumSource class (0 none, 1 dielectric, 2 on a domain edge, 3 conductor)
    const float *area;              // [G] node Area
    double *sigma;                  // [G] Sigma: surface charge density where SumSource sets it
    int *dq_n;                      // dielectric crossings queued by Move for the Sort phase
    int dq_cap;
    int *dq_k;                      // [dq_cap] (cell << 7) | (species << 4) | direction
    float4 *dq_v;                   // [dq_cap] offset after the wrap and velocity (x, y, vx, vy)
    DevSpecies sp[DMAXSP];
    // field
    float *Ex, *Ey, *phi, *phi_p;   // [G]
    const float *lap;               // [cond_numr*G]
    const float *st;                // [5*G] stencil per node: W,S,C,N,E (0 off the unknowns)
    const float *st_sym;            // [5*G] row-scaled symmetric stencil (refinement mode)
    const float *row_scale;         // [G] 1/d_i used to symmetrise (refinement mode)
    float *pf_x, *pf_r, *pf_p, *pf_ap; // [G] FP32 PCG vectors
    float *pf_p2;                   // [G] the second search-direction buffer (directions alternate)
    float *pcg_halo;                // [2 x ngy x CTAs] each CTA's copy of the directions of its neighbours' nodes
    double *x64, *b64;              // [G] FP64 solution and right-hand side
    double *dots;                   // scratch for cluster reductions [64]
    double *pcg_part;               // [2 x 2 x CTAs] CTA totals of the cooperative grid solve (null: cluster)
    double *den;                    // [nsp*G]
    double *source;                 // [G]
    double4 *cw[DMAXSP];            // [C] per-cell corner weight sums
    double *ave_den, *ave_phi;      // [nsp*G], [G]
    double *ave_src, *ave_ex, *ave_ey; // [G] time sums of the charge source and of E
    // sources (src/cuda_Field.cu:10-20)
    int src_num;
    int src_mid[DMAXSRC];
    float src_dc[DMAXSRC], src_ac[DMAXSRC], src_2pif[DMAXSRC], src_rphase[DMAXSRC];
    int efield_flag[DMAXCOND];
    float *src_amp;                 // [src_num] AC amplitudes in use (the power controller revises them)
    // power-driven sources (null pw without any)
    PowerState *pw;
    unsigned int *cond_step;        // [nsp*cond_numr] particles absorbed per conductor in this step
    const int *cond_nodes;          // [n_cond_nodes] node | (conductor index << 24), nodes with a CondID
    int n_cond_nodes;
    int cond_src_num[DMAXCOND], cond_power_id[DMAXCOND];
    float src_power[DMAXSRC];
    int pd_intv;
    float pd_ratio;
    // external circuit (null cs without one)
    CircuitState *cs;
    int circuit_mode;                                   // hp_case_opts.circuit_mode
    float cc_a[HP_CIRCUIT_MAX * 5];                     // coefficients per conductor (src/Efield.c:70-78)
    float lap_sig[HP_CIRCUIT_MAX * HP_CIRCUIT_MAX];     // [j * HP_CIRCUIT_MAX + i]: conductor i in Laplace basis j
    // collisions
    const float *xsec;              // [n_logx * xw]
    int n_logx, xw;
    float idlogx;
    float sigv[32];                 // sigma-v maxima per (projectile, target): 3 Ar, 20 O2, 25 Ar/O2
    float th[96];                   // CollF.Th_e per reaction channel
    float mofm[96];
    int mcc_stride;                 // counters per cell in mcc_count (8 for Ar, 72 for the oxygen sets)
    int mcc_all_species;            // O2 set: 0 electrons only (the reference's launch), 1 every species
    float *prob;                    // [3*C]: electron P1, P2; ion P (Ar); P2 follows the Ar* density
    const float *back_vel1;         // [G]
    const float *back_den1, *back_den2, *back_vel2; // [G] (back_den2, back_vel2: oxygen sets)
    float *fluid_den;               // [nfsp*G] metastable / radical densities at the nodes (the MCC's input)
    const float *vsave;
    int nvel, mcc_n;
    float dt_mcc;                   // electron collision sub-step (DT_MCCn sub-cycles)
    uint64_t seed;
    // bookkeeping
    int64_t *tstep;                 // device step counter
    uint32_t *status;
    float *cond_charge;             // [nsp*cond_numr]
    unsigned int *mcc_count;        // [C*mcc_stride] collisions per cell and channel
    int *pcg_iters;                 // [2]: inner, outer of the last solve
    int64_t *ave_count;
    unsigned long long *eedf;       // [HP_EEDF_BINS+1] electron energy histogram since the last reset
    int eedf_every;                 // 0: off; k: sample every k-th step
    unsigned long long *pushes;     // [64] particles pushed by Move, spread over 32 counters, then
                                    // those of them whose slot changed (their vz was rewritten)
    unsigned long long *far_key;    // [nsp*C*HP_FAR_BUCKET] movers arriving from beyond the 3x3 neighbourhood
    int *far_in;                    // [nsp*C] entries in each bucket (cleared by Sort)
    int move_mode;                  // 0 one cell crossing per step (reference), 1 cross until inside a cell
    // separable inner solve (field_mode 2): rectangle of unknowns and scratch
    int fs_i0, fs_j0, fs_nx, fs_ny, fs_passes;
    float *fs_x;                    // [ny*nx] residual of the symmetrised system
    float *fs_a1, *fs_y;            // [ny*nx] products
    const float *fs_V, *fs_Vt, *fs_W, *fs_Wt, *fs_inv;
    double *fs_res;                 // [2]: final ||r||, ||b||
    // fluid species (metastables, radicals): the continuity solve of
    // src/cuda_Fluid.cu:34-167 and the source cycle of
    // src/cuda_Diagnostic.cu:268-330, 548-743.  nfsp 0 or fluid_on 0: the
    // densities stay at their initial values.
    int nfsp, fluid_on, n_ave, nxl, nyl, tnrct;
    float dtc, denscale0;           // continuity step dt x TimeStep_Conti; electron Denscale
    float *fden, *fsrc;             // [nfsp*C] cell densities and sources (m^-3, m^-3 s^-1)
    float *fflx, *ffly;             // [nfsp*ngx*ncy] x-face fluxes at i*ncy+j, [nfsp*ncx*ngy] y-face at i*ngy+j
    const int *fl_xl, *fl_yl;       // [3*nxl] x lines (x1, x2, y); [3*nyl] y lines (x, y1, y2)
    const float *fl_xfg, *fl_yfg;   // wall factors of every line: [nfsp*lines] fg1, then [nfsp*lines] fg2
    const float *gax, *gbx;         // [nfsp*ngx*ncy] Gummel coefficients of the x faces
    const float *gay, *gby;         // [nfsp*ncx*ngy] of the y faces
    const int *plasma;              // [C] PlasmaRegion
    double *fl_sum;                 // [G] electron density summed over the averaging window
    unsigned int *fl_base;          // [C*mcc_stride] collision tallies at the last average
    float rate_f[96], rr[96];       // tally -> rate factor and CollF.RR per reaction channel
    // solver controls
    int field_mode, pcg_max_iter;
    float pcg_tol2;
    double pcg_rtol;
};

} // namespace hp
