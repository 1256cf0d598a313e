/*
 * oracle.h -- CPU checker for the PIC/MCC step (test infrastructure only).
 *
 * Nothing in the product links or calls this: tests/, the smoke check and
 * bench.py's CPU baseline use it to compute the expected result of each
 * operator on the same inputs the GPU sees.  It restates the reference's
 * per-step algorithm (the files cited in oracle.cpp) on a plain host data
 * layout: per species, particles in cell order with a count per cell (CSR).
 *
 * Two precisions:
 *   or_sim_new(..., precision = 32): the single-precision form the GPU
 *     kernels compute, operation for operation (same reduction trees, same
 *     elementary functions from include/hp_math.h, no fused multiply-adds),
 *     so results are expected to be bit-identical;
 *   precision = 64: the same algorithm with every particle, field and
 *     solver quantity in double and libm functions: the FP64 reference the
 *     mixed-precision GPU runs are compared with over whole RF cycles.
 */
#ifndef HP_ORACLE_H
#define HP_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_case {
    int ngx, ngy, ncx, ncy, nsp, cond_numr, n_unknowns;
    float dt_dx, dt_dy, dt, dx, dy, idx, idy, hdx, hdy, idxy;
    const int *sidx, *boundary, *face, *cond_id;
    const float *eps;        /* [C] EPS0 * eps_r */
    const float *dep_factor; /* [G] */
    float Ascale[5], q_density[5], Escale[5];
    /* collisions (Ar set) */
    const float *xsec;
    int n_logx, xw;
    float idlogx;
    float sigv[32], th[96];
    const float *prob; /* [3*C] */
    const float *back_vel1;
    const float *vsave;
    int nvel, mcc_n;
    uint64_t seed;
    /* field */
    const float *st, *st_sym, *row_scale; /* [5*G], [5*G], [G] node layout */
    const float *lap;                     /* [cond_numr*G] */
    int src_num, src_mid[8], efield_flag[8];
    float src_dc[8], src_ac[8], src_2pif[8], src_rphase[8];
    float pcg_tol2;
    int pcg_max_iter, field_mode;
    double pcg_rtol;
    /* launch shape the GPU used for the PCG reductions */
    int pcg_cluster, pcg_block;
    /* field_mode 2: separable inverse on the rectangle of unknowns */
    int fs_i0, fs_j0, fs_nx, fs_ny, fs_passes;
    const float *fs_V, *fs_Vt, *fs_W, *fs_Wt, *fs_inv;
    /* cell crossings per push: 0 one (reference), 1 until inside a cell */
    int move_mode;
    /* reaction set (0 Ar, 2 Ar/O2) and what the oxygen sets need */
    int gas, mcc_stride, mcc_all_species;
    int eedf_every; /* electron energy histogram every k-th step in or_run with accumulation (0 off) */
    float dt_mcc, np2c[5];
    const float *back_den1, *back_den2, *back_vel2;
    /* 1-2-1 density smoothing in Deposit (DensitySmoothing passes) */
    int n_smt;
    const int *dens_region; /* [G] */
    /* dielectric surface charge: present when n_diel > 0 */
    int n_diel;
    const int *sig_mode; /* [G] SumSource class: 0 none, 1 dielectric, 2 on a domain edge, 3 conductor */
    const float *area;   /* [G] node Area */
    /* power-driven sources: present when n_power > 0 */
    int n_power;
    float src_power[8];
    int cond_src_num[8], cond_power_id[8];
    int pd_intv;
    float pd_ratio;
    /* fluid species: the continuity solve (src/cuda_Fluid.cu) and its sources
     * (src/cuda_Diagnostic.cu:548-743); fluid_on 0 holds the densities at
     * their initial values */
    int nfsp, fluid_on, n_ave, nxl, nyl, tnrct;
    float dtc, denscale0;
    const float *fluid_cell_den;        /* [nfsp*C] initial density per cell */
    const float *fluid_den;             /* [nfsp*G] initial density per node (MCC input) */
    const int *xl, *yl;                 /* [3*nxl] x1, x2, yy; [3*nyl] xx, y1, y2 */
    const float *xl_fg, *yl_fg;         /* [2*nfsp*nxl]: fg1 block, then fg2 block (same for y) */
    const float *gax, *gbx, *gay, *gby; /* [nfsp*ngx*ncy], [nfsp*ncx*ngy] Gummel coefficients */
    const float *flux_x0, *flux_y0;     /* initial fluxes, same layouts */
    const int *plasma;                  /* [C] PlasmaRegion */
    float rate_f[96], rr[96];           /* rate factor per channel (tally -> m^-3 s^-1), CollF.RR */
    /* external circuit (src/cuda_Field.cu:43-103): present when external != 0 */
    int external;
    float cc_a[20];    /* [4*5] coefficients per conductor */
    float lap_sig[16]; /* [j*4 + i] charge on conductor i of the Laplace basis of conductor j */
    int circuit_mode;   /* hp_case_opts.circuit_mode */
} or_case;

typedef struct or_sim or_sim;

or_sim *or_sim_new(const or_case *c, int precision);
void or_sim_free(or_sim *s);
/* particles of species isp in cell order: counts[C], arrays of sum(counts) */
void or_set_particles(or_sim *s, int isp, const int *counts, const float *x, const float *y, const float *vx,
                      const float *vy, const float *vz);
size_t or_num_particles(or_sim *s, int isp);
void or_get_particles(or_sim *s, int isp, int *counts, float *x, float *y, float *vx, float *vy, float *vz);
/* double-precision copy of the particle state (precision 64) */
void or_get_particles_d(or_sim *s, int isp, int *counts, double *x, double *y, double *vx, double *vy, double *vz);
size_t or_num_movers(or_sim *s, int isp);
void or_get_movers(or_sim *s, int isp, int *counts, float *x, float *y, float *vx, float *vy, float *vz,
                   int8_t *codes);
/* node fields: which 0 Ex, 1 Ey, 2 phi, 3 phi_pois (float[G]); 4 den (double[nsp*G]);
 * 5 source (double[G]); 6 b (double[G]); 7 x (double[G]);
 * 8 dielectric surface weights (int64[nsp*G], HP_SIGMA_FRAC_BITS fraction bits); 9 Sigma (double[G]);
 * 10 AC amplitudes in use (float[src_num]); 11 fluid density per cell (float[nfsp*C]); 12 fluid density
 * per node (float[nfsp*G]); 13 fluid source per cell (float[nfsp*C]); 14 fluid x fluxes
 * (float[nfsp*ngx*ncy]); 15 fluid y fluxes (float[nfsp*ncx*ngy]) */
void or_get_grid(or_sim *s, int which, void *out);
/* hp_circuit.h: the reference's cofactor inverse (m: n x n, row stride 4) and one circuit step */
void or_circuit_inverse(float *m, int n);
void or_circuit_step(int nc, const float *cc, const float *lap, const float *vt, const float *qconv,
                     const float *surf, const float *pois_new, float *q, float *phi, float *pois, int mode);
void or_set_grid(or_sim *s, int which, const void *in);
void or_get_counters(or_sim *s, float *cond_charge, unsigned *mcc_count, int *pcg_iters);
/* 1 once a move_mode 1 walk reached its crossing bound (the particle was absorbed) */
int or_walk_bound_hit(or_sim *s);
/* most movers from beyond the 3x3 neighbourhood that one cell received in the last Move */
int or_far_max(or_sim *s);
/* the shared elementary functions (include/hp_math.h), for accuracy tests:
 * fn 0 exp, 1 log, 2 log10, 3 pow(x, y), 4 sin(2 pi x), 5 cos(2 pi x), 6 tan (x in [0, pi/2)), 7 atan */
void or_math(int fn, const float *x, const float *y, float *out, int n);

/* operators (reference order: Field, Move, SortBoundary, MCC, Deposit) */
void or_field(or_sim *s, int64_t tstep);
void or_move(or_sim *s);
void or_sort(or_sim *s);
void or_mcc(or_sim *s, int64_t tstep);
/* DEPOSIT (with the deck's smoothing passes) and the initial Deposit_Basic (without) */
void or_deposit(or_sim *s);
void or_deposit_basic(or_sim *s);
/* n full steps from tstep+1; accumulates node averages when ave != 0 */
void or_run(or_sim *s, int64_t tstep0, int nsteps, int accumulate);
void or_get_averages(or_sim *s, double *ave_den, double *ave_phi, int64_t *count);
/* running sums of the charge source and of Ex, Ey (double[G] each) */
void or_get_field_averages(or_sim *s, double *ave_src, double *ave_ex, double *ave_ey);
/* the electron energy histogram: 201 counts (0.25 eV bins, last = overflow) */
void or_get_eedf(or_sim *s, unsigned long long *h);
/* Scripted uniforms, for pinning the oracle against the reference's own MCC
 * code: u holds the draw lists of nkeys keys back to back, start[nkeys + 1]
 * their offsets; key = cell (flags bit 0 clear) or species * Csize + cell
 * (bit 0 set).  Every MCC draw (null-collision tests included) is then taken
 * in order from its key's list; flags bits 1, 2, 3 take the two draws passed
 * to one anewvel, maxwellv, newvel_ionsc call right to left (the pair mask,
 * bits 0-2 of flags >> 1).  u = NULL goes back to Philox.
 * or_script_overrun counts the draws asked for beyond a list's end (those
 * yield 1.0). */
void or_set_script(or_sim *s, int flags, const float *u, const int64_t *start, int nkeys);
long long or_script_overrun(or_sim *s);
/* the MCC's cross-section lookup: channel ch at energies engy[n] (eV) */
void or_xsec(or_sim *s, int ch, const float *engy, float *out, int n);
/* scattering kinematics with given uniforms, out[3n] = new velocity:
 * kind 0 anewvel:      in[7n] = energy, vel, unit direction x, y, z, rand1, rand2
 * kind 1 newvel_ionsc: in[6n] = relative velocity x, y, z, its magnitude, rand1, rand2
 * kind 2 maxwellv:     in[4n] = vsave sample, thermal speed, Rphi, Rthe */
void or_kinematics(or_sim *s, int kind, const float *in, float *out, int n);
/* One collision of a particle of species isp (velocity v[3]) with target t
 * of the Ar/O2 or O2 set, drawing from u[nu] (pair_rl: the pair mask of
 * or_set_script): ch the reaction channel (-1 none), keep
 * whether the particle stays (with velocity vout[3]), bsp[2] the species born
 * (-1 none) with velocities bv[6], kill whether an O- is removed.  Returns 1
 * when the list ran out. */
int or_collide_oxy(or_sim *s, int isp, int t, const float *v, float bv1, float bv2, const float *u, int nu,
                   int pair_rl, int *ch, int *keep, float *vout, int *bsp, float *bv, int *kill);
/* only the continuity solve (src/cuda_Fluid.cu:34-42), nsteps times, with
 * the fluid sources of grid 13 as they are */
void or_fluid_sweeps(or_sim *s, int nsteps);
/* hp_fluid_sources at n nodes: R[n*tnrct] rates in (neutral channels filled,
 * out), fden[nfsp*n], eden[n] (0.25 x the averaged electron density), bd1,
 * bd2[n], rr[tnrct]; S[nfsp*n] out */
void or_fluid_sources(int gas, int n, int tnrct, int nfsp, float *R, const float *fden, const float *eden,
                      const float *bd1, const float *bd2, const float *rr, float *S);
int or_num_threads(void);
void or_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
