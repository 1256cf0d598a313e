/*
 * hpic.h -- C ABI of the B200 PIC/MCC step library (libhpic.so).
 *
 * The reference runs one discharge case per process through global
 * `void (*op)(void)` operator pointers bound by start_cuda()
 * (inc/main.h:25-32, src/cuda_start.cu:2-34) and called by main_cuda()
 * (src/cuda_main.cu:112-183) in the order
 *     PCG_SOLVER; EFIELD; MOVE; SORT_BOUNDARY; MCC; DEPOSIT.
 * This header keeps those entry points, one per operator, but every call
 * takes an explicit case handle and a CUDA stream instead of process
 * globals, returns a status instead of calling exit(), and never
 * synchronises the device implicitly.  No torch or CUDA types appear in the
 * signatures; `stream` is a cudaStream_t passed as void* (NULL = legacy
 * default stream).
 *
 * Ownership: the caller owns hp_case / hp_batch / hp_server handles; the
 * library owns every device allocation behind them.  Calls on distinct
 * handles may come from different host threads.
 */
#ifndef HPIC_H
#define HPIC_H

#include <stddef.h>
#include <stdint.h>

/* electron energy distribution (HP_GRID_EEDF): bins of HP_EEDF_DE eV from 0,
 * then one overflow bin */
/* Dielectric surface charge is kept per (species, node) as particle weight in
 * fixed point with this many fraction bits, so that its sums do not depend on
 * the order of the additions. */
#define HP_SIGMA_FRAC_BITS 28
#define HP_EEDF_BINS 200
#define HP_EEDF_DE 0.25f

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
typedef enum hp_status {
    HP_OK = 0,
    HP_ERR_ARG = 1,         /* bad argument (NULL handle, index out of range) */
    HP_ERR_DECK = 2,        /* deck failed the reference's validation rules (src/start.c:19-1430) */
    HP_ERR_CUDA = 3,        /* a CUDA runtime call failed; hp_last_error() has the text */
    HP_ERR_OOM = 4,         /* device or host allocation failed */
    HP_ERR_UNSUPPORTED = 5, /* deck feature outside this library's path (see hp_last_error) */
    HP_ERR_DEVICE = 6,      /* the case's device status word is non-zero (hp_case_status) */
    HP_ERR_CAPACITY = 7,    /* batch/server admission refused: memory or slot budget */
    HP_ERR_NO_CUDA = 8      /* no CUDA device: this library has no CPU fallback */
} hp_status;

/* Bits of the per-case device status word.  The reference has no error
 * reporting (checkCudaErrors/gpuErrchk call exit(), src/cuda_main.cu:2-9) and
 * silently halves an overfull cell (ReArgPtcls, src/cuda_Sortboundary.cu:23-40);
 * here the kernels set a bit and the host decides. */
#define HP_STATUS_CELL_OVERFLOW 0x1u /* a cell's slot pool is full (reference: ReArg condition) */
#define HP_STATUS_NONFINITE 0x2u     /* NaN/Inf in the field solve (reference: src/cuda_main.cu:227) */
#define HP_STATUS_PCG_NOCONV 0x4u    /* PCG hit its iteration cap */
#define HP_STATUS_WAIT_TIMEOUT 0x8u  /* a bounded device-side wait gave up */
#define HP_STATUS_WALK_BOUND 0x10u   /* move_mode 1: a particle crossed more cells than the domain spans
                                        (non-finite velocity); it was absorbed */
#define HP_STATUS_SURFACE_OVERFLOW 0x20u /* more dielectric crossings in one step than the case's queue holds;
                                            the excess left no surface charge */

/* Text of the last error raised on the calling host thread. */
const char *hp_last_error(void);

/* ---------------------------------------------------------------- set-up */
/* Host-side case description: the deck read and every table the step
 * consumes, built without touching a GPU.  It restates InputRead,
 * Geometry_setting, Source_setting, FieldSolverSetting and GasSetting
 * (src/main.c:45-49, src/start.c, src/load.c:121-246, src/Particle.c) plus
 * the set-up parts of main_cuda (Set_NullCollisionTime_cuda,
 * PCG_SOLVER_Laplace, Calculate_*GasPara). */
typedef struct hp_setup hp_setup;
struct hp_case_opts;
hp_status hp_setup_build(const char *deck_json, size_t deck_len, const struct hp_case_opts *opts, hp_setup **out);
void hp_setup_destroy(hp_setup *s);
/* The initial particle load of species isp.  layout 0: cell-sorted, offsets
 * in [0,1) and counts[Csize]; layout 1: the reference's load order with
 * global cell coordinates x = i + offset (its HCP arrays, inc/def.h:109-117)
 * and cells[] = i*ngy + j. */
hp_status hp_setup_get_particles(const hp_setup *s, int isp, int layout, int *counts_or_cells, float *x, float *y,
                                 float *vx, float *vy, float *vz, size_t cap, size_t *n_out);

/* ---------------------------------------------------------------- cases */
typedef struct hp_case hp_case;

typedef struct hp_case_opts {
    uint64_t seed;       /* loader seed (Park-Miller, src/Particle.c:211-226) and Philox key */
    int cap_per_cell;    /* particle slots per cell per species; 0 = Max_np / Gsize of the deck */
    int field_mode;      /* 0: reference rule, FP32 Jacobi-PCG to r'z < tol^2 (src/cuda_Field.cu:942-1072);
                            1: FP32 Jacobi-PCG inner solve with FP64 residual refinement to pcg_rtol;
                            2: FP64 refinement whose inner solve is the separable (tensor-product
                               eigenbasis) inverse of the operator, run as FP32 GEMMs; falls back to
                               1 when the operator is not separable */
    double pcg_rtol;     /* field_mode 1: ||b - A x||_2 / ||b||_2 target (default 1e-8) */
    int pcg_max_iter;    /* 0 = 100000, the reference's cap */
    int o2_all_species;  /* O2 gas: 0 = reference launch (electrons only, src/cuda_mcc.cu:76-77), 1 = all species */
    int device;          /* CUDA device ordinal */
    int gas_temp_mode;   /* background-gas temperature field: 0 = the reference's solve, whose matrix
                            leaves out the Neumann doubling on the x = 0 edge (src/load.c:171-237, Atemp)
                            and so cools the gas toward that wall; 1 = the same solve on the potential
                            operator, which keeps equal wall temperatures uniform */
    int move_mode;       /* cell crossings per push: 0 = one (the reference's wrap, src/cuda_Move.cu:227-255,
                            whose multi-cell loop is commented out, so a particle faster than a cell per
                            step keeps an offset outside [0,1) and its later gathers read the wrong
                            cell); 1 = cross cell by cell, with the boundary rule of every cell entered,
                            until the offset is inside a cell */
    int fs_passes;       /* field_mode 2: FP64 refinement passes per solve; 0 = 2 when pcg_rtol >= 1e-10
                            (each pass gains ~6 digits), else 3 */
    int eedf_every;      /* electron energy distribution (HP_GRID_EEDF): 0 = off, k = sample every k-th step */
    int gpu_load;        /* 1 = generate the initial particles on the device at case creation (same
                            Park-Miller draws and cell order as the host load; a cos() in the Maxwellian
                            may differ in its last double bit, so rare vx/vy differ by one float ulp);
                            0 = the reference's host load (default) */
    int fluid_fixed;     /* fluid species (Ar*, the O2 metastables and O atoms): 0 = the reference's
                            continuity solve, fed every AverageIter + 1 steps by the averaged collision
                            rates (src/cuda_Fluid.cu:34-167, src/cuda_Diagnostic.cu:268-330); 1 = hold
                            them at their initial densities */
    int circuit_mode;    /* external circuit (R/L/C on a conductor): 0 = the reference's update
                            (src/cuda_Field.cu:49-80), which divides V - K_t (a voltage minus a charge)
                            by cc0, advances every conductor's circuit charge with the history term K_t
                            of the last conductor and carries only the Poisson part of a conductor's
                            charge from step to step; 1 = a charge balance: V / cc0 - K_t, each
                            conductor's own K_t, and its whole charge (Laplace and Poisson parts)
                            carried, changed only by the circuit and the absorbed particles */
} hp_case_opts;

/* Default options. */
void hp_case_opts_default(hp_case_opts *opts);

/* Build a case from a JSON deck in the reference's format (the text, not a
 * path).  Replaces InputRead + Geometry_setting + Source_setting +
 * FieldSolverSetting + GasSetting (src/main.c:45-49) and main_cuda's
 * Set_*_cuda uploads (src/cuda_main.cu:17-27), including the initial
 * Deposit_Basic (src/cuda_main.cu:28). */
hp_status hp_case_create(const char *deck_json, size_t deck_len, const hp_case_opts *opts, hp_case **out);
hp_status hp_case_destroy(hp_case *c);

typedef struct hp_case_info {
    int ngx, ngy, ncx, ncy, Gsize, Csize;
    int nsp, main_gas, cond_numr, n_unknowns;
    int cap[8];            /* slots per cell, per species */
    int mcc_subcycles;     /* DT_MCCn (src/cuda_mcc.cu:258-266) */
    double dt, dx, dy;
    int64_t tstep;         /* steps taken */
    size_t device_bytes;   /* device memory held by the case (of a set-up: the estimate the server admits by) */
    int pcg_cluster;       /* CTAs per case in the field-solve cluster */
    int pcg_block;         /* threads per CTA in the field solve */
    int field_mode;        /* solver in use: 2 falls back to 1 when the operator is not separable */
    int mcc_stride;        /* collision counters per cell in HP_GRID_MCC_COUNT (8 Ar, 72 O2 and Ar/O2) */
    int n_smt;             /* 1-2-1 density smoothing passes per Deposit (the deck's DensitySmoothing) */
    int n_dielectric;      /* DielectricSpec blocks (surface charge kept when > 0) */
    int n_sources;         /* Source entries */
    int power_driven;      /* 1 when a conductor has a power-driven source (Power(W) != 0) */
    int n_reactions;       /* TnRct: reaction channels of the gas's collision set */
    int n_fluid;           /* nfsp: fluid species (1 Ar: Ar*; 4 O2: O2(a), O2(b), O, O(1D); 5 Ar/O2: Ar* first) */
    int circuit;           /* 1 when a conductor has an R/L/C external circuit (the reference's External_Flag) */
} hp_case_info;
hp_status hp_case_get_info(const hp_case *c, hp_case_info *out);
hp_status hp_setup_get_info(const hp_setup *s, hp_case_info *out);
/* Build a case from an existing set-up (uploads its tables and particles). */
hp_status hp_case_create_from_setup(const hp_setup *s, const hp_case_opts *opts, hp_case **out);

/* Device status word (HP_STATUS_* bits); synchronises on the case's last stream. */
hp_status hp_case_status(hp_case *c, uint32_t *status);

/* Step counter used by hp_Field (V(t) at t = tstep*dt) and by the MCC
 * random streams.  hp_step advances it by one before each step, like the
 * reference's `t += dt; tstep++` (src/cuda_main.cu:114-115). */
hp_status hp_case_set_tstep(hp_case *c, int64_t tstep);

/* ------------------------------------------- per-step operators (drop-in) */
/* PCG_SOLVER (src/cuda_Field.cu:133-181) followed by EFIELD =
 * Efield_cuda_Basic (src/cuda_Field.cu:2-42): Poisson solve with warm start,
 * potential assembly phi = sum_k V_k(t) phi_Lap,k + phi_Pois, E at nodes. */
hp_status hp_Field(hp_case *c, void *stream);
/* MOVE = Move_cuda -> MoveE_Basic (src/cuda_Move.cu:181-270). */
hp_status hp_Move(hp_case *c, void *stream);
/* SORT_BOUNDARY = SortBounndary_cuda -> SortBoundary_Basic
 * (src/cuda_Sortboundary.cu:4-13,41-258). */
hp_status hp_SortBoundary(hp_case *c, void *stream);
/* MCC = MCC_Ar_cuda / MCC_O2_cuda / MCC_ArO2_cuda by the deck's gas
 * (src/cuda_mcc.cu:2-20). */
hp_status hp_MCC(hp_case *c, void *stream);
/* DEPOSIT = Deposit_cuda (src/cuda_Deposit.cu:3-20): CIC density, boundary
 * scaling, rho/eps0, PCG right-hand side. */
hp_status hp_Deposit(hp_case *c, void *stream);
/* No counterpart in the reference.  The charge deposit of hp_Deposit for
 * callers that cannot let a library allocate device memory (a host that
 * budgets or pools every byte of the GPU itself, or a timed loop that must not
 * hit cudaMalloc's implicit device synchronisation): it allocates nothing and
 * writes the boundary-scaled node densities GPG.den of every species into
 * den_out (device memory, nsp * Gsize doubles, species-major), leaving the
 * case's own density, source and right-hand side untouched.  Its per-cell
 * scratch is one fixed array inside the library, 2^19 (species x cells)
 * entries (16 MiB), held on every GPU that loads the library until the
 * process exits; larger cases get HP_ERR_CAPACITY, and a case that belongs
 * to a batch gets HP_ERR_ARG (the batch steps it on its own stream).  Each
 * call outside stream capture looks up that array's device address with the
 * case's device current (and puts the caller's current device back), so the
 * first call on a device must come before any stream capture.  All calls
 * share the one array: calls whose work overlaps on the GPU (other streams,
 * other host threads) race and must be ordered by the caller.  Every scratch
 * entry a call reads it has written first. */
hp_status hp_Deposit_noalloc(hp_case *c, double *den_out, void *stream);
/* n steps of the main loop body (src/cuda_main.cu:114-183 without the
 * diagnostics and dump calls), fused where results allow; replayed from a
 * CUDA graph after the first call on a stream.  A case with fluid species
 * runs each step's continuity sweeps on a stream of its own, forked from and
 * joined back into `stream` within the step. */
hp_status hp_step(hp_case *c, int nsteps, void *stream);
/* Kernels launched by one hp_step (the kernel nodes of its captured graph;
 * 0 before the first hp_step).  No reference counterpart: launch accounting
 * for benchmarks. */
hp_status hp_step_kernels(const hp_case *c, int *n);

/* ------------------------------------------------- state interchange (host) */
/* Particles of species isp in cell-sorted order.  counts[Csize] receives the
 * particles per cell (cell = i*ncy + j); x, y are in-cell offsets in [0,1)
 * as in GCP (inc/def.h:118-127).  Arrays must hold `cap` entries; n_out
 * receives the total.  Synchronous. */
hp_status hp_get_particles(hp_case *c, int isp, int *counts, float *x, float *y, float *vx, float *vy,
                           float *vz, size_t cap, size_t *n_out);
hp_status hp_set_particles(hp_case *c, int isp, const int *counts, const float *x, const float *y,
                           const float *vx, const float *vy, const float *vz);
/* Movers parked by hp_Move and not yet re-binned by hp_SortBoundary: per
 * cell, in the order Move found them, with their wrapped offsets and the
 * direction code (di+1)*3 + (dj+1) of the cell they left through
 * (reference: the relative CellID of src/cuda_Move.cu:227-255). */
hp_status hp_get_movers(hp_case *c, int isp, int *counts, float *x, float *y, float *vx, float *vy, float *vz,
                        int8_t *codes, size_t cap, size_t *n_out);

/* Per-node / per-unknown arrays.  Synchronous. */
typedef enum hp_grid_field {
    HP_GRID_EX = 0,      /* float[Gsize]  GGA.Ex */
    HP_GRID_EY = 1,      /* float[Gsize]  GGA.Ey */
    HP_GRID_PHI = 2,     /* float[Gsize]  TotPotential */
    HP_GRID_PHI_POIS = 3,/* float[Gsize]  dev_phi (Poisson part) */
    HP_GRID_DEN = 4,     /* double[nsp*Gsize] GPG.den (boundary-scaled weight count) */
    HP_GRID_SOURCE = 5,  /* double[Gsize] dev_Source = rho/eps0 */
    HP_GRID_PCG_X = 6,   /* double[N] unknown vector (warm start) */
    HP_GRID_PCG_B = 7,   /* double[N] right-hand side */
    HP_GRID_AVE_DEN = 8, /* double[nsp*Gsize] running sum of den since hp_reset_averages */
    HP_GRID_AVE_PHI = 9, /* double[Gsize] running sum of TotPotential */
    HP_GRID_COND_CHARGE = 10, /* float[nsp*CondNUMR] absorbed particles per conductor */
    HP_GRID_MCC_COUNT = 11,   /* uint32[Csize*mcc_stride] collisions per cell and channel since creation */
    HP_GRID_EEDF = 12,        /* uint64[HP_EEDF_BINS + 1] electron energy histogram (HP_EEDF_DE eV bins,
                                 last = above HP_EEDF_BINS * HP_EEDF_DE eV),
                                 sampled every eedf_every steps since hp_reset_averages; no reference
                                 counterpart (the reference computes no EEDF) */
    HP_GRID_AVE_SOURCE = 13,  /* double[Gsize] running sum of the charge source rho/eps0 (the reference's
                                 ave_Source, src/cuda_SaveDump.cu:91-92) */
    HP_GRID_AVE_EX = 14,      /* double[Gsize] running sums of Ex and Ey (ave_Ex, ave_Ey) */
    HP_GRID_AVE_EY = 15,
    HP_GRID_SURFACE_CHARGE = 16, /* int64[nsp*Gsize] dielectric surface charge per species and node, in
                                    particle weights with HP_SIGMA_FRAC_BITS fraction bits (the reference's
                                    GPG.sigma); 0 bytes in a case without dielectric blocks */
    HP_GRID_SIGMA = 17,       /* double[Gsize] Sigma (the reference's dev_Sigma): the surface charge density
                                 SumSource sets at dielectric nodes (src/cuda_Deposit.cu:35-104) and
                                 Cond_Sigma at conductor and Dirichlet face nodes (src/cuda_Field.cu:500-558);
                                 0 bytes in a case with neither dielectrics nor power-driven sources */
    HP_GRID_SOURCE_AC = 18,   /* float[number of sources] AC amplitudes in use (V): the deck's, as revised by
                                 the power controller of power-driven sources */
    HP_GRID_POWER_STATE = 19, /* the power controller's state (opaque bytes; 0 bytes without power-driven
                                 sources), carried by checkpoints */
    /* fluid species, f = 0 .. nfsp-1 (Fluid_sp, src/Fluid.c:3-75); cell (i, j) at i*ncy + j */
    HP_GRID_FLUID_CELL_DEN = 20, /* float[nfsp*Csize] densities in the cells (GFC.den, m^-3) */
    HP_GRID_FLUID_DEN = 21,      /* float[nfsp*Gsize] densities at the nodes, the collisions' targets (Fluid_Den) */
    HP_GRID_FLUID_SOURCE = 22,   /* float[nfsp*Csize] sources of the last average (GFC.Source, m^-3 s^-1) */
    HP_GRID_FLUID_FLUX_X = 23,   /* float[nfsp*ngx*ncy] x-face fluxes at i*ncy + j (GFC.flux_x) */
    HP_GRID_FLUID_FLUX_Y = 24,   /* float[nfsp*ncx*ngy] y-face fluxes at i*ngy + j (GFC.flux_y) */
    HP_GRID_FLUID_STATE = 25,    /* the averaging window: electron density sum (double[Gsize]), tallies at
                                  the last average (uint32[Csize*mcc_stride]) and the collision
                                  probabilities (float[3*Csize]); carried by checkpoints */
    HP_GRID_CIRCUIT = 26         /* external circuit (0 bytes without one), float[28] (HP_CIRCUIT_MAX = 4): the
                                  circuit charge q(t-1..t-4) per conductor (4 rows of HP_CIRCUIT_MAX), the
                                  absorbed charge of the last step, the conductor potentials and the
                                  Poisson-part surface charges of the last solve (src/cuda_Field.cu:43-103) */
} hp_grid_field;
hp_status hp_get_grid(hp_case *c, hp_grid_field f, void *out, size_t bytes);
hp_status hp_set_grid(hp_case *c, hp_grid_field f, const void *in, size_t bytes);
/* Running averages (N_ave accumulation, src/cuda_Diagnostic.cu:505-547):
 * the sums above and the number of accumulated steps. */
hp_status hp_reset_averages(hp_case *c);
/* Averaged collision rates as the reference's ave_MCC_rate
 * (src/cuda_Diagnostic.cu:548-632): out[node * TnRct + channel], collisions
 * per m^3 and s since hp_reset_averages (Denscale of the projectile over
 * steps x dt), at the lower-left node of the cell they happened in.  `count`
 * is the capacity of out in floats (Gsize x TnRct; TnRct = hp_case_info
 * .n_reactions). */
hp_status hp_get_mcc_rates(hp_case *c, float *out, size_t count);

/* ------------------------------------------------------------ checkpoint */
/* Checkpoint of a case: the reference's V000 dump (V000_DUMP,
 * src/cuda_SaveDump.cu:5-106; readable by V000_LoadDUMP, src/load.c:5-120)
 * followed by an "HPICX001" extension holding the exact state a resumed run
 * needs (step counter and seed that key the random streams, particles as
 * in-cell offsets, field-solver warm start, charge grid, running sums,
 * tallies).  hp_case_load restores it into a case created from the same
 * deck and options, so that the run continues bit for bit as if it had not
 * stopped.  Not for a case inside a batch. */
hp_status hp_case_save(hp_case *c, const char *path);
hp_status hp_case_load(hp_case *c, const char *path);
hp_status hp_get_average_count(hp_case *c, int64_t *n);

/* Field-solver iteration count of the last hp_Field (reference: *FIter). */
hp_status hp_last_pcg_iters(hp_case *c, int *inner, int *outer);
/* field_mode 2: ||b - A x|| / ||b|| after the last solve (-1 in other modes). */
hp_status hp_last_field_residual(hp_case *c, double *rel);
/* Particles advanced by Move since the case was created (the unit of the
 * particle-pushes/s metric). */
hp_status hp_case_pushes(hp_case *c, int64_t *pushes);
/* Cumulative count of pushed particles whose slot changed in Move (they
 * rewrite all five components; a particle that keeps its slot rewrites four:
 * vz does not change in a push).  Feeds the push's algorithmic bytes
 * (32 B per particle + 8 B per slot change).  No reference counterpart. */
hp_status hp_case_slot_changes(hp_case *c, int64_t *changes);

/* The reference's own device structs (inc/def.h), field for field: a host
 * that keeps the reference's GCP / GPG / GGA arrays exchanges a case's state
 * through them.  Particle k of the cell whose lower-left node is
 * ID = i*ngy + j sits at gcp[ID + k*Gsize] (k < mpnc, the reference's MPNC;
 * src/cuda_Move.cu:195) with gpg[ID].PtNumInCell of them; x, y are offsets in
 * the cell.  hp_export_gcp writes a species' particles (every record of the
 * Gsize*mpnc block: unused slots zero, CellID the node ID), and with gpg
 * non-NULL its Gsize GPG records: PtNumInCell, MaxPtNumInCell = mpnc, den (the
 * charge grid's boundary-scaled count), ave_den (the average since
 * hp_reset_averages) and sigma (the dielectric surface charge in particle
 * weights); the collision counters are 0.  HP_ERR_CAPACITY when a cell holds
 * more than mpnc.  hp_import_gcp replaces a species' particles by those of a
 * GCP block and its GPG counts (as hp_set_particles).  hp_export_gga fills
 * Gsize GGA records from the case's tables and fields (Lap_Pot is
 * TotPotential - Pois_Pot). */
typedef struct hp_gcp {
    int CellID;
    float x, y, vx, vy, vz;
} hp_gcp;
typedef struct hp_gpg {
    int PtNumInCell, PtNumMoveInterCell, MaxPtNumInCell, PtNumMCCInCell, PtNullMCCInCell;
    float den, smt_den, sum_den, ave_den, sigma;
} hp_gpg;
typedef struct hp_gga {
    int Boundary, CondID, Face, DensRegion;
    float Area, Temp, BackDen1, BackVel1, BackDen2, BackVel2, Lap_Pot, Pois_Pot, Ex, Ey;
} hp_gga;
hp_status hp_export_gcp(hp_case *c, int isp, int mpnc, hp_gcp *gcp, hp_gpg *gpg);
hp_status hp_import_gcp(hp_case *c, int isp, int mpnc, const hp_gcp *gcp, const hp_gpg *gpg);
hp_status hp_export_gga(hp_case *c, hp_gga *gga);

/* Per-kernel device times of nsteps steps run operator by operator on
 * `stream` (not the captured graph of hp_step): every kernel launch is
 * bracketed by CUDA events, and the entries sum each kernel's launches and
 * milliseconds, in the order the kernels first ran.  *n = the number of
 * kernels; at most cap entries are written.  Not inside a stream capture;
 * one profile at a time per process.  The measurement tool behind the bench's
 * per-kernel rooflines (the reference times whole operators with events,
 * src/cuda_main.cu:112-236). */
typedef struct hp_kernel_stat {
    char name[32];
    int launches;
    double ms;
} hp_kernel_stat;
hp_status hp_profile_step(hp_case *c, int nsteps, void *stream, hp_kernel_stat *out, int cap, int *n);

/* Case tables (constant over a run), for checkers and tools.  `what`:
 * 0 StructureIndex int[(ncx+2)(ncy+2)], 1 A_idx int[Gsize], 2 node Boundary int[Gsize],
 * 3 node Face int[Gsize], 4 node CondID int[Gsize], 5 node Area float[Gsize],
 * 6 BackDen1 float[Gsize], 7 BackVel1 float[Gsize], 8 Laplace basis float[CondNUMR*Gsize],
 * 9 stencil float[5*N] (W,S,C,N,E per unknown, 0 where absent), 10 vsave float[nvel],
 * 11 cross-section table float[N_LOGX*(2+nch)], 12 CollF float[4*TnRct],
 * 13 sigma-v max float[n], 14 node DensRegion int[Gsize], 15 MCC probabilities float[3*Gsize],
 * 16 cell eps_r float[Csize], 17 BackDen2 float[Gsize], 18 BackVel2 float[Gsize],
 * 39 SumSource node class int[Gsize] (0 none, 1 dielectric, 2 dielectric on a
 * domain edge: Sigma doubled, 3 conductor: surface charge cleared),
 * 40 power-driven sources float[2 + nsrc + 2*CondNUMR]: steps between
 * revisions, VoltageUpDownRatio, target power per source, then per conductor
 * its number of power-driven sources and the first one's index,
 * 56 external circuit float[5*CondNUMR + CondNUMR^2] (empty without one): the
 * coefficients CC_a per conductor (src/Efield.c:70-78), then the charge on
 * conductor i of the Laplace basis of conductor k at k*CondNUMR + i
 * (Lap_SIG_Sol, src/cuda_Field.cu:207-216). */
hp_status hp_get_table(hp_case *c, int what, void *out, size_t bytes, size_t *bytes_needed);
hp_status hp_setup_get_table(const hp_setup *s, int what, void *out, size_t bytes, size_t *bytes_needed);

/* ------------------------------------------------------------- batches */
/* Many independent cases advanced together: one launch per phase over all
 * cases, each step captured as a CUDA graph.  Cases keep their own handles;
 * a case belongs to at most one batch at a time. */
typedef struct hp_batch hp_batch;
hp_status hp_batch_create(hp_case *const *cases, int n, hp_batch **out);
hp_status hp_batch_destroy(hp_batch *b);
hp_status hp_batch_step(hp_batch *b, int nsteps, void *stream);
/* Kernels launched by one hp_batch_step (0 before the first).  No reference
 * counterpart. */
hp_status hp_batch_step_kernels(const hp_batch *b, int *n);
/* Per-phase launch shape chosen by the autotuner (hp_batch_autotune) or set here. */
typedef struct hp_tune {
    int warps_per_block_particles; /* Move/Sort/Deposit: warps per CTA (one warp per cell), 1..16 */
    int pcg_block;                 /* PCG: threads per CTA */
    int pcg_cluster_max;           /* PCG: largest cluster per case */
    int move_unroll;               /* Move: chunks of 32 particles loaded per iteration: 1 (with a one-chunk
                                      prefetch), 2 or 4 */
    int mcc_cells_per_warp;        /* MCC (Ar): consecutive cells per warp sharing collision batches: 1, 2, 4, 8
                                      or 16 */
} hp_tune;
hp_status hp_batch_set_tune(hp_batch *b, const hp_tune *t);
hp_status hp_batch_get_tune(hp_batch *b, hp_tune *t);
/* The same launch shapes for a single case (hp_step re-captures its graph).
 * No reference counterpart. */
hp_status hp_case_set_tune(hp_case *c, const hp_tune *t);
hp_status hp_case_get_tune(const hp_case *c, hp_tune *t);
/* Time candidate launch shapes on the batch itself (state is saved and restored). */
hp_status hp_batch_autotune(hp_batch *b, void *stream);

/* ------------------------------------------------------------- serving */
typedef struct hp_server hp_server;
typedef struct hp_server_opts {
    size_t mem_budget_bytes;   /* admission cap on the total device footprint */
    int max_slots;             /* cases resident at once */
    int steps_per_launch;      /* steps between admission points */
    hp_case_opts case_opts;
} hp_server_opts;
/* Defaults: 150 GiB budget, 64 slots, 50 steps per round, hp_case_opts_default. */
void hp_server_opts_default(hp_server_opts *o);
hp_status hp_server_create(const hp_server_opts *o, hp_server **out);
hp_status hp_server_destroy(hp_server *s);
/* Queue a request: deck text and the number of steps to run.  Returns a
 * request id.  Never blocks on the device. */
hp_status hp_server_submit(hp_server *s, const char *deck_json, size_t len, int64_t nsteps, uint64_t seed,
                           int64_t *request_id);
/* Run one scheduling round: admit queued requests that fit, advance every
 * resident case by steps_per_launch (or fewer, to finish exactly), retire
 * finished cases.  Returns the number of requests still queued or running. */
hp_status hp_server_poll(hp_server *s, void *stream, int *pending);
typedef struct hp_result {
    int64_t request_id;
    int error;                 /* HP_OK, or why the request was not run (bad deck, over the budget, ...) */
    uint32_t status;           /* device status word at retirement */
    int64_t steps;
    int64_t particle_pushes;   /* sum over steps of particles advanced */
    double t_submit, t_admit, t_done; /* host clock, seconds */
    int ngx, ngy, nsp;
} hp_result;
/* Pop one finished result; time-averaged n_s (nsp*Gsize) and phi (Gsize)
 * are copied when the pointers are non-NULL.  *got = 0 when none is ready. */
hp_status hp_server_take_result(hp_server *s, hp_result *r, double *ave_den, size_t den_cap,
                                double *ave_phi, size_t phi_cap, int *got);

/* ------------------------------------------------------------- several GPUs
 * Cases -> devices for the batched and served forms on the GPUs of one node
 * (no counterpart in the reference, which runs one case on one GPU).  Cases
 * have no exchange step, so they shard by case: each device runs its share
 * as a batch and the host gathers the results.  Longest-first greedy: cases
 * in decreasing weight (ties: lower index) go to the device with the least
 * weight so far among those whose remaining budget holds the case's bytes
 * (ties: lower device).  weight: work per step (particles); bytes: device
 * footprint (hp_case_info.device_bytes of the set-up); budget: bytes per
 * device, NULL for none.  device_of[k] = -1 and HP_ERR_CAPACITY for a case
 * that fits nowhere (the others are still placed).  Host only: needs no GPU. */
hp_status hp_partition_cases(const double *weight, const size_t *bytes, int ncases, int ndevices,
                             const size_t *budget, int *device_of);

#ifdef __cplusplus
}
#endif
#endif /* HPIC_H */
