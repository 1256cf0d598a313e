// setup.hpp -- host-side case description: everything the per-step
// operators consume, built from a deck by build_setup() (setup.cpp).
//
// Field names follow the reference: GGA node arrays (inc/def.h:86-102),
// GCA cell arrays (inc/def.h:103-108), Species scalars (inc/def.h:142-169),
// CollF (inc/def.h:236-243), the cross-section tables (inc/def.h:244-392).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hp {

constexpr int MAXSP = 5;
constexpr double EPS0 = 8.8542e-12;  // inc/def.h:6
constexpr double CQ = 1.602e-19;     // inc/def.h:9
constexpr double NperTORR = 8.3221e20; // inc/def.h:12
constexpr double AMU = 1.66053e-27;  // inc/def.h:13
constexpr double DBLMIN = 1e-200;    // inc/def.h:11
constexpr double MPI = 3.14159265358979323846;

enum { BC_DIRICHLET = 1, BC_NEUMANN = 2, BC_CONDUCTOR = 3, BC_DIELECTRIC = 4 };
enum { F_LEFT = 0, F_RIGHT, F_UP, F_DOWN, F_UL, F_UR, F_LL, F_LR, F_NONE };
enum { GAS_AR = 0, GAS_O2 = 1, GAS_ARO2 = 2 };

struct SpeciesP {
    std::string name;
    int loadtype = 0;
    float x_center = 0, x_fall = 0, y_center = 0, y_fall = 0;
    int S_ID = 0;
    float InitDens = 0, Temp = 0, np2c = 0;
    int Ratio = 0, MAXNP = 0;
    float mass = 0, q = 0, q_density = 0, vti = 0, qm = 0, Escale = 0, Ascale = 0, Denscale = 0, MCCscale = 0;
    int np = 0;
};

struct BackGP {
    std::string name;
    float Ratio = 0, Pres = 0, Temp = 0, mass = 0, InitDens = 0;
};

struct FluidP {
    std::string name;
    float InitDens = 0, Temp = 0, mass = 0, Vel = 0, Gamma1 = 0;
};

struct CollFP {
    float Flag = 0, mofM = 0, Th_e = 0, RR = 0;
};

struct Setup {
    // --- deck scalars (src/start.c:19-1430) ---
    float xlength = 0, ylength = 0, zlength = 0;
    int ngx = 0, ngy = 0, ncx = 0, ncy = 0, Gsize = 0, Csize = 0;
    float dx = 0, dy = 0, idx = 0, idy = 0, idxy = 0, hdx = 0, hdy = 0;
    float dt = 0, dt_dx = 0, dt_dy = 0;
    int DT_PIC = 0;
    float PCGtol = 0, PCGtol2 = 0;
    int N_ave = 0, N_smt = 0;
    int main_gas = 0, nsp = 0, nfsp = 0, nBG = 0;
    float total_pressure = 0;
    SpeciesP sp[MAXSP];
    BackGP bg[2];
    FluidP fg[MAXSP];
    int cond_num = 0, cond_numr = 0;
    std::vector<int> cond_mid, cond_x0, cond_x1, cond_y0, cond_y1;
    std::vector<float> cond_temp;
    std::vector<float> cond_R, cond_L, cond_C;     // per ConductorSpec line
    bool external = false;                         // an R/L/C circuit on some conductor (External_Flag)
    std::vector<float> cc_a;                       // [cond_numr*5] circuit coefficients (src/Efield.c:70-78)
    std::vector<float> lap_sig;                    // [cond_numr*cond_numr] charge on conductor i of Laplace basis k at k*n+i
    int src_num = 0;
    std::vector<int> src_mid;
    std::vector<float> src_dc, src_ac, src_freq, src_2pifreq, src_rphase;
    std::vector<int> efield_flag; // per conductor (src/Efield.c:34-60)
    std::vector<float> src_power; // per source: target power (W), 0 for a voltage source
    std::vector<int> cond_src_num, cond_power_id; // per conductor: power-driven sources, the first one's index
    int pd_intv = 0;              // steps between amplitude revisions (PowerDrivenOption.Interval x DT_PIC)
    float pd_ratio = 0.05f;       // PowerDrivenOption.VoltageUpDownRatio
    bool power_driven() const {
        for (int n : cond_src_num)
            if (n > 0) return true;
        return false;
    }
    int diel_num = 0;             // DielectricSpec blocks
    std::vector<int> diel_mid, diel_x0, diel_x1, diel_y0, diel_y1;
    std::vector<float> diel_eps;
    float max_freq = 0;

    // --- geometry (src/start.c:1432-1642) ---
    std::vector<int> boundary, cond_id, face, dens_region; // [Gsize]
    std::vector<float> area, temp;                         // [Gsize]
    std::vector<int> plasma_region;                        // [Csize]
    std::vector<float> eps_r;                              // [Csize]
    std::vector<int> sidx;                                 // [(ncx+2)*(ncy+2)] StructureIndex
    std::vector<float> dep_factor;                         // [Gsize] DepositBoundary scale
    std::vector<int> sig_mode; // [Gsize] SumSource class: 0 none, 1 dielectric, 2 dielectric edge (x2), 3 conductor

    // --- field solver (src/start.c:1911-1998, src/load.c:121-246) ---
    int n_unknowns = 0;
    std::vector<int> a_idx;                        // [Gsize] 1-based, 0 = not an unknown
    std::vector<float> a_val, ta_val, matm;        // CSR values (reference layout)
    std::vector<int> ai, aj;                       // CSR 1-based
    std::vector<float> cond_b;                     // [cond_numr * N]
    std::vector<float> temp_b;                     // [N]
    std::vector<float> stencil;                    // [5*N]  W,S,C,N,E of A per unknown (0 = absent)
    std::vector<int> unk_node;                     // [N] node of each unknown
    std::vector<float> lap_basis;                  // [cond_numr * Gsize] Laplace solutions
    std::vector<float> back_den1, back_vel1, back_den2, back_vel2; // [Gsize]
    std::vector<float> node_temp;                  // [Gsize] gas temperature (K) after the solve

    // --- collisions (src/start.c:1003-1429, src/PhysicsData.c, src/cuda_mcc.cu:202-513) ---
    int TnRct = 0, n_logx = 0, n_cx = 0;
    float idlogx = 0;
    std::vector<CollFP> collf;      // [TnRct]
    std::vector<float> xsec;        // [n_logx * (2 + n_cx)] rows (xe, xee, cx_0..)
    std::vector<float> sigv;        // sigma-v max per target
    int mcc_n = 1;                  // DT_MCCn
    float dt_mcc = 0;
    std::vector<float> fluid_den;   // [nfsp * Gsize] metastable/radical densities at the nodes (MCC input)
    std::vector<float> vsave;       // Maxwellian speed table (src/Particle.c:176-210)
    int nvel = 0;

    // --- continuity solve of the fluid species (src/Fluid.c:3-256, src/cuda_Fluid.cu:3-349) ---
    int DT_CONTI = 1;
    float dtc = 0;                  // dt * TimeStep_Conti (src/Efield.c:8)
    int fluid_loadtype = 0;         // the neutral species' load (uniform, exponential, cosine)
    float fluid_x_center = 0, fluid_x_fall = 0, fluid_y_center = 0, fluid_y_fall = 0;
    std::vector<float> fluid_cell_den;  // [nfsp * Csize] initial density per cell
    // lines of plasma cells: x lines (x1, x2, yy) and y lines (xx, y1, y2)
    // with the wall factors fg1, fg2 of each species ([nfsp * lines])
    std::vector<int> xl_x1, xl_x2, xl_yy, yl_xx, yl_y1, yl_y2;
    std::vector<float> xl_fg1, xl_fg2, yl_fg1, yl_fg2;
    std::vector<float> fluid_D;     // [nfsp * Csize] diffusion coefficient
    // Gummel coefficients: x faces [nfsp][ngx*ncy] at i*ncy + j (i in 0..ncx),
    // y faces [nfsp][ncx*ngy] at i*ngy + j (j in 0..ncy)
    std::vector<float> gax, gbx, gay, gby;
    std::vector<float> flux_x0, flux_y0; // initial fluxes (Set_Fluid_cuda)
    // per reaction channel: the factor that turns a channel's tally over one
    // averaging window into a rate (m^-3 s^-1), as Average_*_MCC_rate
    // (src/cuda_Diagnostic.cu:548-633) scales by the projectile's Denscale
    std::vector<float> fluid_rate_f;    // [TnRct]

    // --- initial particles (src/Particle.c:3-175), cell-sorted ---
    std::vector<int> p_count[MAXSP];                       // [Csize]
    std::vector<float> p_x[MAXSP], p_y[MAXSP], p_vx[MAXSP], p_vy[MAXSP], p_vz[MAXSP];
    // the same load in the reference's HCP order (load order, global cell units)
    std::vector<float> h_x[MAXSP], h_y[MAXSP], h_vx[MAXSP], h_vy[MAXSP], h_vz[MAXSP];
    std::vector<int> h_cell[MAXSP];
    int cap[MAXSP] = {0};                                  // slots per cell
    uint64_t seed = 1;
    // a load left to the device (BuildOpts::defer_load): the loading cells in
    // load order, particles per loading cell, and the generator state at the
    // species' first draw; p_count etc. stay empty
    bool load_deferred = false;
    std::vector<int> load_cells[MAXSP];
    long load_seed[MAXSP] = {0};
    // first particle of each loading cell (prefix of the counts; size cells + 1)
    std::vector<long long> load_start[MAXSP];
};

struct BuildOpts {
    uint64_t seed = 1;
    int cap_per_cell = 0;
    int gas_temp_mode = 0; // 0 reference temperature operator, 1 potential operator (uniform for equal walls)
    bool defer_load = false; // leave the particle load to the device (hp_case_opts.gpu_load)
};

// Throws std::runtime_error with a message; the message starts with
// "deck:" for reference validation failures and "unsupported:" for deck
// features outside this library.
void build_setup(const char *json, size_t len, const BuildOpts &o, Setup &s);

} // namespace hp
