// setup.cpp -- case builder: deck -> every table the per-step operators read.
//
// This is a restatement of the reference's host setup, in the order its
// main() runs it (src/main.c:45-49): InputRead, Geometry_setting,
// Source_setting, FieldSolverSetting, GasSetting, followed by the parts of
// main_cuda's set-up that produce step inputs (Set_NullCollisionTime_cuda,
// PCG_SOLVER_Laplace with the gas-temperature solve and Calculate_*GasPara).
// Arithmetic keeps the reference's float/double mix so that tables compare
// bit-exactly with the reference's own set-up code (tests/test_setup.py).
#include "setup.hpp"
#include "hp_circuit.h"
#include "json.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <thread>

#include <dlfcn.h>

namespace hp {

namespace {

[[noreturn]] void deck_fail(const std::string &m) { throw std::runtime_error("deck: " + m); }
[[noreturn]] void unsupported(const std::string &m) { throw std::runtime_error("unsupported: " + m); }

float fnum(const JVal &o, const char *k) { return (float)o.number(k); }
int inum(const JVal &o, const char *k) { return (int)o.number(k); }
int ivnzc(const JVal &o, const char *k) { // src/start.c IVnZC
    int v = (int)o.number(k);
    if (v == 0) deck_fail(std::string("\"") + k + "\" = 0");
    return v;
}
float fvnzc(const JVal &o, const char *k) { // src/start.c FVnZC
    float v = (float)o.number(k);
    if (v == 0.0f) deck_fail(std::string("\"") + k + "\" = 0");
    return v;
}

// Park-Miller minimal standard generator with Schrage's decomposition
// (S. K. Park, K. W. Miller, CACM 31(10), 1988), as the reference's frand()
// (src/Particle.c:211-226), including its division by 2^31-2.
struct ParkMiller {
    long seed;
    float next() {
        const long a = 16807, m = 2147483647, q = 127773, r = 2836;
        long hi = seed / q;
        long lo = seed - q * hi;
        seed = a * lo - r * hi;
        if (seed <= 0) seed = seed + m;
        return (float)(seed / 2147483646.0);
    }
};

// The generator's state k draws ahead: seed * 16807^k mod (2^31 - 1), by
// square-and-multiply.  Each loaded particle takes exactly five draws, so the
// load splits over threads with every thread starting at its own offset and
// the result identical to the sequential loop.
long pm_skip(long seed, unsigned long long k) {
    const unsigned long long m = 2147483647ull;
    unsigned long long a = 16807, r = 1;
    while (k) {
        if (k & 1) r = r * a % m;
        a = a * a % m;
        k >>= 1;
    }
    return (long)(r * (unsigned long long)seed % m);
}

template <class F> void par_range(long long n, F f) {
    const unsigned hw = std::thread::hardware_concurrency();
    const int T = (int)std::max<long long>(1, std::min<long long>(hw ? hw : 1, n / 65536));
    if (T <= 1) {
        f(0LL, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < T; t++) th.emplace_back([&, t] { f(n * t / T, n * (t + 1) / T); });
    for (auto &x : th) x.join();
}

// F(v) = -2 v e^{-v^2}/sqrt(pi) + erf(v): the Maxwellian speed CDF
// (src/Particle.c:227-230), float argument, double evaluation.
float maxwell_cdf(float v) {
    // C semantics: exp and erf of the float promoted to double
    return (float)(-2 * v * exp((double)(-v * v)) / sqrt(MPI) + erf((double)v));
}

// The cells SetParticleLoad (src/Particle.c:3-175) fills, in its order, and
// the prefix of their counts (start[q] = first particle of cell lc[q]):
// UNIFORM n_per_cell in the window; EXPONETIAL and COSINE n_per_cell scaled
// by a Gaussian or cosine profile of the cell centre over every plasma cell
// (at least Ratio); NP_RATIO Ratio per cell in the window (strict upper bounds).
void load_cells(const Setup &s, const SpeciesP &p, const SpeciesP &l, std::vector<int> &lc,
                std::vector<long long> &start) {
    const int n_per_cell = (int)(p.InitDens * s.dx * s.dy * s.zlength / p.np2c);
    const float x_left = l.x_center, x_right = l.x_fall, y_top = l.y_center, y_bottom = l.y_fall;
    const float y0 = y_top / s.dy, y1 = y_bottom / s.dy - 1;
    const float x0 = x_left / s.dx, x1 = x_right / s.dx - 1;
    lc.clear();
    start.assign(1, 0);
    for (int i = 0; i < s.ncx; i++)
        for (int j = 0; j < s.ncy; j++) {
            if (s.plasma_region[(size_t)i * s.ncy + j] != 1) continue;
            int num = 0;
            const float xx = (float)i * s.dx + s.dx / 2, yy = (float)j * s.dy + s.dy / 2;
            switch (l.loadtype) {
            case 0: num = (i >= x0 && i <= x1 && j >= y0 && j <= y1) ? n_per_cell : 0; break;
            case 1: {
                // C semantics: the float arguments promoted to double
                const float ax = -1 * ((xx - x_left) / x_right) * ((xx - x_left) / x_right);
                const float ay = -1 * ((yy - y_bottom) / y_top) * ((yy - y_bottom) / y_top);
                const float wv = (float)(::exp((double)ax) * ::exp((double)ay));
                num = (int)(n_per_cell * wv);
                if (num < 1) num = p.Ratio;
                break;
            }
            case 2: {
                float wv;
                if (xx >= 0.06) wv = 0;
                else wv = (float)(::cos((xx - x_left) * MPI / 2 / x_right) * ::cos((yy - y_bottom) * MPI / 2 / y_top));
                num = (int)(n_per_cell * wv);
                if (num < 1) num = p.Ratio;
                break;
            }
            default: num = (i >= x0 && i < x1 && j >= y0 && j < y1) ? p.Ratio : 0; break;
            }
            if (num <= 0) continue;
            lc.push_back(i * s.ncy + j);
            start.push_back(start.back() + num);
        }
}

void build_vsave(Setup &s) { // src/Particle.c:183-201
    const float NVTS = 3.3f;
    int nvel = (int)(1. / (1 - maxwell_cdf((float)NVTS)));
    float dv = (float)(sqrt(MPI) / (4.0 * nvel));
    s.vsave.assign((size_t)nvel, 0.0f);
    int i = 0;
    for (int n = 0; n < nvel; n++) {
        float rr = (float)((1.0 * n) / nvel);
        while (maxwell_cdf(i * dv) < rr) i++;
        s.vsave[(size_t)n] = (float)(sqrt(2.0) * i * dv);
    }
    s.nvel = nvel;
}

void maxwellv(const Setup &s, ParkMiller &pm, float vti, float &vx, float &vy, float &vz) { // src/Particle.c:203-209
    int n = (int)((s.nvel - 1) * pm.next());
    float aphi = (float)(2 * MPI * pm.next());
    float costheta = 1 - 2 * pm.next();
    float sintheta = (float)sqrt((double)(1 - costheta * costheta));
    vx = (float)(vti * s.vsave[(size_t)n] * sintheta * cos((double)aphi));
    vy = (float)(vti * s.vsave[(size_t)n] * sintheta * sin((double)aphi));
    vz = (float)(vti * s.vsave[(size_t)n] * costheta);
}

// ---------------------------------------------------------------- deck
void read_geometry(const JVal &root, Setup &s, std::vector<int> &bx0, std::vector<int> &bx1, std::vector<int> &by0,
                   std::vector<int> &by1, std::vector<int> &bbc, std::vector<float> &btemp) {
    const JVal &geo = root.object("Geometry");
    const JVal &spec = geo.object("SystemSpec");
    s.xlength = fnum(spec, "X_length(m)");
    s.ylength = fnum(spec, "Y_length(m)");
    s.zlength = fnum(spec, "Z_length(m)");
    s.ngx = inum(spec, "NumGridx");
    s.ngy = inum(spec, "NumGridy");
    if (s.ngx < 3 || s.ngy < 3) deck_fail("NumGridx/NumGridy must be at least 3");
    const auto &bcs = geo.array("BoundaryCondition");
    if (bcs.size() < 4) deck_fail("\"BoundaryCondition\" is too small!(BoundaryNum>=4)"); // src/start.c:53-56
    for (size_t i = 0; i < bcs.size(); i++) {
        const JVal &b = bcs[i];
        int x0 = inum(b, "X0"), x1 = inum(b, "X1"), y0 = inum(b, "Y0"), y1 = inum(b, "Y1"), bc = inum(b, "B.C");
        if (x0 > x1) deck_fail("BoundaryCondition line " + std::to_string(i + 1) + ": X0 > X1");
        if (x1 >= s.ngx) deck_fail("BoundaryCondition line " + std::to_string(i + 1) + ": X1 >= NumGridx");
        if (y0 > y1) deck_fail("BoundaryCondition line " + std::to_string(i + 1) + ": Y0 > Y1");
        if (y1 >= s.ngy) deck_fail("BoundaryCondition line " + std::to_string(i + 1) + ": Y1 >= NumGridy");
        if (bc > 4) deck_fail("BoundaryCondition line " + std::to_string(i + 1) + ": B.C > 4");
        bx0.push_back(x0); bx1.push_back(x1); by0.push_back(y0); by1.push_back(y1); bbc.push_back(bc);
        btemp.push_back(fnum(b, "Temp"));
    }
    const auto &cs = geo.array("ConductorSpec");
    s.cond_num = (int)cs.size();
    if (s.cond_num < 2) deck_fail("\"Conductor\" is too small!(CondNum>=2)");
    if (s.cond_num > 100) deck_fail("\"Conductor\" is too large!(CondNum<100)");
    std::vector<int> ids; // src/start.c:109-144 M_ID ordering rules
    for (auto &c : cs) {
        int id = inum(c, "M_ID");
        if (id == 0) deck_fail("\"M_ID\" > 0");
        if (ids.empty()) {
            if (id != 1) deck_fail("First \"M_ID\" must be 1");
            ids.push_back(id);
        } else {
            if (ids.back() > id) deck_fail("\"M_ID\" must be written in order.");
            if (std::find(ids.begin(), ids.end(), id) == ids.end()) ids.push_back(id);
        }
    }
    s.cond_numr = (int)ids.size();
    int external = 0;
    for (size_t i = 0; i < cs.size(); i++) {
        const JVal &c = cs[i];
        int x0 = inum(c, "X0"), x1 = inum(c, "X1"), y0 = inum(c, "Y0"), y1 = inum(c, "Y1");
        if (x0 > x1 || x1 >= s.ngx || y0 > y1 || y1 >= s.ngy)
            deck_fail("ConductorSpec line " + std::to_string(i + 1) + ": bad extent");
        s.cond_mid.push_back(inum(c, "M_ID"));
        s.cond_x0.push_back(x0); s.cond_x1.push_back(x1); s.cond_y0.push_back(y0); s.cond_y1.push_back(y1);
        s.cond_temp.push_back(fnum(c, "Temp"));
        float R = fnum(c, "R(Ohm)"), L = fnum(c, "L(H)"), C = fnum(c, "C(F)");
        s.cond_R.push_back(R);
        s.cond_L.push_back(L);
        s.cond_C.push_back(C);
        if (!(L < 1e-30f && R < 1e-30f && C >= 1)) external = 1; // src/start.c:173-177
    }
    s.external = external != 0;
    if (s.external && s.cond_numr > HP_CIRCUIT_MAX)
        unsupported("external circuit with more than " + std::to_string(HP_CIRCUIT_MAX) + " conductors");
    const auto &src = geo.array("Source");
    s.src_num = (int)src.size();
    s.max_freq = 0.0f;
    for (size_t i = 0; i < src.size(); i++) {
        const JVal &c = src[i];
        int mid = inum(c, "M_ID");
        if (std::find(s.cond_mid.begin(), s.cond_mid.end(), mid) == s.cond_mid.end())
            deck_fail("Source line " + std::to_string(i + 1) + " is no matching Conductor");
        float dc = fnum(c, "DC(V)"), pw = fnum(c, "Power(W)"), ac = fnum(c, "AC(V)"), fr = fnum(c, "Freq(1/s)");
        float ph = fnum(c, "Phase(deg)");
        if (dc == 0 && pw == 0 && ac == 0) deck_fail("Source line " + std::to_string(i + 1) + " is error");
        s.src_mid.push_back(mid);
        s.src_power.push_back(pw);
        s.src_dc.push_back(dc);
        s.src_ac.push_back(ac);
        s.src_freq.push_back(fr);
        s.src_2pifreq.push_back((float)(2 * MPI * fr));
        s.src_rphase.push_back((float)(MPI / 180 * ph));
        if (fr != 0) s.max_freq = std::max(s.max_freq, fr);
    }
    // dielectric blocks (src/start.c:226-300): M_ID > 0, non-decreasing, none
    // shared with a conductor; node extents inside the grid; Epsilon = eps_r
    const auto &diel = geo.array("DielectricSpec");
    s.diel_num = (int)diel.size();
    int last_id = 0;
    for (size_t i = 0; i < diel.size(); i++) {
        const JVal &c = diel[i];
        const std::string line = "DielectricSpec line " + std::to_string(i + 1);
        int id = inum(c, "M_ID");
        if (id == 0) deck_fail("\"M_ID\" > 0");
        if (i > 0 && last_id > id) deck_fail("\"M_ID\" must be written in order.");
        last_id = id;
        if (std::find(s.cond_mid.begin(), s.cond_mid.end(), id) != s.cond_mid.end())
            deck_fail(line + ": M_ID is duplicated with a conductor");
        // StructureIndex holds a dielectric as its M_ID in 1..99 (src/start.c:1778)
        if (id < 0 || id > 99) deck_fail(line + ": M_ID must be in 1..99");
        int x0 = inum(c, "X0"), x1 = inum(c, "X1"), y0 = inum(c, "Y0"), y1 = inum(c, "Y1");
        if (x0 > x1) deck_fail(line + ": X0 > X1");
        if (x1 >= s.ngx) deck_fail(line + ": X1 >= NumGridx");
        if (y0 > y1) deck_fail(line + ": Y0 > Y1");
        if (y1 >= s.ngy) deck_fail(line + ": Y1 >= NumGridy");
        s.diel_mid.push_back(id);
        s.diel_x0.push_back(x0); s.diel_x1.push_back(x1); s.diel_y0.push_back(y0); s.diel_y1.push_back(y1);
        s.diel_eps.push_back(fnum(c, "Epsilon"));
    }
}

void read_species_block(const JVal &cs, const char *key, SpeciesP &p, float mass, float q) {
    const JVal &o = cs.object(key);
    p.name = key;
    p.S_ID = inum(o, "S_ID");
    p.InitDens = fnum(o, "Density");
    p.Temp = fnum(o, "Temp(eV)");
    p.np2c = fnum(o, "np2c");
    p.Ratio = inum(o, "Ratio");
    p.MAXNP = inum(o, "Max_np");
    p.mass = mass;
    p.q = q;
}

void read_load(const JVal &o, int &type, float &x0, float &x1, float &y0, float &y1, bool charged) {
    type = inum(o, "Loadtype");
    const JVal &lp = o.object("LoadPosition(m)");
    x0 = fnum(lp, "X0"); x1 = fnum(lp, "X1"); y0 = fnum(lp, "Y0"); y1 = fnum(lp, "Y1");
    if (type == 4) { // SMARTLOAD: accepted by the reader, rejected by the loader
    } else if (type == 0) {
        if (x0 >= x1 || y0 >= y1) deck_fail("Load position error (UNIFORM)");
    } else if (type == 1 || type == 2) {
        if (x0 * x1 * y0 * y1 < 0) deck_fail("Load position error");
    } else if (type == 3 && charged) {
    } else {
        deck_fail("\"Loadtype\" is error");
    }
}

void read_fluid(const JVal &ns, const char *key, FluidP &f, float mass) {
    const JVal &o = ns.object(key);
    f.name = key;
    f.InitDens = fnum(o, "Density");
    f.Temp = fnum(o, "Temp(eV)");
    f.mass = mass;
    f.Vel = (float)sqrt(f.Temp * 1.38e-23 / f.mass);
    f.Gamma1 = fnum(o, "Quenching");
}

void read_gas(const JVal &root, Setup &s) {
    const JVal &g = root.object("GasSpecies");
    s.main_gas = inum(g, "Type(0:Ar,1:O2,2:Ar/O2)");
    switch (s.main_gas) {
    case GAS_AR: s.nsp = 2; s.nfsp = 1; s.nBG = 1; break;
    case GAS_O2: s.nsp = 4; s.nfsp = 4; s.nBG = 1; break;
    case GAS_ARO2: s.nsp = 5; s.nfsp = 5; s.nBG = 2; break;
    default: deck_fail("\"Type\" is error in GasSpecies.");
    }
    s.total_pressure = fnum(g, "TotalPres(Torr)");
    const JVal &bgo = g.object("Background");
    const JVal &ns = g.object("NeutralSpecies");
    const JVal &cs = g.object("ChargeSpecies");
    const float me = (float)(5.485799486e-4 * AMU);
    const float mAr = (float)(39.950 * AMU), mArIon = (float)(39.9500 * AMU);
    const float mO2 = (float)(32.0000 * AMU), mO = (float)(16.0000 * AMU);
    const float qe = (float)(-1.0 * CQ), qi = (float)(1.0 * CQ);
    if (s.main_gas == GAS_AR) {
        BackGP &b = s.bg[0];
        b.name = "Argon"; b.Ratio = 1.0f; b.Pres = s.total_pressure;
        b.Temp = fnum(bgo.object("Argon"), "Temp(eV)");
        b.mass = mAr;
        b.InitDens = (float)(NperTORR * b.Pres / (b.Temp + DBLMIN));
        read_load(ns, s.fluid_loadtype, s.fluid_x_center, s.fluid_x_fall, s.fluid_y_center, s.fluid_y_fall, false);
        read_fluid(ns, "Ar*", s.fg[0], mAr);
        read_load(cs, s.sp[0].loadtype, s.sp[0].x_center, s.sp[0].x_fall, s.sp[0].y_center, s.sp[0].y_fall, true);
        read_species_block(cs, "Electron", s.sp[0], me, qe);
        read_species_block(cs, "Ar+", s.sp[1], mArIon, qi);
    } else if (s.main_gas == GAS_O2) {
        BackGP &b = s.bg[0];
        b.name = "Oxygen"; b.Ratio = 1.0f; b.Pres = s.total_pressure;
        b.Temp = fnum(bgo.object("Oxygen"), "Temp(eV)");
        b.mass = mO2;
        b.InitDens = (float)(NperTORR * b.Pres / (b.Temp + DBLMIN));
        read_load(ns, s.fluid_loadtype, s.fluid_x_center, s.fluid_x_fall, s.fluid_y_center, s.fluid_y_fall, false);
        read_fluid(ns, "O2A", s.fg[0], mO2);
        read_fluid(ns, "O2B", s.fg[1], mO2);
        read_fluid(ns, "OP", s.fg[2], mO);
        read_fluid(ns, "OD", s.fg[3], mO);
        read_load(cs, s.sp[0].loadtype, s.sp[0].x_center, s.sp[0].x_fall, s.sp[0].y_center, s.sp[0].y_fall, true);
        read_species_block(cs, "Electron", s.sp[0], me, qe);
        read_species_block(cs, "O2+", s.sp[1], mO2, qi);
        read_species_block(cs, "O+", s.sp[2], mO, qi);
        read_species_block(cs, "O-", s.sp[3], mO, qe);
    } else {
        float f1 = fnum(bgo.object("Argon"), "Ratio");
        float f2 = fnum(bgo.object("Oxygen"), "Ratio");
        f2 = f2 / (f1 + f2);
        BackGP &a = s.bg[0], &o = s.bg[1];
        a.name = "Argon"; a.Temp = fnum(bgo.object("Argon"), "Temp(eV)"); a.mass = mAr;
        o.name = "Oxygen"; o.Temp = fnum(bgo.object("Oxygen"), "Temp(eV)"); o.mass = mO2;
        a.Ratio = (float)(1.0 - f2);
        a.Pres = s.total_pressure * a.Ratio;
        o.Ratio = f2;
        o.Pres = s.total_pressure * o.Ratio;
        a.InitDens = (float)(NperTORR * a.Pres / (a.Temp + DBLMIN));
        o.InitDens = (float)(NperTORR * o.Pres / (o.Temp + DBLMIN));
        read_load(ns, s.fluid_loadtype, s.fluid_x_center, s.fluid_x_fall, s.fluid_y_center, s.fluid_y_fall, false);
        read_fluid(ns, "Ar*", s.fg[0], mAr);
        read_fluid(ns, "O2A", s.fg[1], mO2);
        read_fluid(ns, "O2B", s.fg[2], mO2);
        read_fluid(ns, "OP", s.fg[3], mO);
        read_fluid(ns, "OD", s.fg[4], mO);
        read_load(cs, s.sp[0].loadtype, s.sp[0].x_center, s.sp[0].x_fall, s.sp[0].y_center, s.sp[0].y_fall, true);
        read_species_block(cs, "Electron", s.sp[0], me, qe);
        read_species_block(cs, "Ar+", s.sp[1], mArIon, qi);
        read_species_block(cs, "O2+", s.sp[2], mO2, qi);
        read_species_block(cs, "O+", s.sp[3], mO, qi);
        read_species_block(cs, "O-", s.sp[4], mO, qe);
    }
}

void read_method(const JVal &root, Setup &s) { // src/start.c:732-747
    const JVal &m = root.object("SimulationMethod");
    s.DT_PIC = ivnzc(m, "TimeStep_PIC");
    s.DT_CONTI = ivnzc(m, "TimeStep_Conti");
    s.PCGtol = fvnzc(m, "PCGMarginOfError");
    s.PCGtol2 = s.PCGtol * s.PCGtol;
    ivnzc(m, "HistoryMax");
    ivnzc(m, "HistoryDivide");
    s.N_ave = ivnzc(m, "AverageIter");
    s.N_smt = inum(m, "DensitySmoothing");
    if (s.N_smt < 0) s.N_smt = 0;
    ivnzc(m, "ParticleLimit");
    if (inum(m, "ConstB_Flag")) unsupported("constant magnetic field (ConstB_Flag)");
    // ContinuitySteadyState (src/start.c:773-786) switches the continuity
    // solve of each fluid species off once its mean density settles
    if (m.has("ContinuitySteadyState") && inum(m.object("ContinuitySteadyState"), "Flag"))
        unsupported("ContinuitySteadyState (the continuity solve runs every step here)");
    // power-driven sources (src/start.c:786-790): the amplitude is revised
    // every Interval RF periods, by at most VoltageUpDownRatio upwards
    const JVal &pd = m.object("PowerDrivenOption");
    s.pd_intv = (int)((float)s.DT_PIC * fnum(pd, "Interval"));
    if (s.pd_intv == 0) s.pd_intv = 5 * s.DT_PIC;
    s.pd_ratio = fnum(pd, "VoltageUpDownRatio");
    if (s.pd_ratio == 0.0f) s.pd_ratio = 0.05f;
}

// ---------------------------------------------------------------- tables
// Tables live in data/ beside lib/ of the package; HPIC_DATA_DIR overrides.
std::string data_path(const char *file) {
    const char *env = getenv("HPIC_DATA_DIR");
    std::string dir;
    if (env && *env) {
        dir = env;
    } else {
        Dl_info info;
        if (dladdr((void *)&data_path, &info) && info.dli_fname) {
            std::string so = info.dli_fname;
            size_t cut = so.find_last_of('/');
            std::string libdir = cut == std::string::npos ? std::string(".") : so.substr(0, cut);
            dir = libdir + "/../data";
        }
    }
    if (!dir.empty() && dir.back() != '/') dir += '/';
    return dir + file;
}

void load_xsec(Setup &s) {
    const char *file = s.main_gas == GAS_AR ? "xsec_ar.txt" : s.main_gas == GAS_O2 ? "xsec_o2.txt" : "xsec_aro2.txt";
    std::ifstream in(data_path(file));
    if (!in) throw std::runtime_error(std::string("cannot open cross-section table ") + data_path(file));
    std::vector<std::string> lines;
    std::string line;
    while (std::getline(in, line))
        if (!line.empty() && line[0] != '#') lines.push_back(line);
    if (lines.size() < 3) throw std::runtime_error("bad cross-section table");
    int nlog, ncx, tn;
    float idl;
    {
        std::istringstream h(lines[0]);
        h >> nlog >> ncx >> tn >> idl;
    }
    if (tn != s.TnRct) throw std::runtime_error("cross-section table reaction count mismatch");
    std::vector<float> th(tn), rr(tn);
    {
        std::istringstream a(lines[1]);
        for (int i = 0; i < tn; i++) a >> th[i];
        std::istringstream b(lines[2]);
        for (int i = 0; i < tn; i++) b >> rr[i];
    }
    s.n_logx = nlog;
    s.n_cx = ncx;
    s.idlogx = idl;
    s.xsec.assign((size_t)nlog * (2 + ncx), 0.0f);
    for (int r = 0; r < nlog; r++) {
        std::istringstream rs(lines[3 + r]);
        for (int k = 0; k < 2 + ncx; k++) {
            float v;
            rs >> v;
            // the reference multiplies each resampled channel by its deck flag
            // (src/PhysicsData.c, e.g. :1615); flags are 0 or 1 in practice
            s.xsec[(size_t)r * (2 + ncx) + k] = k < 2 ? v : s.collf[(size_t)(k - 2)].Flag * v;
        }
    }
    for (int i = 0; i < tn; i++) {
        s.collf[(size_t)i].Th_e = th[i];
        s.collf[(size_t)i].RR = s.collf[(size_t)i].Flag != 0.0f && rr[i] != 0.0f ? s.collf[(size_t)i].Flag * rr[i] : 0.0f;
    }
}

void read_collisions(const JVal &root, Setup &s) { // src/start.c:1003-1057
    const JVal &co = root.object("Collision_On_Off");
    if (s.main_gas == GAS_AR) {
        s.TnRct = 10;
        s.collf.assign(10, CollFP());
        const JVal &a = co.object("ArgonCase");
        const char *keys[10] = {"0.e+Ar>e+Ar", "1.e+Ar>e+Ar*", "2.e+Ar>e+Ar*m", "3.e+Ar>2e+Ar^", "4.e+Ar*m>2e+Ar^",
                                "5.Ar+Ar^>Ar^+Ar", "6.Ar+Ar^>Ar+Ar^", "7.e+Ar*m>e+Ar", "8.Ar*m+Ar>e+Ar^+Ar",
                                "9.Ar+Ar*m>Ar+Ar"};
        for (int i = 0; i < 10; i++) s.collf[(size_t)i].Flag = fnum(a, keys[i]);
        float me = s.sp[0].mass, mi = s.sp[1].mass, mb = s.bg[0].mass, mf = s.fg[0].mass;
        float mofm[10] = {me / mb, me / mb, me / mb, me / mb, me / mf, mb / mi, mb / mi, me / mf, mf / mb, mb / mf};
        for (int i = 0; i < 10; i++) s.collf[(size_t)i].mofM = mofm[i];
    } else {
        // the O2 (67 channels) and Ar/O2 (88) sets: deck keys and mofM mass
        // pairs as the reference's reader lists them (src/start.c, the
        // "OxygenCase" / "Argon/OxygenCase" blocks), from data/channels_*.txt
        const bool aro2 = s.main_gas == GAS_ARO2;
        std::ifstream in(data_path(aro2 ? "channels_aro2.txt" : "channels_o2.txt"));
        if (!in) throw std::runtime_error("cannot open the reaction channel list");
        const JVal &a = co.object(aro2 ? "Argon/OxygenCase" : "OxygenCase");
        s.TnRct = aro2 ? 88 : 67;
        s.collf.assign((size_t)s.TnRct, CollFP());
        auto mass = [&](const std::string &m) -> float {
            if (m == "-") return 0.0f;
            const int k = std::atoi(m.c_str() + 2);
            if (m.compare(0, 2, "SP") == 0) return s.sp[k].mass;
            if (m.compare(0, 2, "BG") == 0) return s.bg[k].mass;
            return s.fg[k].mass;
        };
        std::string line;
        int nread = 0;
        while (std::getline(in, line)) {
            if (line.empty() || line[0] == '#') continue;
            std::istringstream ls(line);
            int k;
            std::string key, num, den;
            std::getline(ls >> k >> std::ws, key, '\t');
            ls >> num >> den;
            if (k < 0 || k >= s.TnRct) throw std::runtime_error("bad reaction channel list");
            s.collf[(size_t)k].Flag = fnum(a, key.c_str());
            const float md = mass(den);
            s.collf[(size_t)k].mofM = md != 0.0f ? mass(num) / md : 0.0f;
            nread++;
        }
        if (nread != s.TnRct) throw std::runtime_error("bad reaction channel list");
    }
    for (auto &c : s.collf)
        if (c.Flag < 0) c.Flag = 0.0f;
    load_xsec(s);
}

// ---------------------------------------------------------------- geometry

void geometry(Setup &s, const std::vector<int> &bx0, const std::vector<int> &bx1, const std::vector<int> &by0,
              const std::vector<int> &by1, const std::vector<int> &bbc, const std::vector<float> &btemp) {
    const int ngx = s.ngx, ngy = s.ngy;
    s.Gsize = ngx * ngy;
    s.ncx = ngx - 1;
    s.ncy = ngy - 1;
    s.Csize = s.ncx * s.ncy;
    const int ncx = s.ncx, ncy = s.ncy, G = s.Gsize;
    s.dx = s.xlength / ncx;
    s.dy = s.ylength / ncy;
    s.idx = 1 / s.dx;
    s.idy = 1 / s.dy;
    s.idxy = (float)(1.5 / (s.dx + s.dy));
    s.hdx = (float)(0.5 / s.dx);
    s.hdy = (float)(0.5 / s.dy);
    s.boundary.assign(G, 0);
    s.cond_id.assign(G, 0);
    s.temp.assign(G, 0.0f);
    s.face.assign(G, F_NONE);
    s.area.assign(G, (float)(s.dy * s.zlength));
    s.dens_region.assign(G, 0);
    s.plasma_region.assign(s.Csize, 1);
    s.eps_r.assign(s.Csize, 1.0f);
    // boundary lines (src/start.c:1491-1506)
    for (int j = 0; j < ngy; j++)
        for (int i = 0; i < ngx; i++) {
            int ID = i * ngy + j;
            for (size_t k = 0; k < bx0.size(); k++) {
                if (i >= bx0[k] && i <= bx1[k] && j >= by0[k] && j <= by1[k]) {
                    if (bbc[k] == BC_DIRICHLET) {
                        s.boundary[ID] = BC_DIRICHLET;
                        s.temp[ID] = btemp[k];
                    } else if (s.boundary[ID] != BC_DIRICHLET && bbc[k] == BC_NEUMANN) {
                        s.boundary[ID] = BC_NEUMANN;
                        s.temp[ID] = btemp[k];
                    }
                }
            }
        }
    // dielectrics (src/start.c:1507-1520)
    for (int k = 0; k < s.diel_num; k++)
        for (int i = s.diel_x0[k]; i <= s.diel_x1[k]; i++)
            for (int j = s.diel_y0[k]; j <= s.diel_y1[k]; j++) {
                int ID = i * ngy + j;
                if (s.boundary[ID] == 0) s.boundary[ID] = BC_DIELECTRIC;
                if (i < s.diel_x1[k] && j < s.diel_y1[k]) {
                    int CID = i * ncy + j;
                    s.plasma_region[CID] = 0;
                    s.eps_r[CID] = s.diel_eps[k];
                }
            }
    // conductors (src/start.c:1521-1537)
    for (int k = 0; k < s.cond_num; k++)
        for (int i = s.cond_x0[k]; i <= s.cond_x1[k]; i++)
            for (int j = s.cond_y0[k]; j <= s.cond_y1[k]; j++) {
                int ID = i * ngy + j;
                s.cond_id[ID] = s.cond_mid[k];
                if (s.boundary[ID] == 0 || s.boundary[ID] == BC_DIELECTRIC) {
                    s.boundary[ID] = BC_CONDUCTOR;
                    s.temp[ID] = s.cond_temp[k];
                }
                if (i < s.cond_x1[k] && j < s.cond_y1[k]) {
                    int CID = i * ncy + j;
                    s.plasma_region[CID] = 0;
                    s.eps_r[CID] = 0.0f;
                }
            }
    for (int i = 0; i < ncx; i++) // src/start.c:1539-1550
        for (int j = 0; j < ncy; j++)
            if (s.plasma_region[i * ncy + j] == 1) {
                int ID = i * ngy + j;
                s.dens_region[ID] = s.dens_region[ID + 1] = s.dens_region[ID + ngy] = s.dens_region[ID + ngy + 1] = 1;
            }
    // interior faces (src/start.c:1553-1626); eps_r is read into ints there
    for (int i = 1; i < ngx - 1; i++)
        for (int j = 1; j < ngy - 1; j++) {
            int ID = i * ngy + j, CID = i * ncy + j;
            int P1 = (int)s.eps_r[CID], P2 = (int)s.eps_r[CID - ncy], P3 = (int)s.eps_r[CID - 1],
                P4 = (int)s.eps_r[CID - ncy - 1];
            // dielectric and conductor nodes share the rule and the areas
            // (Face_To_Area, src/start.c:2053-2083)
            if (s.boundary[ID] != BC_CONDUCTOR && s.boundary[ID] != BC_DIELECTRIC) continue;
            int f = -1;
            if ((P2 == 1 && P1 == 1 && P4 == 1) || (P2 != 0 && P1 != 0 && P4 != 0 && P3 == 0)) f = F_UL;
            else if ((P2 == 1 && P1 == 1 && P3 == 1) || (P2 != 0 && P1 != 0 && P3 != 0 && P4 == 0)) f = F_UR;
            else if ((P2 == 1 && P1 == 1 && P4 != 1 && P3 != 1) || (P2 != 0 && P1 != 0 && P4 == 0 && P3 == 0)) f = F_UP;
            else if ((P4 == 1 && P3 == 1 && P2 == 1) || (P2 != 0 && P4 != 0 && P3 != 0 && P1 == 0)) f = F_LL;
            else if ((P4 == 1 && P3 == 1 && P1 == 1) || (P1 != 0 && P4 != 0 && P3 != 0 && P2 == 0)) f = F_LR;
            else if ((P4 == 1 && P3 == 1 && P1 != 1 && P2 != 1) || (P4 != 0 && P3 != 0 && P1 == 0 && P2 == 0)) f = F_DOWN;
            else if ((P4 == 1 && P2 == 1 && P1 != 1 && P3 != 1) || (P4 != 0 && P2 != 0 && P1 == 0 && P3 == 0)) f = F_LEFT;
            else if ((P4 != 1 && P2 != 1 && P1 == 1 && P3 == 1) || (P4 == 0 && P2 == 0 && P1 != 0 && P3 != 0)) f = F_RIGHT;
            if (f >= 0) {
                s.face[ID] = f;
                s.area[ID] = (f == F_UP || f == F_DOWN) ? s.dx * s.zlength
                             : (f == F_LEFT || f == F_RIGHT) ? s.dy * s.zlength
                                                             : (float)(0.5 * (s.dx + s.dy) * s.zlength);
            }
        }
    auto set = [&](int ID, int f, bool xarea) {
        s.face[ID] = f;
        s.area[ID] = xarea ? s.dx * s.zlength : s.dy * s.zlength;
    };
    // the last domain corner (src/start.c:1770-1774) reads vec_G[Gsize], one
    // past the array; that read is taken as CondID 0 here (what the
    // reference's heap held in the golden runs)
    auto cid = [&](int ID) { return ID >= 0 && ID < G ? s.cond_id[ID] : 0; };
    // left/right domain edges (src/start.c:1628-1691)
    for (int j = 1; j < ncy; j++) {
        int ID = j;
        if (s.boundary[ID] == BC_DIRICHLET) {
            set(ID, F_RIGHT, false);
            if (cid(ID + 1) == 0 && cid(ID - 1) != 0 && cid(ngy + ID) != 0) set(ID, F_UP, true);
            else if (cid(ID + 1) != 0 && cid(ID - 1) == 0 && cid(ngy + ID) != 0) set(ID, F_DOWN, true);
            else if (cid(ID + 1) != 0 && cid(ID - 1) != 0 && cid(ngy + ID) != 0) set(ID, F_NONE, false);
            else if (cid(ID + 1) == 0 && cid(ID - 1) == 0 && cid(ngy + ID) != 0) set(ID, F_NONE, false);
        } else if (s.boundary[ID] == BC_NEUMANN) {
            set(ID, F_NONE, false);
            if (cid(ID + 1) == 0 && cid(ID - 1) != 0 && cid(ngy + ID) != 0) set(ID, F_UP, true);
            else if (cid(ID + 1) != 0 && cid(ID - 1) == 0 && cid(ngy + ID) != 0) set(ID, F_DOWN, true);
            else if (cid(ID + 1) != 0 && cid(ID - 1) != 0 && cid(ngy + ID) == 0) set(ID, F_RIGHT, false);
        }
        ID = ncx * ngy + j;
        if (s.boundary[ID] == BC_DIRICHLET) {
            set(ID, F_LEFT, false);
            if (cid(ID + 1) == 0 && cid(ID - 1) != 0 && cid(ID - ngy) != 0) set(ID, F_UP, true);
            else if (cid(ID + 1) != 0 && cid(ID - 1) == 0 && cid(ID - ngy) != 0) set(ID, F_DOWN, true);
            else if (cid(ID + 1) != 0 && cid(ID - 1) != 0 && cid(ID - ngy) != 0) set(ID, F_NONE, false);
            else if (cid(ID + 1) == 0 && cid(ID - 1) == 0 && cid(ID - ngy) != 0) set(ID, F_NONE, false);
        } else if (s.boundary[ID] == BC_NEUMANN) {
            set(ID, F_NONE, false);
            if (cid(ID + 1) == 0 && cid(ID - 1) != 0 && cid(ID - ngy) != 0) set(ID, F_UP, true);
            else if (cid(ID + 1) != 0 && cid(ID - 1) == 0 && cid(ID - ngy) != 0) set(ID, F_DOWN, true);
            else if (cid(ID + 1) != 0 && cid(ID - 1) != 0 && cid(ID - ngy) == 0) set(ID, F_LEFT, false);
        }
    }
    // bottom/top domain edges (src/start.c:1692-1754)
    for (int i = 1; i < ncx; i++) {
        int ID = i * ngy;
        if (s.boundary[ID] == BC_DIRICHLET) {
            set(ID, F_UP, true);
            if (cid(ID + ngy) == 0 && cid(ID - ngy) != 0 && cid(ID + 1) != 0) set(ID, F_RIGHT, false);
            else if (cid(ID + ngy) != 0 && cid(ID - ngy) == 0 && cid(ID + 1) != 0) set(ID, F_LEFT, false);
            else if (cid(ID + ngy) != 0 && cid(ID - ngy) != 0 && cid(ID + 1) != 0) set(ID, F_NONE, false);
            else if (cid(ID + ngy) == 0 && cid(ID - ngy) == 0 && cid(ID + 1) != 0) set(ID, F_NONE, false);
        } else if (s.boundary[ID] == BC_NEUMANN) {
            set(ID, F_NONE, false);
            if (cid(ID + ngy) == 0 && cid(ID - ngy) != 0 && cid(ID + 1) != 0) set(ID, F_RIGHT, false);
            else if (cid(ID + ngy) != 0 && cid(ID - ngy) == 0 && cid(ID + 1) != 0) set(ID, F_LEFT, false);
            else if (cid(ID + ngy) != 0 && cid(ID - ngy) != 0 && cid(ID + 1) == 0) set(ID, F_UP, true);
        }
        ID = i * ngy + ncy;
        if (s.boundary[ID] == BC_DIRICHLET) {
            set(ID, F_DOWN, true);
            if (cid(ID + ngy) == 0 && cid(ID - ngy) != 0 && cid(ID - 1) != 0) set(ID, F_RIGHT, false);
            else if (cid(ID + ngy) != 0 && cid(ID - ngy) == 0 && cid(ID - 1) != 0) set(ID, F_LEFT, false);
            else if (cid(ID + ngy) != 0 && cid(ID - ngy) != 0 && cid(ID - 1) != 0) set(ID, F_NONE, false);
            else if (cid(ID + ngy) == 0 && cid(ID - ngy) == 0 && cid(ID - 1) != 0) set(ID, F_NONE, false);
        } else if (s.boundary[ID] == BC_NEUMANN) {
            set(ID, F_NONE, false);
            if (cid(ID + ngy) == 0 && cid(ID - ngy) != 0 && cid(ID - 1) != 0) set(ID, F_RIGHT, false);
            else if (cid(ID + ngy) != 0 && cid(ID - ngy) == 0 && cid(ID - 1) != 0) set(ID, F_LEFT, false);
            else if (cid(ID + ngy) != 0 && cid(ID - ngy) != 0 && cid(ID - 1) == 0) set(ID, F_DOWN, true);
        }
    }
    // domain corners (src/start.c:1755-1774)
    auto corner = [&](int ID, int f) {
        if (s.boundary[ID] == BC_DIRICHLET && cid(ID + 1) == 0) {
            s.face[ID] = f;
            s.area[ID] = (float)(0.5 * (s.dx + s.dy) * s.zlength);
        }
    };
    corner(0, F_UR);
    corner(ncx * ngy, F_UL);
    corner(ncy, F_LR);
    corner(ncx * ngy + ncy, F_LL);
    // StructureIndex on the (ncx+2) x (ncy+2) ghost grid (src/start.c:1776-1851)
    const int SY = ncy + 2;
    std::vector<int> SI((size_t)(ncx + 2) * SY, 0);
    auto si = [&](int a, int b) -> int & { return SI[(size_t)a * SY + b]; };
    for (int i = 0; i < ncx; i++)
        for (int j = 0; j < ncy; j++) {
            si(i + 1, j + 1) = 0;
            for (int k = 0; k < s.diel_num; k++)
                if (i >= s.diel_x0[k] && i < s.diel_x1[k] && j >= s.diel_y0[k] && j < s.diel_y1[k])
                    si(i + 1, j + 1) = s.diel_mid[k];
            for (int k = 0; k < s.cond_num; k++)
                if (i >= s.cond_x0[k] && i < s.cond_x1[k] && j >= s.cond_y0[k] && j < s.cond_y1[k])
                    si(i + 1, j + 1) = 100 + s.cond_mid[k];
        }
    for (int i = 1; i < ngx; i++) {
        if ((s.boundary[(i - 1) * ngy] == BC_NEUMANN || s.boundary[i * ngy] == BC_NEUMANN) && si(i, 1) == 0)
            si(i, 0) = -s.boundary[(i - 1) * ngy] - 2;
        else
            si(i, 0) = si(i, 1) ? si(i, 1) : -1;
        if ((s.boundary[(i - 1) * ngy + ncy] == BC_NEUMANN || s.boundary[i * ngy + ncy] == BC_NEUMANN) && si(i, ngy - 1) == 0)
            si(i, ngy) = -s.boundary[(i - 1) * ngy + ncy] - 6;
        else
            si(i, ngy) = si(i, ngy - 1) ? si(i, ngy - 1) : -1;
    }
    for (int j = 1; j < ngy; j++) {
        if ((s.boundary[j - 1] == BC_NEUMANN || s.boundary[j] == BC_NEUMANN) && si(1, j) == 0)
            si(0, j) = -s.boundary[j - 1];
        else
            si(0, j) = si(1, j) ? si(1, j) : -1;
        if ((s.boundary[ncx * ngy + j - 1] == BC_NEUMANN || s.boundary[ncx * ngy + j] == BC_NEUMANN) && si(ngx - 1, j) == 0)
            si(ngx, j) = -s.boundary[ncx * ngy + j] - 4;
        else
            si(ngx, j) = si(ngx - 1, j) ? si(ngx - 1, j) : -1;
    }
    si(0, 0) = -s.boundary[0];
    si(ncx + 1, 0) = -s.boundary[(ncx - 1) * ngy];
    si(0, ncy + 1) = -s.boundary[ngy + ncy];
    si(ncx + 1, ncy + 1) = -s.boundary[(ncy - 1) * ngy + ncy]; // the reference's index, kept as written
    s.sidx = SI;
    // DepositBoundary scale per node (src/cuda_Deposit.cu:277-288)
    s.dep_factor.assign(G, 1.0f);
    for (int ID = 0; ID < G; ID++) {
        float f = 1.0f;
        int fc = s.face[ID];
        if (fc == F_LEFT || fc == F_RIGHT || fc == F_UP || fc == F_DOWN) f *= 2;
        else if (fc == F_UL || fc == F_LL || fc == F_UR || fc == F_LR) f *= 4;
        if (s.boundary[ID] == BC_NEUMANN) f *= 2;
        else if (s.boundary[ID] == BC_DIRICHLET && fc != F_NONE && s.cond_id[ID] != 0) f *= 2;
        s.dep_factor[ID] = f;
    }
    // SumSource's node classes (src/cuda_Deposit.cu:35-104): on the domain
    // edges the node looks at its inward neighbour (x edges first), inside at
    // itself; a dielectric there adds its surface charge (Sigma = factor x
    // charge / Area), a conductor clears it
    s.sig_mode.assign(G, 0);
    if (s.diel_num > 0)
        for (int ID = 0; ID < G; ID++) {
            const int x = ID / ngy, y = ID % ngy;
            int nb = ID, edge = 1;
            if (x == 0) nb = ID + ngy;
            else if (x == ngx - 1) nb = ID - ngy;
            else if (y == 0) nb = ID + 1;
            else if (y == ngy - 1) nb = ID - 1;
            else edge = 0;
            if (s.boundary[nb] == BC_DIELECTRIC) s.sig_mode[ID] = edge ? 2 : 1;
            else if (s.boundary[nb] == BC_CONDUCTOR) s.sig_mode[ID] = 3;
        }
}

// ---------------------------------------------------------------- field solver matrix
void field_matrix(Setup &s) {
    const int ngx = s.ngx, ngy = s.ngy, ncx = s.ncx, ncy = s.ncy;
    s.a_idx.assign(s.Gsize, 0);
    int n = 1;
    for (int i = 0; i < ngx; i++) // src/start.c:1919-1928
        for (int j = 0; j < ngy; j++) {
            int G = i * ngy + j;
            if (!s.cond_id[G] && s.boundary[G] != BC_DIRICHLET) s.a_idx[G] = n++;
        }
    const int N = n - 1;
    s.n_unknowns = N;
    s.a_val.assign(5 * (size_t)N, 0.0f);
    s.ta_val.assign(5 * (size_t)N, 0.0f);
    s.ai.assign(N + 1, 0);
    s.aj.assign(5 * (size_t)N, 0);
    s.matm.assign(N, 0.0f);
    s.cond_b.assign((size_t)s.cond_numr * N, 0.0f);
    s.temp_b.assign(N, 0.0f);
    s.stencil.assign(5 * (size_t)N, 0.0f);
    s.unk_node.assign(N, 0);
    float dydx = (float)(0.5 * s.dy / s.dx);
    float dxdy = (float)(0.5 * s.dx / s.dy);
    auto epsr = [&](int a, int b) { return s.eps_r[(size_t)a * ncy + b]; };
    int m = 0, l = 0;
    s.ai[0] = 1;
    for (int i = 0; i < ngx; i++)
        for (int j = 0; j < ngy; j++) {
            if (!s.a_idx[i * ngy + j]) continue;
            int x1, y1, x2, y2;
            x1 = (i == 0) ? i : i - 1; y1 = (j == ncy) ? j - 1 : j; y2 = (j == 0) ? j : j - 1;
            float LEFT = dydx * (epsr(x1, y1) + epsr(x1, y2));
            x1 = (i == ncx) ? i - 1 : i; y1 = (j == ncy) ? j - 1 : j; y2 = (j == 0) ? j : j - 1;
            float RIGHT = dydx * (epsr(x1, y1) + epsr(x1, y2));
            y1 = (j == ncy) ? j - 1 : j; x1 = (i == ncx) ? i - 1 : i; x2 = (i == 0) ? i : i - 1;
            float UP = dxdy * (epsr(x1, y1) + epsr(x2, y1));
            y1 = (j == 0) ? j : j - 1; x1 = (i == ncx) ? i - 1 : i; x2 = (i == 0) ? i : i - 1;
            float DOWN = dxdy * (epsr(x1, y1) + epsr(x2, y1));
            int LEFT_NBC = (i == 0) ? 2 : 1, RIGHT_NBC = (i == ncx) ? 2 : 1;
            int UP_NBC = (j == ncy) ? 2 : 1, DOWN_NBC = (j == 0) ? 2 : 1;
            float *st = &s.stencil[5 * (size_t)l];
            s.unk_node[l] = i * ngy + j;
            auto nb = [&](int G, float coef, float aval, float tval, int slot) {
                if (s.cond_id[G]) {
                    s.cond_b[(size_t)(s.cond_id[G] - 1) * N + l] += coef;
                    s.temp_b[l] += coef * s.temp[G];
                } else if (s.boundary[G] == BC_DIRICHLET) {
                    s.temp_b[l] += coef * s.temp[G];
                } else {
                    s.a_val[m] = aval;
                    s.aj[m] = s.a_idx[G];
                    s.ta_val[m] = tval;
                    st[slot] = aval;
                    m++;
                }
            };
            if (i) nb((i - 1) * ngy + j, LEFT, (-LEFT) * RIGHT_NBC, (-LEFT) * RIGHT_NBC, 0);
            if (j) nb(i * ngy + j - 1, DOWN, (-DOWN) * UP_NBC, (-DOWN), 1);
            float C = LEFT + DOWN + UP + RIGHT;
            s.a_val[m] = C;
            s.matm[l] = 1 / C;
            s.aj[m] = s.a_idx[i * ngy + j];
            s.ta_val[m] = LEFT + DOWN + UP + RIGHT;
            st[2] = C;
            m++;
            if (j != ncy) nb(i * ngy + j + 1, UP, (-UP) * DOWN_NBC, (-UP), 3);
            if (i != ncx) nb((i + 1) * ngy + j, RIGHT, (-RIGHT) * LEFT_NBC, (-RIGHT), 4);
            l++;
            s.ai[l] = m + 1;
        }
    s.a_val.resize(m);
    s.ta_val.resize(m);
    s.aj.resize(m);
}

// BiCGSTAB in double (H. A. van der Vorst, SIAM J. Sci. Stat. Comput. 13,
// 1992) with Jacobi scaling, for the set-up solves.  The reference runs its
// FP32 PCG to its loose absolute tolerance there (src/cuda_Field.cu:182-236);
// solving to 1e-12 relative gives the limit that PCG approaches.
std::vector<double> setup_solve(const Setup &s, const std::vector<float> &vals, const std::vector<double> &b) {
    const int N = s.n_unknowns;
    auto matvec = [&](const std::vector<double> &x, std::vector<double> &y) {
        for (int r = 0; r < N; r++) {
            double acc = 0;
            for (int k = s.ai[r] - 1; k < s.ai[r + 1] - 1; k++) acc += (double)vals[k] * x[(size_t)s.aj[k] - 1];
            y[r] = acc;
        }
    };
    std::vector<double> dinv(N);
    for (int r = 0; r < N; r++) {
        double d = 0;
        for (int k = s.ai[r] - 1; k < s.ai[r + 1] - 1; k++)
            if (s.aj[k] - 1 == r) d = vals[k];
        dinv[r] = d != 0 ? 1.0 / d : 1.0;
    }
    std::vector<double> x(N, 0.0), r(b), rh(b), p(N, 0.0), v(N, 0.0), sv(N), t(N), y(N), z(N);
    double bn = 0;
    for (double q : b) bn += q * q;
    bn = sqrt(bn);
    if (bn == 0) return x;
    double rho = 1, alpha = 1, omega = 1;
    for (int it = 0; it < 20000; it++) {
        double rho1 = 0;
        for (int i = 0; i < N; i++) rho1 += rh[i] * r[i];
        if (rho1 == 0) break;
        double beta = (rho1 / rho) * (alpha / omega);
        for (int i = 0; i < N; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        for (int i = 0; i < N; i++) y[i] = dinv[i] * p[i];
        matvec(y, v);
        double rv = 0;
        for (int i = 0; i < N; i++) rv += rh[i] * v[i];
        alpha = rho1 / rv;
        for (int i = 0; i < N; i++) sv[i] = r[i] - alpha * v[i];
        for (int i = 0; i < N; i++) z[i] = dinv[i] * sv[i];
        matvec(z, t);
        double tt = 0, ts = 0;
        for (int i = 0; i < N; i++) { tt += t[i] * t[i]; ts += t[i] * sv[i]; }
        omega = tt > 0 ? ts / tt : 0;
        double rn = 0;
        for (int i = 0; i < N; i++) {
            x[i] += alpha * y[i] + omega * z[i];
            r[i] = sv[i] - omega * t[i];
            rn += r[i] * r[i];
        }
        rho = rho1;
        if (sqrt(rn) <= 1e-12 * bn || omega == 0) break;
    }
    return x;
}

// External circuit, Source_setting's coefficients (src/Efield.c:70-78): per
// conductor id (the last ConductorSpec line of an M_ID sets them), in the
// reference's mixed precision -- the terms with a double literal in double,
// the integer-literal ones in float, 1/C in float.
void circuit_coefficients(Setup &s) {
    s.cc_a.assign((size_t)s.cond_numr * 5, 0.0f);
    const double dtd = (double)s.dt;
    for (size_t i = 0; i < s.cond_mid.size(); i++) {
        const float L = s.cond_L[i], R = s.cond_R[i], C = s.cond_C[i], dt = s.dt;
        float *a = &s.cc_a[(size_t)(s.cond_mid[i] - 1) * 5];
        a[0] = (float)(2.25 * (double)L / dtd / dtd + 1.5 * (double)R / dtd + (double)(1 / C));
        a[1] = -6 * L / dt / dt - 2 * R / dt;
        a[2] = (float)(5.5 * (double)L / dtd / dtd + .5 * (double)R / dtd);
        a[3] = -2 * L / dt / dt;
        a[4] = (float)(.25 * (double)L / dtd / dtd);
    }
}

// The charge each conductor carries in each Laplace basis (PCG_SOLVER_Laplace,
// src/cuda_Field.cu:207-216): Cond_Sigma_Lap (src/cuda_Field.cu:448-499) at
// the conductor and Dirichlet face nodes, times the node Area, summed per
// CondID in node order in float.  lap_sig[k * cond_numr + i]: basis k,
// conductor i.
void circuit_laplace_charges(Setup &s) {
    const int ngx = s.ngx, ngy = s.ngy, G = s.Gsize, nc = s.cond_numr;
    std::vector<float> eps((size_t)s.Csize);
    for (int k = 0; k < s.Csize; k++) eps[k] = (float)(EPS0 * s.eps_r[k]);
    s.lap_sig.assign((size_t)nc * nc, 0.0f);
    const double dx = (double)s.dx, dy = (double)s.dy;
    for (int k = 0; k < nc; k++) {
        const float *P = &s.lap_basis[(size_t)k * G];
        for (int n = 0; n < G; n++) {
            if (!s.cond_id[n]) continue;
            const int b = s.boundary[n], f = s.face[n];
            float sig = 0.0f; // the reference clears the buffer before the kernel
            if ((b == 3 || b == 1) && f != 8) {
                const int x = n / ngy, y = n - x * ngy;
                int eT = x * (ngy - 1) + y;
                int eL = x ? eT - ngy + 1 : eT;
                int eD = y ? eT - 1 : eT;
                const int eX = eL + eD - eT;
                const int xo = (x == ngx - 1) ? ngy - 1 : 0, yo = (y == ngy - 1) ? 1 : 0;
                eT -= xo + yo;
                eL -= yo;
                eD -= xo;
                const int pL = x ? n - ngy : n, pR = (x == ngx - 1) ? n : n + ngy;
                const int pD = y ? n - 1 : n, pU = (y == ngy - 1) ? n : n + 1;
                auto up = [&] { return 0.5 * (double)(eps[eT] + eps[eL]) * (double)(P[n] - P[pU]) / dy; };
                auto down = [&] { return 0.5 * (double)(eps[eD] + eps[eX]) * (double)(P[n] - P[pD]) / dy; };
                auto left = [&] { return 0.5 * (double)(eps[eL] + eps[eX]) * (double)(P[n] - P[pL]) / dx; };
                auto right = [&] { return 0.5 * (double)(eps[eT] + eps[eD]) * (double)(P[n] - P[pR]) / dx; };
                switch (f) {
                case 2: sig = (float)up(); break;
                case 3: sig = (float)down(); break;
                case 0: sig = (float)left(); break;
                case 1: sig = (float)right(); break;
                case 4: sig = (float)(up() + left()); break;
                case 5: sig = (float)(up() + right()); break;
                case 6: sig = (float)(down() + left()); break;
                case 7: sig = (float)(down() + right()); break;
                default: break;
                }
            }
            float &acc = s.lap_sig[(size_t)k * nc + (s.cond_id[n] - 1)];
            acc += sig * s.area[n];
        }
    }
}

void laplace_and_gas(Setup &s, int gas_temp_mode) {
    const int N = s.n_unknowns, G = s.Gsize;
    // Laplace basis: conductor k at 1 V, the others at 0 V (src/cuda_Field.cu:192-219)
    // the cond_numr + 1 independent solves run on their own threads
    s.lap_basis.assign((size_t)s.cond_numr * G, 0.0f);
    std::vector<std::vector<double>> xs((size_t)s.cond_numr + 1);
    std::vector<std::thread> th;
    for (int k = 0; k < s.cond_numr; k++)
        th.emplace_back([&, k] {
            std::vector<double> b(N);
            for (int i = 0; i < N; i++) b[i] = s.cond_b[(size_t)k * N + i];
            xs[(size_t)k] = setup_solve(s, s.a_val, b);
        });
    // gas temperature: TA x = temp_b (src/cuda_Field.cu:221-233)
    th.emplace_back([&] {
        std::vector<double> b(N);
        for (int i = 0; i < N; i++) b[i] = s.temp_b[i];
        xs[(size_t)s.cond_numr] = setup_solve(s, gas_temp_mode == 1 ? s.a_val : s.ta_val, b);
    });
    for (auto &t : th) t.join();
    for (int k = 0; k < s.cond_numr; k++) {
        const std::vector<double> &x = xs[(size_t)k];
        float *phi = &s.lap_basis[(size_t)k * G];
        for (int g = 0; g < G; g++) {
            if (s.a_idx[g]) phi[g] = (float)x[(size_t)s.a_idx[g] - 1];
            else if (s.cond_id[g] == k + 1) phi[g] = 1.0f;
        }
    }
    {
        const std::vector<double> &x = xs[(size_t)s.cond_numr];
        s.node_temp = s.temp;
        for (int g = 0; g < G; g++)
            if (s.a_idx[g]) s.node_temp[g] = (float)x[(size_t)s.a_idx[g] - 1];
    }
    s.back_den1.assign(G, 0.0f);
    s.back_vel1.assign(G, 0.0f);
    s.back_den2.assign(G, 0.0f);
    s.back_vel2.assign(G, 0.0f);
    for (int g = 0; g < G; g++) { // src/cuda_Field.cu:661-678
        if (!s.dens_region[g]) continue;
        float T = s.node_temp[g];
        if (s.main_gas == GAS_AR || s.main_gas == GAS_O2) {
            s.back_den1[g] = (float)(NperTORR * s.bg[0].Pres / (T * 8.6142e-5 + DBLMIN));
            s.back_vel1[g] = (float)sqrt(T * 1.38e-23 / s.bg[0].mass);
        } else {
            s.back_den1[g] = (float)(NperTORR * s.bg[0].Pres / (T * 8.6142e-5 + DBLMIN));
            s.back_vel1[g] = (float)sqrt(T * 1.38e-23 / s.bg[0].mass);
            s.back_den2[g] = (float)(NperTORR * s.bg[1].Pres / (T * 8.6142e-5 + DBLMIN));
            s.back_vel2[g] = (float)sqrt(T * 1.38e-23 / s.bg[1].mass);
        }
    }
}

// ---------------------------------------------------------------- fluid species
// Ar_meta_omega (src/cuda_Fluid.cu:299-320): the collision integral of
// metastable Ar.  The reference's loop has no break, so every tabulated point
// above the argument overwrites the result and the last interval (50..100)
// decides; kept as written.
float ar_meta_omega(float value) {
    static const float tstar[27] = {0.250f, 0.267f, 0.286f, 0.308f, 0.333f, 0.364f, 0.400f, 0.444f, 0.500f,
                                    0.571f, 0.667f, 0.800f, 1.000f, 1.330f, 2.000f, 2.500f, 2.860f, 3.330f,
                                    4.000f, 5.000f, 6.670f, 10.00f, 12.50f, 16.67f, 25.00f, 50.00f, 100.0f};
    static const float omega[27] = {1.8714f, 1.8344f, 1.7962f, 1.7560f, 1.7142f, 1.6702f, 1.6238f, 1.5748f, 1.5228f,
                                    1.4676f, 1.4090f, 1.3466f, 1.2802f, 1.2096f, 1.1348f, 1.1042f, 1.0888f, 1.0738f,
                                    1.0592f, 1.0450f, 1.0318f, 1.0198f, 1.0154f, 1.0112f, 1.0072f, 1.0034f, 1.000f};
    float temp2 = 0.0f; // the reference's DBL_MIN (1e-200) as a float
    if (value < tstar[0]) temp2 = omega[0];
    else if (value > tstar[26]) temp2 = omega[26];
    else
        for (int i = 1; i < 27; i++)
            if (value < tstar[i]) {
                const float temp1 = (value - tstar[i - 1]) / (tstar[i] - tstar[i - 1]);
                temp2 = omega[i] * temp1 + omega[i - 1] * (1 - temp1);
            }
    return temp2;
}

// Sync_Fluid_GFCtoGFG_forDen (src/cuda_Fluid.cu:321-339): node (i, j) takes
// cell (i, j)'s density; a cell of the last column or row also writes node
// (i+1, j+1), as the reference does.
void fluid_cells_to_nodes(const Setup &s, const std::vector<float> &cell, std::vector<float> &node) {
    const int G = s.Gsize, C = s.Csize, ncy = s.ncy, ngy = s.ngy;
    node.assign((size_t)s.nfsp * G, 0.0f);
    for (int f = 0; f < s.nfsp; f++)
        for (int i = 0; i < s.ncx; i++)
            for (int j = 0; j < ncy; j++) {
                const float v = cell[(size_t)f * C + i * ncy + j];
                node[(size_t)f * G + i * ngy + j] = v;
                if (i == s.ncx - 1 || j == ncy - 1) node[(size_t)f * G + (i + 1) * ngy + j + 1] = v;
            }
}

// Fluid_Setting, Set_Con_Region and Set_Con_Boundary (src/Fluid.c:3-224),
// then Set_Fluid_cuda's diffusion coefficients, Gummel coefficients and
// initial fluxes (src/cuda_Fluid.cu:3-33,54-95,185-298).
void fluid_setting(Setup &s) {
    const int F = s.nfsp, C = s.Csize, ncx = s.ncx, ncy = s.ncy, ngy = s.ngy, ngx = s.ngx;
    s.dtc = s.dt * (float)s.DT_CONTI; // src/Efield.c:8
    s.fluid_cell_den.assign((size_t)F * C, 0.0f);
    for (int f = 0; f < F; f++)
        for (int i = 0; i < ncx; i++)
            for (int j = 0; j < ncy; j++) {
                const int c = i * ncy + j;
                if (s.plasma_region[c] == 0) continue;
                const float xx = (float)i * s.dx, yy = (float)j * s.dy;
                float v = s.fg[f].InitDens;
                if (s.fluid_loadtype == 1) {
                    const float ax = (xx - s.fluid_x_center) / s.fluid_x_fall, ay = (yy - s.fluid_y_center) / s.fluid_y_fall;
                    const float wv = (float)(::exp((double)(-1 * ax * ax)) * ::exp((double)(-1 * ay * ay)));
                    v = s.fg[f].InitDens * wv;
                } else if (s.fluid_loadtype == 2) {
                    const float wv = (float)std::fabs(::cos((double)(xx - s.fluid_x_center) * MPI / 2 / s.fluid_x_fall) *
                                                      ::cos((double)(yy - s.fluid_y_center) * MPI / 2 / s.fluid_y_fall));
                    v = s.fg[f].InitDens * wv;
                }
                s.fluid_cell_den[(size_t)f * C + c] = v;
            }
    fluid_cells_to_nodes(s, s.fluid_cell_den, s.fluid_den);
    // lines of consecutive plasma cells (PlasmaRegion 1): x lines row by row,
    // y lines column by column
    auto plasma = [&](int i, int j) { return s.plasma_region[(size_t)i * ncy + j] == 1; };
    s.xl_x1.clear(); s.xl_x2.clear(); s.xl_yy.clear(); s.yl_xx.clear(); s.yl_y1.clear(); s.yl_y2.clear();
    for (int j = 0; j < ncy; j++)
        for (int i = 0; i < ncx; i++) {
            if (!plasma(i, j)) continue;
            if (i == 0 || !plasma(i - 1, j)) { s.xl_x1.push_back(i); s.xl_yy.push_back(j); }
            if (i == ncx - 1 || !plasma(i + 1, j)) s.xl_x2.push_back(i);
        }
    for (int i = 0; i < ncx; i++)
        for (int j = 0; j < ncy; j++) {
            if (!plasma(i, j)) continue;
            if (j == 0 || !plasma(i, j - 1)) { s.yl_xx.push_back(i); s.yl_y1.push_back(j); }
            if (j == ncy - 1 || !plasma(i, j + 1)) s.yl_y2.push_back(j);
        }
    const int nx = (int)s.xl_x1.size(), ny = (int)s.yl_xx.size();
    // wall factors: Gamma1 ("Quenching"), 0 on a Neumann wall of the domain
    s.xl_fg1.assign((size_t)F * nx, 0.0f); s.xl_fg2.assign((size_t)F * nx, 0.0f);
    s.yl_fg1.assign((size_t)F * ny, 0.0f); s.yl_fg2.assign((size_t)F * ny, 0.0f);
    auto neu = [&](int g) { return s.boundary[g] == BC_NEUMANN; };
    for (int f = 0; f < F; f++) {
        const float g1 = s.fg[f].Gamma1;
        for (int k = 0; k < nx; k++) {
            const int x1 = s.xl_x1[k], x2 = s.xl_x2[k], yy = s.xl_yy[k];
            const int a = x1 * ngy + yy, a1 = x1 * ngy + yy + 1, b = (x2 + 1) * ngy + yy, b1 = (x2 + 1) * ngy + yy + 1;
            s.xl_fg1[(size_t)f * nx + k] = ((neu(a) || neu(a1)) && x1 == 0) ? 0.0f : g1;
            s.xl_fg2[(size_t)f * nx + k] = ((neu(b) || neu(b1)) && x2 == ncx - 1) ? 0.0f : g1;
        }
        for (int k = 0; k < ny; k++) {
            const int xx = s.yl_xx[k], y1 = s.yl_y1[k], y2 = s.yl_y2[k];
            const int a = xx * ngy + y1, a1 = (xx + 1) * ngy + y1, b = xx * ngy + y2 + 1, b1 = (xx + 1) * ngy + y2 + 1;
            s.yl_fg1[(size_t)f * ny + k] = ((neu(a) || neu(a1)) && y1 == 0) ? 0.0f : g1;
            s.yl_fg2[(size_t)f * ny + k] = ((neu(b) || neu(b1)) && y2 == ncy - 1) ? 0.0f : g1;
        }
    }
    // diffusion coefficients (Cal_D_Argon / Cal_D_Oxygen / Cal_D_ArO2) from
    // the gas temperature of the cell's four nodes
    s.fluid_D.assign((size_t)F * C, 0.0f);
    const float P = s.total_pressure;
    for (int f = 0; f < F; f++)
        for (int i = 0; i < ncx; i++)
            for (int j = 0; j < ncy; j++) {
                const int g = i * ngy + j;
                const float *T4 = s.node_temp.data();
                const float T = (float)(0.25 * (double)(T4[g] + T4[g + 1] + T4[g + ngy] + T4[g + ngy + 1]));
                double D;
                if (s.main_gas == GAS_AR) {
                    const float om = ar_meta_omega(T / 124.0f);
                    D = 1.997279e-4 * ::sqrt((double)T / 39.948) * (double)T / (double)(P * 11.682724f * om) * 20;
                } else {
                    // the float square root of a float argument (the reference
                    // is C++: sqrt(float) is the float overload); the
                    // reference's sigma^2 constants are floats
                    const double s0 = (double)0.08559f, s1 = (double)0.10892f, s2 = (double)0.08650f;
                    if (s.main_gas == GAS_O2) {
                        if (f <= 1) D = 2.63e-3 * (double)std::sqrt(T * T * T * 24 / 32 / 32) / (double)P * s2;
                        else D = 2.63e-3 * (double)std::sqrt(T * T * T * 24 / 16 / 16) / (double)P * s1;
                    } else {
                        if (f == 0) D = 2.63e-3 * ::sqrt((double)(T * T * T * 24) / 39.948 / 39.948) / (double)P * s0;
                        else if (f <= 2) D = 2.63e-3 * (double)std::sqrt(T * T * T * 24 / 32 / 32) / (double)P * s2;
                        else D = 2.63e-3 * (double)std::sqrt(T * T * T * 24 / 16 / 16) / (double)P * s1;
                    }
                }
                s.fluid_D[(size_t)f * C + i * ncy + j] = (float)D;
            }
    // Gummel coefficients (calculate_gummel_coef_x/_y; the x interior face
    // averages D[i-1] with itself, as the reference writes it)
    s.gax.assign((size_t)F * ngx * ncy, 0.0f); s.gbx.assign((size_t)F * ngx * ncy, 0.0f);
    s.gay.assign((size_t)F * ncx * ngy, 0.0f); s.gby.assign((size_t)F * ncx * ngy, 0.0f);
    for (int f = 0; f < F; f++) {
        float *ax = &s.gax[(size_t)f * ngx * ncy], *bx = &s.gbx[(size_t)f * ngx * ncy];
        float *ay = &s.gay[(size_t)f * ncx * ngy], *by = &s.gby[(size_t)f * ncx * ngy];
        const float *D = &s.fluid_D[(size_t)f * C];
        const double m = (double)s.fg[f].mass;
        for (int k = 0; k < nx; k++) {
            const int x1 = s.xl_x1[k], x2 = s.xl_x2[k], yy = s.xl_yy[k];
            const double fg1 = s.xl_fg1[(size_t)f * nx + k], fg2 = s.xl_fg2[(size_t)f * nx + k];
            bx[x1 * ncy + yy] = (float)(-fg1 * (-0.25 * ::sqrt((double)s.node_temp[x1 * ngy + yy] * 1.38e-23 / m)));
            ax[x1 * ncy + yy] = 0;
            for (int i = x1 + 1; i <= x2; i++) {
                ax[i * ncy + yy] = (D[(i - 1) * ncy + yy] + D[(i - 1) * ncy + yy]) / 2 / s.dx;
                bx[i * ncy + yy] = ax[i * ncy + yy];
            }
            ax[(x2 + 1) * ncy + yy] = (float)(fg2 * (0.25 * ::sqrt((double)s.node_temp[x2 * ngy + yy] * 1.38e-23 / m)));
            bx[(x2 + 1) * ncy + yy] = 0;
        }
        for (int k = 0; k < ny; k++) {
            const int xx = s.yl_xx[k], y1 = s.yl_y1[k], y2 = s.yl_y2[k];
            const double fg1 = s.yl_fg1[(size_t)f * ny + k], fg2 = s.yl_fg2[(size_t)f * ny + k];
            by[xx * ngy + y1] = (float)(-fg1 * (-0.25 * ::sqrt((double)s.node_temp[xx * ngy + y1] * 1.38e-23 / m)));
            ay[xx * ngy + y1] = 0;
            for (int j = y1 + 1; j <= y2; j++) {
                ay[xx * ngy + j] = (D[xx * ncy + j - 1] + D[xx * ncy + j]) / 2 / s.dy;
                by[xx * ngy + j] = ay[xx * ngy + j];
            }
            ay[xx * ngy + y2 + 1] = (float)(fg2 * (0.25 * ::sqrt((double)s.node_temp[xx * ngy + y2] * 1.38e-23 / m)));
            by[xx * ngy + y2 + 1] = 0;
        }
    }
    // tally -> rate factors (Average_Argon/Oxygen/ArO2_MCC_rate): channel
    // ranges scaled by Denscale / N_ave / dt of their projectile, a few
    // single channels by Denscale x (1 / N_ave / dt), as the reference groups
    // the float operations
    s.fluid_rate_f.assign((size_t)std::max(s.TnRct, 1), 0.0f);
    auto range = [&](int a, int b, int sp) {
        const float t = s.sp[sp].Denscale / (float)s.N_ave / s.dt;
        for (int k = a; k <= b && k < s.TnRct; k++) s.fluid_rate_f[k] = t;
    };
    auto single = [&](int k, int sp) {
        const float t = 1 / (float)s.N_ave / s.dt;
        if (k < s.TnRct) s.fluid_rate_f[k] = s.sp[sp].Denscale * t;
    };
    if (s.main_gas == GAS_AR) {
        range(0, 6, 0);
        range(8, 8, 0);
    } else if (s.main_gas == GAS_O2) {
        range(0, 40, 0); range(41, 46, 3); range(47, 52, 1); range(53, 57, 2);
        single(58, 3);
    } else {
        range(0, 45, 0); range(46, 51, 4); range(52, 59, 2); range(60, 64, 3); range(65, 67, 1);
        single(69, 3); single(70, 3); single(79, 1); single(80, 1); single(81, 0);
    }
    // initial fluxes (Calculate_Flux_x/_y of Set_Fluid_cuda)
    s.flux_x0.assign((size_t)F * ngx * ncy, 0.0f);
    s.flux_y0.assign((size_t)F * ncx * ngy, 0.0f);
    for (int f = 0; f < F; f++) {
        const float *ax = &s.gax[(size_t)f * ngx * ncy], *bx = &s.gbx[(size_t)f * ngx * ncy];
        const float *ay = &s.gay[(size_t)f * ncx * ngy], *by = &s.gby[(size_t)f * ncx * ngy];
        const float *den = &s.fluid_cell_den[(size_t)f * C];
        float *fx = &s.flux_x0[(size_t)f * ngx * ncy], *fy = &s.flux_y0[(size_t)f * ncx * ngy];
        for (int k = 0; k < nx; k++) {
            const int x1 = s.xl_x1[k], x2 = s.xl_x2[k], yy = s.xl_yy[k];
            fx[x1 * ncy + yy] = -s.xl_fg1[(size_t)f * nx + k] * bx[x1 * ncy + yy] * den[x1 * ncy + yy];
            for (int i = x1 + 1; i <= x2; i++)
                fx[i * ncy + yy] = ax[i * ncy + yy] * den[(i - 1) * ncy + yy] - bx[i * ncy + yy] * den[i * ncy + yy];
            fx[(x2 + 1) * ncy + yy] = s.xl_fg2[(size_t)f * nx + k] * ax[(x2 + 1) * ncy + yy] * den[x2 * ncy + yy];
        }
        for (int k = 0; k < ny; k++) {
            const int xx = s.yl_xx[k], y1 = s.yl_y1[k], y2 = s.yl_y2[k];
            fy[xx * ngy + y1] = -s.yl_fg1[(size_t)f * ny + k] * by[xx * ngy + y1] * den[xx * ncy + y1];
            for (int j = y1 + 1; j <= y2; j++)
                fy[xx * ngy + j] = ay[xx * ngy + j] * den[xx * ncy + j - 1] - by[xx * ngy + j] * den[xx * ncy + j];
            fy[xx * ngy + y2 + 1] = s.yl_fg2[(size_t)f * ny + k] * ay[xx * ngy + y2 + 1] * den[xx * ncy + y2];
        }
    }
}

// ---------------------------------------------------------------- species + load
void gas_setting(Setup &s, const BuildOpts &o) { // src/start.c:1999-2051
    // the reference seeds frand() with getpid() (src/main.c:43); any seed in
    // [1, 2^31-2] is used as is, others are folded into that range
    long pm_seed = (o.seed >= 1 && o.seed <= 2147483646ull) ? (long)o.seed : (long)(o.seed % 2147483646ull) + 1;
    ParkMiller pm{pm_seed};
    s.seed = o.seed;
    build_vsave(s);
    for (int isp = 0; isp < s.nsp; isp++) {
        SpeciesP &p = s.sp[isp];
        p.q_density = p.q * p.np2c;
        p.vti = (float)sqrt(CQ * p.Temp / p.mass);
        p.qm = p.q / p.mass;
        p.Escale = (float)(0.5 * p.mass / CQ);
        p.Ascale = p.qm * s.dt;
        p.Denscale = p.np2c / s.dx / s.dy;
        p.MCCscale = 1 / p.np2c * s.dx * s.dy * s.dt;
        int cap = o.cap_per_cell > 0 ? o.cap_per_cell : p.MAXNP / s.Gsize;
        cap = std::max(cap, 32);
        s.cap[isp] = (cap + 31) / 32 * 32;
        // SetParticleLoad (src/Particle.c:3-175) with SP[0]'s load type and
        // window: the loading cells in the reference's order (i outer, j
        // inner), each with its particle count, and the first particle of each
        const SpeciesP &l = s.sp[0];
        if (l.loadtype == 4) unsupported("particle load type SMARTLOAD (the reference exits on it)");
        std::vector<int> lc;
        std::vector<long long> &lstart = s.load_start[isp];
        load_cells(s, p, l, lc, lstart);
        const long long np = lstart.back();
        auto &hx = s.h_x[isp], &hy = s.h_y[isp], &hvx = s.h_vx[isp], &hvy = s.h_vy[isp], &hvz = s.h_vz[isp];
        auto &hc = s.h_cell[isp];
        if (o.defer_load) {
            s.load_deferred = true;
            s.load_cells[isp] = lc;
            s.load_seed[isp] = pm.seed;
            pm.seed = pm_skip(pm.seed, 5ull * (unsigned long long)np);
            p.np = (int)np;
            continue;
        }
        hx.resize(np); hy.resize(np); hvx.resize(np); hvy.resize(np); hvz.resize(np); hc.resize(np);
        const long seed0 = pm.seed;
        par_range(np, [&](long long k0, long long k1) {
            ParkMiller q{pm_skip(seed0, 5ull * (unsigned long long)k0)};
            // the loading cell of particle k0, then walk forward
            size_t li = (size_t)(std::upper_bound(lstart.begin(), lstart.end(), k0) - lstart.begin()) - 1;
            for (long long k = k0; k < k1; k++) {
                while (k >= lstart[li + 1]) li++;
                const int c = lc[li];
                const int i = c / s.ncy, j = c - i * s.ncy;
                float vx, vy, vz;
                maxwellv(s, q, p.vti, vx, vy, vz);
                hx[k] = (float)i + q.next();
                hy[k] = (float)j + q.next();
                hvx[k] = vx; hvy[k] = vy; hvz[k] = vz;
                hc[k] = i * s.ngy + j;
            }
        });
        pm.seed = pm_skip(seed0, 5ull * (unsigned long long)np);
        p.np = (int)hx.size();
        // Copy_HCPtoGCP (src/cuda_Particle.cu:28-58): cell from the integer part
        std::vector<int> &cnt = s.p_count[isp];
        cnt.assign(s.Csize, 0);
        std::vector<int> cell_of(p.np);
        // frand() can return exactly 1.0 (seed 2^31-2), which puts a particle
        // at x = i + 1: the reference then files it under cell i+1, and for
        // the last column or row that "cell" does not exist (its kernels read
        // past the grid).  Such a particle stays in the last cell here, with
        // its offset just below 1.
        std::vector<float> offx(p.np), offy(p.np);
        // stable counting sort by cell, in fixed chunks: per-chunk counts,
        // then each chunk scatters after the chunks before it
        const int NCH = 64;
        const long long npl = p.np;
        std::vector<int> ccount((size_t)NCH * s.Csize, 0);
        auto chunk_lo = [&](int t) { return npl * t / NCH; };
        {
            std::vector<std::thread> th;
            const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
            for (unsigned w = 0; w < hw; w++)
                th.emplace_back([&, w] {
                    for (int t = (int)w; t < NCH; t += (int)hw) {
                        int *cc = &ccount[(size_t)t * s.Csize];
                        for (long long k = chunk_lo(t); k < chunk_lo(t + 1); k++) {
                            int XID = (int)hx[k], YID = (int)hy[k];
                            float ox = hx[k] - XID, oy = hy[k] - YID;
                            if (XID >= s.ncx) { XID = s.ncx - 1; ox = 0.99999994f; }
                            if (YID >= s.ncy) { YID = s.ncy - 1; oy = 0.99999994f; }
                            offx[k] = ox;
                            offy[k] = oy;
                            cell_of[k] = XID * s.ncy + YID;
                            cc[cell_of[k]]++;
                        }
                    }
                });
            for (auto &x : th) x.join();
        }
        // fill[t][c]: where chunk t's first particle of cell c goes
        std::vector<int> start(s.Csize + 1, 0);
        for (int c = 0; c < s.Csize; c++) {
            int tot = 0;
            for (int t = 0; t < NCH; t++) tot += ccount[(size_t)t * s.Csize + c];
            cnt[c] = tot;
            start[c + 1] = start[c] + tot;
        }
        std::vector<int> fill((size_t)NCH * s.Csize);
        for (int c = 0; c < s.Csize; c++) {
            int at = start[c];
            for (int t = 0; t < NCH; t++) {
                fill[(size_t)t * s.Csize + c] = at;
                at += ccount[(size_t)t * s.Csize + c];
            }
        }
        s.p_x[isp].assign(p.np, 0); s.p_y[isp].assign(p.np, 0);
        s.p_vx[isp].assign(p.np, 0); s.p_vy[isp].assign(p.np, 0); s.p_vz[isp].assign(p.np, 0);
        {
            std::vector<std::thread> th;
            const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
            for (unsigned w = 0; w < hw; w++)
                th.emplace_back([&, w] {
                    for (int t = (int)w; t < NCH; t += (int)hw) {
                        int *fl = &fill[(size_t)t * s.Csize];
                        for (long long k = chunk_lo(t); k < chunk_lo(t + 1); k++) {
                            const int d = fl[cell_of[k]]++;
                            s.p_x[isp][d] = offx[k];
                            s.p_y[isp][d] = offy[k];
                            s.p_vx[isp][d] = hvx[k]; s.p_vy[isp][d] = hvy[k]; s.p_vz[isp][d] = hvz[k];
                        }
                    }
                });
            for (auto &x : th) x.join();
        }
    }
}

// sigma-v maximum of one (projectile, target) pair over the table: the sum
// of the listed channels, summed in the reference's groups
// (src/cuda_mcc.cu:277-466), times the projectile speed at each grid energy
struct SigGroup {
    int proj;                 // projectile species
    std::vector<std::vector<int>> parts; // channel groups, summed separately then added
};

float sigv_max(const Setup &s, const SigGroup &g) {
    const int W = 2 + s.n_cx;
    double best = 0.0;
    for (int i = 0; i < s.n_logx; i++) {
        const float *row = &s.xsec[(size_t)i * W];
        float engy = row[1];
        float sig = 0.0f;
        for (size_t p = 0; p < g.parts.size(); p++) {
            float part = 0.0f;
            for (size_t q = 0; q < g.parts[p].size(); q++) part = q ? part + row[2 + g.parts[p][q]] : row[2 + g.parts[p][q]];
            sig = p ? sig + part : part;
        }
        best = std::max(best, sqrt(2 * 1.602e-19 * engy / s.sp[g.proj].mass) * sig);
        best = (float)best;
    }
    return (float)best;
}

std::vector<int> span(int a, int b) {
    std::vector<int> v;
    for (int k = a; k <= b; k++) v.push_back(k);
    return v;
}

void null_collision_oxygen(Setup &s) { // src/cuda_mcc.cu:277-466
    const float prob_cut = 0.08f;
    const bool aro2 = s.main_gas == GAS_ARO2;
    std::vector<SigGroup> g;
    // electron targets: (sigv index, target density) for the sub-cycle count
    std::vector<float> edens;
    if (aro2) {
        g = {{0, {span(0, 3)}}, {0, {{4}}}, {0, {span(5, 9), span(10, 14), span(15, 18)}},
             {0, {span(19, 23), span(24, 26)}}, {0, {span(27, 31), span(32, 34)}}, {0, {{35}}}, {0, {{36}}},
             {0, {span(37, 41), span(42, 43)}}, {0, {span(44, 45)}}, {4, {span(46, 47)}}, {4, {{48}}},
             {4, {{49}}}, {4, {{50}}}, {4, {{51}}}, {2, {{52}}}, {2, {span(53, 55)}}, {2, {{56}}}, {2, {{57}}},
             {2, {span(58, 59)}}, {3, {span(60, 61)}}, {3, {{62}}}, {3, {{63}}}, {3, {{64}}}, {1, {span(65, 66)}},
             {1, {{67}}}};
        edens = {s.bg[0].InitDens, s.fg[0].InitDens, s.bg[1].InitDens, s.fg[1].InitDens, s.fg[2].InitDens,
                 s.sp[4].InitDens, s.sp[2].InitDens, s.fg[3].InitDens, s.fg[4].InitDens};
    } else {
        g = {{0, {span(0, 4), span(5, 9), span(10, 13)}}, {0, {span(14, 18), span(19, 21)}},
             {0, {span(22, 26), span(27, 29)}}, {0, {{30}}}, {0, {{31}}}, {0, {span(32, 36), span(37, 38)}},
             {0, {span(39, 40)}}, {3, {span(41, 42)}}, {3, {{43}}}, {3, {{44}}}, {3, {{45}}}, {3, {{46}}},
             {1, {{47}}}, {1, {span(48, 50)}}, {1, {{51}}}, {1, {{52}}}, {2, {span(53, 54)}}, {2, {{55}}},
             {2, {{56}}}, {2, {{57}}}};
        edens = {s.bg[0].InitDens, s.fg[0].InitDens, s.fg[1].InitDens, s.sp[3].InitDens, s.sp[1].InitDens,
                 s.fg[2].InitDens, s.fg[3].InitDens};
    }
    s.sigv.assign(g.size(), 0.0f);
    for (size_t k = 0; k < g.size(); k++) s.sigv[k] = sigv_max(s, g[k]);
    float col0 = 0.0f;
    for (size_t k = 0; k < edens.size(); k++) {
        const float t = (float)(1.0 - exp((double)(-1 * s.dt * s.sigv[k] * edens[k])));
        col0 = k ? col0 + t : t;
    }
    if (col0 > prob_cut) {
        s.mcc_n = (int)ceil((double)(col0 / prob_cut));
        float ratio = 1 / (float)s.mcc_n;
        s.dt_mcc = s.dt * ratio;
    } else {
        s.mcc_n = 1;
        s.dt_mcc = s.dt;
    }
}

void null_collision(Setup &s) { // src/cuda_mcc.cu:202-276 (Ar)
    const float prob_cut = 0.08f;
    if (s.main_gas != GAS_AR) {
        null_collision_oxygen(s);
        return;
    }
    s.sigv.assign(3, 0.0f);
    const int W = 2 + s.n_cx;
    for (int i = 0; i < s.n_logx; i++) {
        const float *row = &s.xsec[(size_t)i * W];
        float engy = row[1];
        float sig0 = row[2] + row[3] + row[4] + row[5];
        s.sigv[0] = (float)std::max((double)s.sigv[0], sqrt(2 * 1.602e-19 * engy / s.sp[0].mass) * sig0);
        float sig1 = row[6];
        s.sigv[1] = (float)std::max((double)s.sigv[1], sqrt(2 * 1.602e-19 * engy / s.sp[0].mass) * sig1);
        float sig2 = row[7] + row[8];
        s.sigv[2] = (float)std::max((double)s.sigv[2], sqrt(2 * 1.602e-19 * engy / s.sp[1].mass) * sig2);
    }
    float T0 = (float)(1.0 - exp((double)(-1 * s.dt * s.sigv[0] * s.bg[0].InitDens)));
    float T1 = (float)(1.0 - exp((double)(-1 * s.dt * s.sigv[1] * s.fg[0].InitDens)));
    float col0 = T0 + T1;
    if (col0 > prob_cut) {
        s.mcc_n = (int)ceil((double)(col0 / prob_cut));
        float ratio = 1 / (float)s.mcc_n;
        s.dt_mcc = s.dt * ratio;
    } else {
        s.mcc_n = 1;
        s.dt_mcc = s.dt;
    }
}

} // namespace

void build_setup(const char *json, size_t len, const BuildOpts &o, Setup &s) {
    JVal root;
    try {
        root = JParser(json, len).parse();
    } catch (std::exception &e) {
        deck_fail(e.what());
    }
    std::vector<int> bx0, bx1, by0, by1, bbc;
    std::vector<float> btemp;
    read_geometry(root, s, bx0, bx1, by0, by1, bbc, btemp);
    read_gas(root, s);
    read_method(root, s);
    read_collisions(root, s);
    geometry(s, bx0, bx1, by0, by1, bbc, btemp);
    // Source_setting (src/Efield.c:3-66)
    if (s.max_freq == 0.0f) deck_fail("no AC source: the time step is set from the highest source frequency");
    s.dt = (float)(1.0 / s.max_freq / (float)s.DT_PIC);
    s.dt_dx = s.dt / s.dx;
    s.dt_dy = s.dt / s.dy;
    s.efield_flag.assign(s.cond_numr, 0);
    for (int i = 0; i < s.cond_numr; i++) {
        int n = 0;
        for (int j = 0; j < s.src_num; j++)
            if (i + 1 == s.src_mid[j]) n++;
        s.efield_flag[i] = (n > 0 && n < 4) ? 1 : 0;
    }
    // power-driven sources per conductor (src/Efield.c:29-66): the first
    // one's amplitude is what the controller revises; two make the
    // reference's dual-power mode, which revises nothing
    s.cond_src_num.assign(s.cond_numr, 0);
    s.cond_power_id.assign(s.cond_numr, -1);
    for (int i = 0; i < s.cond_numr; i++)
        for (int j = 0; j < s.src_num; j++)
            if (i + 1 == s.src_mid[j] && s.src_power[j] != 0) {
                if (s.cond_src_num[i] == 2) deck_fail("no more than two power-driven sources per conductor");
                if (s.cond_src_num[i] == 0) s.cond_power_id[i] = j;
                s.cond_src_num[i]++;
            }
    if (s.external) circuit_coefficients(s);
    field_matrix(s);
    gas_setting(s, o);
    null_collision(s);
    laplace_and_gas(s, o.gas_temp_mode);
    if (s.external) circuit_laplace_charges(s);
    fluid_setting(s);
}

} // namespace hp
