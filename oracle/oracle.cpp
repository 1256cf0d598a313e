// oracle.cpp -- CPU restatement of the PIC/MCC step (test infrastructure:
// the checker the GPU results are compared with; never shipped).
//
// Follows, operator by operator:
//   Move          src/cuda_Move.cu:181-270
//   SortBoundary  src/cuda_Sortboundary.cu:41-258, codes from src/start.c:1776-1851
//   MCC (Ar)      src/cuda_mcc.cu:97-106,139-201, src/cuda_mccAr.cu:41-232,707-776
//   Deposit       src/cuda_Deposit.cu:3-104,277-325
//   Field         src/cuda_Field.cu:2-42,133-181,500-558,639-660,698-846,942-1072
// with the deterministic ordering this library defines where the reference
// has none (per-particle Philox draws, pull-ordered re-binning).  See
// oracle.h for the two precisions.
#include "oracle.h"

#include <cmath>
#include <cstring>
#include <vector>

#include <algorithm>
#include <atomic>
#include <array>
#include <thread>

#include "hp_fluid.h"
#include "hp_circuit.h"
#include "hp_math.h"
#include "hp_rng.h"
#include "hpic.h"

namespace {

// cells are independent in the MCC and deposit passes: split them over host threads
int g_threads = 0;
int nthreads() {
    if (g_threads <= 0) {
        unsigned h = std::thread::hardware_concurrency();
        g_threads = h ? (int)h : 1;
    }
    return g_threads;
}
template <class F> void par_for(int n, F f) {
    const int T = std::min(nthreads(), std::max(1, n / 64));
    if (T <= 1) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < T; t++)
        th.emplace_back([&, t] {
            for (int i = t; i < n; i += T) f(i);
        });
    for (auto &x : th) x.join();
}

// ---------------------------------------------------------------- math by precision
inline float m_log10(float x) { return hp_log10f(x); }
inline double m_log10(double x) { return std::log10(x); }
inline float m_exp(float x) { return hp_expf(x); }
inline double m_exp(double x) { return std::exp(x); }
inline float m_pow(float b, float e) { return hp_powf(b, e); }
inline double m_pow(double b, double e) { return std::pow(b, e); }
inline void m_sincos_turns(float t, float *s, float *c) { hp_sincos_turns(t, s, c); }
inline void m_sincos_turns(double t, double *s, double *c) {
    *s = std::sin(2.0 * M_PI * t);
    *c = std::cos(2.0 * M_PI * t);
}
inline float m_tan(float y) { return hp_tanf_q1(y); }
inline double m_tan(double y) { return std::tan(y); }
inline float m_atan(float x) { return hp_atanf(x); }
inline double m_atan(double x) { return std::atan(x); }

// the kernels' warp tree: v[l] += v[l ^ o] for o = 16, 8, 4, 2, 1; lane 0
inline double warp_tree(double *v) {
    double t[32];
    for (int o = 16; o > 0; o >>= 1) {
        for (int l = 0; l < 32; l++) t[l] = v[l] + v[l ^ o];
        std::memcpy(v, t, sizeof t);
    }
    return v[0];
}

struct Fate {
    int fi, fj;
    bool absorbed, flipx, flipy;
    int cond;
};

struct SimBase {
    or_case c;
    int G = 0, C = 0, precision = 32;
    std::vector<float> cond_charge;
    std::vector<unsigned> mcc_count;
    int pcg_iters[2] = {0, 0};
    std::vector<double> ave_den, ave_phi, ave_src, ave_ex, ave_ey;
    std::vector<long long> sig; // [nsp*G] dielectric surface weights, fixed point
    std::vector<double> sigma;  // [G] Sigma where SumSource or Cond_Sigma sets it
    std::vector<float> src_amp; // AC amplitudes in use
    std::vector<unsigned> cond_step; // [nsp*cond_numr] absorbed in this step
    struct {
        double surf[8], old[8], old2[8];
        float power[8];
        int count[8];
        int power_init;
    } pw{};
    std::vector<int> cond_list; // nodes with a CondID, in node order
    // external circuit: charge history, absorbed charge of the last step,
    // conductor potentials and Poisson-part surface charges of the last solve
    struct {
        float q[4 * HP_CIRCUIT_MAX], qconv[HP_CIRCUIT_MAX], phi[HP_CIRCUIT_MAX], pois[HP_CIRCUIT_MAX];
    } circ{};
    // Scripted uniforms, for pinning against the reference's own MCC code:
    // when on, every MCC draw (null-collision tests included) is taken in
    // order from a per-key list instead of Philox; key = cell, or species *
    // Csize + cell with by_species.  The reference's kernels, fed the same
    // lists through their curand_uniform calls (one thread per key), then
    // see the same numbers in the same order.  A list that runs out yields
    // 1.0 (no collision) and counts an overrun.
    struct Script {
        bool on = false;
        int by_species = 0;
        int pair_rl = 0; // kinematics calls (PAIR_* bits) whose two draws are taken right to left
        std::vector<float> u;
        std::vector<int64_t> start, pos;
    } script;
    std::atomic<long long> script_overrun{0};
    float u_script(uint32_t species, uint32_t cell) {
        const size_t key = script.by_species ? (size_t)species * (size_t)C + cell : cell;
        if (key + 1 >= script.start.size()) {
            script_overrun++;
            return 1.0f;
        }
        int64_t &p = script.pos[key];
        if (script.start[key] + p >= script.start[key + 1]) {
            script_overrun++;
            return 1.0f;
        }
        return script.u[(size_t)(script.start[key] + p++)];
    }
    // ------------------------------------------------------------ fluid species
    // The continuity solve of the metastable / radical densities
    // (Solve_Continuity_eqn, src/cuda_Fluid.cu:34-167) and the diagnostic
    // cycle that feeds it (Diagnostic_Basic, src/cuda_Diagnostic.cu:268-330):
    // every n_ave + 1 steps the electron density and the collision tallies
    // are averaged into sources; from the first such step on the densities
    // are copied to the nodes (the MCC's input) each step, and from the next
    // one the continuity solve runs each step.  All in float as the reference.
    std::vector<float> fden, fsrc, fflx, ffly, fnode, prob_v, f_gam, f_x;
    std::vector<double> sum_den_e;
    std::vector<unsigned> fl_base;
    void fluid_init() {
        const size_t F = (size_t)c.nfsp, ngx = c.ngx, ncy = c.ncy, ncx = c.ncx, ngy = c.ngy;
        fden.assign(c.fluid_cell_den, c.fluid_cell_den + F * C);
        fsrc.assign(F * C, 0.0f);
        fflx.assign(c.flux_x0, c.flux_x0 + F * ngx * ncy);
        ffly.assign(c.flux_y0, c.flux_y0 + F * ncx * ngy);
        fnode.assign(c.fluid_den, c.fluid_den + F * G);
        prob_v.assign(c.prob, c.prob + 3 * (size_t)C);
        f_gam.assign(F * C, 0.0f);
        f_x.assign(F * C, 0.0f);
        sum_den_e.assign(G, 0.0);
        fl_base.assign((size_t)(c.mcc_stride > 0 ? c.mcc_stride : 8) * C, 0u);
    }
    // tridiag (src/cuda_Fluid.cu:168-184); false where a pivot vanishes
    static bool tridiag(const float *a, const float *b, const float *cc, const float *d, float *x, float *gam, int n) {
        float bet;
        x[0] = d[0] / (bet = b[0]);
        for (int j = 1; j < n; j++) {
            gam[j - 1] = cc[j - 1] / bet;
            bet = b[j] - a[j] * cc[j - 1] / bet;
            x[j] = (d[j] - a[j] * x[j - 1]) / bet;
            if (bet == 0) return false;
        }
        for (int j = n - 2; j >= 0; j--) x[j] -= gam[j] * x[j + 1];
        return true;
    }
    // Solve_Density_x + Calculate_Flux_x of one species (dir 0), or the y
    // pair (dir 1), line by line
    void fluid_sweep(int f, int dir) {
        const int ngx = c.ngx, ngy = c.ngy, ncx = c.ncx, ncy = c.ncy;
        const int nl = dir ? c.nyl : c.nxl;
        const int *L = dir ? c.yl : c.xl;
        const float *fg = dir ? c.yl_fg : c.xl_fg;
        const float *A = dir ? c.gay : c.gax, *B = dir ? c.gby : c.gbx;
        const size_t fo = dir ? (size_t)f * ncx * ngy : (size_t)f * ngx * ncy; // face arrays
        const float *ga_ = A + fo, *gb_ = B + fo;
        float *flux = (dir ? ffly.data() : fflx.data()) + fo;
        const float *other = (dir ? fflx.data() + (size_t)f * ngx * ncy : ffly.data() + (size_t)f * ncx * ngy);
        float *den = fden.data() + (size_t)f * C;
        const float *src = fsrc.data() + (size_t)f * C;
        const float dtc = c.dtc, del_f = dtc / (dir ? c.dy : c.dx), dother = dir ? c.dx : c.dy;
        std::vector<float> a, b, cc, d, x, gam;
        for (int k = 0; k < nl; k++) {
            const int p = L[3 * k], lo = L[3 * k + 1], hi = L[3 * k + 2]; // x: x1, x2, yy; y: xx, y1, y2
            const int first = dir ? lo : p, last = dir ? hi : lo, fixed = dir ? p : hi;
            const int num = last - first + 1;
            a.assign(num, 0); b.assign(num, 0); cc.assign(num, 0); d.assign(num, 0); x.assign(num, 0); gam.assign(num, 0);
            // face index of position q along the line, cell index of q
            auto face = [&](int q) { return dir ? fixed * ngy + q : q * ncy + fixed; };
            auto cell = [&](int q) { return dir ? fixed * ncy + q : q * ncy + fixed; };
            // the other direction's two faces of cell q: an x sweep reads the y
            // faces (q, fixed) and (q, fixed + 1), a y sweep the x faces
            // (fixed, q) and (fixed + 1, q)
            auto olo = [&](int q) { return dir ? fixed * ncy + q : q * ngy + fixed; };
            auto ohi = [&](int q) { return dir ? (fixed + 1) * ncy + q : q * ngy + fixed + 1; };
            for (int i = 0; i < num; i++) {
                const int q = i + first;
                a[i] = -ga_[face(q)] * del_f;
                b[i] = 1 + (ga_[face(q + 1)] + gb_[face(q)]) * del_f;
                cc[i] = -gb_[face(q + 1)] * del_f;
                d[i] = den[cell(q)] + src[cell(q)] * dtc - (other[ohi(q)] - other[olo(q)]) * dtc / dother;
            }
            if (!tridiag(a.data(), b.data(), cc.data(), d.data(), x.data(), gam.data(), num)) continue;
            for (int i = 0; i < num; i++) {
                const int q = i + first;
                den[cell(q)] = (c.plasma[cell(q)] == 1 && x[i] > 1e9f) ? x[i] : 0.0f;
            }
            const float fg1 = fg[(size_t)f * nl + k], fg2 = fg[(size_t)c.nfsp * nl + (size_t)f * nl + k];
            flux[face(first)] = -fg1 * gb_[face(first)] * den[cell(first)];
            for (int q = first + 1; q <= last; q++)
                flux[face(q)] = ga_[face(q)] * den[cell(q - 1)] - gb_[face(q)] * den[cell(q)];
            flux[face(last + 1)] = fg2 * ga_[face(last + 1)] * den[cell(last)];
        }
    }
    void fluid_sweeps() {
        for (int f = 0; f < c.nfsp; f++) {
            fluid_sweep(f, 0);
            fluid_sweep(f, 1);
        }
    }
    // the diagnostic cycle of step t (1-based): accumulate, or average into
    // sources; then, once the first average is in, the node copy (and the Ar
    // collision probability that reads it)
    void fluid_diag(int64_t t, const double *den_e) {
        const int N = c.n_ave;
        const int64_t per = (int64_t)N + 1;
        const int ph = (int)((t - 1) % per);
        const int st = c.mcc_stride > 0 ? c.mcc_stride : 8;
        if (ph < N) {
            for (int g = 0; g < G; g++) sum_den_e[g] += den_e[g];
        } else {
            const float temp = c.denscale0 / (float)N;
            std::vector<float> R(96), S(5);
            float nn[5];
            for (int g = 0; g < G; g++) {
                const int i = g / c.ngy, j = g - i * c.ngy;
                const bool has_cell = i < c.ncx && j < c.ncy;
                const int cell = i * c.ncy + j;
                const float ave = temp * (float)(sum_den_e[g] + den_e[g]);
                sum_den_e[g] = 0.0;
                const float eden = (float)(0.25 * (double)ave);
                std::fill(R.begin(), R.end(), 0.0f);
                if (has_cell)
                    for (int ch = 0; ch < st && ch < c.tnrct; ch++) {
                        const unsigned now = mcc_count[(size_t)cell * st + ch];
                        R[ch] = c.rate_f[ch] * (float)(now - fl_base[(size_t)cell * st + ch]);
                        fl_base[(size_t)cell * st + ch] = now;
                    }
                for (int f = 0; f < 5; f++) nn[f] = f < c.nfsp ? fnode[(size_t)f * G + g] : 0.0f;
                const float bd1 = c.back_den1 ? c.back_den1[g] : 0.0f, bd2 = c.back_den2 ? c.back_den2[g] : 0.0f;
                hp_fluid_sources(c.gas, R.data(), nn, bd1, bd2, eden, c.rr, S.data());
                if (has_cell)
                    for (int f = 0; f < c.nfsp; f++) fsrc[(size_t)f * C + cell] = S[f];
            }
        }
        if (t >= per) fluid_sync();
    }
    void fluid_sync() {
        const int ncy = c.ncy, ngy = c.ngy;
        for (int f = 0; f < c.nfsp; f++)
            for (int i = 0; i < c.ncx; i++)
                for (int j = 0; j < ncy; j++) {
                    const float v = fden[(size_t)f * C + i * ncy + j];
                    fnode[(size_t)f * G + i * ngy + j] = v;
                    if (i == c.ncx - 1 || j == ncy - 1) fnode[(size_t)f * G + (i + 1) * ngy + j + 1] = v;
                }
        if (c.gas == 0)
            for (int cell = 0; cell < C; cell++) {
                const int i = cell / ncy, j = cell - i * ncy, node = i * ngy + j;
                const float e = hp_expf(-1 * c.dt_mcc * c.sigv[1] * fnode[node]);
                prob_v[(size_t)C + cell] = prob_v[cell] + 1.0f - e;
            }
    }
    void fluid(int64_t t, const double *den_e) {
        if (!c.fluid_on || c.nfsp <= 0) return;
        if (t >= (int64_t)c.n_ave + 2) fluid_sweeps();
        fluid_diag(t, den_e);
    }
    virtual void fluid_step(int64_t t) = 0;
    virtual void power(int64_t tstep) = 0;
    int64_t ave_count = 0;
    bool walk_bound_hit = false; // a walk that reached its crossing bound
    std::vector<unsigned long long> eedf = std::vector<unsigned long long>(201, 0ull);
    virtual void eedf_sample() = 0;
    virtual ~SimBase() {}
    virtual void set_particles(int, const int *, const float *, const float *, const float *, const float *,
                               const float *) = 0;
    virtual size_t num(int) = 0;
    virtual void get_particles(int, int *, float *, float *, float *, float *, float *) = 0;
    virtual void get_particles_d(int, int *, double *, double *, double *, double *, double *) = 0;
    virtual size_t num_movers(int) = 0;
    virtual void get_movers(int, int *, float *, float *, float *, float *, float *, int8_t *) = 0;
    virtual void get_grid(int, void *) = 0;
    virtual void set_grid(int, const void *) = 0;
    virtual void field(int64_t) = 0;
    virtual void move() = 0;
    virtual void sort() = 0;
    virtual void mcc(int64_t) = 0;
    virtual void deposit(bool smooth) = 0;
    virtual void accumulate() = 0;
    virtual int far_max() const = 0;
    virtual void xsec_n(int ch, const float *engy, float *out, int n) const = 0;
    virtual void kinematics(int kind, const float *in, float *out, int n) const = 0;
    virtual int collide_oxy(int isp, int t, const float *v, float bv1, float bv2, const float *u, int nu, int pair_rl,
                            int *ch, int *keep, float *vout, int *bsp, float *bv, int *kill) = 0;
};

template <class R> struct Sim : SimBase {
    struct Sp {
        std::vector<int> cnt, start;
        std::vector<R> x, y, vx, vy, vz;
        std::vector<int> mcnt, mstart;
        std::vector<R> mx, my, mvx, mvy, mvz;
        std::vector<int8_t> mcode;
        void restart() {
            start.assign(cnt.size() + 1, 0);
            for (size_t k = 0; k < cnt.size(); k++) start[k + 1] = start[k] + cnt[k];
        }
    } sp[5];
    std::vector<R> Ex, Ey, phi, phi_p;
    std::vector<double> den, source, b64, x64;
    std::vector<float> pf_x;
    std::vector<double> cw[5][4];

    explicit Sim(const or_case &cc, int prec) {
        c = cc;
        precision = prec;
        G = c.ngx * c.ngy;
        C = c.ncx * c.ncy;
        for (int s = 0; s < c.nsp; s++) {
            sp[s].cnt.assign(C, 0);
            sp[s].mcnt.assign(C, 0);
            sp[s].restart();
            for (int q = 0; q < 4; q++) cw[s][q].assign(C, 0.0);
        }
        Ex.assign(G, 0); Ey.assign(G, 0); phi.assign(G, 0); phi_p.assign(G, 0);
        den.assign((size_t)c.nsp * G, 0.0);
        source.assign(G, 0.0); b64.assign(G, 0.0); x64.assign(G, 0.0);
        pf_x.assign(G, 0.0f);
        cond_charge.assign((size_t)c.nsp * c.cond_numr, 0.0f);
        mcc_count.assign((size_t)(c.mcc_stride > 0 ? c.mcc_stride : 8) * C, 0u);
        ave_den.assign((size_t)c.nsp * G, 0.0);
        ave_phi.assign(G, 0.0);
        ave_src.assign(G, 0.0);
        ave_ex.assign(G, 0.0);
        ave_ey.assign(G, 0.0);
        sig.assign((size_t)c.nsp * G, 0);
        sigma.assign(G, 0.0);
        src_amp.assign(c.src_ac, c.src_ac + c.src_num);
        cond_step.assign((size_t)c.nsp * c.cond_numr, 0u);
        for (int n = 0; n < G; n++)
            if (c.cond_id[n]) cond_list.push_back(n);
        fluid_init();
    }
    void fluid_step(int64_t t) override { fluid(t, den.data()); }

    // ------------------------------------------------------------ state
    void set_particles(int s, const int *counts, const float *x, const float *y, const float *vx, const float *vy,
                       const float *vz) override {
        Sp &p = sp[s];
        p.cnt.assign(counts, counts + C);
        p.restart();
        size_t n = (size_t)p.start[C];
        p.x.assign(x, x + n); p.y.assign(y, y + n);
        p.vx.assign(vx, vx + n); p.vy.assign(vy, vy + n); p.vz.assign(vz, vz + n);
    }
    size_t num(int s) override { return sp[s].x.size(); }
    void get_particles(int s, int *counts, float *x, float *y, float *vx, float *vy, float *vz) override {
        Sp &p = sp[s];
        if (counts) std::memcpy(counts, p.cnt.data(), (size_t)C * 4);
        for (size_t k = 0; k < p.x.size(); k++) {
            if (x) x[k] = (float)p.x[k];
            if (y) y[k] = (float)p.y[k];
            if (vx) vx[k] = (float)p.vx[k];
            if (vy) vy[k] = (float)p.vy[k];
            if (vz) vz[k] = (float)p.vz[k];
        }
    }
    void get_particles_d(int s, int *counts, double *x, double *y, double *vx, double *vy, double *vz) override {
        Sp &p = sp[s];
        if (counts) std::memcpy(counts, p.cnt.data(), (size_t)C * 4);
        for (size_t k = 0; k < p.x.size(); k++) {
            x[k] = p.x[k]; y[k] = p.y[k]; vx[k] = p.vx[k]; vy[k] = p.vy[k]; vz[k] = p.vz[k];
        }
    }
    size_t num_movers(int s) override { return sp[s].mx.size(); }
    void get_movers(int s, int *counts, float *x, float *y, float *vx, float *vy, float *vz, int8_t *codes) override {
        Sp &p = sp[s];
        if (counts) std::memcpy(counts, p.mcnt.data(), (size_t)C * 4);
        for (size_t k = 0; k < p.mx.size(); k++) {
            x[k] = (float)p.mx[k]; y[k] = (float)p.my[k];
            vx[k] = (float)p.mvx[k]; vy[k] = (float)p.mvy[k]; vz[k] = (float)p.mvz[k];
            if (codes) codes[k] = p.mcode[k];
        }
    }
    void get_grid(int which, void *out) override {
        float *f = (float *)out;
        double *d = (double *)out;
        switch (which) {
        case 0: for (int n = 0; n < G; n++) f[n] = (float)Ex[n]; break;
        case 1: for (int n = 0; n < G; n++) f[n] = (float)Ey[n]; break;
        case 2: for (int n = 0; n < G; n++) f[n] = (float)phi[n]; break;
        case 3: for (int n = 0; n < G; n++) f[n] = (float)phi_p[n]; break;
        case 4: std::memcpy(d, den.data(), den.size() * 8); break;
        case 5: std::memcpy(d, source.data(), source.size() * 8); break;
        case 6: std::memcpy(d, b64.data(), b64.size() * 8); break;
        case 7:
            if (precision == 32 && c.field_mode == 0) for (int n = 0; n < G; n++) d[n] = pf_x[n];
            else std::memcpy(d, x64.data(), x64.size() * 8);
            break;
        case 8: std::memcpy(out, sig.data(), sig.size() * 8); break;
        case 9: std::memcpy(d, sigma.data(), sigma.size() * 8); break;
        case 10: std::memcpy(f, src_amp.data(), src_amp.size() * 4); break;
        case 11: std::memcpy(f, fden.data(), fden.size() * 4); break;
        case 12: std::memcpy(f, fnode.data(), fnode.size() * 4); break;
        case 13: std::memcpy(f, fsrc.data(), fsrc.size() * 4); break;
        case 14: std::memcpy(f, fflx.data(), fflx.size() * 4); break;
        case 15: std::memcpy(f, ffly.data(), ffly.size() * 4); break;
        case 16: std::memcpy(f, &circ, sizeof circ); break;
        }
    }
    void set_grid(int which, const void *in) override {
        const float *f = (const float *)in;
        const double *d = (const double *)in;
        switch (which) {
        case 0: for (int n = 0; n < G; n++) Ex[n] = f[n]; break;
        case 1: for (int n = 0; n < G; n++) Ey[n] = f[n]; break;
        case 2: for (int n = 0; n < G; n++) phi[n] = f[n]; break;
        case 3: for (int n = 0; n < G; n++) phi_p[n] = f[n]; break;
        case 4: std::memcpy(den.data(), d, den.size() * 8); break;
        case 5: std::memcpy(source.data(), d, source.size() * 8); break;
        case 6: std::memcpy(b64.data(), d, b64.size() * 8); break;
        case 7:
            if (precision == 32 && c.field_mode == 0) for (int n = 0; n < G; n++) pf_x[n] = (float)d[n];
            else std::memcpy(x64.data(), d, x64.size() * 8);
            break;
        case 8: std::memcpy(sig.data(), in, sig.size() * 8); break;
        case 9: std::memcpy(sigma.data(), d, sigma.size() * 8); break;
        case 11: std::memcpy(fden.data(), f, fden.size() * 4); break;
        case 12: std::memcpy(fnode.data(), f, fnode.size() * 4); break;
        case 13: std::memcpy(fsrc.data(), f, fsrc.size() * 4); break;
        case 14: std::memcpy(fflx.data(), f, fflx.size() * 4); break;
        case 15: std::memcpy(ffly.data(), f, ffly.size() * 4); break;
        case 16: std::memcpy(&circ, f, sizeof circ); break;
        }
    }

    // ------------------------------------------------------------ Move
    // Fate of one cell crossing from the ghost code of the cell entered
    // (src/cuda_Sortboundary.cu:70-256; codes from src/start.c:1776-1851).
    Fate fate(int si, int sj, int di, int dj) const {
        Fate f{si + di, sj + dj, false, false, false, -1};
        const int S = c.sidx[(si + 1 + di) * (c.ncy + 2) + (sj + 1 + dj)];
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
            else if (S >= 1) f.cond = -2 - ((di + 1) * 3 + (dj + 1)); // a dielectric: the direction entered
            break;
        }
        if (!f.absorbed && (f.fi < 0 || f.fi >= c.ncx || f.fj < 0 || f.fj >= c.ncy)) f.absorbed = true;
        return f;
    }

    // ------------------------------------------------------------ dielectric surface charge
    // A crossing into a dielectric cell, kept from Move for SortBoundary.
    struct Hit {
        int s, i, j, dir;
        R x, y, vx, vy;
    };
    std::vector<Hit> hits;

    // One share in fixed point; shares that are not finite or reach 2^20 in
    // magnitude, and nodes off the grid, are dropped (the kernels' rule).
    void surface_add(int s, int node, R w) {
        if (node < 0 || node >= G || !(std::fabs(w) < (R)1048576)) return;
        sig[(size_t)s * G + node] += (long long)std::llrint((double)w * (double)(1ll << HP_SIGMA_FRAC_BITS));
    }

    // SortBoundary's dielectric branch (src/cuda_Sortboundary.cu:93-207), on
    // the flat node index as the reference computes it.
    void surface_split(const Hit &h) {
        const int ngy = c.ngy, SY = c.ncy + 2;
        const int di = h.dir / 3 - 1, dj = h.dir % 3 - 1;
        const int T = h.i * ngy + h.j, C_ = T + di * ngy + dj;
        const int g = (h.i + 1 + di) * SY + (h.j + 1 + dj);
        const int *SI = c.sidx;
        const R x = h.x, y = h.y, vx = h.vx, vy = h.vy;
        int pa = 0, pb = 0;
        R a = 0, b = 0, delta;
        switch (h.dir) {
        case 5: delta = x - vx / vy * y; pa = C_; a = 1 - delta; pb = C_ + ngy; b = delta; break;     // top
        case 3: delta = x + vx / vy * (1 - y); pa = T; a = 1 - delta; pb = T + ngy; b = delta; break; // bottom
        case 7: delta = y - vy / vx * x; pa = C_; a = 1 - delta; pb = C_ + 1; b = delta; break;       // right
        case 1: delta = y + vy / vx * (1 - x); pa = T; a = 1 - delta; pb = T + 1; b = delta; break;   // left
        case 8: // up-right: ngy+1
            delta = x - vx / vy * y;
            if (delta >= 0) {
                if (SI[g - 1]) { delta = y - vy / vx * x; pa = C_ - 1; a = -delta; pb = C_; b = 1 + delta; }
                else { pa = C_; a = 1 - delta; pb = C_ + ngy; b = delta; }
            } else {
                if (SI[g - SY]) { pa = T + 1; a = -delta; pb = C_; b = 1 + delta; }
                else { delta = y - vy / vx * x; pa = C_; a = 1 - delta; pb = C_ + 1; b = delta; }
            }
            break;
        case 6: // down-right: ngy-1
            delta = x + vx / vy * (1 - y);
            if (delta >= 0) {
                if (SI[g + 1]) { delta = y - vy / vx * x; pa = C_ + 1; a = 2 - delta; pb = C_ + 2; b = delta - 1; }
                else { pa = C_ + 1; a = 1 - delta; pb = C_ + 1 + ngy; b = delta; }
            } else {
                if (SI[g - SY]) { pa = T; a = -delta; pb = C_ + 1; b = 1 + delta; }
                else { delta = y - vy / vx * x; pa = C_; a = 1 - delta; pb = C_ + 1; b = delta; }
            }
            break;
        case 2: // up-left: -ngy+1
            delta = x - vx / vy * y;
            if (delta < 1) {
                if (SI[g - 1]) { delta = y + vy / vx * (1 - x); pa = C_ + ngy - 1; a = -delta; pb = C_ + ngy; b = 1 + delta; }
                else { pa = C_; a = 1 - delta; pb = C_ + ngy; b = delta; }
            } else {
                if (SI[g + SY]) { pa = T + 1; a = 2 - delta; pb = T + 1 + ngy; b = delta - 1; }
                else { delta = y + vy / vx * (1 - x); pa = T + 1; a = 1 - delta; pb = T + 2; b = delta; }
            }
            break;
        case 0: // down-left: -ngy-1
            delta = x + vx / vy * (1 - y);
            if (delta < 1) {
                if (SI[g + 1]) { delta = y + vy / vx * (1 - x); pa = T; a = 2 - delta; pb = T + 1; b = delta - 1; }
                else { pa = C_; a = 1 - delta; pb = T; b = delta; }
            } else {
                if (SI[g + SY]) { pa = T; a = 2 - delta; pb = T + ngy; b = delta - 1; }
                else { delta = y + vy / vx * (1 - x); pa = T - 1; a = 1 - delta; pb = T; b = delta; }
            }
            break;
        default: return;
        }
        surface_add(h.s, pa, a);
        surface_add(h.s, pb, b);
    }

    // SumSource's surface term (src/cuda_Deposit.cu:40-97)
    double surface_charge(int n) {
        const int m = c.sig_mode[n];
        if (m == 0) return 0.0;
        if (m == 3) {
            for (int s = 0; s < c.nsp; s++) sig[(size_t)s * G + n] = 0;
            return 0.0;
        }
        double q = 0.0;
        for (int s = 0; s < c.nsp; s++)
            q += (double)sig[(size_t)s * G + n] * (1.0 / (double)(1ll << HP_SIGMA_FRAC_BITS)) * (double)c.q_density[s];
        sigma[n] = (m == 2 ? 2.0 : 1.0) * q / (double)c.area[n];
        return q;
    }

    // One wrap per crossing (src/cuda_Move.cu:227-255) and the rule of the
    // cell entered; move_mode 0 stops after one crossing as the reference
    // does, move_mode 1 crosses until the offset is inside a cell (bounded).
    // 0 inside the domain, 1 absorbed, 2 crossing bound hit.
    static R one_below() { return std::nextafter((R)1, (R)0); }
    int walk(int &i, int &j, R &lx, R &ly, R &vx, R &vy, int &cond) const {
        const int maxs = c.move_mode ? 2 * (c.ncx + c.ncy) + 4 : 1;
        for (int st = 0; st < maxs; st++) {
            // the reference computes (float)((double)l -+ 1.0); for a float l
            // the double difference is exact, so one operation in R rounds
            // the same exact value identically
            int di = 0, dj = 0;
            if (ly >= 1) { dj = 1; ly = ly - (R)1; }
            else if (ly < 0) { dj = -1; ly = ly + (R)1; }
            if (lx >= 1) { di = 1; lx = lx - (R)1; }
            else if (lx < 0) { di = -1; lx = lx + (R)1; }
            const Fate f = fate(i, j, di, dj);
            if (f.absorbed) {
                cond = f.cond;
                return 1;
            }
            if (f.flipx) { lx = 1 - lx; vx = -1 * vx; }
            if (f.flipy) { ly = 1 - ly; vy = -1 * vy; }
            // a particle that reaches a wall exactly (offset 0 after the wrap) flips
            // to offset 1, the wall itself, which no cell holds: keep it just inside
            // (move_mode 0 keeps offset 1, as the reference does)
            if (c.move_mode) {
                if (f.flipx && lx == 1) lx = one_below();
                if (f.flipy && ly == 1) ly = one_below();
            }
            i = f.fi;
            j = f.fj;
            if (!(ly >= 1 || ly < 0 || lx >= 1 || lx < 0)) return 0;
        }
        if (c.move_mode) {
            cond = -1;
            return 2;
        }
        return 0;
    }

    // movers beyond the 3x3 neighbourhood: (species, dest) -> (source<<18 | r, mover index)
    std::vector<std::vector<std::pair<uint64_t, size_t>>> far[5];
    int far_max() const override {
        size_t m = 0;
        for (int s = 0; s < c.nsp; s++)
            for (const auto &v : far[s]) m = std::max(m, v.size());
        return (int)m;
    }

    // MoveE_Basic (src/cuda_Move.cu:181-270) with the boundary rules applied
    // per crossing; mover codes: destination (di+1)*3+(dj+1) within the 3x3
    // neighbourhood, 14 beyond it, 15 absorbed.
    void move() override {
        for (int s = 0; s < c.nsp; s++) {
            Sp &p = sp[s];
            std::vector<int> ncnt(C, 0);
            std::vector<R> nx, ny, nvx, nvy, nvz;
            nx.reserve(p.x.size()); ny.reserve(p.x.size()); nvx.reserve(p.x.size()); nvy.reserve(p.x.size());
            nvz.reserve(p.x.size());
            p.mcnt.assign(C, 0);
            p.mx.clear(); p.my.clear(); p.mvx.clear(); p.mvy.clear(); p.mvz.clear(); p.mcode.clear();
            far[s].assign(C, {});
            const R As = (R)c.Ascale[s], dtdx = (R)c.dt_dx, dtdy = (R)c.dt_dy;
            for (int cell = 0; cell < C; cell++) {
                const int i = cell / c.ncy, j = cell - i * c.ncy, node = i * c.ngy + j;
                const R ex_ws = Ex[node], ex_wn = Ex[node + 1], ex_es = Ex[node + c.ngy], ex_en = Ex[node + c.ngy + 1];
                const R ey_ws = Ey[node], ey_wn = Ey[node + 1], ey_es = Ey[node + c.ngy], ey_en = Ey[node + c.ngy + 1];
                for (int q = p.start[cell]; q < p.start[cell + 1]; q++) {
                    R lx = p.x[q], ly = p.y[q];
                    const R vx = p.vx[q], vy = p.vy[q], vz = p.vz[q];
                    // bilinear weights, then fused multiply-adds (as the kernel)
                    const R wx = 1 - lx, wy = 1 - ly;
                    const R w00 = wx * wy, w01 = wx * ly, w10 = lx * wy, w11 = lx * ly;
                    const R del_vx = std::fma(ex_en, w11, std::fma(ex_es, w10, std::fma(ex_wn, w01, ex_ws * w00)));
                    const R del_vy = std::fma(ey_en, w11, std::fma(ey_es, w10, std::fma(ey_wn, w01, ey_ws * w00)));
                    R mvX = std::fma(del_vx, As, vx);
                    R mvY = std::fma(del_vy, As, vy);
                    lx = std::fma(mvX, dtdx, lx);
                    ly = std::fma(mvY, dtdy, ly);
                    if (ly >= 1 || ly < 0 || lx >= 1 || lx < 0) {
                        int fi = i, fj = j, cond = -1, code;
                        const int r = walk(fi, fj, lx, ly, mvX, mvY, cond);
                        if (r) {
                            code = 15;
                            if (cond >= 0 && cond < c.cond_numr) {
                                cond_charge[(size_t)s * c.cond_numr + cond] += 1.0f;
                                if (c.n_power > 0 || c.external) cond_step[(size_t)s * c.cond_numr + cond]++;
                            } else if (cond <= -2 && c.n_diel > 0) hits.push_back({s, fi, fj, -2 - cond, lx, ly, mvX, mvY});
                            if (r == 2) walk_bound_hit = true;
                        } else {
                            const int ddi = fi - i, ddj = fj - j;
                            code = (ddi >= -1 && ddi <= 1 && ddj >= -1 && ddj <= 1) ? (ddi + 1) * 3 + (ddj + 1) : 14;
                        }
                        if (code == 14)
                            far[s][fi * c.ncy + fj].push_back(
                                {((uint64_t)cell << 18) | (uint64_t)p.mcnt[cell], p.mx.size()});
                        p.mcnt[cell]++;
                        p.mx.push_back(lx); p.my.push_back(ly);
                        p.mvx.push_back(mvX); p.mvy.push_back(mvY); p.mvz.push_back(vz);
                        p.mcode.push_back((int8_t)code);
                    } else {
                        ncnt[cell]++;
                        nx.push_back(lx); ny.push_back(ly); nvx.push_back(mvX); nvy.push_back(mvY); nvz.push_back(vz);
                    }
                }
            }
            p.cnt.swap(ncnt);
            p.x.swap(nx); p.y.swap(ny); p.vx.swap(nvx); p.vy.swap(nvy); p.vz.swap(nvz);
            p.restart();
            p.mstart.assign(C + 1, 0);
            for (int k = 0; k < C; k++) p.mstart[k + 1] = p.mstart[k] + p.mcnt[k];
        }
    }

    // ------------------------------------------------------------ SortBoundary
    // Pull order per destination cell: its stayers, the 3x3 source cells'
    // movers addressed to it (sources in increasing cell index, movers in
    // list order), then the far movers in (source, r) order.
    void sort() override {
        for (const Hit &h : hits) surface_split(h);
        hits.clear();
        for (int s = 0; s < c.nsp; s++) {
            Sp &p = sp[s];
            std::vector<int> ncnt(C, 0);
            std::vector<R> nx, ny, nvx, nvy, nvz;
            auto take = [&](size_t q) {
                nx.push_back(p.mx[q]); ny.push_back(p.my[q]); nvx.push_back(p.mvx[q]); nvy.push_back(p.mvy[q]);
                nvz.push_back(p.mvz[q]);
            };
            if (far[s].size() != (size_t)C) far[s].assign(C, {});
            for (int cell = 0; cell < C; cell++) {
                const int i = cell / c.ncy, j = cell - i * c.ncy;
                for (int q = p.start[cell]; q < p.start[cell + 1]; q++) {
                    nx.push_back(p.x[q]); ny.push_back(p.y[q]); nvx.push_back(p.vx[q]); nvy.push_back(p.vy[q]);
                    nvz.push_back(p.vz[q]);
                }
                int out = p.cnt[cell];
                for (int si = i - 1; si <= i + 1; si++) {
                    if (si < 0 || si >= c.ncx) continue;
                    for (int sj = j - 1; sj <= j + 1; sj++) {
                        if (sj < 0 || sj >= c.ncy) continue;
                        const int src = si * c.ncy + sj;
                        const int want = (i - si + 1) * 3 + (j - sj + 1);
                        for (int q = p.mstart[src]; q < p.mstart[src + 1]; q++) {
                            if (p.mcode[q] != want) continue;
                            take((size_t)q);
                            out++;
                        }
                    }
                }
                auto &fl = far[s][cell];
                std::sort(fl.begin(), fl.end());
                for (auto &e : fl) {
                    take(e.second);
                    out++;
                }
                ncnt[cell] = out;
            }
            p.cnt.swap(ncnt);
            p.x.swap(nx); p.y.swap(ny); p.vx.swap(nvx); p.vy.swap(nvy); p.vz.swap(nvz);
            p.restart();
            p.mcnt.assign(C, 0);
            p.mstart.assign(C + 1, 0);
            p.mx.clear(); p.my.clear(); p.mvx.clear(); p.mvy.clear(); p.mvz.clear(); p.mcode.clear();
            far[s].assign(C, {});
        }
    }

    // ------------------------------------------------------------ MCC draws
    // the null-collision test draw and a particle stream's next draw, or the
    // scripted list of the same (species, cell)
    float u_test(uint32_t slot, int cell, uint32_t step, uint32_t species, uint32_t sub) {
        return script.on ? u_script(species, (uint32_t)cell)
                         : hp_test_draw(c.seed, slot, (uint32_t)cell, step, species, sub);
    }
    float nextu(hp_stream &rs) { return script.on ? u_script(rs.ctr.w >> 16, rs.ctr.y) : hp_stream_next(&rs); }
    // one collider's own list (single-collision entry points)
    struct ListStream {
        const float *u;
        int n, pos;
        bool overrun;
        int pair_rl;
    };
    static float nextu(ListStream &ls) {
        if (ls.pos >= ls.n) {
            ls.overrun = true;
            return 1.0f;
        }
        return ls.u[ls.pos++];
    }
    // The two uniforms a collision passes to one kinematics call
    // (anewvel, maxwellv, newvel_ionsc).  C++ leaves the order in which the
    // reference's two curand_uniform() arguments are evaluated open; the
    // Philox streams take the left one first, and a scripted list can be
    // read right to left for the calls whose bit (PAIR_*) is set in the
    // script's pair mask, as the reference's nvcc build evaluates them.
    enum { PAIR_ANEWVEL = 1, PAIR_MAXWELLV = 2, PAIR_IONSC = 4 };
    int pair_rl(const hp_stream &) const { return script.on ? script.pair_rl : 0; }
    static int pair_rl(const ListStream &ls) { return ls.pair_rl; }
    template <class S> void draw2(S &rs, R &a, R &b, int call) {
        const R first = (R)nextu(rs), second = (R)nextu(rs);
        if (pair_rl(rs) & call) { a = second; b = first; }
        else { a = first; b = second; }
    }

    // ------------------------------------------------------------ MCC (Ar)
    R xsec(int ch, R engy) const {
        if (engy == 0) return (R)0;
        const R lengy = m_log10(engy);
        const float *t = c.xsec;
        const int W = c.xw;
        const R xe0 = t[0], xeN = t[(c.n_logx - 1) * W];
        if (lengy < xe0) return t[2 + ch];
        if (lengy > xeN) return (R)t[(c.n_logx - 1) * W + 2 + ch] * (R)0.1f * m_exp((R)(-1 * (lengy - xeN)));
        const R ee1 = (R)c.idlogx * (lengy - xe0);
        int ee2 = (int)ee1;
        if (ee2 > c.n_logx - 2) ee2 = c.n_logx - 2;
        if (ee2 < 0) ee2 = 0;
        const R a1 = ee1 - ee2;
        const R a2 = 1 - a1;
        return a2 * (R)t[ee2 * W + 2 + ch] + a1 * (R)t[(ee2 + 1) * W + 2 + ch];
    }
    static void maxwellv(R &vx, R &vy, R &vz, R vsaven, R vti, R Rphi, R Rthe) {
        R sn, cs;
        m_sincos_turns(Rphi, &sn, &cs);
        const R costheta = 1 - 2 * Rthe;
        const R sintheta = std::sqrt(1 - costheta * costheta);
        vx = vti * vsaven * sintheta * cs;
        vy = vti * vsaven * sintheta * sn;
        vz = vti * vsaven * costheta;
    }
    static void anewvel(R energy, R vel, R &nvx, R &nvy, R &nvz, R rand1, R rand2) {
        R coschi;
        if (energy < (R)1e-30f) coschi = 1;
        else coschi = (R)(((double)energy + 2.0 - 2.0 * (double)m_pow((R)(energy + 1.0), rand1)) / energy);
        const R sinchi = (R)std::sqrt(std::fabs(1.0 - (double)(coschi * coschi)));
        R sinphi, cosphi;
        m_sincos_turns(rand2, &sinphi, &cosphi);
        const R r13 = nvx, r23 = nvy, r33 = nvz;
        R up1, up2, up3;
        if (r33 == (R)1.0f || r33 == (R)-1.0f) { up1 = 0; up2 = 1; up3 = 0; }
        else { up1 = 0; up2 = 0; up3 = 1; }
        R r12 = r23 * up3 - r33 * up2;
        R r22 = r33 * up1 - r13 * up3;
        R r32 = r13 * up2 - r23 * up1;
        const R mag = std::sqrt(r12 * r12 + r22 * r22 + r32 * r32);
        r12 /= mag; r22 /= mag; r32 /= mag;
        const R r11 = r22 * r33 - r32 * r23;
        const R r21 = r32 * r13 - r12 * r33;
        const R r31 = r12 * r23 - r22 * r13;
        nvx = vel * (r11 * sinchi * cosphi + r12 * sinchi * sinphi + r13 * coschi);
        nvy = vel * (r21 * sinchi * cosphi + r22 * sinchi * sinphi + r23 * coschi);
        nvz = vel * (r31 * sinchi * cosphi + r32 * sinchi * sinphi + r33 * coschi);
    }
    static void newvel_ionsc(R &vxs, R &vys, R &vzs, R vel, R rand1, R rand2) {
        const R coschi = std::sqrt(rand1);
        const R sinchi = (R)std::sqrt(std::fabs(1.0 - (double)(coschi * coschi)));
        R sinphi, cosphi;
        m_sincos_turns(rand2, &sinphi, &cosphi);
        const R r13 = vxs / vel, r23 = vys / vel, r33 = vzs / vel;
        R up1, up2, up3;
        if (r33 == (R)1.0f || r33 == (R)-1.0f) { up1 = 0; up2 = 1; up3 = 0; }
        else { up1 = 0; up2 = 0; up3 = 1; }
        R r12 = r23 * up3 - r33 * up2;
        R r22 = r33 * up1 - r13 * up3;
        R r32 = r13 * up2 - r23 * up1;
        const R mag = std::sqrt(r12 * r12 + r22 * r22 + r32 * r32);
        r12 /= mag; r22 /= mag; r32 /= mag;
        const R r11 = r22 * r33 - r32 * r23;
        const R r21 = r32 * r13 - r12 * r33;
        const R r31 = r12 * r23 - r22 * r13;
        vxs = vel * coschi * (r11 * sinchi * cosphi + r12 * sinchi * sinphi + r13 * coschi);
        vys = vel * coschi * (r21 * sinchi * cosphi + r22 * sinchi * sinphi + r23 * coschi);
        vzs = vel * coschi * (r31 * sinchi * cosphi + r32 * sinchi * sinphi + r33 * coschi);
    }

    void xsec_n(int ch, const float *engy, float *out, int n) const override {
        for (int k = 0; k < n; k++) out[k] = (float)xsec(ch, (R)engy[k]);
    }
    void kinematics(int kind, const float *in, float *out, int n) const override {
        for (int k = 0; k < n; k++) {
            R x = 0, y = 0, z = 0;
            if (kind == 0) {
                const float *a = in + 7 * (size_t)k;
                x = a[2]; y = a[3]; z = a[4];
                anewvel((R)a[0], (R)a[1], x, y, z, (R)a[5], (R)a[6]);
            } else if (kind == 1) {
                const float *a = in + 6 * (size_t)k;
                x = a[0]; y = a[1]; z = a[2];
                newvel_ionsc(x, y, z, (R)a[3], (R)a[4], (R)a[5]);
            } else {
                const float *a = in + 4 * (size_t)k;
                maxwellv(x, y, z, (R)a[0], (R)a[1], (R)a[2], (R)a[3]);
            }
            out[3 * (size_t)k] = (float)x;
            out[3 * (size_t)k + 1] = (float)y;
            out[3 * (size_t)k + 2] = (float)z;
        }
    }
    int collide_oxy(int isp, int t, const float *v, float bv1, float bv2, const float *u, int nu, int pair_rl_,
                    int *ch, int *keep, float *vout, int *bsp, float *bv, int *kill) override {
        ListStream ls{u, nu, 0, false, pair_rl_};
        OxyOut o;
        if (isp == 0) oxy_electron((R)v[0], (R)v[1], (R)v[2], t, (R)bv1, ls, o);
        else oxy_ion(isp, (R)v[0], (R)v[1], (R)v[2], t, (R)bv1, (R)bv2, ls, o);
        *ch = o.ch;
        *keep = o.keep ? 1 : 0;
        vout[0] = (float)o.vx; vout[1] = (float)o.vy; vout[2] = (float)o.vz;
        for (int q = 0; q < 2; q++) {
            bsp[q] = o.bsp[q];
            for (int d = 0; d < 3; d++) bv[3 * q + d] = (float)o.bv[q][d];
        }
        *kill = o.kill ? 1 : 0;
        return ls.overrun ? 1 : 0;
    }

    // ------------------------------------------------------------ MCC (Ar/O2)
    // MCC_ArO2_Basic (src/cuda_mcc.cu:21-71), ArO2_Collision_Check and the
    // species handlers (src/cuda_mccArO2.cu:51-1265), with the order this
    // library defines: tests on the counts at the start of the call, species
    // e, Ar+, O2+, O+, O- in turn, colliders in slot order, holes filled from
    // the end of each species (a stable compaction when a species has more
    // than 64 holes in a cell), births appended in collider order, the O-
    // removed by a detachment drawn among the O- present at the start.
    struct OxyOut {
        bool keep = true;
        R vx = 0, vy = 0, vz = 0;
        int bsp[2] = {-1, -1};
        R bv[2][3] = {{0, 0, 0}, {0, 0, 0}};
        bool kill = false;
        float r2 = 0.f;
        int ch = -1;
    };
    static R ox_exp(R x) { return m_exp(x); }
    // 1 - exp(-a b n) accumulated as the reference does: float with 1.0f for
    // electrons, double (its 1.0 literal) for ions
    static R e_acc(R prev, bool first, R ex) { return first ? (R)1.0f - ex : prev + (R)1.0f - ex; }
    static R i_acc(R prev, bool first, R ex) {
        return first ? (R)(1.0 - (double)ex) : (R)((double)prev + 1.0 - (double)ex);
    }

    template <class S> void oxy_electron(R vx, R vy, R vz, int t, R bv1, S &rs, OxyOut &o) {
        // ladders: (channel, action, threshold index or first new species, second new species, gain)
        enum { EL, LO, GA, AT, IO, RE, DE };
        struct Rg { int ch, act, a1, a2; float gain; };
        static const Rg rg[] = {
            {0, EL, 0, 0, 0}, {1, LO, 1, 0, 0}, {2, LO, 2, 0, 0}, {3, IO, 0, 1, 0},
            {4, IO, 0, 1, 0},
            {5, EL, 0, 0, 0}, {6, LO, 6, 0, 0}, {7, LO, 7, 0, 0}, {8, LO, 8, 0, 0}, {9, LO, 9, 0, 0},
            {10, LO, 10, 0, 0}, {11, AT, 0, 0, 0}, {12, LO, 12, 0, 0}, {13, LO, 13, 0, 0}, {14, LO, 14, 0, 0},
            {15, IO, 0, 2, 0}, {16, LO, 11, 0, 0}, {17, IO, 3, 4, 0}, {18, IO, 0, 3, 0},
            {19, IO, 0, 2, 0}, {20, AT, 0, 0, 0}, {21, GA, 0, 0, 0.977f}, {22, GA, 0, 0, 0.977f},
            {23, LO, 23, 0, 0}, {24, LO, 24, 0, 0}, {25, LO, 25, 0, 0}, {26, IO, 0, 3, 0},
            {27, IO, 0, 2, 0}, {28, AT, 0, 0, 0}, {29, GA, 0, 0, 1.627f}, {30, GA, 0, 0, 1.627f},
            {31, LO, 31, 0, 0}, {32, LO, 32, 0, 0}, {33, LO, 33, 0, 0}, {34, IO, 0, 3, 0},
            {35, DE, 0, 0, 0},
            {36, RE, 0, 0, 0},
            {37, LO, 37, 0, 0}, {38, LO, 38, 0, 0}, {39, LO, 39, 0, 0}, {40, LO, 40, 0, 0}, {41, LO, 41, 0, 0},
            {42, IO, 0, 3, 0}, {43, LO, 43, 0, 0},
            {44, IO, 0, 3, 0}, {45, GA, 0, 0, 1.96f},
        };
        static const int start[10] = {0, 4, 5, 19, 27, 35, 36, 37, 44, 46};
        // the O2 set (src/cuda_mccO2.cu:2-429)
        static const Rg rgo[] = {
            {0, EL, 0, 0, 0}, {1, LO, 1, 0, 0}, {2, LO, 2, 0, 0}, {3, LO, 3, 0, 0}, {4, LO, 4, 0, 0},
            {5, LO, 5, 0, 0}, {6, AT, 0, 0, 0}, {7, LO, 7, 0, 0}, {8, LO, 8, 0, 0}, {9, LO, 9, 0, 0},
            {10, IO, 0, 1, 0}, {11, LO, 11, 0, 0}, {12, IO, 2, 3, 0}, {13, IO, 0, 2, 0},
            {14, IO, 0, 1, 0}, {15, AT, 0, 0, 0}, {16, GA, 0, 0, 0.977f}, {17, GA, 0, 0, 0.977f},
            {18, LO, 18, 0, 0}, {19, LO, 19, 0, 0}, {20, LO, 20, 0, 0}, {21, IO, 0, 2, 0},
            {22, IO, 0, 1, 0}, {23, AT, 0, 0, 0}, {24, GA, 0, 0, 1.627f}, {25, GA, 0, 0, 1.627f},
            {26, LO, 26, 0, 0}, {27, LO, 27, 0, 0}, {28, LO, 28, 0, 0}, {29, IO, 0, 2, 0},
            {30, DE, 0, 0, 0},
            {31, RE, 0, 0, 0},
            {32, LO, 32, 0, 0}, {33, LO, 33, 0, 0}, {34, LO, 34, 0, 0}, {35, LO, 35, 0, 0}, {36, LO, 36, 0, 0},
            {37, IO, 0, 2, 0}, {38, LO, 38, 0, 0},
            {39, IO, 0, 2, 0}, {40, GA, 0, 0, 1.96f},
        };
        static const int starto[8] = {0, 14, 22, 30, 31, 32, 39, 41};
        const bool aro2 = c.gas == 2;
        const Rg *ladder = aro2 ? rg : rgo;
        const int *lstart = aro2 ? start : starto;
        const R Esc = (R)c.Escale[0];
        R VX = vx, VY = vy, VZ = vz;
        const R dum = VX * VX + VY * VY + VZ * VZ;
        R vel = std::sqrt(dum);
        VX /= vel; VY /= vel; VZ /= vel;
        R engy = Esc * dum;
        int colltype = 1, i1 = 0, i2 = 0;
        R rengy = 0, vel2 = 0;
        R R1;
        if (aro2) {
            R1 = (R)nextu(rs);
            R1 *= (R)c.sigv[t] / vel;
        } else {
            R1 = (R)nextu(rs) * (R)c.sigv[t] / vel;
        }
        R sum = 0;
        bool hit = false;
        for (int k = lstart[t]; k < lstart[t + 1]; k++) {
            const Rg &r = ladder[k];
            if (!(engy > (R)c.th[r.ch])) continue;
            sum = sum + xsec(r.ch, engy);
            if (!(R1 <= sum)) continue;
            hit = true;
            o.ch = r.ch;
            switch (r.act) {
            case EL: break;
            case LO: engy -= (R)c.th[r.a1]; vel = std::sqrt(std::fabs(engy) / Esc); break;
            case GA: engy += (R)r.gain; vel = std::sqrt(std::fabs(engy) / Esc); break;
            case AT: colltype = 2; break;
            case RE: colltype = 4; break;
            case DE:
                colltype = 5;
                engy -= (R)c.th[r.ch];
                vel = std::sqrt(std::fabs(engy) / Esc);
                break;
            default: {
                colltype = 3;
                engy -= (R)c.th[r.ch];
                if (aro2) {
                    const R u = (R)nextu(rs);
                    rengy = (R)(10.0 * (double)m_tan(u * m_atan((R)(engy / 20.0))));
                    engy -= rengy;
                    vel = std::sqrt(std::fabs(rengy) / Esc);
                    vel2 = std::sqrt(std::fabs(engy) / Esc);
                } else {
                    vel = std::sqrt(std::fabs(engy) / Esc);
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
            R a, b;
            draw2(rs, a, b, PAIR_ANEWVEL);
            anewvel(engy, vel, VX, VY, VZ, a, b);
            o.vx = VX; o.vy = VY; o.vz = VZ;
            break;
        }
        case 2: {
            o.keep = false;
            const int n = (int)((c.nvel - 1) * nextu(rs));
            R a, b;
            draw2(rs, a, b, PAIR_MAXWELLV);
            o.bsp[0] = aro2 ? 4 : 3;
            maxwellv(o.bv[0][0], o.bv[0][1], o.bv[0][2], (R)c.vsave[n], bv1, a, b);
            break;
        }
        case 3: {
            const int isp[2] = {i1, i2};
            for (int q = 0; q < 2; q++) {
                o.bsp[q] = isp[q];
                if (isp[q] == 0) {
                    o.bv[q][0] = VX; o.bv[q][1] = VY; o.bv[q][2] = VZ;
                    if (aro2) {
                        R a, b;
                        draw2(rs, a, b, PAIR_ANEWVEL);
                        anewvel(rengy, vel, o.bv[q][0], o.bv[q][1], o.bv[q][2], a, b);
                    }
                } else {
                    const int n = (int)((c.nvel - 1) * nextu(rs));
                    R a, b;
                    draw2(rs, a, b, PAIR_MAXWELLV);
                    maxwellv(o.bv[q][0], o.bv[q][1], o.bv[q][2], (R)c.vsave[n], bv1, a, b);
                }
            }
            R a, b;
            draw2(rs, a, b, PAIR_ANEWVEL);
            anewvel(engy, aro2 ? vel2 : vel, VX, VY, VZ, a, b);
            o.vx = VX; o.vy = VY; o.vz = VZ;
            break;
        }
        case 4: o.keep = false; break;
        default: {
            o.bsp[0] = 0;
            o.bv[0][0] = VX; o.bv[0][1] = VY; o.bv[0][2] = VZ;
            R a, b;
            draw2(rs, a, b, PAIR_ANEWVEL);
            anewvel(engy, vel, VX, VY, VZ, a, b);
            o.vx = VX; o.vy = VY; o.vz = VZ;
            o.kill = true;
            o.r2 = nextu(rs);
            break;
        }
        }
    }

    template <class S> void oxy_ion(int s, R vx, R vy, R vz, int t, R bv1, R bv2, S &rs, OxyOut &o) {
        enum { NUL, SCAT, CX, TO_OP, TO_ARP, TO_O2P, DET, REC };
        const bool aro2 = c.gas == 2;
        const int OMINUS = aro2 ? 4 : 3, O2P = aro2 ? 2 : 1, OPL = aro2 ? 3 : 2;
        o.keep = true;
        o.vx = vx; o.vy = vy; o.vz = vz;
        const R Esc = (R)c.Escale[s];
        R vnx = 0, vny = 0, vnz = 0, VX, VY, VZ, vel, engy;
        if (s == OMINUS) {
            VX = vx; VY = vy; VZ = vz;
            const R dum = VX * VX + VY * VY + VZ * VZ;
            vel = std::sqrt(dum);
            VX /= vel; VY /= vel; VZ /= vel;
            engy = Esc * dum;
        } else {
            const R vneut = aro2 ? (s == 1 ? (t == 0 ? bv1 : bv2) : (s == 2 ? bv1 : bv2)) : bv1;
            const int n = (int)((c.nvel - 1) * nextu(rs));
            R a, b;
            draw2(rs, a, b, PAIR_MAXWELLV);
            maxwellv(vnx, vny, vnz, (R)c.vsave[n], vneut, a, b);
            VX = vx - vnx; VY = vy - vny; VZ = vz - vnz;
            const R dum = VX * VX + VY * VY + VZ * VZ;
            vel = std::sqrt(dum);
            engy = Esc * dum;
            if (aro2 && s == 1) (void)nextu(rs);
        }
        int sv = 0, nr = 0, ch[3] = {0, 0, 0}, act[3] = {0, 0, 0};
        bool cum = false;
        if (!aro2) {
            switch (s) {
            case 1:
                sv = 12 + t;
                if (t == 0) { nr = 1; ch[0] = 47; act[0] = TO_OP; }
                else if (t == 1) { nr = 3; ch[0] = 48; act[0] = CX; ch[1] = 49; act[1] = SCAT; ch[2] = 50; act[2] = TO_OP; }
                else { nr = 1; ch[0] = 49 + t; act[0] = CX; }
                break;
            case 2:
                sv = 16 + t;
                if (t == 0) { nr = 2; ch[0] = 53; act[0] = TO_O2P; ch[1] = 54; act[1] = SCAT; }
                else if (t == 1) { nr = 1; ch[0] = 55; act[0] = CX; }
                else { nr = 1; ch[0] = 54 + t; act[0] = TO_O2P; }
                break;
            default:
                sv = 9 + t;
                if (t == 0) { nr = 2; ch[0] = 41; act[0] = SCAT; ch[1] = 42; act[1] = DET; cum = true; }
                else if (t == 1) { nr = 1; ch[0] = 43; act[0] = DET; }
                else if (t == 2) { nr = 1; ch[0] = 44; act[0] = REC; }
                else if (t == 3) { nr = 1; ch[0] = 45; act[0] = REC; }
                else { nr = 1; ch[0] = 46; act[0] = DET; }
                break;
            }
        } else
        switch (s) {
        case 1:
            sv = 23 + t;
            if (t == 0) { nr = 2; ch[0] = 65; act[0] = CX; ch[1] = 66; act[1] = SCAT; }
            else { nr = 1; ch[0] = 67; act[0] = SCAT; }
            break;
        case 2:
            sv = 14 + t;
            if (t == 0) { nr = 1; ch[0] = 52; act[0] = TO_OP; }
            else if (t == 1) { nr = 3; ch[0] = 53; act[0] = CX; ch[1] = 54; act[1] = SCAT; ch[2] = 55; act[2] = TO_OP; }
            else if (t == 2) { nr = 1; ch[0] = 56; act[0] = CX; }
            else if (t == 3) { nr = 1; ch[0] = 57; act[0] = CX; }
            else { nr = 2; ch[0] = 58; act[0] = TO_ARP; ch[1] = 59; act[1] = CX; }
            break;
        case 3:
            sv = 19 + t;
            if (t == 0) { nr = 2; ch[0] = 60; act[0] = TO_O2P; ch[1] = 61; act[1] = SCAT; }
            else if (t == 1) { nr = 1; ch[0] = 62; act[0] = CX; }
            else { nr = 1; ch[0] = 61 + t; act[0] = TO_O2P; }
            break;
        default:
            sv = 9 + t;
            if (t == 0) { nr = 2; ch[0] = 46; act[0] = SCAT; ch[1] = 47; act[1] = DET; cum = true; }
            else if (t == 1) { nr = 1; ch[0] = 48; act[0] = DET; }
            else if (t == 2) { nr = 1; ch[0] = 49; act[0] = REC; }
            else if (t == 3) { nr = 1; ch[0] = 50; act[0] = REC; }
            else { nr = 1; ch[0] = 51; act[0] = DET; }
            break;
        }
        const R R1 = (R)nextu(rs) * (R)c.sigv[sv] / vel;
        int what = NUL;
        R sum = 0;
        for (int k = 0; k < nr; k++) {
            if (!(engy > (R)c.th[ch[k]])) continue;
            const R xs = xsec(ch[k], engy);
            sum = (k > 0 && cum) ? sum + xs : xs;
            if (R1 <= sum) { what = act[k]; o.ch = ch[k]; break; }
        }
        auto born = [&](int sp_, R a, R b, R cc) { o.keep = false; o.bsp[0] = sp_; o.bv[0][0] = a; o.bv[0][1] = b; o.bv[0][2] = cc; };
        switch (what) {
        case NUL: break;
        case SCAT: {
            R a, b;
            draw2(rs, a, b, PAIR_IONSC);
            newvel_ionsc(VX, VY, VZ, vel, a, b);
            if (s == OMINUS) { o.vx = VX; o.vy = VY; o.vz = VZ; }
            else { o.vx = VX + vnx; o.vy = VY + vny; o.vz = VZ + vnz; }
            break;
        }
        case CX: o.vx = vnx; o.vy = vny; o.vz = vnz; break;
        case TO_OP: born(OPL, vnx, vny, vnz); break;
        case TO_ARP: born(1, vnx, vny, vnz); break;
        case TO_O2P: born(O2P, vnx, vny, vnz); break;
        case DET: born(0, VX, VY, VZ); break;
        default: o.keep = false; break;
        }
    }

    void mcc_aro2(int64_t tstep) {
        const uint32_t step = (uint32_t)tstep;
        const bool aro2 = c.gas == 2;
        const int NS = aro2 ? 5 : 4, STRIDE = c.mcc_stride, HOLE_CAP = 64, OMINUS = aro2 ? 4 : 3;
        // the reference's O2 launch collides electrons only (src/cuda_mcc.cu:76-77)
        const int NACT = (aro2 || c.mcc_all_species) ? NS : 1;
        struct P5 { std::vector<R> x, y, vx, vy, vz; };
        std::vector<std::array<P5, 5>> out((size_t)C);
        par_for(C, [&](int cell) {
            const int i = cell / c.ncy, j = cell - i * c.ncy, node = i * c.ngy + j, Gn = G;
            const R bd1 = c.back_den1[node], bd2 = aro2 ? (R)c.back_den2[node] : (R)0;
            const R F0 = fnode[node], F1 = fnode[Gn + node], F2 = fnode[2 * Gn + node];
            const R F3 = fnode[3 * Gn + node], F4 = aro2 ? (R)fnode[4 * Gn + node] : (R)0;
            auto xe = [&](R a, R b, R n) { return ox_exp(-1 * a * b * n); };
            auto nq = [&](int s, R sig, R dtx) {
                R t = -1 * dtx;
                t = t * sig;
                t = t * (R)(float)den[(size_t)s * Gn + node];
                t = t * (R)c.np2c[s];
                t = t * (R)c.idx;
                t = t * (R)c.idy;
                return ox_exp(t);
            };
            const R dtm = c.dt_mcc, dt = c.dt;
            const float *sv = c.sigv;
            R p[5][9];
            int np[5] = {9, 2, 5, 4, 5};
            if (!aro2) { // O2Collision_Check (src/cuda_mccO2.cu:867-911)
                np[0] = 7; np[1] = 4; np[2] = 4; np[3] = 5; np[4] = 1;
                R *e = p[0];
                e[0] = e_acc(0, true, xe(dtm, sv[0], bd1));
                e[1] = e_acc(e[0], false, xe(dtm, sv[1], F0));
                e[2] = e_acc(e[1], false, xe(dtm, sv[2], F1));
                e[3] = e_acc(e[2], false, nq(3, sv[3], dtm));
                e[4] = e_acc(e[3], false, nq(1, sv[4], dtm));
                e[5] = e_acc(e[4], false, xe(dtm, sv[5], F2));
                e[6] = e_acc(e[5], false, xe(dtm, sv[6], F3));
                R *a = p[1];
                a[0] = i_acc(0, true, xe(dtm, sv[12], F2));
                a[1] = i_acc(a[0], false, xe(dtm, sv[13], bd1));
                a[2] = i_acc(a[1], false, xe(dtm, sv[14], F0));
                a[3] = i_acc(a[2], false, xe(dtm, sv[15], F1));
                R *b = p[2];
                b[0] = i_acc(0, true, xe(dt, sv[16], bd1));
                b[1] = i_acc(b[0], false, xe(dt, sv[17], F2));
                b[2] = i_acc(b[1], false, xe(dt, sv[18], F0));
                b[3] = i_acc(b[2], false, xe(dt, sv[19], F1));
                R *m = p[3];
                m[0] = i_acc(0, true, xe(dt, sv[7], bd1));
                m[1] = i_acc(m[0], false, xe(dt, sv[8], F2));
                m[2] = i_acc(m[1], false, nq(1, sv[9], dt));
                m[3] = i_acc(m[2], false, nq(2, sv[10], dt));
                m[4] = i_acc(m[3], false, xe(dt, sv[11], F0));
            } else {
                R *e = p[0];
                e[0] = e_acc(0, true, xe(dtm, sv[0], bd1));
                e[1] = e_acc(e[0], false, xe(dtm, sv[1], F0));
                e[2] = e_acc(e[1], false, xe(dtm, sv[2], bd2));
                e[3] = e_acc(e[2], false, xe(dtm, sv[3], F1));
                e[4] = e_acc(e[3], false, xe(dtm, sv[4], F2));
                e[5] = e_acc(e[4], false, nq(4, sv[5], dtm));
                e[6] = e_acc(e[5], false, nq(2, sv[6], dtm));
                e[7] = e_acc(e[6], false, xe(dtm, sv[7], F3));
                e[8] = e_acc(e[7], false, xe(dtm, sv[8], F4));
                R *a = p[1];
                a[0] = i_acc(0, true, xe(dt, sv[23], bd1));
                a[1] = i_acc(a[0], false, xe(dt, sv[24], bd2));
                R *o2 = p[2];
                o2[0] = i_acc(0, true, xe(dt, sv[14], F3));
                o2[1] = i_acc(o2[0], false, xe(dt, sv[15], bd2));
                o2[2] = i_acc(o2[1], false, xe(dt, sv[16], F1));
                o2[3] = i_acc(o2[2], false, xe(dt, sv[17], F2));
                o2[4] = i_acc(o2[3], false, xe(dt, sv[18], bd1));
                R *op = p[3];
                op[0] = i_acc(0, true, xe(dt, sv[19], bd2));
                op[1] = i_acc(op[0], false, xe(dt, sv[20], F3));
                op[2] = i_acc(op[1], false, xe(dt, sv[21], F1));
                op[3] = i_acc(op[2], false, xe(dt, sv[22], F2));
                R *om = p[4];
                om[0] = i_acc(0, true, xe(dt, sv[9], bd2));
                om[1] = i_acc(om[0], false, xe(dt, sv[10], F3));
                om[2] = i_acc(om[1], false, nq(2, sv[11], dt));
                om[3] = i_acc(om[2], false, nq(3, sv[12], dt));
                om[4] = i_acc(om[3], false, xe(dt, sv[13], F1));
            }
            const R bv1 = c.back_vel1[node], bv2 = aro2 ? (R)c.back_vel2[node] : (R)0;
            std::array<P5, 5> &L = out[(size_t)cell];
            std::vector<char> gone[5];
            int n0[5];
            std::vector<int> holes[5];
            for (int s = 0; s < NS; s++) {
                Sp &q = sp[s];
                const int a = q.start[cell], b = q.start[cell + 1];
                L[s].x.assign(q.x.begin() + a, q.x.begin() + b);
                L[s].y.assign(q.y.begin() + a, q.y.begin() + b);
                L[s].vx.assign(q.vx.begin() + a, q.vx.begin() + b);
                L[s].vy.assign(q.vy.begin() + a, q.vy.begin() + b);
                L[s].vz.assign(q.vz.begin() + a, q.vz.begin() + b);
                n0[s] = b - a;
                gone[s].assign((size_t)n0[s], 0);
            }
            unsigned *cnt = &mcc_count[(size_t)cell * STRIDE];
            for (int s = 0; s < NACT; s++) {
                const int nsub = (s == 0 || (!aro2 && s == 1)) ? c.mcc_n : 1;
                const R Tprob = p[s][np[s] - 1];
                for (int k = 0; k < n0[s]; k++) {
                    int t = -1;
                    for (int jj = 0; jj < nsub; jj++) {
                        const float R1 = u_test((uint32_t)k, cell, step, (uint32_t)s, (uint32_t)jj);
                        if ((R)R1 < Tprob) {
                            t = np[s] - 1;
                            for (int q = 0; q < np[s] - 1; q++)
                                if ((R)R1 <= p[s][q]) { t = q; break; }
                            break;
                        }
                    }
                    if (t < 0 || gone[s][(size_t)k]) continue;
                    hp_stream rs;
                    hp_stream_init(&rs, c.seed, (uint32_t)k, (uint32_t)cell, step, (uint32_t)s);
                    OxyOut o;
                    const R vx = L[s].vx[(size_t)k], vy = L[s].vy[(size_t)k], vz = L[s].vz[(size_t)k];
                    if (s == 0) oxy_electron(vx, vy, vz, t, bv1, rs, o);
                    else oxy_ion(s, vx, vy, vz, t, bv1, bv2, rs, o);
                    if (o.ch >= 0) cnt[o.ch]++;
                    const R px = L[s].x[(size_t)k], py = L[s].y[(size_t)k];
                    if (o.keep) {
                        L[s].vx[(size_t)k] = o.vx; L[s].vy[(size_t)k] = o.vy; L[s].vz[(size_t)k] = o.vz;
                    } else {
                        gone[s][(size_t)k] = 1;
                        holes[s].push_back(k);
                    }
                    for (int q = 0; q < 2; q++) {
                        const int t2 = o.bsp[q];
                        if (t2 < 0) continue;
                        L[t2].x.push_back(px); L[t2].y.push_back(py);
                        L[t2].vx.push_back(o.bv[q][0]); L[t2].vy.push_back(o.bv[q][1]); L[t2].vz.push_back(o.bv[q][2]);
                        gone[t2].push_back(0);
                    }
                    if (o.kill) {
                        const int om = OMINUS;
                        int nlive = 0;
                        for (int q = 0; q < n0[om]; q++) nlive += gone[om][(size_t)q] ? 0 : 1;
                        if (nlive > 0) {
                            int pick = 0;
                            if (nlive > 1) {
                                pick = (int)((float)nlive * o.r2);
                                if (pick > nlive - 1) pick = nlive - 1;
                            }
                            for (int q = 0; q < n0[om]; q++) {
                                if (gone[om][(size_t)q]) continue;
                                if (pick-- == 0) {
                                    gone[om][(size_t)q] = 1;
                                    holes[om].push_back(q);
                                    break;
                                }
                            }
                        }
                    }
                }
            }
            for (int s = 0; s < NS; s++) {
                P5 &l = L[s];
                int n = (int)l.x.size();
                if (holes[s].empty()) continue;
                if ((int)holes[s].size() <= HOLE_CAP) {
                    std::vector<int> h = holes[s];
                    std::sort(h.begin(), h.end());
                    for (int hp : h) {
                        while (n > 0 && gone[s][(size_t)n - 1]) n--;
                        if (hp >= n) continue;
                        l.x[(size_t)hp] = l.x[(size_t)n - 1]; l.y[(size_t)hp] = l.y[(size_t)n - 1];
                        l.vx[(size_t)hp] = l.vx[(size_t)n - 1]; l.vy[(size_t)hp] = l.vy[(size_t)n - 1];
                        l.vz[(size_t)hp] = l.vz[(size_t)n - 1];
                        gone[s][(size_t)hp] = 0;
                        n--;
                    }
                    while (n > 0 && gone[s][(size_t)n - 1]) n--;
                } else {
                    int w = 0;
                    for (int k = 0; k < n; k++) {
                        if (gone[s][(size_t)k]) continue;
                        l.x[(size_t)w] = l.x[(size_t)k]; l.y[(size_t)w] = l.y[(size_t)k];
                        l.vx[(size_t)w] = l.vx[(size_t)k]; l.vy[(size_t)w] = l.vy[(size_t)k];
                        l.vz[(size_t)w] = l.vz[(size_t)k];
                        w++;
                    }
                    n = w;
                }
                l.x.resize((size_t)n); l.y.resize((size_t)n); l.vx.resize((size_t)n); l.vy.resize((size_t)n);
                l.vz.resize((size_t)n);
            }
        });
        for (int s = 0; s < NS; s++) {
            Sp &q = sp[s];
            std::vector<R> nx, ny, nvx, nvy, nvz;
            for (int cell = 0; cell < C; cell++) {
                const P5 &l = out[(size_t)cell][(size_t)s];
                nx.insert(nx.end(), l.x.begin(), l.x.end()); ny.insert(ny.end(), l.y.begin(), l.y.end());
                nvx.insert(nvx.end(), l.vx.begin(), l.vx.end()); nvy.insert(nvy.end(), l.vy.begin(), l.vy.end());
                nvz.insert(nvz.end(), l.vz.begin(), l.vz.end());
                q.cnt[cell] = (int)l.x.size();
            }
            q.x.swap(nx); q.y.swap(ny); q.vx.swap(nvx); q.vy.swap(nvy); q.vz.swap(nvz);
            q.restart();
        }
    }

    void mcc(int64_t tstep) override {
        if (c.gas == 1 || c.gas == 2) {
            mcc_aro2(tstep);
            return;
        }
        Sp &el = sp[0], &ion = sp[1];
        const uint32_t step = (uint32_t)tstep;
        std::vector<int> ecnt(C), icnt(C);
        // per-cell outputs, then CSR rebuild
        std::vector<std::vector<R>> enew(C), inew(C); // created particles: x,y,vx,vy,vz
        par_for(C, [&](int cell) {
            const int i = cell / c.ncy, j = cell - i * c.ncy, node = i * c.ngy + j;
            const float P1 = prob_v[cell], P2 = prob_v[C + cell], Pion = prob_v[2 * C + cell];
            const R bvel = c.back_vel1[node];
            unsigned cnt_ch[7] = {0, 0, 0, 0, 0, 0, 0};
            const int ni = ion.cnt[cell];
            for (int k = 0; k < ni; k++) {
                if (u_test((uint32_t)k, cell, step, 1u, 0u) > Pion) continue;
                hp_stream rs;
                hp_stream_init(&rs, c.seed, (uint32_t)k, (uint32_t)cell, step, 1u);
                const int nn = (int)((c.nvel - 1) * nextu(rs));
                R vnx, vny, vnz;
                {
                    R a, b;
                    draw2(rs, a, b, PAIR_MAXWELLV);
                    maxwellv(vnx, vny, vnz, (R)c.vsave[nn], bvel, a, b);
                }
                const size_t q = (size_t)ion.start[cell] + k;
                const R vx = ion.vx[q], vy = ion.vy[q], vz = ion.vz[q];
                R VX = vx - vnx, VY = vy - vnz, VZ = vz - vny;
                const R dum = VX * VX + VY * VY + VZ * VZ;
                const R engy = (R)c.Escale[1] * dum;
                const R vel = std::sqrt(dum);
                const R Rr = (R)nextu(rs) * (R)c.sigv[2] / vel;
                R SumSigma = xsec(5, engy);
                R ox, oy, oz;
                if (Rr <= SumSigma) {
                    ox = vnx; oy = vny; oz = vnz;
                    cnt_ch[5]++;
                } else if (Rr <= (SumSigma += xsec(6, engy))) {
                    R a, b;
                    draw2(rs, a, b, PAIR_IONSC);
                    newvel_ionsc(VX, VY, VZ, vel, a, b);
                    ox = VX + vnx; oy = VY + vny; oz = VZ + vnz;
                    cnt_ch[6]++;
                } else {
                    ox = vx; oy = vy; oz = vz;
                }
                ion.vx[q] = ox; ion.vy[q] = oy; ion.vz[q] = oz;
            }
            const int ne = el.cnt[cell];
            for (int k = 0; k < ne; k++) {
                int colltype = 0;
                float R1 = 0.f;
                for (int jj = 0; jj < c.mcc_n; jj++) {
                    R1 = u_test((uint32_t)k, cell, step, 0u, (uint32_t)jj);
                    if (R1 < P2) { colltype = 1; break; }
                }
                if (!colltype) continue;
                hp_stream rs;
                hp_stream_init(&rs, c.seed, (uint32_t)k, (uint32_t)cell, step, 0u);
                const int target = (R1 <= P1) ? 0 : 1;
                const size_t q = (size_t)el.start[cell] + k;
                R VX = el.vx[q], VY = el.vy[q], VZ = el.vz[q];
                const R dum = VX * VX + VY * VY + VZ * VZ;
                R vel = std::sqrt(dum);
                VX /= vel; VY /= vel; VZ /= vel;
                R engy = (R)c.Escale[0] * dum;
                R rengy = 0, vel2 = 0;
                const R Esc = (R)c.Escale[0];
                auto ionize = [&](float th) {
                    colltype = 2;
                    engy -= (R)th;
                    const R u = nextu(rs);
                    rengy = (R)(10.0 * (double)m_tan(u * m_atan((R)(engy / 20.0))));
                    engy -= rengy;
                    vel = std::sqrt(std::fabs(rengy) / Esc);
                    vel2 = std::sqrt(std::fabs(engy) / Esc);
                };
                if (target == 0) {
                    const R R2 = (R)nextu(rs) * (R)c.sigv[0] / vel;
                    R SumSigma = xsec(0, engy);
                    if (R2 <= SumSigma) {
                        colltype = 0;
                        cnt_ch[0]++;
                    } else if (engy > (R)c.th[1] && R2 <= (SumSigma += xsec(1, engy))) {
                        colltype = 0;
                        engy -= (R)c.th[1];
                        vel = std::sqrt(std::fabs(engy) / Esc);
                        cnt_ch[1]++;
                    } else if (engy > (R)c.th[2] && R2 <= (SumSigma += xsec(2, engy))) {
                        colltype = 0;
                        engy -= (R)c.th[2];
                        vel = std::sqrt(std::fabs(engy) / Esc);
                        cnt_ch[2]++;
                    } else if (engy > (R)c.th[3] && R2 <= (SumSigma += xsec(3, engy))) {
                        ionize(c.th[3]);
                        cnt_ch[3]++;
                    }
                } else {
                    const R R2 = (R)nextu(rs) * (R)c.sigv[1] / vel;
                    const R SumSigma = xsec(4, engy);
                    if (engy > (R)c.th[4] && R2 <= SumSigma) {
                        ionize(c.th[4]);
                        cnt_ch[4]++;
                    }
                }
                if (colltype == 0) {
                    R a, b;
                    draw2(rs, a, b, PAIR_ANEWVEL);
                    anewvel(engy, vel, VX, VY, VZ, a, b);
                    el.vx[q] = VX; el.vy[q] = VY; el.vz[q] = VZ;
                } else if (colltype == 2) {
                    R nevx = VX, nevy = VY, nevz = VZ;
                    {
                        R a, b;
                        draw2(rs, a, b, PAIR_ANEWVEL);
                        anewvel(rengy, vel, nevx, nevy, nevz, a, b);
                    }
                    R nivx = VX, nivy = VY, nivz = VZ;
                    {
                        const int nn = (int)((c.nvel - 1) * nextu(rs));
                        R a, b;
                        draw2(rs, a, b, PAIR_MAXWELLV);
                        maxwellv(nivx, nivy, nivz, (R)c.vsave[nn], bvel, a, b);
                    }
                    {
                        R a, b;
                        draw2(rs, a, b, PAIR_ANEWVEL);
                        anewvel(engy, vel2, VX, VY, VZ, a, b);
                    }
                    el.vx[q] = VX; el.vy[q] = VY; el.vz[q] = VZ;
                    const R px = el.x[q], py = el.y[q];
                    R e5[5] = {px, py, nevx, nevy, nevz};
                    R i5[5] = {px, py, nivx, nivy, nivz};
                    enew[cell].insert(enew[cell].end(), e5, e5 + 5);
                    inew[cell].insert(inew[cell].end(), i5, i5 + 5);
                }
            }
            for (int ch = 0; ch < 7; ch++) mcc_count[(size_t)cell * 8 + ch] += cnt_ch[ch];
        });
        auto append = [&](Sp &p, std::vector<std::vector<R>> &add) {
            std::vector<R> nx, ny, nvx, nvy, nvz;
            for (int cell = 0; cell < C; cell++) {
                for (int q = p.start[cell]; q < p.start[cell + 1]; q++) {
                    nx.push_back(p.x[q]); ny.push_back(p.y[q]); nvx.push_back(p.vx[q]); nvy.push_back(p.vy[q]);
                    nvz.push_back(p.vz[q]);
                }
                const std::vector<R> &a = add[cell];
                for (size_t k = 0; k < a.size(); k += 5) {
                    nx.push_back(a[k]); ny.push_back(a[k + 1]); nvx.push_back(a[k + 2]); nvy.push_back(a[k + 3]);
                    nvz.push_back(a[k + 4]);
                }
                p.cnt[cell] += (int)(a.size() / 5);
            }
            p.x.swap(nx); p.y.swap(ny); p.vx.swap(nvx); p.vy.swap(nvy); p.vz.swap(nvz);
            p.restart();
        };
        append(el, enew);
        append(ion, inew);
    }

    // ------------------------------------------------------------ Deposit
    // Smooth_121_x/_y (src/cuda_Deposit.cu:105-170) in double, as the kernels
    double smooth_121(const std::vector<double> &v, size_t o, int id, int at, int last, int step) const {
        const int *dr = c.dens_region;
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
        const double l = a1 ? (double)a1 * v[o + (size_t)(id - step)] : 0.0;
        const double r = a3 ? (double)a3 * v[o + (size_t)(id + step)] : 0.0;
        return 0.25 * (l + (double)(2 * a2) * v[o + (size_t)id] + r);
    }

    void deposit(bool smooth) override {
        for (int s = 0; s < c.nsp; s++) {
            Sp &p = sp[s];
            par_for(C, [&](int cell) {
                R lane[4][32];
                for (int q = 0; q < 4; q++)
                    for (int l = 0; l < 32; l++) lane[q][l] = 0;
                const int n = p.cnt[cell];
                for (int k = 0; k < n; k++) {
                    const int l = k & 31;
                    const R lx = p.x[(size_t)p.start[cell] + k], ly = p.y[(size_t)p.start[cell] + k];
                    lane[0][l] += (1 - lx) * (1 - ly);
                    lane[1][l] += (1 - lx) * ly;
                    lane[2][l] += lx * (1 - ly);
                    lane[3][l] += lx * ly;
                }
                for (int q = 0; q < 4; q++) {
                    double v[32];
                    for (int l = 0; l < 32; l++) v[l] = (double)lane[q][l];
                    cw[s][q][cell] = warp_tree(v);
                }
            });
        }
        for (int n = 0; n < G; n++) {
            const int i = n / c.ngy, j = n - i * c.ngy, ncy = c.ncy;
            for (int s = 0; s < c.nsp; s++) {
                double d = 0.0;
                if (i < c.ncx && j < ncy) d += cw[s][0][i * ncy + j];
                if (i < c.ncx && j > 0) d += cw[s][1][i * ncy + j - 1];
                if (i > 0 && j < ncy) d += cw[s][2][(i - 1) * ncy + j];
                if (i > 0 && j > 0) d += cw[s][3][(i - 1) * ncy + j - 1];
                d *= (double)c.dep_factor[n];
                den[(size_t)s * G + n] = d;
            }
        }
        if (smooth && c.n_smt > 0) {
            std::vector<double> smt(den.size());
            for (int pass = 0; pass < c.n_smt; pass++) {
                for (int s = 0; s < c.nsp; s++)
                    for (int n = 0; n < G; n++)
                        smt[(size_t)s * G + n] = smooth_121(den, (size_t)s * G, n, n / c.ngy, c.ngx - 1, c.ngy);
                for (int s = 0; s < c.nsp; s++)
                    for (int n = 0; n < G; n++)
                        den[(size_t)s * G + n] = smooth_121(smt, (size_t)s * G, n, n % c.ngy, c.ngy - 1, 1);
            }
        }
        for (int n = 0; n < G; n++) {
            double sum = 0.0;
            for (int s = 0; s < c.nsp; s++) sum += den[(size_t)s * G + n] * (double)c.q_density[s];
            if (c.n_diel > 0) sum += surface_charge(n);
            const double src = sum / 8.8542e-12;
            source[n] = src;
            b64[n] = c.st[2 * G + n] != 0.0f ? src : 0.0;
        }
    }

    // ------------------------------------------------------------ Field
    float spmv_f(const float *st, int n, const std::vector<float> &v) const {
        float out = 0.0f;
        const float cw_ = st[n], cs = st[G + n], cc = st[2 * G + n], cn = st[3 * G + n], ce = st[4 * G + n];
        if (cw_ != 0.0f) out += cw_ * v[n - c.ngy];
        if (cs != 0.0f) out += cs * v[n - 1];
        out += cc * v[n];
        if (cn != 0.0f) out += cn * v[n + 1];
        if (ce != 0.0f) out += ce * v[n + c.ngy];
        return out;
    }
    double spmv_d(const float *st, int n, const std::vector<double> &v) const {
        double out = 0.0;
        const float cw_ = st[n], cs = st[G + n], cc = st[2 * G + n], cn = st[3 * G + n], ce = st[4 * G + n];
        if (cw_ != 0.0f) out += (double)cw_ * v[n - c.ngy];
        if (cs != 0.0f) out += (double)cs * v[n - 1];
        out += (double)cc * v[n];
        if (cn != 0.0f) out += (double)cn * v[n + 1];
        if (ce != 0.0f) out += (double)ce * v[n + c.ngy];
        return out;
    }

    // Cluster reduction of the GPU PCG: thread partials (nodes lo+t, lo+t+T, ...),
    // warp trees, warps in order, CTAs in rank order.  f(n, acc) adds node n.
    template <class F> double cluster_reduce(F f) const {
        const int CS = c.pcg_cluster, T = c.pcg_block, nw = T / 32;
        const int per = (G + CS - 1) / CS;
        double total = 0.0;
        for (int r = 0; r < CS; r++) {
            const int lo = r * per, hi = std::min(G, lo + per);
            double block = 0.0;
            for (int w = 0; w < nw; w++) {
                double v[32];
                for (int l = 0; l < 32; l++) {
                    double part = 0.0;
                    for (int n = lo + w * 32 + l; n < hi; n += T) f(n, part);
                    v[l] = part;
                }
                block += warp_tree(v);
            }
            total += block;
        }
        return total;
    }

    // C[m][n] = sum_k A[m][k] B[k][n], accumulated in k order from zero with
    // separate multiply and add roundings, as the GPU's grouped GEMM
    static void gemm(const float *A, const float *B, float *Cm, int M, int N, int K) {
        std::vector<float> acc((size_t)N);
        for (int m = 0; m < M; m++) {
            std::fill(acc.begin(), acc.end(), 0.0f);
            for (int k = 0; k < K; k++) {
                const float a = A[(size_t)m * K + k];
                const float *b = B + (size_t)k * N;
                for (int n = 0; n < N; n++) acc[n] = acc[n] + a * b[n];
            }
            std::copy(acc.begin(), acc.end(), Cm + (size_t)m * N);
        }
    }

    void field_fast() {
        const float *st = c.st;
        const int nx = c.fs_nx, ny = c.fs_ny;
        const size_t nxy = (size_t)nx * ny;
        std::vector<float> X(nxy), A1(nxy), Y(nxy), E(nxy);
        for (int pass = 0; pass < c.fs_passes; pass++) {
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    const int node = (c.fs_i0 + i) * c.ngy + (c.fs_j0 + j);
                    const double r64 = b64[node] - spmv_d(st, node, x64);
                    X[(size_t)j * nx + i] = (float)(r64 * (double)c.row_scale[node]);
                }
            gemm(X.data(), c.fs_V, A1.data(), ny, nx, nx);
            gemm(c.fs_Wt, A1.data(), Y.data(), ny, nx, ny);
            for (size_t k = 0; k < nxy; k++) Y[k] = Y[k] * c.fs_inv[k];
            gemm(Y.data(), c.fs_Vt, A1.data(), ny, nx, nx);
            gemm(c.fs_W, A1.data(), E.data(), ny, nx, ny);
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) x64[(size_t)(c.fs_i0 + i) * c.ngy + (c.fs_j0 + j)] += (double)E[(size_t)j * nx + i];
        }
        for (int n = 0; n < G; n++) phi_p[n] = st[2 * G + n] != 0.0f ? (float)x64[n] : 0.0f;
        pcg_iters[0] = c.fs_passes;
        pcg_iters[1] = c.fs_passes;
    }

    void field_f32() {
        if (c.field_mode == 2) {
            field_fast();
            return;
        }
        const float *st = c.st;
        std::vector<float> x = pf_x, r(G, 0.0f), p(G, 0.0f), ap(G, 0.0f);
        int iters = 0, outer = 0;
        const int maxit = c.pcg_max_iter;
        if (c.field_mode == 0) {
            for (int n = 0; n < G; n++) {
                const float cc = st[2 * G + n];
                if (cc == 0.0f) continue;
                const float ax = spmv_f(st, n, x);
                const float rr = -1.0f * ax + (float)b64[n];
                r[n] = rr;
                p[n] = (1 / cc) * rr;
            }
            double rz = cluster_reduce([&](int n, double &a) {
                const float cc = st[2 * G + n];
                if (cc != 0.0f) a += (double)(r[n] * ((1 / cc) * r[n]));
            });
            int iter = 1;
            while (rz > (double)c.pcg_tol2 && iter <= maxit) {
                for (int n = 0; n < G; n++)
                    if (st[2 * G + n] != 0.0f) ap[n] = spmv_f(st, n, p);
                const double pap = cluster_reduce([&](int n, double &a) {
                    if (st[2 * G + n] != 0.0f) a += (double)(p[n] * ap[n]);
                });
                const float alpha = (pap != 0.0) ? (float)rz / (float)pap : 0.0f;
                for (int n = 0; n < G; n++) {
                    const float cc = st[2 * G + n];
                    if (cc == 0.0f) continue;
                    x[n] = alpha * p[n] + x[n];
                    r[n] = -alpha * ap[n] + r[n];
                }
                const double rznew = cluster_reduce([&](int n, double &a) {
                    const float cc = st[2 * G + n];
                    if (cc != 0.0f) a += (double)(r[n] * ((1 / cc) * r[n]));
                });
                if (!(rznew == rznew) || std::isinf(rznew)) break;
                const float beta = (rz != 0.0) ? (float)rznew / (float)rz : 0.0f;
                for (int n = 0; n < G; n++) {
                    const float cc = st[2 * G + n];
                    if (cc != 0.0f) p[n] = beta * p[n] + (1 / cc) * r[n];
                }
                rz = rznew;
                iter++;
            }
            iters = iter;
            pf_x = x;
            for (int n = 0; n < G; n++) phi_p[n] = st[2 * G + n] != 0.0f ? x[n] : 0.0f;
        } else {
            const float *ss = c.st_sym;
            double bb = cluster_reduce([&](int n, double &a) { a += b64[n] * b64[n]; });
            const double target = c.pcg_rtol * c.pcg_rtol * bb;
            for (outer = 0; outer < 12; outer++) {
                std::vector<double> r64(G, 0.0);
                for (int n = 0; n < G; n++) {
                    const float cc = st[2 * G + n];
                    if (cc == 0.0f) continue;
                    r64[n] = b64[n] - spmv_d(st, n, x64);
                    const float rs = (float)(r64[n] * (double)c.row_scale[n]);
                    r[n] = rs;
                    x[n] = 0.0f;
                    p[n] = (1 / ss[2 * G + n]) * rs;
                }
                const double rr = cluster_reduce([&](int n, double &a) {
                    if (st[2 * G + n] != 0.0f) a += r64[n] * r64[n];
                });
                double rz = cluster_reduce([&](int n, double &a) {
                    if (st[2 * G + n] != 0.0f) a += (double)(r[n] * ((1 / ss[2 * G + n]) * r[n]));
                });
                if (!(rr == rr) || rr <= target || bb == 0.0) break;
                const double rz0 = rz;
                int iter = 0;
                while (rz > 1e-10 * rz0 && iter < maxit) {
                    for (int n = 0; n < G; n++)
                        if (ss[2 * G + n] != 0.0f) ap[n] = spmv_f(ss, n, p);
                    const double pap = cluster_reduce([&](int n, double &a) {
                        if (ss[2 * G + n] != 0.0f) a += (double)(p[n] * ap[n]);
                    });
                    const float alpha = (pap != 0.0) ? (float)(rz / pap) : 0.0f;
                    for (int n = 0; n < G; n++) {
                        if (ss[2 * G + n] == 0.0f) continue;
                        x[n] = alpha * p[n] + x[n];
                        r[n] = -alpha * ap[n] + r[n];
                    }
                    const double rznew = cluster_reduce([&](int n, double &a) {
                        const float cc = ss[2 * G + n];
                        if (cc != 0.0f) a += (double)(r[n] * ((1 / cc) * r[n]));
                    });
                    const float beta = (rz != 0.0) ? (float)(rznew / rz) : 0.0f;
                    for (int n = 0; n < G; n++) {
                        const float cc = ss[2 * G + n];
                        if (cc != 0.0f) p[n] = beta * p[n] + (1 / cc) * r[n];
                    }
                    rz = rznew;
                    iter++;
                }
                iters += iter;
                for (int n = 0; n < G; n++)
                    if (st[2 * G + n] != 0.0f) x64[n] += (double)x[n];
            }
            for (int n = 0; n < G; n++) phi_p[n] = st[2 * G + n] != 0.0f ? (float)x64[n] : 0.0f;
        }
        pcg_iters[0] = iters;
        pcg_iters[1] = outer;
    }

    // FP64 reference solve: Jacobi-PCG on the symmetric form D^-1 A, in double,
    // warm-started, to ||r|| <= 1e-11 ||b||.
    void field_f64() {
        const float *st = c.st, *ss = c.st_sym;
        std::vector<double> r(G, 0.0), p(G, 0.0), ap(G, 0.0), z(G, 0.0);
        double bb = 0.0;
        for (int n = 0; n < G; n++) bb += b64[n] * b64[n];
        double rz = 0.0, rr = 0.0;
        for (int n = 0; n < G; n++) {
            if (st[2 * G + n] == 0.0f) continue;
            const double res = b64[n] - spmv_d(st, n, x64);
            rr += res * res;
            r[n] = res * (double)c.row_scale[n];
            z[n] = r[n] / (double)ss[2 * G + n];
            p[n] = z[n];
            rz += r[n] * z[n];
        }
        int it = 0;
        const double tol2 = 1e-22 * bb;
        while (rr > tol2 && bb > 0 && it < 200000) {
            double pap = 0.0;
            for (int n = 0; n < G; n++) {
                if (ss[2 * G + n] == 0.0f) continue;
                ap[n] = spmv_d(ss, n, p);
                pap += p[n] * ap[n];
            }
            const double alpha = rz / pap;
            double rznew = 0.0;
            for (int n = 0; n < G; n++) {
                if (ss[2 * G + n] == 0.0f) continue;
                x64[n] += alpha * p[n];
                r[n] -= alpha * ap[n];
                z[n] = r[n] / (double)ss[2 * G + n];
                rznew += r[n] * z[n];
            }
            const double beta = rznew / rz;
            for (int n = 0; n < G; n++)
                if (ss[2 * G + n] != 0.0f) p[n] = z[n] + beta * p[n];
            rz = rznew;
            it++;
            if ((it & 31) == 0) { // true residual of the unscaled system
                rr = 0.0;
                for (int n = 0; n < G; n++) {
                    if (st[2 * G + n] == 0.0f) continue;
                    const double res = b64[n] - spmv_d(st, n, x64);
                    rr += res * res;
                }
            }
        }
        pcg_iters[0] = it;
        pcg_iters[1] = 1;
        for (int n = 0; n < G; n++) phi_p[n] = st[2 * G + n] != 0.0f ? (R)x64[n] : (R)0;
    }

    R cond_sigma(int n, int eT, int eL, int eD, int eX, int pL, int pR, int pD, int pU) const {
        const int b = c.boundary[n], f = c.face[n];
        if (b == 2) return c.n_diel > 0 ? (R)sigma[n] : (R)0; // Sigma left by SumSource
        if (!((b == 3 || b == 1) && f != 8)) return 0;
        R SumSig = 0;
        for (int s = 0; s < c.nsp; s++) SumSig += (R)den[(size_t)s * G + n] * (R)c.q_density[s];
        const R *P = phi_p.data();
        auto E = [&](int k) { return (R)c.eps[k]; };
        const R hdx = c.hdx, hdy = c.hdy, idxy = c.idxy;
        switch (f) {
        case 2: return hdy * (E(eT) + E(eL)) * (P[n] - P[pU]) - hdx * SumSig;
        case 3: return hdy * (E(eD) + E(eX)) * (P[n] - P[pD]) - hdx * SumSig;
        case 0: return hdx * (E(eL) + E(eX)) * (P[n] - P[pL]) - hdy * SumSig;
        case 1: return hdx * (E(eT) + E(eD)) * (P[n] - P[pR]) - hdy * SumSig;
        case 4: return hdy * (E(eT) + E(eL)) * (P[n] - P[pU]) + hdx * (E(eL) + E(eX)) * (P[n] - P[pL]) - idxy * SumSig;
        case 5: return hdy * (E(eT) + E(eL)) * (P[n] - P[pU]) + hdx * (E(eT) + E(eD)) * (P[n] - P[pR]) - idxy * SumSig;
        case 6: return hdy * (E(eD) + E(eX)) * (P[n] - P[pD]) + hdx * (E(eL) + E(eX)) * (P[n] - P[pL]) - idxy * SumSig;
        case 7: return hdy * (E(eD) + E(eX)) * (P[n] - P[pD]) + hdx * (E(eT) + E(eD)) * (P[n] - P[pR]) - idxy * SumSig;
        default: return 0;
        }
    }

    void field(int64_t tstep) override {
        if (precision == 32) field_f32();
        else field_f64();
        // potential assembly
        const double time = (double)tstep * (double)c.dt;
        std::vector<R> vk(c.cond_numr, 0);
        for (int k = 0; k < c.cond_numr; k++) {
            R v = 0;
            if (c.efield_flag[k])
                for (int q = 0; q < c.src_num; q++)
                    if (c.src_mid[q] == k + 1)
                        v = (R)((double)v + ((double)c.src_dc[q] +
                                             (double)src_amp[q] * std::sin((double)c.src_2pif[q] * time + (double)c.src_rphase[q])));
            vk[k] = v;
        }
        if (c.external) circuit(vk);
        for (int n = 0; n < G; n++) {
            R tot = 0;
            for (int k = 0; k < c.cond_numr; k++) tot += vk[k] * (R)c.lap[(size_t)k * G + n];
            tot += 1 * phi_p[n];
            phi[n] = tot;
        }
        // E at nodes
        const int ngx = c.ngx, ngy = c.ngy;
        const R idx = c.idx, idy = c.idy, hdx = c.hdx, hdy = c.hdy, dx = c.dx, dy = c.dy;
        const R half = (R)0.5f;
        for (int n = 0; n < G; n++) {
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
            const R *P = phi.data();
            auto E = [&](int k) { return (R)c.eps[k]; };
            const int f = c.face[n], b = c.boundary[n];
            R ex, ey;
            bool write = true;
            // Cond_Sigma's Sigma at conductor and Dirichlet face nodes (the power controller's input)
            if ((c.n_power > 0 || c.n_diel > 0 || c.external) && (b == 3 || b == 1) && f != 8)
                sigma[n] = (double)cond_sigma(n, eT, eL, eD, eX, pL, pR, pD, pU);
            if (f == 0) {
                if (b == 3 || b == 2 || b == 1) {
                    ex = (R)-2.0f * cond_sigma(n, eT, eL, eD, eX, pL, pR, pD, pU) / (E(eL) + E(eX));
                    ey = 0;
                } else if (b == 4 || b >= 100) {
                    ex = idx * (P[pL] - P[n]);
                    ey = hdy * (P[pD] - P[pU]);
                } else {
                    ex = half * (E(eT) + E(eD)) * (P[pR] - P[n]) * idx;
                    ex -= (half * dx / dy) * E(eT) * (P[n] - P[pU]) * idy;
                    ex -= (half * dx / dy) * E(eD) * (P[n] - P[pD]) * idy;
                    ex /= -half * (E(eL) + E(eX));
                    ey = hdy * (P[pD] - P[pU]);
                }
            } else if (f == 1) {
                if (b == 3 || b == 2 || b == 1) {
                    ex = (R)2.0f * cond_sigma(n, eT, eL, eD, eX, pL, pR, pD, pU) / (E(eT) + E(eD));
                    ey = 0;
                } else if (b == 4 || b >= 100) {
                    ex = idx * (P[n] - P[pR]);
                    ey = hdy * (P[pD] - P[pU]);
                } else {
                    ex = half * (E(eL) + E(eX)) * (P[pL] - P[n]) * idx;
                    ex -= (half * dx / dy) * E(eL) * (P[n] - P[pU]) * idy;
                    ex -= (half * dx / dy) * E(eX) * (P[n] - P[pD]) * idy;
                    ex /= half * (E(eT) + E(eD));
                    ey = hdy * (P[pD] - P[pU]);
                }
            } else if (f == 2) {
                if (b == 3 || b == 2 || b == 1) {
                    ex = 0;
                    ey = (R)2.0f * cond_sigma(n, eT, eL, eD, eX, pL, pR, pD, pU) / (E(eT) + E(eL));
                } else if (b == 4 || b >= 100) {
                    ex = hdx * (P[pL] - P[pR]);
                    ey = idy * (P[n] - P[pU]);
                } else {
                    ex = hdx * (P[pL] - P[pR]);
                    ey = half * (E(eD) + E(eX)) * (P[pD] - P[n]) * idy;
                    ey -= (half * dy / dx) * E(eD) * (P[n] - P[pR]) * idx;
                    ey -= (half * dy / dx) * E(eX) * (P[n] - P[pL]) * idx;
                    ey /= half * (E(eT) + E(eL));
                }
            } else if (f == 3) {
                if (b == 3 || b == 2 || b == 1) {
                    ex = 0;
                    ey = (R)-2.0f * cond_sigma(n, eT, eL, eD, eX, pL, pR, pD, pU) / (E(eD) + E(eX));
                } else if (b == 4 || b >= 100) {
                    ex = hdx * (P[pL] - P[pR]);
                    ey = idy * (P[pD] - P[n]);
                } else {
                    ex = hdx * (P[pL] - P[pR]);
                    ey = half * (E(eT) + E(eL)) * (P[pU] - P[n]) * idy;
                    ey -= (half * dy / dx) * E(eT) * (P[n] - P[pR]) * idx;
                    ey -= (half * dy / dx) * E(eL) * (P[n] - P[pL]) * idx;
                    ey /= -half * (E(eD) + E(eX));
                }
            } else if (f >= 4 && f <= 7) {
                const bool solid = (b == 3 || b == 1 || b == 4);
                if (!solid) { ex = hdx * (P[pL] - P[pR]); ey = hdy * (P[pD] - P[pU]); }
                else if (f == 4) { ex = idx * (P[pL] - P[n]); ey = idy * (P[n] - P[pU]); }
                else if (f == 5) { ex = idx * (P[n] - P[pR]); ey = idy * (P[n] - P[pU]); }
                else if (f == 6) { ex = idx * (P[pL] - P[n]); ey = idy * (P[pD] - P[n]); }
                else { ex = idx * (P[n] - P[pR]); ey = idy * (P[pD] - P[n]); }
            } else if (b == 2) {
                if (x == 0 || x == ngx - 1) { ex = 0; ey = hdy * (P[pD] - P[pU]); }
                else if (y == 0 || y == ngy - 1) { ex = hdx * (P[pL] - P[pR]); ey = 0; }
                else { write = false; ex = ey = 0; }
            } else {
                ex = hdx * (P[pL] - P[pR]);
                ey = hdy * (P[pD] - P[pU]);
            }
            if (write) { Ex[n] = ex; Ey[n] = ey; }
        }
    }

    // Efield_cuda's circuit (src/cuda_Field.cu:43-81) as the kernel computes
    // it: the surface charge of this step's Poisson part per conductor
    // (Cond_Sigma on phi_p x Area, FP64, list entry q added to partial q % 256,
    // the partials reduced by halving, rounded to float), then the circuit
    // solve of hp_circuit.h; vk becomes the conductors' potentials.
    template <class V> void circuit(V &vk) {
        const int nc = c.cond_numr, ngx = c.ngx, ngy = c.ngy;
        std::vector<double> part((size_t)256 * 8, 0.0);
        for (size_t q = 0; q < cond_list.size(); q++) {
            const int n = cond_list[q];
            const int b = c.boundary[n], f = c.face[n];
            double sg = 0.0;
            if ((b == 3 || b == 1) && f != 8) {
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
                sg = (double)(float)cond_sigma(n, eT, eL, eD, eX, pL, pR, pD, pU);
            }
            part[(q % 256) * 8 + (c.cond_id[n] - 1)] += sg * (double)c.area[n];
        }
        for (int h = 128; h > 0; h >>= 1)
            for (int t = 0; t < h; t++)
                for (int k = 0; k < nc; k++) part[(size_t)t * 8 + k] += part[(size_t)(t + h) * 8 + k];
        float vt[HP_CIRCUIT_MAX], surf[HP_CIRCUIT_MAX], pois[HP_CIRCUIT_MAX];
        for (int i = 0; i < nc; i++) {
            vt[i] = (float)vk[i];
            surf[i] = (float)pw.surf[i];
            pois[i] = (float)part[i];
        }
        hp_circuit_step(nc, c.cc_a, c.lap_sig, vt, circ.qconv, surf, pois, circ.q, circ.phi, circ.pois, c.circuit_mode);
        for (int i = 0; i < nc; i++) vk[i] = circ.phi[i];
    }

    // The reference's power controller (src/cuda_Diagnostic.cu:365-420) as
    // the kernel computes it: surface charge per conductor in FP64, list entry
    // q added to partial q % 256, the 256 partials reduced by halving.
    void power(int64_t tstep) override {
        if (c.n_power <= 0 && !c.external) return;
        const int nc = c.cond_numr;
        std::vector<double> part((size_t)256 * 8, 0.0);
        for (size_t q = 0; q < cond_list.size(); q++) {
            const int n = cond_list[q];
            part[(q % 256) * 8 + (c.cond_id[n] - 1)] += sigma[n] * (double)c.area[n];
        }
        for (int h = 128; h > 0; h >>= 1)
            for (int t = 0; t < h; t++)
                for (int k = 0; k < nc; k++) part[(size_t)t * 8 + k] += part[(size_t)(t + h) * 8 + k];
        const double time = (double)tstep * (double)c.dt;
        for (int i = 0; i < nc; i++) {
            pw.old2[i] = pw.old[i];
            pw.old[i] = pw.surf[i];
            pw.surf[i] = part[i];
            float cond_current = 0.0f, q_conv = 0.0f;
            for (int s = 0; s < c.nsp; s++) {
                unsigned &cnt = cond_step[(size_t)s * nc + i];
                cond_current += c.q_density[s] * (float)cnt / c.dt;
                q_conv -= c.q_density[s] * (float)cnt; // the circuit's convective charge
                cnt = 0;
            }
            if (c.external) circ.qconv[i] = q_conv;
            const float dis_current = (float)(0.5 * (3.0 * pw.surf[i] - 4.0 * pw.old[i] + pw.old2[i]) / (double)c.dt);
            const float current = dis_current - cond_current;
            if (c.cond_src_num[i] != 1) continue;
            float phi_now = 0.0f; // V_t: the conductor's voltage at this step (float, as the kernels)
            if (c.efield_flag[i])
                for (int q = 0; q < c.src_num; q++)
                    if (c.src_mid[q] == i + 1)
                        phi_now = (float)((double)phi_now + ((double)c.src_dc[q] +
                                          (double)src_amp[q] * std::sin((double)c.src_2pif[q] * time + (double)c.src_rphase[q])));
            pw.power[i] += phi_now * current;
            pw.count[i]++;
            if (pw.count[i] != c.pd_intv) continue;
            pw.power[i] /= (float)pw.count[i];
            pw.count[i] = 0;
            const int q = c.cond_power_id[i];
            if (pw.power[i] > 0) phi_now = src_amp[q] * hp_powf(std::fabs(c.src_power[q] / pw.power[i]), 0.2f);
            if (pw.power_init) {
                if (phi_now > (1.0f + c.pd_ratio) * src_amp[q]) src_amp[q] = (float)((double)src_amp[q] * 1.05);
                else src_amp[q] = phi_now;
            }
            pw.power[i] = 0.0f;
            pw.power_init++;
        }
    }

    void accumulate() override {
        for (size_t k = 0; k < den.size(); k++) ave_den[k] += den[k];
        for (int n = 0; n < G; n++) ave_phi[n] += (double)phi[n];
        for (int n = 0; n < G; n++) ave_src[n] += source[n];
        for (int n = 0; n < G; n++) ave_ex[n] += (double)Ex[n];
        for (int n = 0; n < G; n++) ave_ey[n] += (double)Ey[n];
        ave_count++;
    }
    // electron energy histogram (the library's EEDF: 200 bins of 0.25 eV and
    // an overflow bin), E = Escale |v|^2 as the MCC computes it
    void eedf_sample() override {
        const Sp &e = sp[0];
        const R Esc = (R)c.Escale[0], top = (R)(200 * 0.25f), inv = (R)(1.0f / 0.25f);
        for (size_t k = 0; k < e.vx.size(); k++) {
            const R v = e.vx[k] * e.vx[k] + e.vy[k] * e.vy[k] + e.vz[k] * e.vz[k];
            const R en = Esc * v;
            const int b = en < top ? (int)(en * inv) : 200;
            eedf[(size_t)b]++;
        }
    }
};

} // namespace

struct or_sim {
    SimBase *impl;
};

extern "C" {

or_sim *or_sim_new(const or_case *c, int precision) {
    or_sim *s = new or_sim;
    if (precision == 64) s->impl = new Sim<double>(*c, 64);
    else s->impl = new Sim<float>(*c, 32);
    return s;
}
void or_sim_free(or_sim *s) {
    if (!s) return;
    delete s->impl;
    delete s;
}
void or_set_particles(or_sim *s, int isp, const int *counts, const float *x, const float *y, const float *vx,
                      const float *vy, const float *vz) {
    s->impl->set_particles(isp, counts, x, y, vx, vy, vz);
}
size_t or_num_particles(or_sim *s, int isp) { return s->impl->num(isp); }
void or_get_particles(or_sim *s, int isp, int *counts, float *x, float *y, float *vx, float *vy, float *vz) {
    s->impl->get_particles(isp, counts, x, y, vx, vy, vz);
}
void or_get_particles_d(or_sim *s, int isp, int *counts, double *x, double *y, double *vx, double *vy, double *vz) {
    s->impl->get_particles_d(isp, counts, x, y, vx, vy, vz);
}
size_t or_num_movers(or_sim *s, int isp) { return s->impl->num_movers(isp); }
void or_get_movers(or_sim *s, int isp, int *counts, float *x, float *y, float *vx, float *vy, float *vz,
                   int8_t *codes) {
    s->impl->get_movers(isp, counts, x, y, vx, vy, vz, codes);
}
void or_get_grid(or_sim *s, int which, void *out) { s->impl->get_grid(which, out); }
void or_set_grid(or_sim *s, int which, const void *in) { s->impl->set_grid(which, in); }
void or_math(int fn, const float *x, const float *y, float *out, int n) {
    for (int k = 0; k < n; k++) {
        float s_, c_;
        switch (fn) {
        case 0: out[k] = hp_expf(x[k]); break;
        case 1: out[k] = hp_logf(x[k]); break;
        case 2: out[k] = hp_log10f(x[k]); break;
        case 3: out[k] = hp_powf(x[k], y[k]); break;
        case 4: hp_sincos_turns(x[k], &s_, &c_); out[k] = s_; break;
        case 5: hp_sincos_turns(x[k], &s_, &c_); out[k] = c_; break;
        case 6: out[k] = hp_tanf_q1(x[k]); break;
        default: out[k] = hp_atanf(x[k]); break;
        }
    }
}
int or_walk_bound_hit(or_sim *s) { return s->impl->walk_bound_hit ? 1 : 0; }
int or_far_max(or_sim *s) { return s->impl->far_max(); }
void or_get_counters(or_sim *s, float *cond_charge, unsigned *mcc_count, int *pcg_iters) {
    SimBase *b = s->impl;
    if (cond_charge) std::memcpy(cond_charge, b->cond_charge.data(), b->cond_charge.size() * 4);
    if (mcc_count) std::memcpy(mcc_count, b->mcc_count.data(), b->mcc_count.size() * 4);
    if (pcg_iters) { pcg_iters[0] = b->pcg_iters[0]; pcg_iters[1] = b->pcg_iters[1]; }
}
void or_set_script(or_sim *s, int flags, const float *u, const int64_t *start, int nkeys) {
    SimBase *b = s->impl;
    b->script_overrun = 0;
    if (!u || nkeys <= 0) {
        b->script = SimBase::Script();
        return;
    }
    b->script.on = true;
    b->script.by_species = flags & 1;
    b->script.pair_rl = (flags >> 1) & 7;
    b->script.start.assign(start, start + nkeys + 1);
    b->script.u.assign(u, u + start[nkeys]);
    b->script.pos.assign((size_t)nkeys, 0);
}
long long or_script_overrun(or_sim *s) { return s->impl->script_overrun.load(); }
void or_xsec(or_sim *s, int ch, const float *engy, float *out, int n) { s->impl->xsec_n(ch, engy, out, n); }
void or_kinematics(or_sim *s, int kind, const float *in, float *out, int n) { s->impl->kinematics(kind, in, out, n); }
int or_collide_oxy(or_sim *s, int isp, int t, const float *v, float bv1, float bv2, const float *u, int nu,
                   int pair_rl, int *ch, int *keep, float *vout, int *bsp, float *bv, int *kill) {
    return s->impl->collide_oxy(isp, t, v, bv1, bv2, u, nu, pair_rl, ch, keep, vout, bsp, bv, kill);
}
void or_fluid_sources(int gas, int n, int tnrct, int nfsp, float *R, const float *fden, const float *eden,
                      const float *bd1, const float *bd2, const float *rr, float *S) {
    std::vector<float> r(96), rrv(96, 0.0f);
    std::copy(rr, rr + std::min(tnrct, 96), rrv.begin());
    for (int g = 0; g < n; g++) {
        std::fill(r.begin(), r.end(), 0.0f);
        std::copy(R + (size_t)g * tnrct, R + (size_t)g * tnrct + std::min(tnrct, 96), r.begin());
        float nn[5] = {0, 0, 0, 0, 0}, out[5] = {0, 0, 0, 0, 0};
        for (int f = 0; f < nfsp && f < 5; f++) nn[f] = fden[(size_t)f * n + g];
        hp_fluid_sources(gas, r.data(), nn, bd1[g], bd2[g], eden[g], rrv.data(), out);
        std::copy(r.begin(), r.begin() + std::min(tnrct, 96), R + (size_t)g * tnrct);
        for (int f = 0; f < nfsp && f < 5; f++) S[(size_t)f * n + g] = out[f];
    }
}
void or_fluid_sweeps(or_sim *s, int nsteps) {
    for (int k = 0; k < nsteps; k++) s->impl->fluid_sweeps();
}
void or_field(or_sim *s, int64_t tstep) { s->impl->field(tstep); }
void or_move(or_sim *s) { s->impl->move(); }
void or_sort(or_sim *s) { s->impl->sort(); }
void or_mcc(or_sim *s, int64_t tstep) { s->impl->mcc(tstep); }
void or_deposit(or_sim *s) { s->impl->deposit(true); }
void or_deposit_basic(or_sim *s) { s->impl->deposit(false); }
void or_run(or_sim *s, int64_t tstep0, int nsteps, int accumulate) {
    for (int k = 1; k <= nsteps; k++) {
        const int64_t t = tstep0 + k;
        s->impl->field(t);
        s->impl->move();
        s->impl->sort();
        s->impl->mcc(t);
        s->impl->deposit(true);
        s->impl->fluid_step(t);
        if (accumulate) {
            s->impl->accumulate();
            const int ev = s->impl->c.eedf_every;
            if (ev > 0 && t % ev == 0) s->impl->eedf_sample();
        }
        s->impl->power(t);
    }
}
void or_get_eedf(or_sim *s, unsigned long long *h) { std::memcpy(h, s->impl->eedf.data(), 201 * 8); }
void or_get_field_averages(or_sim *s, double *ave_src, double *ave_ex, double *ave_ey) {
    SimBase *b = s->impl;
    if (ave_src) std::memcpy(ave_src, b->ave_src.data(), b->ave_src.size() * 8);
    if (ave_ex) std::memcpy(ave_ex, b->ave_ex.data(), b->ave_ex.size() * 8);
    if (ave_ey) std::memcpy(ave_ey, b->ave_ey.data(), b->ave_ey.size() * 8);
}
void or_get_averages(or_sim *s, double *ave_den, double *ave_phi, int64_t *count) {
    SimBase *b = s->impl;
    if (ave_den) std::memcpy(ave_den, b->ave_den.data(), b->ave_den.size() * 8);
    if (ave_phi) std::memcpy(ave_phi, b->ave_phi.data(), b->ave_phi.size() * 8);
    if (count) *count = b->ave_count;
}
int or_num_threads(void) { return nthreads(); }
// the circuit arithmetic of hp_circuit.h, for checking it against the
// reference's own cofactor and a transcription of Efield_cuda
void or_circuit_inverse(float *m, int n) { hp_ci_inverse(m, n); }
void or_circuit_step(int nc, const float *cc, const float *lap, const float *vt, const float *qconv,
                     const float *surf, const float *pois_new, float *q, float *phi, float *pois, int mode) {
    hp_circuit_step(nc, cc, lap, vt, qconv, surf, pois_new, q, phi, pois, mode);
}
void or_set_threads(int n) { g_threads = n; }

} // extern "C"
