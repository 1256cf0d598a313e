// checkpoint.cu -- checkpoint and resume of one case.
//
// The file starts with the reference's V000 dump (V000_DUMP,
// src/cuda_SaveDump.cu:5-106; read back by V000_LoadDUMP, src/load.c:5-120),
// field for field, so that the reference's loader and its post-processing
// read it: time, step counters, gas, every particle as (CellID, x, y, vx, vy,
// vz) with x, y in grid units, the fluid species (Conti_Flag, densities,
// sources, fluxes), (empty) history, per-node densities, background gas,
// potentials, fields and their time averages.  Quantities this library does
// not model are written as the reference's neutral values: no history
// records, MCC rates 0 (the exact per-cell tallies are in the extension).
// The dielectric surface charge goes out as the reference's float sigma per
// (species, node).
//
// An extension block follows ("HPICX003"): everything a resumed run needs to
// continue bit for bit -- the step counter that keys the Philox streams, the
// case seed, the particles as in-cell offsets in the device's cell order,
// the field solver's warm start, the charge grid and right-hand side, the
// running sums, tallies and histogram, the fluid species and their averaging
// window.  hp_case_load reads the V000 part only to check it against the
// case, then restores the extension.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.hpp"

using namespace hp;

namespace {

struct File {
    FILE *f = nullptr;
    bool ok = true;
    ~File() {
        if (f) fclose(f);
    }
    void put(const void *p, size_t n) {
        if (ok && n && fwrite(p, 1, n, f) != n) ok = false;
    }
    void get(void *p, size_t n) {
        if (ok && n && fread(p, 1, n, f) != n) ok = false;
    }
    void skip(size_t n) {
        if (ok && n && fseek(f, (long)n, SEEK_CUR) != 0) ok = false;
    }
    template <class T> void put1(T v) { put(&v, sizeof v); }
    template <class T> T get1() {
        T v{};
        get(&v, sizeof v);
        return v;
    }
    void zeros(size_t n) {
        static const char z[4096] = {};
        while (n && ok) {
            const size_t k = n < sizeof z ? n : sizeof z;
            put(z, k);
            n -= k;
        }
    }
};

const char MAGIC[8] = {'H', 'P', 'I', 'C', 'X', '0', '0', '4'};
// the extension's format version; the magic's last digits carry the same number
constexpr uint32_t EXT_VERSION = 4u;
const char TAIL[8] = {'H', 'P', 'I', 'C', 'E', 'N', 'D', '1'};
// grid fields carried by the extension, in file order
const hp_grid_field EXT_GRIDS[] = {HP_GRID_EX,         HP_GRID_EY,          HP_GRID_PHI,     HP_GRID_PHI_POIS,
                                   HP_GRID_DEN,        HP_GRID_SOURCE,      HP_GRID_PCG_X,   HP_GRID_PCG_B,
                                   HP_GRID_AVE_DEN,    HP_GRID_AVE_PHI,     HP_GRID_AVE_SOURCE, HP_GRID_AVE_EX,
                                   HP_GRID_AVE_EY,     HP_GRID_COND_CHARGE, HP_GRID_MCC_COUNT, HP_GRID_EEDF,
                                   HP_GRID_SURFACE_CHARGE, HP_GRID_SIGMA, HP_GRID_SOURCE_AC, HP_GRID_POWER_STATE,
                                   HP_GRID_FLUID_CELL_DEN, HP_GRID_FLUID_DEN, HP_GRID_FLUID_SOURCE,
                                   HP_GRID_FLUID_FLUX_X, HP_GRID_FLUID_FLUX_Y, HP_GRID_FLUID_STATE,
                                   HP_GRID_CIRCUIT};

template <class T> std::vector<T> fetch(hp_case *c, hp_grid_field f) {
    void *p = nullptr;
    size_t nb = 0;
    std::vector<T> v;
    if (hpi_grid_ptr(c, f, &p, &nb) != HP_OK || nb == 0) return v;
    v.resize(nb / sizeof(T));
    if (cudaMemcpy(v.data(), p, nb, cudaMemcpyDeviceToHost) != cudaSuccess) v.clear();
    return v;
}

struct Particles {
    std::vector<int> cnt;
    std::vector<float> a[5];
};

hp_status get_species(hp_case *c, int isp, Particles &P) {
    size_t n = 0;
    P.cnt.assign(c->s.Csize, 0);
    hp_status st = hp_get_particles(c, isp, P.cnt.data(), nullptr, nullptr, nullptr, nullptr, nullptr, 0, &n);
    if (st != HP_OK) return st;
    for (auto &v : P.a) v.resize(n ? n : 1);
    return hp_get_particles(c, isp, P.cnt.data(), P.a[0].data(), P.a[1].data(), P.a[2].data(), P.a[3].data(),
                            P.a[4].data(), n, &n);
}

// the V000 part (src/cuda_SaveDump.cu:5-106)
hp_status write_v000(hp_case *c, File &F, int64_t tstep, int64_t ave_count, const std::vector<Particles> &ps,
                     const std::vector<double> &den, const std::vector<double> &ave_den,
                     const std::vector<float> &phi, const std::vector<float> &phi_p, const std::vector<float> &ex,
                     const std::vector<float> &ey, const std::vector<double> &ave_phi,
                     const std::vector<double> &ave_src, const std::vector<double> &ave_ex,
                     const std::vector<double> &ave_ey, const std::vector<long long> &sig) {
    const Setup &s = c->s;
    const int G = s.Gsize, ngy = s.ngy, ncy = s.ncy;
    F.put1<double>((double)tstep * (double)s.dt); // t
    F.put1<int32_t>((int32_t)tstep);
    F.put1<int32_t>(0); // cstep: no continuity steps
    F.put1<int32_t>(s.main_gas);
    for (int isp = 0; isp < s.nsp; isp++) {
        const Particles &P = ps[(size_t)isp];
        F.put1<float>(s.sp[isp].np2c);
        size_t np = 0;
        for (int v : P.cnt) np += (size_t)v;
        F.put1<int32_t>((int32_t)np);
        // Copy_GCPtoHCP (src/cuda_Particle.cu:70-98): CellID is the node of the
        // cell's lower-left corner, x = XID + offset in float
        std::vector<char> buf;
        buf.reserve(24 * 65536);
        size_t q = 0;
        for (int cell = 0; cell < s.Csize; cell++) {
            const int i = cell / ncy, j = cell - i * ncy;
            const int32_t cid = i * ngy + j;
            for (int k = 0; k < P.cnt[(size_t)cell]; k++, q++) {
                const float rec[5] = {(float)i + P.a[0][q], (float)j + P.a[1][q], P.a[2][q], P.a[3][q], P.a[4][q]};
                const size_t at = buf.size();
                buf.resize(at + 24);
                std::memcpy(&buf[at], &cid, 4);
                std::memcpy(&buf[at + 4], rec, 20);
                if (buf.size() >= 24 * 65536) {
                    F.put(buf.data(), buf.size());
                    buf.clear();
                }
            }
        }
        F.put(buf.data(), buf.size());
    }
    // fluid: Conti_Flag (set from the first average on), then per fluid
    // species den and Source row by row interleaved ([ncx][ncy] each),
    // flux_x[ngx][ncy], flux_y[ncx][ngy]
    {
        const auto fden = fetch<float>(c, HP_GRID_FLUID_CELL_DEN), fsrc = fetch<float>(c, HP_GRID_FLUID_SOURCE);
        const auto fx = fetch<float>(c, HP_GRID_FLUID_FLUX_X), fy = fetch<float>(c, HP_GRID_FLUID_FLUX_Y);
        const bool on = c->h.fluid_on && tstep >= (int64_t)c->h.n_ave + 1;
        F.put1<int32_t>(on ? 1 : 0);
        const size_t C = (size_t)s.Csize, nfx = (size_t)s.ngx * ncy, nfy = (size_t)s.ncx * ngy;
        for (int f = 0; f < s.nfsp; f++) {
            for (int i = 0; i < s.ncx; i++) {
                F.put(&fden[(size_t)f * C + (size_t)i * ncy], (size_t)ncy * 4);
                F.put(&fsrc[(size_t)f * C + (size_t)i * ncy], (size_t)ncy * 4);
            }
            F.put(&fx[(size_t)f * nfx], nfx * 4);
            F.put(&fy[(size_t)f * nfy], nfy * 4);
        }
    }
    // history: hist_count 0, dHIST, no records (every array has hist_count
    // entries), then hist_ave_count 0
    F.put1<int32_t>(0);
    F.put1<int32_t>(0);
    F.put1<int32_t>(0);
    // per (species, node): den, ave_den, sigma
    {
        std::vector<float> rec((size_t)s.nsp * G * 3);
        for (size_t k = 0; k < (size_t)s.nsp * G; k++) {
            rec[3 * k] = (float)den[k];
            rec[3 * k + 1] = ave_count > 0 ? (float)(ave_den[k] / (double)ave_count) : 0.f;
            rec[3 * k + 2] = sig.empty() ? 0.f : (float)((double)sig[k] / (double)(1ll << HP_SIGMA_FRAC_BITS));
        }
        F.put(rec.data(), rec.size() * 4);
    }
    // per node: Temp, BackVel1, BackDen1, BackVel2, BackDen2, Lap_Pot, Pois_Pot, Ex, Ey
    {
        auto at = [](const std::vector<float> &v, int n) { return v.empty() ? 0.f : v[(size_t)n]; };
        std::vector<float> rec((size_t)G * 9);
        for (int n = 0; n < G; n++) {
            float *r = &rec[(size_t)n * 9];
            r[0] = at(s.node_temp, n);
            r[1] = at(s.back_vel1, n);
            r[2] = at(s.back_den1, n);
            r[3] = at(s.back_vel2, n);
            r[4] = at(s.back_den2, n);
            r[5] = phi[(size_t)n] - phi_p[(size_t)n]; // the Laplace part of the potential
            r[6] = phi_p[(size_t)n];
            r[7] = ex[(size_t)n];
            r[8] = ey[(size_t)n];
        }
        F.put(rec.data(), rec.size() * 4);
    }
    // TotPotential, ave_Potential, ave_Source, ave_Sigma, ave_Ex, ave_Ey
    F.put(phi.data(), (size_t)G * 4);
    auto put_ave = [&](const std::vector<double> &sum) {
        std::vector<float> v((size_t)G, 0.f);
        if (ave_count > 0)
            for (int n = 0; n < G; n++) v[(size_t)n] = (float)(sum[(size_t)n] / (double)ave_count);
        F.put(v.data(), v.size() * 4);
    };
    put_ave(ave_phi);
    put_ave(ave_src);
    F.zeros((size_t)G * 4);
    put_ave(ave_ex);
    put_ave(ave_ey);
    // ave_MCC_rate[TnRct][Gsize]
    F.zeros((size_t)s.TnRct * G * 4);
    return F.ok ? HP_OK : (hpi::set_error("checkpoint write failed"), HP_ERR_ARG);
}

// bytes of the V000 part for this case and these particle counts
size_t v000_bytes(const Setup &s, const std::vector<int64_t> &np) {
    const size_t G = (size_t)s.Gsize;
    size_t b = 8 + 4 + 4 + 4;
    for (int isp = 0; isp < s.nsp; isp++) b += 4 + 4 + 24 * (size_t)np[(size_t)isp];
    b += 4 + (size_t)s.nfsp * 4 * ((size_t)s.ncx * s.ncy * 2 + (size_t)s.ngx * s.ncy + (size_t)s.ncx * s.ngy);
    b += 12;
    b += (size_t)s.nsp * G * 12 + G * 36 + G * 24 + (size_t)s.TnRct * G * 4;
    return b;
}

} // namespace

extern "C" {

hp_status hp_case_save(hp_case *c, const char *path) {
    if (!c || !path) return HP_ERR_ARG;
    if (c->batch) return hpi::set_error("case belongs to a batch"), HP_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess || cudaStreamSynchronize(c->last_stream) != cudaSuccess)
        return hpi::cuda_fail(cudaGetLastError(), "checkpoint sync");
    const Setup &s = c->s;
    int64_t tstep = 0, ave_count = 0;
    uint32_t status = 0;
    unsigned long long pushes[64];
    if (cudaMemcpy(&tstep, c->h.tstep, 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&ave_count, c->h.ave_count, 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&status, c->h.status, 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(pushes, c->h.pushes, sizeof pushes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return hpi::cuda_fail(cudaGetLastError(), "checkpoint read-back");
    std::vector<Particles> ps((size_t)s.nsp);
    for (int isp = 0; isp < s.nsp; isp++) {
        hp_status st = get_species(c, isp, ps[(size_t)isp]);
        if (st != HP_OK) return st;
    }
    const auto den = fetch<double>(c, HP_GRID_DEN), ave_den = fetch<double>(c, HP_GRID_AVE_DEN);
    const auto phi = fetch<float>(c, HP_GRID_PHI), phi_p = fetch<float>(c, HP_GRID_PHI_POIS);
    const auto ex = fetch<float>(c, HP_GRID_EX), ey = fetch<float>(c, HP_GRID_EY);
    const auto ave_phi = fetch<double>(c, HP_GRID_AVE_PHI), ave_src = fetch<double>(c, HP_GRID_AVE_SOURCE);
    const auto ave_ex = fetch<double>(c, HP_GRID_AVE_EX), ave_ey = fetch<double>(c, HP_GRID_AVE_EY);
    const auto sig = fetch<long long>(c, HP_GRID_SURFACE_CHARGE);
    if (phi.size() != (size_t)s.Gsize || ave_ey.size() != (size_t)s.Gsize)
        return hpi::cuda_fail(cudaGetLastError(), "checkpoint grid read-back");
    File F;
    F.f = fopen(path, "wb");
    if (!F.f) return hpi::set_error(std::string("cannot open ") + path), HP_ERR_ARG;
    hp_status st = write_v000(c, F, tstep, ave_count, ps, den, ave_den, phi, phi_p, ex, ey, ave_phi, ave_src,
                              ave_ex, ave_ey, sig);
    if (st != HP_OK) return st;
    // extension
    F.put(MAGIC, 8);
    F.put1<uint32_t>(EXT_VERSION);
    F.put1<int32_t>(s.nsp);
    F.put1<int32_t>(s.Gsize);
    F.put1<int32_t>(s.Csize);
    F.put1<int32_t>(c->opts.field_mode);
    F.put1<int64_t>(tstep);
    F.put1<uint64_t>(c->h.seed);
    F.put1<int64_t>(ave_count);
    F.put1<uint32_t>(status);
    for (int isp = 0; isp < s.nsp; isp++) {
        const Particles &P = ps[(size_t)isp];
        size_t np = 0;
        for (int v : P.cnt) np += (size_t)v;
        F.put1<int64_t>((int64_t)np);
        F.put(P.cnt.data(), P.cnt.size() * 4);
        for (int a = 0; a < 5; a++) F.put(P.a[a].data(), np * 4);
    }
    for (hp_grid_field g : EXT_GRIDS) {
        void *p = nullptr;
        size_t nb = 0;
        if ((st = hpi_grid_ptr(c, g, &p, &nb)) != HP_OK) return st;
        std::vector<char> b(nb);
        if (nb && cudaMemcpy(b.data(), p, nb, cudaMemcpyDeviceToHost) != cudaSuccess)
            return hpi::cuda_fail(cudaGetLastError(), "checkpoint grid");
        F.put1<int32_t>((int32_t)g);
        F.put1<uint64_t>((uint64_t)nb);
        F.put(b.data(), nb);
    }
    F.put(pushes, sizeof pushes);
    F.put(TAIL, 8);
    return F.ok ? HP_OK : (hpi::set_error("checkpoint write failed"), HP_ERR_ARG);
}

hp_status hp_case_load(hp_case *c, const char *path) {
    if (!c || !path) return HP_ERR_ARG;
    if (c->batch) return hpi::set_error("case belongs to a batch"), HP_ERR_ARG;
    const Setup &s = c->s;
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) return hpi::set_error(std::string("cannot open ") + path), HP_ERR_ARG;
    auto bad = [&](const std::string &why) { return hpi::set_error("checkpoint " + std::string(path) + ": " + why), HP_ERR_ARG; };
    // V000 part: check it belongs to this case, note the particle counts
    F.skip(16);
    const int32_t gas = F.get1<int32_t>();
    if (!F.ok) return bad("truncated");
    if (gas != s.main_gas) return bad("gas species do not match");
    std::vector<int64_t> np((size_t)s.nsp);
    for (int isp = 0; isp < s.nsp; isp++) {
        F.skip(4); // np2c
        np[(size_t)isp] = F.get1<int32_t>();
        if (!F.ok || np[(size_t)isp] < 0) return bad("truncated particle section");
        F.skip(24 * (size_t)np[(size_t)isp]);
    }
    if (fseek(F.f, (long)v000_bytes(s, np), SEEK_SET) != 0) return bad("truncated");
    char magic[8];
    F.get(magic, 8);
    if (!F.ok || std::memcmp(magic, MAGIC, 8) != 0)
        return bad("no " + std::string(MAGIC, 8) + " extension after the V000 part");
    const uint32_t ver = F.get1<uint32_t>();
    const int32_t nsp = F.get1<int32_t>(), G = F.get1<int32_t>(), C = F.get1<int32_t>(), fm = F.get1<int32_t>();
    if (!F.ok || ver != EXT_VERSION) return bad("unknown extension version");
    if (nsp != s.nsp || G != s.Gsize || C != s.Csize) return bad("grid or species do not match the case");
    if (fm != c->opts.field_mode) return bad("field_mode differs from the case's");
    const int64_t tstep = F.get1<int64_t>();
    const uint64_t seed = F.get1<uint64_t>();
    const int64_t ave_count = F.get1<int64_t>();
    const uint32_t status = F.get1<uint32_t>();
    std::vector<Particles> ps((size_t)s.nsp);
    for (int isp = 0; isp < s.nsp; isp++) {
        Particles &P = ps[(size_t)isp];
        const int64_t n = F.get1<int64_t>();
        if (!F.ok || n < 0 || n != np[(size_t)isp]) return bad("particle counts differ between the two parts");
        P.cnt.resize((size_t)C);
        F.get(P.cnt.data(), (size_t)C * 4);
        if (!F.ok) return bad("truncated particles");
        int64_t total = 0;
        for (int32_t k : P.cnt) {
            if (k < 0) return bad("negative cell count");
            total += k;
        }
        if (total != n) return bad("cell counts do not sum to the particle count");
        for (int a = 0; a < 5; a++) {
            P.a[a].resize(n ? (size_t)n : 1);
            F.get(P.a[a].data(), (size_t)n * 4);
        }
        if (!F.ok) return bad("truncated particles");
    }
    std::vector<std::vector<char>> grids;
    for (hp_grid_field g : EXT_GRIDS) {
        void *p = nullptr;
        size_t nb = 0;
        hp_status st = hpi_grid_ptr(c, g, &p, &nb);
        if (st != HP_OK) return st;
        const int32_t id = F.get1<int32_t>();
        const uint64_t fb = F.get1<uint64_t>();
        if (!F.ok || id != (int32_t)g || fb != (uint64_t)nb) return bad("grid section does not match the case");
        grids.emplace_back(nb);
        F.get(grids.back().data(), nb);
    }
    unsigned long long pushes[64];
    F.get(pushes, sizeof pushes);
    char tail[8];
    F.get(tail, 8);
    if (!F.ok || std::memcmp(tail, TAIL, 8) != 0) return bad("truncated extension");
    // everything read: now change the case
    if (cudaSetDevice(c->device) != cudaSuccess || cudaStreamSynchronize(c->last_stream) != cudaSuccess)
        return hpi::cuda_fail(cudaGetLastError(), "checkpoint sync");
    for (int isp = 0; isp < s.nsp; isp++) {
        Particles &P = ps[(size_t)isp];
        hp_status st = hp_set_particles(c, isp, P.cnt.data(), P.a[0].data(), P.a[1].data(), P.a[2].data(),
                                        P.a[3].data(), P.a[4].data());
        if (st != HP_OK) return st;
    }
    size_t k = 0;
    for (hp_grid_field g : EXT_GRIDS) {
        void *p = nullptr;
        size_t nb = 0;
        hpi_grid_ptr(c, g, &p, &nb);
        if (nb && cudaMemcpy(p, grids[k].data(), nb, cudaMemcpyHostToDevice) != cudaSuccess)
            return hpi::cuda_fail(cudaGetLastError(), "checkpoint grid restore");
        k++;
    }
    if (cudaMemcpy(c->h.tstep, &tstep, 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->h.ave_count, &ave_count, 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->h.status, &status, 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->h.pushes, pushes, sizeof pushes, cudaMemcpyHostToDevice) != cudaSuccess)
        return hpi::cuda_fail(cudaGetLastError(), "checkpoint counters");
    if (seed != c->h.seed) { // the dump's Philox key: the descriptor carries it
        c->h.seed = seed;
        if (cudaMemcpy(c->d_case, &c->h, sizeof(DevCase), cudaMemcpyHostToDevice) != cudaSuccess)
            return hpi::cuda_fail(cudaGetLastError(), "checkpoint seed");
    }
    return HP_OK;
}

} // extern "C"
