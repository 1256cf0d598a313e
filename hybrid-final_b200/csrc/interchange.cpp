// interchange.cpp -- a case's state in the reference's own device structs
// (inc/def.h: GCP particles, GPG per-(species, node) data, GGA per-node
// data), for a host that keeps them.
//
// The reference stores particle k of the cell whose lower-left node is
// ID = i*ngy + j at GCP[ID + k*Gsize] inside each species' block of
// MPNC*Gsize records (src/cuda_Move.cu:195), with GPG[isp*Gsize + ID].
// PtNumInCell of them; offsets are in cell units, as here.  These calls
// convert between that layout and the library's slot pool through the plain
// array calls (hp_get/set_particles, hp_get_grid, hp_get_table).
#include <cstring>
#include <vector>

#include "capi_internal.hpp"

using hpi::set_error;

namespace {

// node ID of cell c (cell = i*ncy + j, node = i*ngy + j)
inline int node_of(const hp_case_info &in, int c) {
    const int i = c / in.ncy, j = c - i * in.ncy;
    return i * in.ngy + j;
}

template <class T> hp_status grid_to(hp_case *c, hp_grid_field f, std::vector<T> &v, size_t n) {
    v.assign(n, T(0));
    return n ? hp_get_grid(c, f, v.data(), n * sizeof(T)) : HP_OK;
}

template <class T> hp_status table_to(hp_case *c, int what, std::vector<T> &v) {
    size_t nb = 0;
    hp_status st = hp_get_table(c, what, nullptr, 0, &nb);
    if (st != HP_OK) return st;
    v.assign(nb / sizeof(T), T(0));
    return nb ? hp_get_table(c, what, v.data(), nb, &nb) : HP_OK;
}

} // namespace

extern "C" {

hp_status hp_export_gcp(hp_case *c, int isp, int mpnc, hp_gcp *gcp, hp_gpg *gpg) {
    hp_case_info in;
    if (!c || !gcp || mpnc <= 0) return set_error("hp_export_gcp: bad arguments"), HP_ERR_ARG;
    hp_status st = hp_case_get_info(c, &in);
    if (st != HP_OK) return st;
    if (isp < 0 || isp >= in.nsp) return set_error("hp_export_gcp: bad species"), HP_ERR_ARG;
    const int C = in.Csize, G = in.Gsize;
    std::vector<int> counts(C);
    size_t n = 0;
    if ((st = hp_get_particles(c, isp, counts.data(), nullptr, nullptr, nullptr, nullptr, nullptr, 0, &n)) != HP_OK)
        return st;
    for (int cell = 0; cell < C; cell++)
        if (counts[cell] > mpnc) return set_error("hp_export_gcp: a cell holds more particles than mpnc"), HP_ERR_CAPACITY;
    std::vector<float> a[5];
    for (auto &v : a) v.resize(n ? n : 1);
    if ((st = hp_get_particles(c, isp, counts.data(), a[0].data(), a[1].data(), a[2].data(), a[3].data(),
                               a[4].data(), n, &n)) != HP_OK)
        return st;
    std::memset(gcp, 0, sizeof(hp_gcp) * (size_t)mpnc * G);
    size_t q = 0;
    for (int cell = 0; cell < C; cell++) {
        const int id = node_of(in, cell);
        for (int k = 0; k < counts[cell]; k++, q++) {
            hp_gcp &p = gcp[(size_t)id + (size_t)k * G];
            p.CellID = id;
            p.x = a[0][q];
            p.y = a[1][q];
            p.vx = a[2][q];
            p.vy = a[3][q];
            p.vz = a[4][q];
        }
    }
    if (!gpg) return HP_OK;
    std::vector<double> den, ave;
    std::vector<long long> sig;
    int64_t nave = 0;
    if ((st = grid_to(c, HP_GRID_DEN, den, (size_t)in.nsp * G)) != HP_OK) return st;
    if ((st = grid_to(c, HP_GRID_AVE_DEN, ave, (size_t)in.nsp * G)) != HP_OK) return st;
    if ((st = grid_to(c, HP_GRID_SURFACE_CHARGE, sig, in.n_dielectric ? (size_t)in.nsp * G : 0)) != HP_OK) return st;
    if ((st = hp_get_average_count(c, &nave)) != HP_OK) return st;
    std::memset(gpg, 0, sizeof(hp_gpg) * (size_t)G);
    for (int cell = 0; cell < C; cell++) {
        const int id = node_of(in, cell);
        gpg[id].PtNumInCell = counts[cell];
        gpg[id].MaxPtNumInCell = mpnc;
    }
    for (int g = 0; g < G; g++) {
        const size_t k = (size_t)isp * G + g;
        gpg[g].den = (float)den[k];
        gpg[g].ave_den = nave > 0 ? (float)(ave[k] / (double)nave) : 0.0f;
        if (!sig.empty()) gpg[g].sigma = (float)((double)sig[k] / (double)(1LL << HP_SIGMA_FRAC_BITS));
    }
    return HP_OK;
}

hp_status hp_import_gcp(hp_case *c, int isp, int mpnc, const hp_gcp *gcp, const hp_gpg *gpg) {
    hp_case_info in;
    if (!c || !gcp || !gpg || mpnc <= 0) return set_error("hp_import_gcp: bad arguments"), HP_ERR_ARG;
    hp_status st = hp_case_get_info(c, &in);
    if (st != HP_OK) return st;
    if (isp < 0 || isp >= in.nsp) return set_error("hp_import_gcp: bad species"), HP_ERR_ARG;
    const int C = in.Csize, G = in.Gsize;
    std::vector<int> counts(C);
    size_t n = 0;
    for (int cell = 0; cell < C; cell++) {
        const int k = gpg[node_of(in, cell)].PtNumInCell;
        if (k < 0 || k > mpnc) return set_error("hp_import_gcp: PtNumInCell outside 0..mpnc"), HP_ERR_ARG;
        counts[cell] = k;
        n += (size_t)k;
    }
    std::vector<float> a[5];
    for (auto &v : a) v.resize(n ? n : 1);
    size_t q = 0;
    for (int cell = 0; cell < C; cell++) {
        const int id = node_of(in, cell);
        for (int k = 0; k < counts[cell]; k++, q++) {
            const hp_gcp &p = gcp[(size_t)id + (size_t)k * G];
            a[0][q] = p.x;
            a[1][q] = p.y;
            a[2][q] = p.vx;
            a[3][q] = p.vy;
            a[4][q] = p.vz;
        }
    }
    return hp_set_particles(c, isp, counts.data(), a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data());
}

hp_status hp_export_gga(hp_case *c, hp_gga *gga) {
    hp_case_info in;
    if (!c || !gga) return set_error("hp_export_gga: bad arguments"), HP_ERR_ARG;
    hp_status st = hp_case_get_info(c, &in);
    if (st != HP_OK) return st;
    const size_t G = (size_t)in.Gsize;
    std::vector<int> bnd, cid, face, dr;
    std::vector<float> area, temp, bd1, bv1, bd2, bv2, phi, phip, ex, ey;
    if ((st = table_to(c, 2, bnd)) != HP_OK || (st = table_to(c, 4, cid)) != HP_OK ||
        (st = table_to(c, 3, face)) != HP_OK || (st = table_to(c, 14, dr)) != HP_OK ||
        (st = table_to(c, 5, area)) != HP_OK || (st = table_to(c, 27, temp)) != HP_OK ||
        (st = table_to(c, 6, bd1)) != HP_OK || (st = table_to(c, 7, bv1)) != HP_OK ||
        (st = table_to(c, 17, bd2)) != HP_OK || (st = table_to(c, 18, bv2)) != HP_OK)
        return st;
    if ((st = grid_to(c, HP_GRID_PHI, phi, G)) != HP_OK || (st = grid_to(c, HP_GRID_PHI_POIS, phip, G)) != HP_OK ||
        (st = grid_to(c, HP_GRID_EX, ex, G)) != HP_OK || (st = grid_to(c, HP_GRID_EY, ey, G)) != HP_OK)
        return st;
    auto at = [](const std::vector<float> &v, size_t g) { return g < v.size() ? v[g] : 0.0f; };
    for (size_t g = 0; g < G; g++) {
        hp_gga &r = gga[g];
        r.Boundary = bnd[g];
        r.CondID = cid[g];
        r.Face = face[g];
        r.DensRegion = dr[g];
        r.Area = area[g];
        r.Temp = at(temp, g);
        r.BackDen1 = at(bd1, g);
        r.BackVel1 = at(bv1, g);
        r.BackDen2 = at(bd2, g);
        r.BackVel2 = at(bv2, g);
        r.Pois_Pot = phip[g];
        r.Lap_Pot = phi[g] - phip[g]; // TotPotential = Lap_Pot + Pois_Pot (src/cuda_Field.cu:27-35)
        r.Ex = ex[g];
        r.Ey = ey[g];
    }
    return HP_OK;
}

} // extern "C"
