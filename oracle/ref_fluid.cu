// ref_fluid.cu -- checker only: runs the reference's own host-side
// continuity solve (src/Fluid.c, src/cuda_Fluid.cu, compiled unedited by
// oracle/Makefile) for ref_dump, and writes its state.  Nothing in the
// product links this.
//
// rf_fluid(outdir, temps, src, nsteps): installs the gas temperature of
// every node (the reference solves it on the GPU before Set_Fluid_cuda),
// then runs Fluid_Setting (regions, wall factors, initial density), the
// diffusion coefficients (Cal_D_Argon / _Oxygen / _ArO2), the Gummel
// coefficients and the initial fluxes as Set_Fluid_cuda does, and writes
// them; with src (float[nfsp*Csize], cell order) it sets the sources and
// runs Solve_Continuity_eqn nsteps times, then writes densities and fluxes.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "cuda_Fluid.cuh"

extern "C" void Fluid_Setting(); // src/Fluid.c

namespace {
void wr(const std::string &dir, const char *name, const void *p, size_t bytes) {
    const std::string path = dir + "/" + name + ".bin";
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) { std::perror(path.c_str()); std::exit(2); }
    if (bytes && std::fwrite(p, 1, bytes, f) != bytes) { std::perror(path.c_str()); std::exit(2); }
    std::fclose(f);
}
// a [sx][sy] float** matrix of every fluid species, flattened species by species
std::vector<float> flat(float **GFC::*m, int sx, int sy) {
    std::vector<float> v;
    for (int f = 0; f < nfsp; f++)
        for (int i = 0; i < sx; i++)
            for (int j = 0; j < sy; j++) v.push_back((Fluid_sp[f].*m)[i][j]);
    return v;
}
} // namespace

extern "C" int rf_fluid(const char *outdir, const float *temps, const float *src, int nsteps) {
    const std::string d(outdir);
    for (int g = 0; g < Gsize; g++) vec_G[g].Temp = temps[g];
    Fluid_Setting();
    if (MainGas == ARGON) Cal_D_Argon(vec_C, vec_G, Fluid_sp);
    else if (MainGas == OXYGEN) Cal_D_Oxygen(vec_C, vec_G, Fluid_sp);
    else Cal_D_ArO2(vec_C, vec_G, Fluid_sp);
    calculate_gummel_coef_x();
    calculate_gummel_coef_y();
    for (int f = 0; f < nfsp; f++) {
        Calculate_Flux_x(f);
        Calculate_Flux_y(f);
    }
    std::vector<int> xl, yl;
    std::vector<float> xfg, yfg;
    for (int k = 0; k < Conti_xnum; k++) {
        xl.push_back(Conti_x[0].x1[k]); xl.push_back(Conti_x[0].x2[k]); xl.push_back(Conti_x[0].yy[k]);
    }
    for (int k = 0; k < Conti_ynum; k++) {
        yl.push_back(Conti_y[0].xx[k]); yl.push_back(Conti_y[0].y1[k]); yl.push_back(Conti_y[0].y2[k]);
    }
    for (int f = 0; f < nfsp; f++) for (int k = 0; k < Conti_xnum; k++) xfg.push_back(Conti_x[f].fg1[k]);
    for (int f = 0; f < nfsp; f++) for (int k = 0; k < Conti_xnum; k++) xfg.push_back(Conti_x[f].fg2[k]);
    for (int f = 0; f < nfsp; f++) for (int k = 0; k < Conti_ynum; k++) yfg.push_back(Conti_y[f].fg1[k]);
    for (int f = 0; f < nfsp; f++) for (int k = 0; k < Conti_ynum; k++) yfg.push_back(Conti_y[f].fg2[k]);
    wr(d, "fl_xlines", xl.data(), xl.size() * 4);
    wr(d, "fl_ylines", yl.data(), yl.size() * 4);
    wr(d, "fl_xl_fg", xfg.data(), xfg.size() * 4);
    wr(d, "fl_yl_fg", yfg.data(), yfg.size() * 4);
    std::vector<float> v;
    v = flat(&GFC::D, ncx, ncy); wr(d, "fl_D", v.data(), v.size() * 4);
    v = flat(&GFC::den, ncx, ncy); wr(d, "fl_den0", v.data(), v.size() * 4);
    v = flat(&GFC::gummel_ax, ngx, ncy); wr(d, "fl_gax", v.data(), v.size() * 4);
    v = flat(&GFC::gummel_bx, ngx, ncy); wr(d, "fl_gbx", v.data(), v.size() * 4);
    v = flat(&GFC::gummel_ay, ncx, ngy); wr(d, "fl_gay", v.data(), v.size() * 4);
    v = flat(&GFC::gummel_by, ncx, ngy); wr(d, "fl_gby", v.data(), v.size() * 4);
    v = flat(&GFC::flux_x, ngx, ncy); wr(d, "fl_flux_x0", v.data(), v.size() * 4);
    v = flat(&GFC::flux_y, ncx, ngy); wr(d, "fl_flux_y0", v.data(), v.size() * 4);
    Sync_Fluid_GFCtoGFG_forDen(Fluid_sp, Fluid_Den);
    {
        std::vector<float> n;
        for (int k = 0; k < nfsp * Gsize; k++) n.push_back(Fluid_Den[k].n);
        wr(d, "fl_node_den0", n.data(), n.size() * 4);
    }
    if (!src) return 0;
    for (int f = 0; f < nfsp; f++)
        for (int i = 0; i < ncx; i++)
            for (int j = 0; j < ncy; j++) Fluid_sp[f].Source[i][j] = src[(size_t)f * Csize + i * ncy + j];
    for (int k = 0; k < nsteps; k++) Solve_Continuity_eqn();
    v = flat(&GFC::den, ncx, ncy); wr(d, "fl_den", v.data(), v.size() * 4);
    v = flat(&GFC::flux_x, ngx, ncy); wr(d, "fl_flux_x", v.data(), v.size() * 4);
    v = flat(&GFC::flux_y, ncx, ngy); wr(d, "fl_flux_y", v.data(), v.size() * 4);
    return 0;
}
