// capi.cu -- C ABI of libhpic: case lifecycle, operators, interchange, batches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "capi_internal.hpp"
#include "prof.cuh"

using namespace hp;

namespace hpi {

thread_local std::string g_err;

void set_error(const std::string &m) { g_err = m; }

bool tune_valid(const hp_tune &t) {
    if (t.warps_per_block_particles < 1 || t.warps_per_block_particles > 16) return false;
    if (t.pcg_block < 64 || t.pcg_block > 512 || (t.pcg_block & 31)) return false;
    if (t.pcg_cluster_max < 1 || t.pcg_cluster_max > 16 || (t.pcg_cluster_max & (t.pcg_cluster_max - 1)))
        return false;
    const int g = t.mcc_cells_per_warp;
    if (g != 1 && g != 2 && g != 4 && g != 8 && g != 16) return false;
    return t.move_unroll == 1 || t.move_unroll == 2 || t.move_unroll == 4;
}

int count_kernel_nodes(cudaGraph_t g) {
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
    int k = 0;
    for (size_t q = 0; q < n; q++) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[q], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
    }
    return k;
}

hp_status cuda_fail(cudaError_t e, const char *what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return HP_ERR_CUDA;
}

hp_status fast_plan_build(hp_case *const *cases, const std::vector<int> &idx, FastPlanDev &out) {
    out = FastPlanDev();
    const int n = (int)idx.size();
    if (n == 0) return HP_OK;
    std::vector<int> items(n + 1, 0);
    std::vector<GemmProb> st[4];
    int tiles[4] = {0, 0, 0, 0};
    for (int q = 0; q < n; q++) {
        const hp::DevCase &h = cases[q]->h;
        const int nx = h.fs_nx, ny = h.fs_ny;
        items[q + 1] = items[q] + nx * ny;
        const int tn = (nx + FS_TILE - 1) / FS_TILE, tm = (ny + FS_TILE - 1) / FS_TILE;
        out.plan.final_chunks = std::max(out.plan.final_chunks, (h.G + FS_CHUNK - 1) / FS_CHUNK);
        GemmProb g[4];
        std::memset(g, 0, sizeof g);
        // A1 = X V ; Y = (W^T A1) .* inv ; A2 = Y V^T ; x64 += W A2
        g[0] = GemmProb{ny, nx, nx, h.fs_x, h.fs_V, h.fs_a1, nullptr, nullptr, 0, 0, 0, 0, tn, 0};
        g[1] = GemmProb{ny, nx, ny, h.fs_Wt, h.fs_a1, h.fs_y, h.fs_inv, nullptr, 0, 0, 0, 1, tn, 0};
        g[2] = GemmProb{ny, nx, nx, h.fs_y, h.fs_Vt, h.fs_a1, nullptr, nullptr, 0, 0, 0, 0, tn, 0};
        g[3] = GemmProb{ny, nx, ny, h.fs_W, h.fs_a1, nullptr, nullptr, h.x64, h.ngy, h.fs_i0, h.fs_j0, 2, tn, 0};
        for (int k = 0; k < 4; k++) {
            g[k].tile_start = tiles[k];
            tiles[k] += tm * tn;
            st[k].push_back(g[k]);
        }
    }
    cudaError_t e;
    if ((e = cudaMalloc(&out.d_list, sizeof(int) * n)) != cudaSuccess) return cuda_fail(e, "fast plan");
    if ((e = cudaMalloc(&out.d_items, sizeof(int) * (n + 1))) != cudaSuccess) return cuda_fail(e, "fast plan");
    if ((e = cudaMalloc(&out.d_probs, sizeof(GemmProb) * 4 * n)) != cudaSuccess) return cuda_fail(e, "fast plan");
    cudaMemcpy(out.d_list, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(out.d_items, items.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    for (int k = 0; k < 4; k++) {
        e = cudaMemcpy(out.d_probs + (size_t)k * n, st[k].data(), sizeof(GemmProb) * n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "fast plan");
        out.plan.probs[k] = out.d_probs + (size_t)k * n;
        out.plan.ntiles[k] = tiles[k];
    }
    out.plan.list = out.d_list;
    out.plan.item_start = out.d_items;
    out.plan.n = n;
    out.plan.items = items[n];
    out.plan.passes = cases[0]->h.fs_passes > 0 ? cases[0]->h.fs_passes : 3;
    return HP_OK;
}

void fast_plan_free(FastPlanDev &f) {
    cudaFree(f.d_list);
    cudaFree(f.d_items);
    cudaFree(f.d_probs);
    f = FastPlanDev();
}

} // namespace hpi

using hpi::cuda_fail;
using hpi::set_error;

#define CK(call)                                                                                                       \
    do {                                                                                                               \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);                                                           \
    } while (0)

namespace {

hp_status from_exception(const std::exception &e) {
    std::string m = e.what();
    set_error(m);
    if (m.rfind("deck:", 0) == 0) return HP_ERR_DECK;
    if (m.rfind("unsupported:", 0) == 0) return HP_ERR_UNSUPPORTED;
    return HP_ERR_ARG;
}

BuildOpts build_opts(const hp_case_opts *o) {
    BuildOpts b;
    if (o) {
        b.seed = o->seed;
        b.cap_per_cell = o->cap_per_cell;
        b.gas_temp_mode = o->gas_temp_mode;
        b.defer_load = o->gpu_load != 0;
    }
    return b;
}

void fill_info(const Setup &s, hp_case_info *out) {
    std::memset(out, 0, sizeof(*out));
    out->ngx = s.ngx; out->ngy = s.ngy; out->ncx = s.ncx; out->ncy = s.ncy;
    out->Gsize = s.Gsize; out->Csize = s.Csize;
    out->nsp = s.nsp; out->main_gas = s.main_gas; out->cond_numr = s.cond_numr; out->n_unknowns = s.n_unknowns;
    for (int i = 0; i < s.nsp && i < 8; i++) out->cap[i] = s.cap[i];
    out->mcc_subcycles = s.mcc_n;
    out->dt = s.dt; out->dx = s.dx; out->dy = s.dy;
    out->mcc_stride = s.main_gas == GAS_AR ? 8 : 72;
    out->n_smt = s.N_smt;
    out->n_dielectric = s.diel_num;
    out->n_sources = s.src_num;
    out->power_driven = s.power_driven() ? 1 : 0;
    out->n_reactions = s.TnRct;
    out->n_fluid = s.nfsp;
    out->circuit = s.external ? 1 : 0;
}

// Collision probability per cell from its lower-left node
// (src/cuda_mccAr.cu:57-58 for electrons with dt_mcc, :189 for ions with dt).
std::vector<float> cell_probabilities(const Setup &s) {
    std::vector<float> p((size_t)3 * s.Csize, 0.0f);
    if (s.main_gas != GAS_AR) return p;
    for (int c = 0; c < s.Csize; c++) {
        int i = c / s.ncy, j = c % s.ncy, node = i * s.ngy + j;
        float P1 = 1.0f - std::exp(-1 * s.dt_mcc * s.sigv[0] * s.back_den1[node]);
        float P2 = P1 + 1.0f - std::exp(-1 * s.dt_mcc * s.sigv[1] * s.fluid_den[node]);
        float Pi = 1.0f - std::exp(-1 * s.dt * s.sigv[2] * s.back_den1[node]);
        p[c] = P1;
        p[(size_t)s.Csize + c] = P2;
        p[(size_t)2 * s.Csize + c] = Pi;
    }
    return p;
}

// Node-layout operator (W,S,C,N,E per node, 0 off the unknowns) and its
// row-scaled symmetric form D^-1 A, with D = 2 per Neumann edge doubling
// (the NBC factors of src/load.c:161-164).
void node_stencils(const Setup &s, std::vector<float> &st, std::vector<float> &sym, std::vector<float> &scale) {
    const int G = s.Gsize;
    st.assign((size_t)5 * G, 0.0f);
    sym.assign((size_t)5 * G, 0.0f);
    scale.assign(G, 1.0f);
    for (int u = 0; u < s.n_unknowns; u++) {
        int n = s.unk_node[u];
        int i = n / s.ngy, j = n % s.ngy;
        float dscale = (float)(((i == 0 || i == s.ncx) ? 2 : 1) * ((j == 0 || j == s.ncy) ? 2 : 1));
        for (int k = 0; k < 5; k++) {
            float a = s.stencil[(size_t)5 * u + k];
            st[(size_t)k * G + n] = a;
            sym[(size_t)k * G + n] = a / dscale;
        }
        scale[n] = 1.0f / dscale;
    }
}

template <class T> hp_status dalloc(hp_case *c, T **p, size_t count) {
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        set_error(std::string("cudaMalloc of ") + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
        return HP_ERR_OOM;
    }
    c->allocs.push_back(*p);
    c->alloc_bytes.push_back(bytes);
    c->bytes += bytes;
    e = cudaMemset(*p, 0, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemset");
    return HP_OK;
}

template <class T> hp_status dupload(hp_case *c, T **p, const std::vector<T> &v) {
    hp_status st = dalloc(c, p, v.size());
    if (st != HP_OK) return st;
    if (!v.empty()) CK(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return HP_OK;
}

#define TRY(x)                                                                                                         \
    do {                                                                                                               \
        hp_status s_ = (x);                                                                                            \
        if (s_ != HP_OK) return s_;                                                                                    \
    } while (0)

// Counts per cell and CSR arrays from the host: the arrays go to the device
// as they are (one copy each) and a kernel files them into the slot pool.
hp_status upload_particles(hp_case *c, int isp, const int *counts, const float *x, const float *y, const float *vx,
                           const float *vy, const float *vz) {
    const Setup &s = c->s;
    const int C = s.Csize, cap = c->h.sp[isp].cap;
    std::vector<int> start(C + 1, 0);
    for (int cell = 0; cell < C; cell++) {
        const int n = counts[cell];
        if (n < 0 || 2 * n > cap) {
            set_error("cell " + std::to_string(cell) + " holds " + std::to_string(n) +
                      " particles; the slot pool takes at most " + std::to_string(cap / 2));
            return HP_ERR_CAPACITY;
        }
        start[cell + 1] = start[cell] + n;
    }
    const size_t total = (size_t)start[C];
    int *d_start = nullptr;
    float *d_src = nullptr;
    CK(cudaMalloc(&d_start, sizeof(int) * (size_t)(C + 1)));
    cudaError_t e = cudaMalloc(&d_src, sizeof(float) * std::max<size_t>(5 * total, 1));
    if (e != cudaSuccess) {
        cudaFree(d_start);
        return cuda_fail(e, "cudaMalloc (particle upload)");
    }
    const float *arr[5] = {x, y, vx, vy, vz};
    e = cudaMemcpy(d_start, start.data(), sizeof(int) * (size_t)(C + 1), cudaMemcpyHostToDevice);
    for (int a = 0; a < 5 && e == cudaSuccess && total; a++)
        e = cudaMemcpy(d_src + (size_t)a * total, arr[a], sizeof(float) * total, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_scatter(c->h.sp[isp], C, d_start, d_src, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(d_start);
    cudaFree(d_src);
    if (e != cudaSuccess) return cuda_fail(e, "particle upload");
    return HP_OK;
}

hp_status build_device(hp_case *c) {
    const Setup &s = c->s;
    DevCase &h = c->h;
    std::memset(&h, 0, sizeof(h));
    const int G = s.Gsize, C = s.Csize;
    if (s.nsp > DMAXSP || s.cond_numr > DMAXCOND || s.src_num > DMAXSRC) {
        set_error("case exceeds the library's species/conductor/source limits");
        return HP_ERR_UNSUPPORTED;
    }
    h.ngx = s.ngx; h.ngy = s.ngy; h.ncx = s.ncx; h.ncy = s.ncy; h.G = G; h.C = C; h.nsp = s.nsp;
    h.gas = s.main_gas; h.cond_numr = s.cond_numr; h.n_unknowns = s.n_unknowns;
    h.dt_dx = s.dt_dx; h.dt_dy = s.dt_dy; h.dt = s.dt;
    h.dx = s.dx; h.dy = s.dy; h.idx = s.idx; h.idy = s.idy; h.hdx = s.hdx; h.hdy = s.hdy; h.idxy = s.idxy;
    TRY(dupload(c, (int **)&h.sidx, s.sidx));
    TRY(dupload(c, (int **)&h.boundary, s.boundary));
    TRY(dupload(c, (int **)&h.face, s.face));
    TRY(dupload(c, (int **)&h.cond_id, s.cond_id));
    {
        std::vector<float> eps(C);
        for (int k = 0; k < C; k++) eps[k] = (float)(EPS0 * s.eps_r[k]); // src/cuda_Field.cu:289-291
        TRY(dupload(c, (float **)&h.eps, eps));
    }
    TRY(dupload(c, (float **)&h.dep_factor, s.dep_factor));
    h.n_smt = s.N_smt;
    TRY(dupload(c, (int **)&h.dens_region, s.dens_region));
    if (s.N_smt > 0) TRY(dalloc(c, &h.smt, (size_t)s.nsp * G));
    if (s.diel_num > 0) {
        TRY(dalloc(c, &h.sig, (size_t)s.nsp * G));
        TRY(dupload(c, (int **)&h.sig_mode, s.sig_mode));
        // the crossings one step can queue: every particle a cell next to a
        // dielectric cell can hold (the mover half of its slots), per species
        long long adj = 0;
        for (int i = 0; i < s.ncx; i++)
            for (int j = 0; j < s.ncy; j++) {
                if (s.plasma_region[(size_t)i * s.ncy + j] != 1) continue;
                bool near = false;
                for (int a = -1; a <= 1 && !near; a++)
                    for (int b = -1; b <= 1 && !near; b++) {
                        const int S = s.sidx[(size_t)(i + 1 + a) * (s.ncy + 2) + (j + 1 + b)];
                        near = S >= 1 && S < 100;
                    }
                adj += near;
            }
        long long cap = 0;
        for (int isp = 0; isp < s.nsp; isp++) cap += adj * ((s.cap[isp] + 1) / 2);
        cap = std::max(cap, 4096LL);
        if (cap > (1LL << 30)) return set_error("dielectric crossing queue above 2^30 entries"), HP_ERR_ARG;
        h.dq_cap = (int)cap;
        TRY(dalloc(c, &h.dq_n, 1));
        TRY(dalloc(c, &h.dq_k, (size_t)cap));
        TRY(dalloc(c, &h.dq_v, (size_t)cap));
        if ((long long)C >= (1LL << 24)) return set_error("dielectric decks hold at most 2^24 cells"), HP_ERR_ARG;
    }
    if (c->opts.move_mode != 0 && c->opts.move_mode != 1) return set_error("move_mode must be 0 or 1"), HP_ERR_ARG;
    if (c->opts.circuit_mode != 0 && c->opts.circuit_mode != 1)
        return set_error("circuit_mode must be 0 or 1"), HP_ERR_ARG;
    for (int isp = 0; isp < s.nsp; isp++) {
        // a far mover's key holds its rank r < cap/2 in 18 bits
        if (s.cap[isp] > (1 << 19)) return set_error("cap_per_cell above 2^19"), HP_ERR_ARG;
    }
    for (int isp = 0; isp < s.nsp; isp++) {
        DevSpecies &sp = h.sp[isp];
        sp.cap = s.cap[isp];
        sp.Ascale = s.sp[isp].Ascale;
        sp.q_density = s.sp[isp].q_density;
        sp.Escale = s.sp[isp].Escale;
        sp.np2c = s.sp[isp].np2c;
        size_t nslot = (size_t)C * sp.cap;
        TRY(dalloc(c, &sp.x, nslot));
        TRY(dalloc(c, &sp.y, nslot));
        TRY(dalloc(c, &sp.vx, nslot));
        TRY(dalloc(c, &sp.vy, nslot));
        TRY(dalloc(c, &sp.vz, nslot));
        TRY(dalloc(c, &sp.code, nslot));
        TRY(dalloc(c, &sp.cnt, C));
        TRY(dalloc(c, &sp.nmov, C));
        TRY(dalloc(c, &sp.dcount, (size_t)C * 9));
        TRY(dalloc(c, &h.cw[isp], C));
    }
    TRY(dalloc(c, &h.Ex, G));
    TRY(dalloc(c, &h.Ey, G));
    TRY(dalloc(c, &h.phi, G));
    TRY(dalloc(c, &h.phi_p, G));
    TRY(dupload(c, (float **)&h.lap, s.lap_basis));
    {
        std::vector<float> st, sym, scale;
        node_stencils(s, st, sym, scale);
        TRY(dupload(c, (float **)&h.st, st));
        TRY(dupload(c, (float **)&h.st_sym, sym));
        TRY(dupload(c, (float **)&h.row_scale, scale));
    }
    TRY(dalloc(c, &h.pf_x, G));
    TRY(dalloc(c, &h.pf_r, G));
    TRY(dalloc(c, &h.pf_p, G));
    TRY(dalloc(c, &h.pf_p2, G));
    // one halo of 2 x ngy directions per CTA, for up to 16 cluster CTAs or one per 1024 nodes
    TRY(dalloc(c, &h.pcg_halo, (size_t)2 * s.ngy * std::max(16, (G + 1023) / 1024)));
    TRY(dalloc(c, &h.pf_ap, G));
    TRY(dalloc(c, &h.x64, G));
    TRY(dalloc(c, &h.b64, G));
    TRY(dalloc(c, &h.dots, 64));
    TRY(dalloc(c, &h.den, (size_t)s.nsp * G));
    TRY(dalloc(c, &h.source, G));
    TRY(dalloc(c, &h.ave_den, (size_t)s.nsp * G));
    TRY(dalloc(c, &h.ave_phi, G));
    TRY(dalloc(c, &h.ave_src, G));
    TRY(dalloc(c, &h.ave_ex, G));
    TRY(dalloc(c, &h.ave_ey, G));
    h.src_num = s.src_num;
    for (int k = 0; k < s.src_num; k++) {
        h.src_mid[k] = s.src_mid[k];
        h.src_dc[k] = s.src_dc[k];
        h.src_ac[k] = s.src_ac[k];
        h.src_2pif[k] = s.src_2pifreq[k];
        h.src_rphase[k] = s.src_rphase[k];
    }
    for (int k = 0; k < s.cond_numr; k++) h.efield_flag[k] = s.efield_flag[k];
    TRY(dupload(c, (float **)&h.src_amp, std::vector<float>(s.src_ac.begin(), s.src_ac.end())));
    // the power controller's surface charge and absorbed counts also feed the external circuit
    if (s.power_driven() || s.external) {
        for (int k = 0; k < s.src_num; k++) h.src_power[k] = s.src_power[k];
        for (int k = 0; k < s.cond_numr; k++) {
            h.cond_src_num[k] = s.cond_src_num[k];
            h.cond_power_id[k] = s.cond_power_id[k];
        }
        h.pd_intv = s.pd_intv;
        h.pd_ratio = s.pd_ratio;
        TRY(dalloc(c, &h.pw, 1));
        TRY(dalloc(c, &h.cond_step, (size_t)s.nsp * s.cond_numr));
        std::vector<int> cn;
        for (int n = 0; n < G; n++)
            if (s.cond_id[n]) cn.push_back(n | ((s.cond_id[n] - 1) << 24));
        if (G >= (1 << 24)) return set_error("power-driven and circuit decks hold at most 2^24 nodes"), HP_ERR_ARG;
        h.n_cond_nodes = (int)cn.size();
        TRY(dupload(c, (int **)&h.cond_nodes, cn));
    }
    if (s.external) { // src/cuda_Field.cu:43-103
        TRY(dalloc(c, &h.cs, 1));
        h.circuit_mode = c->opts.circuit_mode;
        const int nc = s.cond_numr;
        for (int i = 0; i < nc; i++) {
            for (int q = 0; q < 5; q++) h.cc_a[i * 5 + q] = s.cc_a[(size_t)i * 5 + q];
            for (int j = 0; j < nc; j++) h.lap_sig[j * HP_CIRCUIT_MAX + i] = s.lap_sig[(size_t)j * nc + i];
        }
    }
    if (s.power_driven() || s.diel_num > 0 || s.external) {
        TRY(dupload(c, (float **)&h.area, s.area));
        TRY(dalloc(c, &h.sigma, (size_t)G));
    }
    TRY(dupload(c, (float **)&h.xsec, s.xsec));
    h.n_logx = s.n_logx;
    h.xw = 2 + s.n_cx;
    h.idlogx = s.idlogx;
    if (s.sigv.size() > 32 || s.TnRct > 96) return set_error("reaction set larger than the device tables"), HP_ERR_UNSUPPORTED;
    for (size_t k = 0; k < s.sigv.size(); k++) h.sigv[k] = s.sigv[k];
    for (int k = 0; k < s.TnRct; k++) {
        h.th[k] = s.collf[k].Th_e;
        h.mofm[k] = s.collf[k].mofM;
    }
    h.mcc_stride = s.main_gas == GAS_AR ? 8 : 72;
    h.mcc_all_species = c->opts.o2_all_species ? 1 : 0;
    TRY(dupload(c, (float **)&h.back_den1, s.back_den1));
    if (s.main_gas != GAS_AR) {
        TRY(dupload(c, (float **)&h.back_den2, s.back_den2));
        TRY(dupload(c, (float **)&h.back_vel2, s.back_vel2));
    }
    // fluid species and the state of their averaging window: the electron
    // density sum, the tallies at the last average and the collision
    // probabilities (one block, HP_GRID_FLUID_STATE)
    c->prob = cell_probabilities(s);
    {
        const int F = s.nfsp, st = h.mcc_stride;
        c->fl_state_bytes = (size_t)G * 8 + (size_t)C * st * 4 + (size_t)3 * C * 4;
        TRY(dalloc(c, &c->fl_state, c->fl_state_bytes));
        h.fl_sum = (double *)c->fl_state;
        h.fl_base = (unsigned int *)(c->fl_state + (size_t)G * 8);
        h.prob = (float *)(c->fl_state + (size_t)G * 8 + (size_t)C * st * 4);
        CK(cudaMemcpy(h.prob, c->prob.data(), (size_t)3 * C * 4, cudaMemcpyHostToDevice));
        h.nfsp = F;
        h.fluid_on = (F > 0 && !c->opts.fluid_fixed) ? 1 : 0;
        h.n_ave = s.N_ave;
        h.tnrct = s.TnRct;
        h.dtc = s.dtc;
        h.denscale0 = s.sp[0].Denscale;
        h.nxl = (int)s.xl_x1.size();
        h.nyl = (int)s.yl_xx.size();
        for (int k = 0; k < s.TnRct && k < 96; k++) {
            h.rate_f[k] = s.fluid_rate_f[k];
            h.rr[k] = s.collf[k].RR;
        }
        if (F > 0) {
            if (h.fluid_on && (fluid_sweep_warps(s.ncx) == 0 || fluid_sweep_warps(s.ncy) == 0))
                return set_error("grid too wide for the fluid sweep"), HP_ERR_UNSUPPORTED;
            if (h.fluid_on && s.N_ave < 1) return set_error("AverageIter must be at least 1"), HP_ERR_UNSUPPORTED;
            std::vector<int> xl, yl;
            for (int k = 0; k < h.nxl; k++) { xl.push_back(s.xl_x1[k]); xl.push_back(s.xl_x2[k]); xl.push_back(s.xl_yy[k]); }
            for (int k = 0; k < h.nyl; k++) { yl.push_back(s.yl_xx[k]); yl.push_back(s.yl_y1[k]); yl.push_back(s.yl_y2[k]); }
            std::vector<float> xfg(s.xl_fg1), yfg(s.yl_fg1);
            xfg.insert(xfg.end(), s.xl_fg2.begin(), s.xl_fg2.end());
            yfg.insert(yfg.end(), s.yl_fg2.begin(), s.yl_fg2.end());
            TRY(dupload(c, &h.fluid_den, s.fluid_den));
            TRY(dupload(c, &h.fden, s.fluid_cell_den));
            TRY(dalloc(c, &h.fsrc, (size_t)F * C));
            TRY(dupload(c, &h.fflx, s.flux_x0));
            TRY(dupload(c, &h.ffly, s.flux_y0));
            TRY(dupload(c, (int **)&h.fl_xl, xl));
            TRY(dupload(c, (int **)&h.fl_yl, yl));
            TRY(dupload(c, (float **)&h.fl_xfg, xfg));
            TRY(dupload(c, (float **)&h.fl_yfg, yfg));
            TRY(dupload(c, (float **)&h.gax, s.gax));
            TRY(dupload(c, (float **)&h.gbx, s.gbx));
            TRY(dupload(c, (float **)&h.gay, s.gay));
            TRY(dupload(c, (float **)&h.gby, s.gby));
            TRY(dupload(c, (int **)&h.plasma, s.plasma_region));
        }
    }
    TRY(dupload(c, (float **)&h.back_vel1, s.back_vel1));
    TRY(dupload(c, (float **)&h.vsave, s.vsave));
    h.nvel = s.nvel;
    h.mcc_n = s.mcc_n;
    h.dt_mcc = s.dt_mcc;
    if (s.mcc_n < 1 || s.mcc_n > 2047) return set_error("MCC subcycle count outside 1..2047"), HP_ERR_UNSUPPORTED;
    h.seed = c->opts.seed;
    TRY(dalloc(c, &h.tstep, 1));
    TRY(dalloc(c, &h.status, 1));
    TRY(dalloc(c, &h.cond_charge, (size_t)s.nsp * s.cond_numr));
    TRY(dalloc(c, &h.mcc_count, (size_t)h.mcc_stride * C));
    TRY(dalloc(c, &h.pcg_iters, 2));
    TRY(dalloc(c, &h.ave_count, 1));
    TRY(dalloc(c, &h.eedf, HP_EEDF_BINS + 1));
    h.eedf_every = c->opts.eedf_every > 0 ? c->opts.eedf_every : 0;
    TRY(dalloc(c, &h.pushes, 64));
    TRY(dalloc(c, &h.far_in, (size_t)s.nsp * C));
    TRY(dalloc(c, &h.far_key, (size_t)s.nsp * C * HP_FAR_BUCKET));
    h.move_mode = c->opts.move_mode;
    h.field_mode = c->opts.field_mode;
    if (h.field_mode == 2) {
        // separable inner solve when the operator allows it, else mode 1
        if (build_fast_solver(s, c->fs)) {
            const size_t nxy = (size_t)c->fs.nx * c->fs.ny;
            h.fs_i0 = c->fs.i0; h.fs_j0 = c->fs.j0; h.fs_nx = c->fs.nx; h.fs_ny = c->fs.ny;
            {
                const double rtol = c->opts.pcg_rtol > 0 ? c->opts.pcg_rtol : 1e-8;
                c->fs_passes = c->opts.fs_passes > 0 ? c->opts.fs_passes : (rtol >= 1e-10 ? 2 : 3);
            }
            h.fs_passes = c->fs_passes;
            TRY(dupload(c, (float **)&h.fs_V, c->fs.V));
            TRY(dupload(c, (float **)&h.fs_Vt, c->fs.Vt));
            TRY(dupload(c, (float **)&h.fs_W, c->fs.W));
            TRY(dupload(c, (float **)&h.fs_Wt, c->fs.Wt));
            TRY(dupload(c, (float **)&h.fs_inv, c->fs.inv_eig));
            TRY(dalloc(c, &h.fs_x, nxy));
            TRY(dalloc(c, &h.fs_a1, nxy));
            TRY(dalloc(c, &h.fs_y, nxy));
            TRY(dalloc(c, &h.fs_res, 2 + 2 * (size_t)((G + FS_CHUNK - 1) / FS_CHUNK)));
        } else {
            h.field_mode = 1;
        }
    }
    h.pcg_max_iter = c->opts.pcg_max_iter > 0 ? c->opts.pcg_max_iter : 100000;
    h.pcg_tol2 = s.PCGtol2;
    h.pcg_rtol = c->opts.pcg_rtol > 0 ? c->opts.pcg_rtol : 1e-8;
    // a PCG case too large for a 16-CTA cluster solves over the whole GPU
    // (cooperative launch); its CTA totals need 2 x 2 doubles per CTA
    const int grid_ctas = h.field_mode != 2 ? pcg_grid_ctas(G, c->lc.pcg_block) : 0;
    if (grid_ctas > 0) TRY(dalloc(c, &h.pcg_part, 4 * (size_t)((G + 1023) / 1024)));
    TRY(dalloc(c, &c->d_list0, 1));
    TRY(dalloc(c, &c->d_case, 1));
    CK(cudaMemcpy(c->d_case, &h, sizeof(h), cudaMemcpyHostToDevice));
    {
        // particles, cells, nodes, fluid x lines, fluid y lines
        const int nx = h.fluid_on ? s.nfsp * h.nxl : 0, ny = h.fluid_on ? s.nfsp * h.nyl : 0;
        std::vector<int> items = {0, s.nsp * C, 0, C, 0, G, 0, nx, 0, ny};
        TRY(dupload(c, &c->d_items, items));
        c->fplan_fluid.xl_items = c->d_items + 6;
        c->fplan_fluid.yl_items = c->d_items + 8;
        c->fplan_fluid.n_x = nx;
        c->fplan_fluid.n_y = ny;
        c->fplan_fluid.len_x = s.ncx;
        c->fplan_fluid.len_y = s.ncy;
        c->fplan_fluid.any = h.fluid_on != 0;
    }
    for (int isp = 0; isp < s.nsp; isp++) {
        if (s.load_deferred) TRY(hpi::device_load(c, isp));
        else
            TRY(upload_particles(c, isp, s.p_count[isp].data(), s.p_x[isp].data(), s.p_y[isp].data(),
                                 s.p_vx[isp].data(), s.p_vy[isp].data(), s.p_vz[isp].data()));
    }
    c->pcg_cluster = grid_ctas > 0 ? grid_ctas : pcg_cluster_for_nodes(G);
    if (h.field_mode == 2) {
        hp_case *one[1] = {c};
        TRY(hpi::fast_plan_build(one, std::vector<int>{0}, c->fplan));
    }
    return HP_OK;
}

cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }


hp_status op_field(hp_case *c, cudaStream_t st) {
    PcgGroup g{c->pcg_cluster, c->lc.pcg_block, c->d_list0, 1};
    const bool fast = c->h.field_mode == 2;
    cudaError_t e = launch_field(c->d_case, c->d_items + 4, 1, c->s.Gsize, &g, fast ? 0 : 1,
                                 fast ? &c->fplan.plan : nullptr, st, c->h.cs != nullptr);
    return e == cudaSuccess ? HP_OK : cuda_fail(e, "field");
}
hp_status op_move(hp_case *c, cudaStream_t st) {
    cudaError_t e = launch_move(c->d_case, c->d_items, 1, c->s.nsp * c->s.Csize, c->lc, st);
    return e == cudaSuccess ? HP_OK : cuda_fail(e, "move");
}
hp_status op_sort(hp_case *c, cudaStream_t st) {
    cudaError_t e = launch_sort(c->d_case, c->d_items, 1, c->s.nsp * c->s.Csize, c->lc, st, c->s.diel_num > 0);
    return e == cudaSuccess ? HP_OK : cuda_fail(e, "sort");
}
hp_status op_mcc(hp_case *c, cudaStream_t st) {
    if (c->s.main_gas == GAS_ARO2 || c->s.main_gas == GAS_O2) {
        cudaError_t e = launch_mcc_oxy(c->d_case, c->d_items + 2, 1, c->s.Csize, c->s.main_gas, st);
        return e == cudaSuccess ? HP_OK : cuda_fail(e, "mcc");
    }
    if (c->s.main_gas != GAS_AR) {
        set_error("MCC for this gas is not built");
        return HP_ERR_UNSUPPORTED;
    }
    cudaError_t e = launch_mcc_ar(c->d_case, c->d_items + 2, 1, c->s.Csize, c->lc, st);
    return e == cudaSuccess ? HP_OK : cuda_fail(e, "mcc");
}
// smooth: DEPOSIT = Deposit_cuda with its DensitySmoothing passes
// (src/cuda_start.cu:32, src/cuda_Deposit.cu:3-20); the initial deposit
// before the loop is Deposit_Basic, without them (src/cuda_main.cu:28)
hp_status op_deposit(hp_case *c, cudaStream_t st, bool smooth) {
    cudaError_t e = launch_deposit(c->d_case, c->d_items, c->d_items + 4, 1, c->s.nsp * c->s.Csize, c->s.Gsize,
                                   c->lc, st, smooth ? c->s.N_smt : 0);
    return e == cudaSuccess ? HP_OK : cuda_fail(e, "deposit");
}

hp_status one_step(hp_case *c, cudaStream_t st) {
    cudaError_t e = launch_advance(c->d_case, 1, st);
    if (e != cudaSuccess) return cuda_fail(e, "advance");
    if (c->fplan_fluid.any) {
        e = fluid_begin(c->d_case, 1, c->fplan_fluid, c->fl_fork, st);
        if (e != cudaSuccess) return cuda_fail(e, "fluid");
    }
    TRY(op_field(c, st));
    TRY(op_move(c, st));
    TRY(op_sort(c, st));
    TRY(op_mcc(c, st));
    TRY(op_deposit(c, st, true));
    if (c->fplan_fluid.any) {
        e = fluid_end(c->d_case, c->d_items + 4, 1, c->s.Gsize, c->fplan_fluid, c->fl_fork, st);
        if (e != cudaSuccess) return cuda_fail(e, "fluid");
    }
    e = launch_accumulate(c->d_case, c->d_items + 4, 1, c->s.Gsize, st);
    if (e == cudaSuccess && c->h.eedf_every > 0) e = launch_eedf(c->d_case, c->d_items + 2, 1, c->s.Csize, st);
    if (e == cudaSuccess && c->h.pw) e = launch_power(c->d_case, 1, st);
    return e == cudaSuccess ? HP_OK : cuda_fail(e, "accumulate");
}

int check_cuda_device(int dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return -1;
    if (dev < 0 || dev >= n) return -2;
    return 0;
}

} // namespace

// ======================================================================== C ABI
extern "C" {

const char *hp_last_error(void) { return hpi::g_err.c_str(); }

void hp_case_opts_default(hp_case_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->seed = 1;
    o->field_mode = 0;
    o->pcg_rtol = 1e-8;
    o->pcg_max_iter = 0;
    o->o2_all_species = 0;
    o->device = 0;
}

hp_status hp_setup_build(const char *deck, size_t len, const hp_case_opts *opts, hp_setup **out) {
    if (!deck || !out) return set_error("null argument"), HP_ERR_ARG;
    hp_setup *s = new hp_setup();
    hp_case_opts_default(&s->opts);
    if (opts) s->opts = *opts;
    try {
        build_setup(deck, len, build_opts(&s->opts), s->s);
    } catch (const std::exception &e) {
        delete s;
        return from_exception(e);
    }
    *out = s;
    return HP_OK;
}

void hp_setup_destroy(hp_setup *s) { delete s; }

hp_status hp_setup_get_info(const hp_setup *s, hp_case_info *out) {
    if (!s || !out) return HP_ERR_ARG;
    fill_info(s->s, out);
    out->device_bytes = hpi::estimate_device_bytes(s->s, s->opts); // what a case built from it will hold
    return HP_OK;
}

hp_status hp_setup_get_particles(const hp_setup *su, int isp, int layout, int *cells, float *x, float *y, float *vx,
                                 float *vy, float *vz, size_t cap, size_t *n_out) {
    if (!su || isp < 0 || isp >= su->s.nsp) return set_error("bad species"), HP_ERR_ARG;
    const Setup &s = su->s;
    if (s.load_deferred)
        return set_error("this set-up leaves the particle load to the device (gpu_load): read the case's particles"),
               HP_ERR_ARG;
    size_t n = (size_t)s.sp[isp].np;
    if (n_out) *n_out = n;
    if (cap < n) return set_error("output arrays too small"), HP_ERR_ARG;
    if (layout == 0) {
        if (cells) std::memcpy(cells, s.p_count[isp].data(), (size_t)s.Csize * sizeof(int));
        std::memcpy(x, s.p_x[isp].data(), n * 4); std::memcpy(y, s.p_y[isp].data(), n * 4);
        std::memcpy(vx, s.p_vx[isp].data(), n * 4); std::memcpy(vy, s.p_vy[isp].data(), n * 4);
        std::memcpy(vz, s.p_vz[isp].data(), n * 4);
    } else {
        if (cells) std::memcpy(cells, s.h_cell[isp].data(), n * sizeof(int));
        std::memcpy(x, s.h_x[isp].data(), n * 4); std::memcpy(y, s.h_y[isp].data(), n * 4);
        std::memcpy(vx, s.h_vx[isp].data(), n * 4); std::memcpy(vy, s.h_vy[isp].data(), n * 4);
        std::memcpy(vz, s.h_vz[isp].data(), n * 4);
    }
    return HP_OK;
}

static hp_status table_of(const Setup &s, const std::vector<float> *prob, const FastSolver *fs, int what, void *out,
                          size_t bytes, size_t *needed) {
    const void *src = nullptr;
    size_t nb = 0;
    std::vector<float> tmpf;
    std::vector<int> tmpi;
    switch (what) {
    case 0: src = s.sidx.data(); nb = s.sidx.size() * 4; break;
    case 1: src = s.a_idx.data(); nb = s.a_idx.size() * 4; break;
    case 2: src = s.boundary.data(); nb = s.boundary.size() * 4; break;
    case 3: src = s.face.data(); nb = s.face.size() * 4; break;
    case 4: src = s.cond_id.data(); nb = s.cond_id.size() * 4; break;
    case 5: src = s.area.data(); nb = s.area.size() * 4; break;
    case 6: src = s.back_den1.data(); nb = s.back_den1.size() * 4; break;
    case 7: src = s.back_vel1.data(); nb = s.back_vel1.size() * 4; break;
    case 8: src = s.lap_basis.data(); nb = s.lap_basis.size() * 4; break;
    case 9: src = s.stencil.data(); nb = s.stencil.size() * 4; break;
    case 10: src = s.vsave.data(); nb = s.vsave.size() * 4; break;
    case 11: src = s.xsec.data(); nb = s.xsec.size() * 4; break;
    case 12:
        for (auto &cf : s.collf) { tmpf.push_back(cf.Flag); tmpf.push_back(cf.mofM); tmpf.push_back(cf.Th_e); tmpf.push_back(cf.RR); }
        src = tmpf.data(); nb = tmpf.size() * 4; break;
    case 13: src = s.sigv.data(); nb = s.sigv.size() * 4; break;
    case 14: src = s.dens_region.data(); nb = s.dens_region.size() * 4; break;
    case 15:
        if (prob) { src = prob->data(); nb = prob->size() * 4; }
        else { tmpf = cell_probabilities(s); src = tmpf.data(); nb = tmpf.size() * 4; }
        break;
    case 16: src = s.eps_r.data(); nb = s.eps_r.size() * 4; break;
    case 17: src = s.back_den2.data(); nb = s.back_den2.size() * 4; break;
    case 18: src = s.back_vel2.data(); nb = s.back_vel2.size() * 4; break;
    // reference-layout matrix and set-up vectors (src/load.c:121-246)
    case 19: src = s.a_val.data(); nb = s.a_val.size() * 4; break;
    case 20: src = s.ai.data(); nb = s.ai.size() * 4; break;
    case 21: src = s.aj.data(); nb = s.aj.size() * 4; break;
    case 22: src = s.matm.data(); nb = s.matm.size() * 4; break;
    case 23: src = s.cond_b.data(); nb = s.cond_b.size() * 4; break;
    case 24: src = s.temp_b.data(); nb = s.temp_b.size() * 4; break;
    case 25: src = s.ta_val.data(); nb = s.ta_val.size() * 4; break;
    case 26: // species scalars: 16 floats per species
        for (int i = 0; i < s.nsp; i++) {
            const SpeciesP &p = s.sp[i];
            float v[16] = {p.np2c, p.mass, p.q, p.q_density, p.vti, p.qm, p.Escale, p.Ascale, p.Denscale, p.MCCscale,
                           (float)p.MAXNP, p.Temp, p.InitDens, (float)p.np, (float)s.cap[i], 0.0f};
            tmpf.insert(tmpf.end(), v, v + 16);
        }
        src = tmpf.data(); nb = tmpf.size() * 4; break;
    case 27: src = s.node_temp.data(); nb = s.node_temp.size() * 4; break;
    case 28: src = s.dep_factor.data(); nb = s.dep_factor.size() * 4; break;
    case 29: src = s.fluid_den.data(); nb = s.fluid_den.size() * 4; break;
    case 30: // scalars: dt, dt_mcc, PCGtol, dx, dy, idx, idy, hdx, hdy, idxy, zlength, mcc_n, nvel, TnRct, n_logx, idlogx
    {
        float v[16] = {s.dt, s.dt_mcc, s.PCGtol, s.dx, s.dy, s.idx, s.idy, s.hdx, s.hdy, s.idxy, s.zlength,
                       (float)s.mcc_n, (float)s.nvel, (float)s.TnRct, (float)s.n_logx, s.idlogx};
        tmpf.assign(v, v + 16);
        src = tmpf.data(); nb = tmpf.size() * 4; break;
    }
    case 31: // sources: per source mid, dc, ac, 2pif, rphase; then efield flags
        for (int k = 0; k < s.src_num; k++) {
            tmpf.push_back((float)s.src_mid[k]); tmpf.push_back(s.src_dc[k]); tmpf.push_back(s.src_ac[k]);
            tmpf.push_back(s.src_2pifreq[k]); tmpf.push_back(s.src_rphase[k]);
        }
        for (int k = 0; k < s.cond_numr; k++) tmpf.push_back((float)s.efield_flag[k]);
        src = tmpf.data(); nb = tmpf.size() * 4; break;
    case 32: src = s.unk_node.data(); nb = s.unk_node.size() * 4; break;
    // separable inverse of field_mode 2: 33 int[6] {ok, i0, j0, nx, ny, 0};
    // 34 V, 35 V^T (nx*nx); 36 W, 37 W^T (ny*ny); 38 1/(lambda_i+theta_j) (ny*nx)
    case 33:
        tmpi = {fs && fs->ok ? 1 : 0, fs ? fs->i0 : 0, fs ? fs->j0 : 0, fs ? fs->nx : 0, fs ? fs->ny : 0, 0};
        src = tmpi.data(); nb = tmpi.size() * 4; break;
    case 34: if (fs) { src = fs->V.data(); nb = fs->V.size() * 4; } break;
    case 35: if (fs) { src = fs->Vt.data(); nb = fs->Vt.size() * 4; } break;
    case 36: if (fs) { src = fs->W.data(); nb = fs->W.size() * 4; } break;
    case 37: if (fs) { src = fs->Wt.data(); nb = fs->Wt.size() * 4; } break;
    case 38: if (fs) { src = fs->inv_eig.data(); nb = fs->inv_eig.size() * 4; } break;
    case 39: src = s.sig_mode.data(); nb = s.sig_mode.size() * 4; break;
    case 40: // power-driven sources: pd_intv, pd_ratio, target power per source, (count, first) per conductor
        tmpf.push_back((float)s.pd_intv);
        tmpf.push_back(s.pd_ratio);
        for (int k = 0; k < s.src_num; k++) tmpf.push_back(s.src_power[k]);
        for (int k = 0; k < s.cond_numr; k++) {
            tmpf.push_back((float)s.cond_src_num[k]);
            tmpf.push_back((float)s.cond_power_id[k]);
        }
        src = tmpf.data(); nb = tmpf.size() * 4; break;
    // fluid species (continuity solve)
    case 41: src = s.fluid_cell_den.data(); nb = s.fluid_cell_den.size() * 4; break;
    case 42:
        for (size_t k = 0; k < s.xl_x1.size(); k++) { tmpi.push_back(s.xl_x1[k]); tmpi.push_back(s.xl_x2[k]); tmpi.push_back(s.xl_yy[k]); }
        src = tmpi.data(); nb = tmpi.size() * 4; break;
    case 43:
        for (size_t k = 0; k < s.yl_xx.size(); k++) { tmpi.push_back(s.yl_xx[k]); tmpi.push_back(s.yl_y1[k]); tmpi.push_back(s.yl_y2[k]); }
        src = tmpi.data(); nb = tmpi.size() * 4; break;
    case 44:
        tmpf = s.xl_fg1; tmpf.insert(tmpf.end(), s.xl_fg2.begin(), s.xl_fg2.end());
        src = tmpf.data(); nb = tmpf.size() * 4; break;
    case 45:
        tmpf = s.yl_fg1; tmpf.insert(tmpf.end(), s.yl_fg2.begin(), s.yl_fg2.end());
        src = tmpf.data(); nb = tmpf.size() * 4; break;
    case 46: src = s.gax.data(); nb = s.gax.size() * 4; break;
    case 47: src = s.gbx.data(); nb = s.gbx.size() * 4; break;
    case 48: src = s.gay.data(); nb = s.gay.size() * 4; break;
    case 49: src = s.gby.data(); nb = s.gby.size() * 4; break;
    case 50: src = s.flux_x0.data(); nb = s.flux_x0.size() * 4; break;
    case 51: src = s.flux_y0.data(); nb = s.flux_y0.size() * 4; break;
    case 52: src = s.fluid_D.data(); nb = s.fluid_D.size() * 4; break;
    case 53: // fluid scalars: dtc, N_ave, TimeStep_Conti, nfsp, x lines, y lines
        tmpf = {s.dtc, (float)s.N_ave, (float)s.DT_CONTI, (float)s.nfsp, (float)s.xl_x1.size(), (float)s.yl_xx.size()};
        src = tmpf.data(); nb = tmpf.size() * 4; break;
    case 54: src = s.fluid_rate_f.data(); nb = s.fluid_rate_f.size() * 4; break;
    case 55: src = s.plasma_region.data(); nb = s.plasma_region.size() * 4; break;
    case 56: // external circuit: CC_a per conductor, then Lap_SIG_Sol by basis
        tmpf = s.cc_a;
        tmpf.insert(tmpf.end(), s.lap_sig.begin(), s.lap_sig.end());
        src = tmpf.data(); nb = tmpf.size() * 4; break;
    default: set_error("unknown table id"); return HP_ERR_ARG;
    }
    if (needed) *needed = nb;
    if (!out) return HP_OK;
    if (bytes < nb) return set_error("output buffer too small"), HP_ERR_ARG;
    if (nb) std::memcpy(out, src, nb);
    return HP_OK;
}

hp_status hp_setup_get_table(const hp_setup *s, int what, void *out, size_t bytes, size_t *needed) {
    if (!s) return HP_ERR_ARG;
    if (what >= 33 && what <= 38 && !s->fs_built) {
        hp_setup *m = const_cast<hp_setup *>(s);
        try {
            build_fast_solver(m->s, m->fs);
        } catch (const std::exception &e) {
            return from_exception(e);
        }
        m->fs_built = true;
    }
    return table_of(s->s, nullptr, &s->fs, what, out, bytes, needed);
}

hp_status hp_get_table(hp_case *c, int what, void *out, size_t bytes, size_t *needed) {
    if (!c) return HP_ERR_ARG;
    return table_of(c->s, &c->prob, &c->fs, what, out, bytes, needed);
}

static hp_status case_from(Setup s, const hp_case_opts *opts, hp_case **out) {
    hp_case_opts o;
    hp_case_opts_default(&o);
    if (opts) o = *opts;
    int chk = check_cuda_device(o.device);
    if (chk == -1) return set_error("no CUDA device: libhpic has no CPU path"), HP_ERR_NO_CUDA;
    if (chk == -2) return set_error("device ordinal out of range"), HP_ERR_ARG;
    CK(cudaSetDevice(o.device));
    hp_case *c = new hp_case();
    c->s = std::move(s);
    c->opts = o;
    c->device = o.device;
    hp_status st = build_device(c);
    if (st == HP_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaStreamCreate");
    }
    if (st == HP_OK && c->fplan_fluid.n_x + c->fplan_fluid.n_y > 0) {
        cudaError_t e = fluid_fork_create(c->fl_fork);
        if (e != cudaSuccess) st = cuda_fail(e, "fluid side stream");
    }
    if (st == HP_OK) st = op_deposit(c, c->own_stream, false); // Deposit_Basic before the loop (src/cuda_main.cu:28)
    if (st == HP_OK) {
        cudaError_t e = cudaStreamSynchronize(c->own_stream);
        if (e != cudaSuccess) st = cuda_fail(e, "initial deposit");
    }
    if (st != HP_OK) {
        hp_case_destroy(c);
        return st;
    }
    c->last_stream = c->own_stream;
    *out = c;
    return HP_OK;
}

hp_status hp_case_create(const char *deck, size_t len, const hp_case_opts *opts, hp_case **out) {
    if (!deck || !out) return set_error("null argument"), HP_ERR_ARG;
    hp_case_opts o;
    hp_case_opts_default(&o);
    if (opts) o = *opts;
    int chk = check_cuda_device(o.device);
    if (chk == -1) return set_error("no CUDA device: libhpic has no CPU path"), HP_ERR_NO_CUDA;
    Setup s;
    try {
        build_setup(deck, len, build_opts(&o), s);
    } catch (const std::exception &e) {
        return from_exception(e);
    }
    return case_from(std::move(s), &o, out);
}

hp_status hp_case_create_from_setup(const hp_setup *su, const hp_case_opts *opts, hp_case **out) {
    if (!su || !out) return HP_ERR_ARG;
    hp_case_opts o = su->opts;
    if (opts) o = *opts;
    return case_from(su->s, &o, out);
}
} // extern "C"

namespace hpi {
hp_status case_from_setup_owned(hp::Setup &&s, const hp_case_opts &o, hp_case **out) {
    hp_status st = case_from(std::move(s), &o, out);
    if (st != HP_OK) return st;
    // the initial load now lives on the device
    hp::Setup &h = (*out)->s;
    for (int k = 0; k < hp::MAXSP; k++) {
        std::vector<float>().swap(h.p_x[k]); std::vector<float>().swap(h.p_y[k]);
        std::vector<float>().swap(h.p_vx[k]); std::vector<float>().swap(h.p_vy[k]);
        std::vector<float>().swap(h.p_vz[k]);
        std::vector<float>().swap(h.h_x[k]); std::vector<float>().swap(h.h_y[k]);
        std::vector<float>().swap(h.h_vx[k]); std::vector<float>().swap(h.h_vy[k]);
        std::vector<float>().swap(h.h_vz[k]); std::vector<int>().swap(h.h_cell[k]);
    }
    return HP_OK;
}

size_t estimate_device_bytes(const hp::Setup &s, const hp_case_opts &o) {

    const size_t G = (size_t)s.Gsize, C = (size_t)s.Csize, nsp = (size_t)s.nsp;
    size_t b = 0;
    for (int k = 0; k < s.nsp; k++) {
        const size_t cap = (size_t)s.cap[k]; // already sized by the cap_per_cell option
        b += C * cap * 21 + C * (4 + 4 + 36 + 32);         // slots, counts, dcount, corner sums
    }
    b += nsp * C * (4 + 8 * HP_FAR_BUCKET) + 8 * C * 4;  // far buckets, channel counts
    b += G * (16 * 4 + 8 * 8 + 16 * nsp) + C * 16 + (size_t)s.cond_numr * G * 4;
    b += s.xsec.size() * 4 + s.vsave.size() * 4 + 3 * C * 4;
    if (o.field_mode == 2) b += 2 * ((size_t)s.ngx * s.ngx + (size_t)s.ngy * s.ngy) * 4 + 5 * G * 4;
    return b + b / 16 + (1u << 20); // allocation rounding and small arrays
}
} // namespace hpi

extern "C" {

hp_status hp_case_destroy(hp_case *c) {
    if (!c) return HP_OK;
    cudaSetDevice(c->device);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->own_stream) {
        cudaStreamSynchronize(c->own_stream);
        cudaStreamDestroy(c->own_stream);
    }
    fluid_fork_destroy(c->fl_fork);
    cudaDeviceSynchronize();
    for (void *p : c->allocs) cudaFree(p);
    hpi::fast_plan_free(c->fplan);
    delete c;
    return HP_OK;
}

hp_status hp_case_get_info(const hp_case *c, hp_case_info *out) {
    if (!c || !out) return HP_ERR_ARG;
    fill_info(c->s, out);
    out->device_bytes = c->bytes;
    out->pcg_cluster = c->pcg_cluster;
    out->field_mode = c->h.field_mode;
    out->mcc_stride = c->h.mcc_stride;
    out->pcg_block = c->lc.pcg_block;
    int64_t t = 0;
    cudaMemcpy(&t, c->h.tstep, 8, cudaMemcpyDeviceToHost);
    out->tstep = t;
    return HP_OK;
}

hp_status hp_case_status(hp_case *c, uint32_t *status) {
    if (!c || !status) return HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    CK(cudaMemcpy(status, c->h.status, 4, cudaMemcpyDeviceToHost));
    return HP_OK;
}

hp_status hp_case_set_tstep(hp_case *c, int64_t t) {
    if (!c) return HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    CK(cudaMemcpy(c->h.tstep, &t, 8, cudaMemcpyHostToDevice));
    return HP_OK;
}

#define OP_BODY(fn)                                                                                                    \
    if (!c) return HP_ERR_ARG;                                                                                         \
    if (c->batch) return set_error("case belongs to a batch"), HP_ERR_ARG;                                             \
    CK(cudaSetDevice(c->device));                                                                                      \
    hp_status st_ = fn(c, as_stream(stream));                                                                          \
    c->last_stream = as_stream(stream);                                                                                \
    return st_;

hp_status hp_Field(hp_case *c, void *stream) { OP_BODY(op_field) }
hp_status hp_Move(hp_case *c, void *stream) { OP_BODY(op_move) }
hp_status hp_SortBoundary(hp_case *c, void *stream) { OP_BODY(op_sort) }
hp_status hp_MCC(hp_case *c, void *stream) { OP_BODY(op_mcc) }
static hp_status op_deposit_step(hp_case *c, cudaStream_t st) { return op_deposit(c, st, true); }
hp_status hp_Deposit(hp_case *c, void *stream) { OP_BODY(op_deposit_step) }

hp_status hp_step(hp_case *c, int nsteps, void *stream) {
    if (!c || nsteps < 0) return HP_ERR_ARG;
    if (c->batch) return set_error("case belongs to a batch"), HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = as_stream(stream);
    if (!c->graph) {
        // capture one step on the case's own stream, after the caller's work
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CK(cudaEventRecord(ev, st));
        CK(cudaStreamWaitEvent(c->own_stream, ev, 0));
        CK(cudaEventDestroy(ev));
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(c->own_stream, cudaStreamCaptureModeThreadLocal));
        hp_status s1 = one_step(c, c->own_stream);
        cudaError_t e = cudaStreamEndCapture(c->own_stream, &g);
        if (s1 != HP_OK) return s1;
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        c->graph_kernels = hpi::count_kernel_nodes(g);
        e = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        CK(cudaStreamSynchronize(c->own_stream));
    }
    for (int k = 0; k < nsteps; k++) CK(cudaGraphLaunch(c->graph, st));
    c->last_stream = st;
    return HP_OK;
}

hp_status hp_profile_step(hp_case *c, int nsteps, void *stream, hp_kernel_stat *out, int cap, int *n) {
    if (!c || nsteps < 1 || !n || cap < 0 || (cap > 0 && !out)) return HP_ERR_ARG;
    if (c->batch) return set_error("case belongs to a batch"), HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = as_stream(stream);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return set_error("hp_profile_step cannot run inside a stream capture"), HP_ERR_ARG;
    std::vector<std::string> names;
    std::vector<int> launches;
    std::vector<double> ms;
    prof::begin();
    hp_status s1 = HP_OK;
    for (int k = 0; k < nsteps && s1 == HP_OK; k++) s1 = one_step(c, st);
    prof::mark_slow(st, nullptr); // closes the last kernel
    const bool ok = prof::end(names, launches, ms);
    c->last_stream = st;
    if (s1 != HP_OK) return s1;
    if (!ok) return cuda_fail(cudaGetLastError(), "profile events");
    *n = (int)names.size();
    for (int k = 0; k < (int)names.size() && k < cap; k++) {
        std::memset(out[k].name, 0, sizeof out[k].name);
        std::strncpy(out[k].name, names[k].c_str(), sizeof out[k].name - 1);
        out[k].launches = launches[k];
        out[k].ms = ms[k];
    }
    return HP_OK;
}

hp_status hp_case_set_tune(hp_case *c, const hp_tune *t) {
    if (!c || !t) return HP_ERR_ARG;
    if (c->batch) return set_error("case belongs to a batch: tune the batch"), HP_ERR_ARG;
    if (!hpi::tune_valid(*t)) return set_error("hp_tune out of range"), HP_ERR_ARG;
    c->lc.warps_per_block = t->warps_per_block_particles;
    c->lc.pcg_block = t->pcg_block;
    c->lc.pcg_cluster_max = t->pcg_cluster_max;
    c->lc.move_unroll = t->move_unroll;
    c->lc.mcc_cells = t->mcc_cells_per_warp;
    {
        const int gp = c->h.pcg_part ? pcg_grid_ctas(c->s.Gsize, t->pcg_block) : 0;
        c->pcg_cluster = gp > 0 ? gp : std::min(pcg_cluster_for_nodes(c->s.Gsize), t->pcg_cluster_max);
    }
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
        c->graph_kernels = 0;
    }
    return HP_OK;
}

hp_status hp_case_get_tune(const hp_case *c, hp_tune *t) {
    if (!c || !t) return HP_ERR_ARG;
    t->warps_per_block_particles = c->lc.warps_per_block;
    t->pcg_block = c->lc.pcg_block;
    t->pcg_cluster_max = c->lc.pcg_cluster_max;
    t->move_unroll = c->lc.move_unroll;
    t->mcc_cells_per_warp = c->lc.mcc_cells;
    return HP_OK;
}

hp_status hp_step_kernels(const hp_case *c, int *n) {
    if (!c || !n) return HP_ERR_ARG;
    *n = c->graph_kernels;
    return HP_OK;
}

hp_status hp_get_particles(hp_case *c, int isp, int *counts, float *x, float *y, float *vx, float *vy, float *vz,
                           size_t cap, size_t *n_out) {
    if (!c || isp < 0 || isp >= c->s.nsp) return HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    const int C = c->s.Csize;
    const DevSpecies &sp = c->h.sp[isp];
    std::vector<int> cnt(C);
    CK(cudaMemcpy(cnt.data(), sp.cnt, (size_t)C * 4, cudaMemcpyDeviceToHost));
    size_t total = 0;
    for (int v : cnt) total += (size_t)v;
    if (n_out) *n_out = total;
    if (counts) std::memcpy(counts, cnt.data(), (size_t)C * 4);
    if (!x) return HP_OK;
    if (cap < total) return set_error("output arrays too small"), HP_ERR_ARG;
    const size_t ns = (size_t)C * sp.cap;
    std::vector<float> b(ns);
    float *outs[5] = {x, y, vx, vy, vz};
    float *srcs[5] = {sp.x, sp.y, sp.vx, sp.vy, sp.vz};
    for (int a = 0; a < 5; a++) {
        if (!outs[a]) continue;
        CK(cudaMemcpy(b.data(), srcs[a], ns * 4, cudaMemcpyDeviceToHost));
        size_t q = 0;
        for (int cell = 0; cell < C; cell++)
            for (int k = 0; k < cnt[cell]; k++) outs[a][q++] = b[(size_t)cell * sp.cap + k];
    }
    return HP_OK;
}

hp_status hp_get_movers(hp_case *c, int isp, int *counts, float *x, float *y, float *vx, float *vy, float *vz,
                        int8_t *codes, size_t cap, size_t *n_out) {
    if (!c || isp < 0 || isp >= c->s.nsp) return HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    const int C = c->s.Csize;
    const DevSpecies &sp = c->h.sp[isp];
    std::vector<int> m(C);
    CK(cudaMemcpy(m.data(), sp.nmov, (size_t)C * 4, cudaMemcpyDeviceToHost));
    size_t total = 0;
    for (int v : m) total += (size_t)v;
    if (n_out) *n_out = total;
    if (counts) std::memcpy(counts, m.data(), (size_t)C * 4);
    if (!x) return HP_OK;
    if (cap < total) return set_error("output arrays too small"), HP_ERR_ARG;
    const size_t ns = (size_t)C * sp.cap;
    std::vector<float> b(ns);
    float *outs[5] = {x, y, vx, vy, vz};
    float *srcs[5] = {sp.x, sp.y, sp.vx, sp.vy, sp.vz};
    for (int a = 0; a < 5; a++) {
        CK(cudaMemcpy(b.data(), srcs[a], ns * 4, cudaMemcpyDeviceToHost));
        size_t q = 0;
        for (int cell = 0; cell < C; cell++)
            for (int r = 0; r < m[cell]; r++) outs[a][q++] = b[(size_t)cell * sp.cap + sp.cap - 1 - r];
    }
    if (codes) {
        std::vector<int8_t> cb(ns);
        CK(cudaMemcpy(cb.data(), sp.code, ns, cudaMemcpyDeviceToHost));
        size_t q = 0;
        for (int cell = 0; cell < C; cell++)
            for (int r = 0; r < m[cell]; r++) codes[q++] = cb[(size_t)cell * sp.cap + sp.cap - 1 - r];
    }
    return HP_OK;
}

hp_status hp_set_particles(hp_case *c, int isp, const int *counts, const float *x, const float *y, const float *vx,
                           const float *vy, const float *vz) {
    if (!c || isp < 0 || isp >= c->s.nsp || !counts) return HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    return upload_particles(c, isp, counts, x, y, vx, vy, vz);
}

static hp_status grid_ptr(hp_case *c, hp_grid_field f, void **p, size_t *nb) {
    const int G = c->s.Gsize, nsp = c->s.nsp;
    switch (f) {
    case HP_GRID_EX: *p = c->h.Ex; *nb = (size_t)G * 4; break;
    case HP_GRID_EY: *p = c->h.Ey; *nb = (size_t)G * 4; break;
    case HP_GRID_PHI: *p = c->h.phi; *nb = (size_t)G * 4; break;
    case HP_GRID_PHI_POIS: *p = c->h.phi_p; *nb = (size_t)G * 4; break;
    case HP_GRID_DEN: *p = c->h.den; *nb = (size_t)nsp * G * 8; break;
    case HP_GRID_SOURCE: *p = c->h.source; *nb = (size_t)G * 8; break;
    case HP_GRID_PCG_X:
        if (c->opts.field_mode == 0) { *p = c->h.pf_x; *nb = (size_t)G * 4; }
        else { *p = c->h.x64; *nb = (size_t)G * 8; }
        break;
    case HP_GRID_PCG_B: *p = c->h.b64; *nb = (size_t)G * 8; break;
    case HP_GRID_AVE_DEN: *p = c->h.ave_den; *nb = (size_t)nsp * G * 8; break;
    case HP_GRID_AVE_PHI: *p = c->h.ave_phi; *nb = (size_t)G * 8; break;
    case HP_GRID_AVE_SOURCE: *p = c->h.ave_src; *nb = (size_t)G * 8; break;
    case HP_GRID_AVE_EX: *p = c->h.ave_ex; *nb = (size_t)G * 8; break;
    case HP_GRID_AVE_EY: *p = c->h.ave_ey; *nb = (size_t)G * 8; break;
    case HP_GRID_COND_CHARGE: *p = c->h.cond_charge; *nb = (size_t)nsp * c->s.cond_numr * 4; break;
    case HP_GRID_MCC_COUNT: *p = c->h.mcc_count; *nb = (size_t)c->h.mcc_stride * c->s.Csize * 4; break;
    case HP_GRID_EEDF: *p = c->h.eedf; *nb = (size_t)(HP_EEDF_BINS + 1) * 8; break;
    case HP_GRID_SURFACE_CHARGE: *p = c->h.sig; *nb = c->h.sig ? (size_t)nsp * G * 8 : 0; break;
    case HP_GRID_SIGMA: *p = c->h.sigma; *nb = c->h.sigma ? (size_t)G * 8 : 0; break;
    case HP_GRID_SOURCE_AC: *p = c->h.src_amp; *nb = (size_t)c->s.src_num * 4; break;
    case HP_GRID_POWER_STATE: *p = c->h.pw; *nb = c->h.pw ? sizeof(PowerState) : 0; break;
    case HP_GRID_FLUID_CELL_DEN: *p = c->h.fden; *nb = (size_t)c->s.nfsp * c->s.Csize * 4; break;
    case HP_GRID_FLUID_DEN: *p = c->h.fluid_den; *nb = (size_t)c->s.nfsp * G * 4; break;
    case HP_GRID_FLUID_SOURCE: *p = c->h.fsrc; *nb = (size_t)c->s.nfsp * c->s.Csize * 4; break;
    case HP_GRID_FLUID_FLUX_X: *p = c->h.fflx; *nb = (size_t)c->s.nfsp * c->s.ngx * c->s.ncy * 4; break;
    case HP_GRID_FLUID_FLUX_Y: *p = c->h.ffly; *nb = (size_t)c->s.nfsp * c->s.ncx * c->s.ngy * 4; break;
    case HP_GRID_FLUID_STATE: *p = c->fl_state; *nb = c->fl_state_bytes; break;
    case HP_GRID_CIRCUIT: *p = c->h.cs; *nb = c->h.cs ? sizeof(CircuitState) : 0; break;
    default: return set_error("unknown grid field"), HP_ERR_ARG;
    }
    return HP_OK;
}

// device address and size of a grid field, for the checkpoint writer
hp_status hpi_grid_ptr(hp_case *c, hp_grid_field f, void **p, size_t *nb) { return grid_ptr(c, f, p, nb); }

hp_status hp_get_grid(hp_case *c, hp_grid_field f, void *out, size_t bytes) {
    if (!c || !out) return HP_ERR_ARG;
    void *p;
    size_t nb;
    TRY(grid_ptr(c, f, &p, &nb));
    if (bytes < nb) return set_error("output buffer too small (" + std::to_string(nb) + " needed)"), HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    if (nb) CK(cudaMemcpy(out, p, nb, cudaMemcpyDeviceToHost));
    return HP_OK;
}

hp_status hp_set_grid(hp_case *c, hp_grid_field f, const void *in, size_t bytes) {
    if (!c || !in) return HP_ERR_ARG;
    void *p;
    size_t nb;
    TRY(grid_ptr(c, f, &p, &nb));
    if (bytes != nb) return set_error("input size mismatch (" + std::to_string(nb) + " expected)"), HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    if (nb) CK(cudaMemcpy(p, in, nb, cudaMemcpyHostToDevice));
    return HP_OK;
}

hp_status hp_reset_averages(hp_case *c) {
    if (!c) return HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    CK(cudaMemset(c->h.ave_den, 0, (size_t)c->s.nsp * c->s.Gsize * 8));
    CK(cudaMemset(c->h.ave_phi, 0, (size_t)c->s.Gsize * 8));
    CK(cudaMemset(c->h.ave_src, 0, (size_t)c->s.Gsize * 8));
    CK(cudaMemset(c->h.ave_ex, 0, (size_t)c->s.Gsize * 8));
    CK(cudaMemset(c->h.ave_ey, 0, (size_t)c->s.Gsize * 8));
    CK(cudaMemset(c->h.ave_count, 0, 8));
    CK(cudaMemset(c->h.eedf, 0, (HP_EEDF_BINS + 1) * 8));
    c->mcc_base.resize((size_t)c->h.mcc_stride * c->s.Csize);
    CK(cudaMemcpy(c->mcc_base.data(), c->h.mcc_count, c->mcc_base.size() * 4, cudaMemcpyDeviceToHost));
    return HP_OK;
}

// The reference's averaged collision rates (Average_Argon/Oxygen/ArO2_MCC_rate,
// src/cuda_Diagnostic.cu:548-632): per node (the lower-left node of the cell
// the collision happened in) and reaction channel, the collisions since
// hp_reset_averages times Denscale of the channel's projectile species over
// (steps accumulated x dt), in the reference's float arithmetic.  Channels
// without a tally here (Ar 7-8, Ar/O2 68 and 71 on) are 0.
hp_status hp_get_mcc_rates(hp_case *c, float *out, size_t count) {
    if (!c || !out) return HP_ERR_ARG;
    const Setup &s = c->s;
    const int T = s.TnRct, G = s.Gsize, C = s.Csize, st = c->h.mcc_stride;
    if (count < (size_t)G * T) return set_error("output buffer too small (Gsize x TnRct floats)"), HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    std::vector<uint32_t> now((size_t)st * C);
    int64_t n = 0;
    CK(cudaMemcpy(now.data(), c->h.mcc_count, now.size() * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&n, c->h.ave_count, 8, cudaMemcpyDeviceToHost));
    std::fill(out, out + (size_t)G * T, 0.0f);
    if (n <= 0) return HP_OK;
    // projectile species of each channel (the reference's scaling ranges)
    std::vector<int> proj(T, -1);
    auto range = [&](int a, int b, int sp) { for (int k = a; k <= b && k < T; k++) proj[k] = sp; };
    if (s.main_gas == GAS_AR) range(0, 6, 0);
    else if (s.main_gas == GAS_O2) { range(0, 40, 0); range(41, 46, 3); range(47, 52, 1); range(53, 57, 2); range(58, 58, 3); }
    else { range(0, 45, 0); range(46, 51, 4); range(52, 59, 2); range(60, 64, 3); range(65, 67, 1); range(69, 70, 3); }
    for (int k = 0; k < T && k < st; k++) {
        if (proj[k] < 0) continue;
        const float temp = s.sp[proj[k]].Denscale / (float)n / s.dt;
        for (int cell = 0; cell < C; cell++) {
            const size_t q = (size_t)cell * st + k;
            const uint32_t cnt = now[q] - (c->mcc_base.empty() ? 0u : c->mcc_base[q]);
            const int i = cell / s.ncy, j = cell - i * s.ncy;
            out[(size_t)(i * s.ngy + j) * T + k] = temp * (float)cnt;
        }
    }
    return HP_OK;
}

hp_status hp_get_average_count(hp_case *c, int64_t *n) {
    if (!c || !n) return HP_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    CK(cudaMemcpy(n, c->h.ave_count, 8, cudaMemcpyDeviceToHost));
    return HP_OK;
}

hp_status hp_case_pushes(hp_case *c, int64_t *pushes) {
    if (!c || !pushes) return HP_ERR_ARG;
    unsigned long long v[32];
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    CK(cudaMemcpy(v, c->h.pushes, sizeof v, cudaMemcpyDeviceToHost));
    int64_t t = 0;
    for (int k = 0; k < 32; k++) t += (int64_t)v[k];
    *pushes = t;
    return HP_OK;
}

hp_status hp_case_slot_changes(hp_case *c, int64_t *changes) {
    if (!c || !changes) return HP_ERR_ARG;
    unsigned long long v[32];
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    CK(cudaMemcpy(v, c->h.pushes + 32, sizeof v, cudaMemcpyDeviceToHost));
    int64_t t = 0;
    for (int k = 0; k < 32; k++) t += (int64_t)v[k];
    *changes = t;
    return HP_OK;
}

hp_status hp_last_field_residual(hp_case *c, double *rel) {
    if (!c || !rel) return HP_ERR_ARG;
    *rel = -1.0;
    if (c->h.field_mode != 2) return HP_OK;
    double v[2];
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    CK(cudaMemcpy(v, c->h.fs_res, sizeof v, cudaMemcpyDeviceToHost));
    *rel = v[1] > 0 ? v[0] / v[1] : 0.0;
    return HP_OK;
}

hp_status hp_last_pcg_iters(hp_case *c, int *inner, int *outer) {
    if (!c) return HP_ERR_ARG;
    int v[2];
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->last_stream));
    CK(cudaMemcpy(v, c->h.pcg_iters, 8, cudaMemcpyDeviceToHost));
    if (inner) *inner = v[0];
    if (outer) *outer = v[1];
    return HP_OK;
}

} // extern "C"
