// ref_kernels.cu -- test harness that runs the reference's own CUDA step code
// on states the tests supply (test infrastructure, never linked into the
// product).
//
// oracle/Makefile target `ref_kernels` compiles the reference's
// src/cuda_Move.cu, cuda_Sortboundary.cu, cuda_Deposit.cu, cuda_Field.cu,
// cuda_mcc.cu, cuda_mccAr.cu, cuda_mccO2.cu, cuda_mccArO2.cu and
// Variables.cu where they lie, unedited, for sm_100a with the reference's own
// flags (-use_fast_math -rdc=true) and the pre-include oracle/ref_shim.h, and
// links them with this file into oracle/_ref/libref_kernels.so.  The entry
// points below take host arrays in the reference's own layout, copy them into
// the reference's structs (GCP, GPG, GGA, GCA, Species, CollF, ...; inc/def.h),
// launch the reference kernel or device function, and copy the result back.
// The tests compare those results with the oracle's restatement on the same
// inputs, which pins the restatement to the reference's code.
//
// Layout of particles (the reference's: inc/def.h GCP, src/cuda_Move.cu:195):
// node ID = i * ngy + j, particle k of (species isp, node ID) at
//   isp * MAXNP + ID + k * Gsize,  MAXNP = mpnc * Gsize,
// where mpnc is the slots per node (the reference's MaxPtNumInCell).
//
// Every entry checks the indices its kernel will form against the buffers on
// the host before the launch (counts within the slots, particles only in
// nodes that own a cell, StructureIndex codes within the conductor list) and
// returns an error instead of launching when one would fall outside.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

// the reference's structs (inc/def.h, through its common header); its other
// headers re-include def.h, so the kernels used here are declared below with
// the signatures of their definitions
#include "xypic.cuh"
// inc/def.h's function-like min/max would shadow std::min/std::max here
#undef min
#undef max

#define RK_HANDLER(name)                                                                                            \
    __device__ void name(int Gsize, int ngy, int TID, int nvel, float *vsave, curandState *states, Species *info,   \
                         GPG *data, GCP *sp, int N_LOGX, float idLOGX, MCC_sigmav *sigv, CollF *info_CX,          \
                         RK_TABLE *CX, int TnRct, float *MCCR, GGA *BG)

// src/cuda_Move.cu:181
__global__ void MoveE_Basic(int Gsize, int ngy, float dt_dx, float dt_dy, Species *info, GCP *sp, GPG *data, GGA *Field);
// src/cuda_Sortboundary.cu:41
__global__ void SortBoundary_Basic(int Gsize, int ngy, int CondNum, float dt_dx, float dt_dy, int *StructureIndex,
                                   Species *info, GCP *sp, GPG *data, GGA *Field, float *Cond, int *ReArgFlag);
// src/cuda_Deposit.cu:35,277,289,318
__global__ void SumSource(int nsp, int Gsize, int ngx, int ngy, Species *info, GGA *vecSet, GPG *data, float *Sigma,
                          float *Source);
__global__ void DepositBoundary(int Gsize, int ngy, int nsp, GGA *vecSet, GPG *data);
__global__ void DepositAtom(int Gsize, int ngy, Species *info, GCP *sp, GPG *data);
__global__ void DepositInitDensity(int Gsize, Species *info, GPG *data);
// src/cuda_Field.cu:500,698,942
__global__ void Cond_Sigma(int ngx, int ngy, float hdx, float hdy, float idxy, float zlength, GGA *vecG, GCA *vecC,
                           Species *info, GPG *data, float *Phi, float *Sigma);
__global__ void VtoEfield(int ngx, int ngy, float dx, float dy, float hdx, float hdy, float idx, float idy,
                          float *Sigma, float *Phi, GPG *data, GCA *vecC, GGA *vecG);
__global__ void PCG_float(int *I, int *J, float *val, float *x, float *M, float *Ax, float *p, float *r, float *Z,
                          int N, int nnz, float tol2, int *Iter, float *d_result);
// src/cuda_mcc.cu:97,139,148,174
__global__ void MCC_Ar_Basic(int Gsize, int Csize, int ngy, int nsp, float dt, int MCCn, float dtm, float idx,
                             float idy, int nvel, float *vsave, curandState *states, int N_LOGX, float idLOGX,
                             MCC_sigmav *sigv, CollF *CollP, ArCollD *CX, int TnRct, float *MCCR, float *Stack,
                             Fluid *infoF, GFG *Fluid, GGA *BG, Species *info, GPG *data, GCP *sp);
__device__ void dev_maxwellv(float *vx_local, float *vy_local, float *vz_local, float vsaven, float vti, float Rphi,
                             float Rthe);
__device__ void dev_anewvel(float energy, float vel, float *n_vx, float *n_vy, float *n_vz, int e_flag,
                            float massrate, float rand1, float rand2);
__device__ void dev_newvel_IONSC(float *vx_sc, float *vy_sc, float *vz_sc, float vel, float rand1, float rand2);
// src/cuda_Diagnostic.cu:634,643,684
__global__ void Argon_Update_Source(int Gsize, int ngy, int TnRct, float *MCCR, CollF *CollP, GPG *SP, GFG *FG,
                                    GFG *FG_S, GGA *BG);
__global__ void Oxygen_Update_Source(int Gsize, int TnRct, float *MCCR, CollF *CollP, GPG *SP, GFG *FG, GFG *FG_S,
                                     GGA *BG);
__global__ void ArO2_Update_Source(int Gsize, int ngy, int TnRct, float *MCCR, CollF *CollP, GPG *SP, GFG *FG,
                                   GFG *FG_S, GGA *BG);
// src/cuda_mccAr.cu:707, src/cuda_mccO2.cu:978, src/cuda_mccArO2.cu:2461
__device__ float Argon_CrossSection(int R, float engy, int N_LOGX, float idLOGX, ArCollD *data);
__device__ float O2_CrossSection(int R, float engy, int N_LOGX, float idLOGX, O2CollD *data);
__device__ float ArO2_CrossSection(int R, float engy, int N_LOGX, float idLOGX, ArO2CollD *data);
// species handlers: src/cuda_mccArO2.cu:51,561,672,843,986 and src/cuda_mccO2.cu:2,430,576,719
#define RK_TABLE ArO2CollD
RK_HANDLER(ArO2_Electron);
RK_HANDLER(ArO2_Ar_ion);
RK_HANDLER(ArO2_O2_ion);
RK_HANDLER(ArO2_O_ion);
RK_HANDLER(ArO2_O_negative);
#undef RK_TABLE
#define RK_TABLE O2CollD
RK_HANDLER(O2_Electron);
RK_HANDLER(O2_O2_ion);
RK_HANDLER(O2_O_ion);
RK_HANDLER(O2_O_negative);
#undef RK_TABLE

// ------------------------------------------------------------ scripted draws
// Each thread's list: u[start[key] .. start[key + 1]), key = global thread
// index (the reference's TID for its per-node MCC kernels).
__device__ const float *g_rk_u;
__device__ const long long *g_rk_start;
__device__ int *g_rk_pos;
__device__ int g_rk_nkeys;
__device__ unsigned long long g_rk_overrun;

__device__ float hp_ref_uniform(curandState *) {
    const int key = (int)(threadIdx.x + blockIdx.x * blockDim.x);
    if (key >= g_rk_nkeys) {
        atomicAdd(&g_rk_overrun, 1ull);
        return 1.0f;
    }
    const int p = g_rk_pos[key];
    const long long at = g_rk_start[key] + p;
    if (at >= g_rk_start[key + 1]) {
        atomicAdd(&g_rk_overrun, 1ull);
        return 1.0f;
    }
    g_rk_pos[key] = p + 1;
    return g_rk_u[at];
}

namespace {

std::string g_err;

struct Fail {
    int code;
};

void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        g_err = std::string(what) + ": " + cudaGetErrorString(e);
        throw Fail{(int)e};
    }
}
void need(bool ok, const std::string &why) {
    if (!ok) {
        g_err = why;
        throw Fail{-1};
    }
}

// device buffers freed when the call returns
struct Arena {
    std::vector<void *> ptrs;
    ~Arena() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T> T *alloc(size_t n) {
        void *p = nullptr;
        ck(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
        ptrs.push_back(p);
        ck(cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T)), "cudaMemset");
        return (T *)p;
    }
    template <class T> T *put(const T *h, size_t n) {
        T *d = alloc<T>(n);
        if (n) ck(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
        return d;
    }
    template <class T> T *put(const std::vector<T> &h) { return put(h.data(), h.size()); }
};
template <class T> void get(std::vector<T> &h, const T *d) {
    if (!h.empty()) ck(cudaMemcpy(h.data(), d, h.size() * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
}

unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

void sync(const char *what) {
    ck(cudaGetLastError(), what);
    ck(cudaDeviceSynchronize(), what);
}

// Optional timing (rk_set_timing): before its checked launch, each timed
// kernel runs `g_reps` more times, every time on a restored copy of its
// inputs, with the launch shape the reference picks at start-up
// (cudaOccupancyMaxPotentialBlockSize over Gsize*nsp threads,
// src/cuda_Init.cu:35-46), bracketed by CUDA events; g_ms[k] is the mean
// time of the k-th timed kernel of the last call.
int g_reps = 0;
float g_ms[8] = {};

template <class K> int ref_block(K kern, long long nthreads) {
    int mingrid = 0, block = 0;
    ck(cudaOccupancyMaxPotentialBlockSize(&mingrid, &block, kern, 0, (int)std::min<long long>(nthreads, 1 << 30)),
       "cudaOccupancyMaxPotentialBlockSize");
    need(block > 0, "no launchable block size");
    return block;
}

template <class T> void restore(T *dst, const T *src, size_t n) {
    if (n) ck(cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice), "cudaMemcpy D2D");
}
template <class T> T *snapshot(Arena &a, const T *d, size_t n) {
    T *p = a.alloc<T>(n);
    restore(p, d, n);
    return p;
}

// events around nk kernels launched back to back on the default stream
struct Timed {
    cudaEvent_t e[9];
    int nk;
    explicit Timed(int n) : nk(n) {
        for (int k = 0; k <= nk; k++) ck(cudaEventCreate(&e[k]), "cudaEventCreate");
        std::fill(g_ms, g_ms + 8, 0.f);
    }
    ~Timed() {
        for (int k = 0; k <= nk; k++) cudaEventDestroy(e[k]);
    }
    void mark(int k) { ck(cudaEventRecord(e[k]), "cudaEventRecord"); }
    void add() {
        ck(cudaEventSynchronize(e[nk]), "cudaEventSynchronize");
        for (int k = 0; k < nk; k++) {
            float t = 0.f;
            ck(cudaEventElapsedTime(&t, e[k], e[k + 1]), "cudaEventElapsedTime");
            g_ms[k] += t / (float)g_reps;
        }
    }
};

template <class F> int guarded(F f) {
    try {
        g_err.clear();
        f();
        return 0;
    } catch (Fail &e) {
        return e.code ? e.code : -1;
    }
}

} // namespace

extern "C" {

// Per-case constants shared by the entry points (host side).
typedef struct rk_case {
    int ngx, ngy, nsp, mpnc;
    float dt_dx, dt_dy;
    float ascale[5], q_density[5], escale[5], np2c[5];
} rk_case;

const char *rk_last_error(void) { return g_err.c_str(); }

/* Timing of the reference kernels: reps > 0 makes rk_move and rk_deposit
 * first run their kernels reps times on restored copies of the inputs with
 * the reference's launch shape, timed with CUDA events (0 turns it off).
 * rk_last_ms copies the mean times of the last timed call: rk_move
 * {MoveE_Basic}; rk_deposit {DepositInitDensity, DepositAtom,
 * DepositBoundary, SumSource}. */
void rk_set_timing(int reps) { g_reps = reps > 0 ? reps : 0; }
void rk_last_ms(float *out8) { std::memcpy(out8, g_ms, sizeof(g_ms)); }

} // extern "C"

namespace {

struct Dims {
    int G, nsp, mpnc;
    long long maxnp;
};
Dims dims(const rk_case *c) {
    need(c->ngx >= 2 && c->ngy >= 2 && c->nsp >= 1 && c->nsp <= 5 && c->mpnc >= 1, "bad case dimensions");
    Dims d;
    d.G = c->ngx * c->ngy;
    d.nsp = c->nsp;
    d.mpnc = c->mpnc;
    d.maxnp = (long long)c->mpnc * d.G;
    return d;
}

std::vector<Species> species(const rk_case *c, const Dims &d) {
    std::vector<Species> s((size_t)d.nsp);
    for (int i = 0; i < d.nsp; i++) {
        std::memset(&s[(size_t)i], 0, sizeof(Species));
        s[(size_t)i].spnum = d.nsp;
        s[(size_t)i].MAXNP = (int)d.maxnp;
        s[(size_t)i].St_num = (int)(i * d.maxnp);
        s[(size_t)i].End_num = (int)((i + 1) * d.maxnp - 1);
        s[(size_t)i].Ascale = c->ascale[i];
        s[(size_t)i].q_density = c->q_density[i];
        s[(size_t)i].Escale = c->escale[i];
        s[(size_t)i].np2c = c->np2c[i];
    }
    return s;
}

// particles only in nodes that own a cell, counts within the slots
void check_counts(const rk_case *c, const Dims &d, const int *pnc, int limit) {
    for (int s = 0; s < d.nsp; s++)
        for (int id = 0; id < d.G; id++) {
            const int n = pnc[(size_t)s * d.G + id];
            const int i = id / c->ngy, j = id % c->ngy;
            need(n >= 0 && n <= limit, "particle count outside [0, " + std::to_string(limit) + "]");
            need(n == 0 || (i < c->ngx - 1 && j < c->ngy - 1), "particles in a node that owns no cell");
        }
}

std::vector<GCP> pack(const Dims &d, const float *x, const float *y, const float *vx, const float *vy,
                      const float *vz, const int *cellid) {
    const size_t n = (size_t)(d.nsp * d.maxnp);
    std::vector<GCP> p(n);
    for (size_t k = 0; k < n; k++) {
        p[k].CellID = cellid ? cellid[k] : 0;
        p[k].x = x[k];
        p[k].y = y[k];
        p[k].vx = vx[k];
        p[k].vy = vy[k];
        p[k].vz = vz[k];
    }
    return p;
}
void unpack(const std::vector<GCP> &p, float *x, float *y, float *vx, float *vy, float *vz, int *cellid) {
    for (size_t k = 0; k < p.size(); k++) {
        if (cellid) cellid[k] = p[k].CellID;
        x[k] = p[k].x;
        y[k] = p[k].y;
        vx[k] = p[k].vx;
        vy[k] = p[k].vy;
        vz[k] = p[k].vz;
    }
}

std::vector<GPG> gpg(const Dims &d, const int *pnc, const int *pnmc) {
    std::vector<GPG> g((size_t)d.nsp * d.G);
    for (size_t k = 0; k < g.size(); k++) {
        std::memset(&g[k], 0, sizeof(GPG));
        g[k].PtNumInCell = pnc ? pnc[k] : 0;
        g[k].PtNumMoveInterCell = pnmc ? pnmc[k] : 0;
        g[k].MaxPtNumInCell = d.mpnc;
    }
    return g;
}

// thread lists of scripted uniforms
struct Script {
    float *u = nullptr;
    long long *start = nullptr;
    int *pos = nullptr;
};
void set_script(Arena &a, const float *u, const long long *start, int nkeys) {
    need(nkeys >= 0 && (nkeys == 0 || start[0] == 0), "bad script offsets");
    for (int k = 0; k < nkeys; k++) need(start[k + 1] >= start[k], "script offsets must not decrease");
    const long long total = nkeys ? start[nkeys] : 0;
    const float *du = a.put(u, (size_t)total);
    const long long *ds = a.put(start, (size_t)nkeys + 1);
    int *dp = a.alloc<int>((size_t)nkeys);
    unsigned long long zero = 0;
    ck(cudaMemcpyToSymbol(g_rk_u, &du, sizeof(du)), "script");
    ck(cudaMemcpyToSymbol(g_rk_start, &ds, sizeof(ds)), "script");
    ck(cudaMemcpyToSymbol(g_rk_pos, &dp, sizeof(dp)), "script");
    ck(cudaMemcpyToSymbol(g_rk_nkeys, &nkeys, sizeof(int)), "script");
    ck(cudaMemcpyToSymbol(g_rk_overrun, &zero, sizeof(zero)), "script");
}
long long script_overrun() {
    unsigned long long v = 0;
    ck(cudaMemcpyFromSymbol(&v, g_rk_overrun, sizeof(v)), "script overrun");
    return (long long)v;
}

__global__ void k_xsec(int gas, int ch, int n_logx, float idlogx, const float *tab, const float *e, float *out, int n) {
    const int k = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= n) return;
    if (gas == 0) out[k] = Argon_CrossSection(ch, e[k], n_logx, idlogx, (ArCollD *)tab);
    else if (gas == 1) out[k] = O2_CrossSection(ch, e[k], n_logx, idlogx, (O2CollD *)tab);
    else out[k] = ArO2_CrossSection(ch, e[k], n_logx, idlogx, (ArO2CollD *)tab);
}

__global__ void k_kin(int kind, const float *in, float *out, int n) {
    const int k = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= n) return;
    float x = 0.f, y = 0.f, z = 0.f;
    if (kind == 0) {
        const float *a = in + 7 * (size_t)k;
        x = a[2]; y = a[3]; z = a[4];
        dev_anewvel(a[0], a[1], &x, &y, &z, 0, 0.f, a[5], a[6]);
    } else if (kind == 1) {
        const float *a = in + 6 * (size_t)k;
        x = a[0]; y = a[1]; z = a[2];
        dev_newvel_IONSC(&x, &y, &z, a[3], a[4], a[5]);
    } else {
        const float *a = in + 4 * (size_t)k;
        dev_maxwellv(&x, &y, &z, a[0], a[1], a[2], a[3]);
    }
    out[3 * (size_t)k] = x;
    out[3 * (size_t)k + 1] = y;
    out[3 * (size_t)k + 2] = z;
}

// one collider per thread: thread ID is node ID of species isp (TID = isp * G + ID)
__global__ void k_oxy(int gas, int isp, int G, int ngy, int nvel, float *vsave, curandState *states, Species *info,
                      GPG *data, GCP *sp, int n_logx, float idlogx, MCC_sigmav *sigv, CollF *collf, void *cx,
                      int tnrct, float *mccr, GGA *bg) {
    const int id = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (id >= G) return;
    const int tid = isp * G + id;
    if (gas == 2) {
        ArO2CollD *t = (ArO2CollD *)cx;
        switch (isp) {
        case 0: ArO2_Electron(G, ngy, tid, nvel, vsave, states, info, data, sp, n_logx, idlogx, sigv, collf, t, tnrct, mccr, bg); break;
        case 1: ArO2_Ar_ion(G, ngy, tid, nvel, vsave, states, info, data, sp, n_logx, idlogx, sigv, collf, t, tnrct, mccr, bg); break;
        case 2: ArO2_O2_ion(G, ngy, tid, nvel, vsave, states, info, data, sp, n_logx, idlogx, sigv, collf, t, tnrct, mccr, bg); break;
        case 3: ArO2_O_ion(G, ngy, tid, nvel, vsave, states, info, data, sp, n_logx, idlogx, sigv, collf, t, tnrct, mccr, bg); break;
        default: ArO2_O_negative(G, ngy, tid, nvel, vsave, states, info, data, sp, n_logx, idlogx, sigv, collf, t, tnrct, mccr, bg); break;
        }
    } else {
        O2CollD *t = (O2CollD *)cx;
        switch (isp) {
        case 0: O2_Electron(G, ngy, tid, nvel, vsave, states, info, data, sp, n_logx, idlogx, sigv, collf, t, tnrct, mccr, bg); break;
        case 1: O2_O2_ion(G, ngy, tid, nvel, vsave, states, info, data, sp, n_logx, idlogx, sigv, collf, t, tnrct, mccr, bg); break;
        case 2: O2_O_ion(G, ngy, tid, nvel, vsave, states, info, data, sp, n_logx, idlogx, sigv, collf, t, tnrct, mccr, bg); break;
        default: O2_O_negative(G, ngy, tid, nvel, vsave, states, info, data, sp, n_logx, idlogx, sigv, collf, t, tnrct, mccr, bg); break;
        }
    }
}

// Replays SortBoundary_Basic's reads and index arithmetic
// (src/cuda_Sortboundary.cu:58-236) on the device state without writing any
// of it: every index is checked before it is used, arrivals are counted in
// `arr`, and out[] receives {movers, SMCID out of range, CID out of range,
// slot out of range, the largest slot, codes seen outside the handled set,
// the smallest and largest cell offset read}.
__global__ void k_sort_probe(int G, int ngy, int nsp, int mpnc, int ns, const int *sidx, const GCP *sp,
                             const GPG *data, int *arr, long long *out) {
    const int TID = (int)(threadIdx.x + blockIdx.x * blockDim.x);
    if (TID >= G * nsp) return;
    const int isp = TID / G, ID = TID % G, x = ID / ngy;
    const int PNMIC = data[TID].PtNumMoveInterCell;
    if (PNMIC <= 0) return;
    const long long maxnp = (long long)mpnc * G;
    long long i = isp * maxnp + ID + (long long)(mpnc - 1) * G;
    for (int k = 0; k < PNMIC && k < mpnc; k++, i -= G) {
        atomicAdd((unsigned long long *)&out[0], 1ull);
        if (i < isp * maxnp || i >= (isp + 1) * maxnp) { atomicAdd((unsigned long long *)&out[3], 1ull); continue; }
        const int MCID = sp[i].CellID;
        atomicMin(&out[6], (long long)MCID);
        atomicMax(&out[7], (long long)MCID);
        int SM;
        if (MCID > 1) SM = (ID + ngy + 2 + x) + (MCID + 1);
        else if (MCID < -1) SM = (ID + ngy + 2 + x) + (MCID - 1);
        else SM = (ID + ngy + 2 + x) + MCID;
        if (SM < 0 || SM >= ns) { atomicAdd((unsigned long long *)&out[1], 1ull); continue; }
        const int S = sidx[SM];
        int sum = 0;
        bool keep = true;
        switch (S) {
        case 0: break;
        case -2: sum = ngy; break;
        case -6: sum = -ngy; break;
        case -4: sum = 1; break;
        case -8: sum = -1; break;
        case -12: sum = ngy + 1; break;
        case -16: sum = 1 - ngy; break;
        case -20: sum = ngy - 1; break;
        case -24: sum = -ngy - 1; break;
        case -1: keep = false; break;
        default:
            keep = false;
            if (S < 100) atomicAdd((unsigned long long *)&out[5], 1ull);
        }
        if (!keep) continue;
        const int CID = TID + MCID + sum;
        if (CID < isp * G || CID >= (isp + 1) * G) { atomicAdd((unsigned long long *)&out[2], 1ull); continue; }
        const int old = data[CID].PtNumInCell + atomicAdd(&arr[CID], 1);
        atomicMax(&out[4], (long long)old);
        if (old >= mpnc) atomicAdd((unsigned long long *)&out[3], 1ull);
    }
}

// a cross-section table with one zero row past its end: the reference's
// lookup reads row ee2 + 1 when log10(E) lands on the last grid point
std::vector<float> padded_table(const float *tab, int n_logx, int width) {
    std::vector<float> t((size_t)(n_logx + 1) * width, 0.f);
    std::memcpy(t.data(), tab, (size_t)n_logx * width * sizeof(float));
    return t;
}
int table_width(int gas) {
    return gas == 0 ? (int)(sizeof(ArCollD) / 4) : gas == 1 ? (int)(sizeof(O2CollD) / 4) : (int)(sizeof(ArO2CollD) / 4);
}

} // namespace

extern "C" {

/* MoveE_Basic (src/cuda_Move.cu:181-270) on the given state.  pnc[nsp*G]
 * in: particles per node; out: stayers.  pnmc[nsp*G] out: movers.  The
 * particle arrays (nsp * mpnc * G each) are updated in place; movers sit at
 * the top slots with CellID the cell offset the reference encodes. */
int rk_move(const rk_case *c, const float *ex, const float *ey, int *pnc, int *pnmc, float *x, float *y, float *vx,
            float *vy, float *vz, int *cellid) {
    return guarded([&] {
        const Dims d = dims(c);
        check_counts(c, d, pnc, d.mpnc);
        Arena a;
        std::vector<Species> info = species(c, d);
        std::vector<GGA> f((size_t)d.G);
        for (int k = 0; k < d.G; k++) {
            std::memset(&f[(size_t)k], 0, sizeof(GGA));
            f[(size_t)k].Ex = ex[k];
            f[(size_t)k].Ey = ey[k];
        }
        std::vector<GCP> sp = pack(d, x, y, vx, vy, vz, cellid);
        std::vector<GPG> g = gpg(d, pnc, nullptr);
        Species *di = a.put(info);
        GGA *df = a.put(f);
        GCP *ds = a.put(sp);
        GPG *dg = a.put(g);
        if (g_reps > 0) {
            const GCP *ds0 = snapshot(a, ds, sp.size());
            const GPG *dg0 = snapshot(a, dg, g.size());
            const long long nt = (long long)d.nsp * d.G;
            const int b = ref_block(MoveE_Basic, nt);
            Timed t(1);
            for (int r = 0; r < g_reps; r++) {
                restore(ds, ds0, sp.size());
                restore(dg, dg0, g.size());
                t.mark(0);
                MoveE_Basic<<<blocks(nt, b), b>>>(d.G, c->ngy, c->dt_dx, c->dt_dy, di, ds, dg, df);
                t.mark(1);
                t.add();
            }
            sync("MoveE_Basic (timed)");
            restore(ds, ds0, sp.size());
            restore(dg, dg0, g.size());
        }
        MoveE_Basic<<<blocks((long long)d.nsp * d.G, 256), 256>>>(d.G, c->ngy, c->dt_dx, c->dt_dy, di, ds, dg, df);
        sync("MoveE_Basic");
        get(sp, ds);
        get(g, dg);
        unpack(sp, x, y, vx, vy, vz, cellid);
        for (size_t k = 0; k < g.size(); k++) {
            pnc[k] = g[k].PtNumInCell;
            pnmc[k] = g[k].PtNumMoveInterCell;
        }
    });
}

/* SortBoundary_Basic (src/cuda_Sortboundary.cu:41-258) after rk_move:
 * movers re-binned by atomics (so their order inside a cell is the arrival
 * order), Neumann reflections, Dirichlet and conductor absorption.
 * sidx[(ngx+1)*(ngy+1)] is the StructureIndex (src/start.c:1776-1851);
 * cond[nsp*cond_num] receives the conductor counts; *rearg the reference's
 * ReArgFlag (it is reported, ReArgPtcls is not run). */
int rk_sortboundary(const rk_case *c, int cond_num, const int *sidx, int *pnc, int *pnmc, float *x, float *y,
                    float *vx, float *vy, float *vz, int *cellid, float *cond, int *rearg) {
    return guarded([&] {
        const Dims d = dims(c);
        check_counts(c, d, pnc, d.mpnc);
        const int ns = (c->ngx + 1) * (c->ngy + 1);
        // SortBoundary_Basic acts on the codes 0, 1-99, 100+, -1, -2, -4, -6,
        // -8, -12, -16, -20, -24 (src/cuda_Sortboundary.cu:90-236).  Others
        // (the -3, -5, -7 the set-up writes next to some corners) leave its
        // destination offset uninitialised, so a mover entering such a cell
        // would be written to an undefined slot: they are passed as -1
        // (absorbed), which is the oracle's defined behaviour for them.
        std::vector<int> code(sidx, sidx + ns);
        for (int k = 0; k < ns; k++) {
            const int v = code[(size_t)k];
            const bool handled = v >= 0 || v == -1 || v == -2 || v == -4 || v == -6 || v == -8 || v == -12 ||
                                 v == -16 || v == -20 || v == -24;
            if (!handled) code[(size_t)k] = -1;
            need(v < 100 || (v >= 101 && v <= 100 + cond_num), "StructureIndex conductor code beyond the list");
            need(v < 1 || v >= 100, "dielectric cells are not supported here");
        }
        // every destination can hold its stayers plus all movers of its 3x3
        // neighbourhood, its own reflected ones included
        int most = 0;
        for (int k = 0; k < d.nsp * d.G; k++) most = std::max(most, pnc[k] + pnmc[k]);
        need(10LL * most < d.mpnc, "slots per node too few for the re-binning");
        Arena a;
        std::vector<Species> info = species(c, d);
        std::vector<GCP> sp = pack(d, x, y, vx, vy, vz, cellid);
        std::vector<GPG> g = gpg(d, pnc, pnmc);
        Species *di = a.put(info);
        GCP *ds = a.put(sp);
        GPG *dg = a.put(g);
        GGA *df = a.alloc<GGA>((size_t)d.G);
        int *dsi = a.put(code);
        float *dc = a.alloc<float>((size_t)d.nsp * std::max(cond_num, 1));
        int *dr = a.alloc<int>(1);
        SortBoundary_Basic<<<blocks((long long)d.nsp * d.G, 256), 256>>>(d.G, c->ngy, cond_num, c->dt_dx, c->dt_dy, dsi, di,
                                                                          ds, dg, df, dc, dr);
        sync("SortBoundary_Basic");
        get(sp, ds);
        get(g, dg);
        unpack(sp, x, y, vx, vy, vz, cellid);
        for (size_t k = 0; k < g.size(); k++) {
            pnc[k] = g[k].PtNumInCell;
            pnmc[k] = g[k].PtNumMoveInterCell;
        }
        std::vector<float> hc((size_t)d.nsp * std::max(cond_num, 1));
        get(hc, dc);
        if (cond) std::memcpy(cond, hc.data(), (size_t)d.nsp * cond_num * sizeof(float));
        if (rearg) ck(cudaMemcpy(rearg, dr, sizeof(int), cudaMemcpyDeviceToHost), "rearg");
    });
}

/* A read-only replay of SortBoundary_Basic's index arithmetic on the same
 * inputs as rk_sortboundary (k_sort_probe); out[8] as described there, and
 * regs_local[2] the reference kernel's registers per thread and local bytes. */
int rk_sort_probe(const rk_case *c, const int *sidx, const int *pnc, const int *pnmc, const int *cellid,
                  long long *out, int *regs_local) {
    return guarded([&] {
        const Dims d = dims(c);
        check_counts(c, d, pnc, d.mpnc);
        const int ns = (c->ngx + 1) * (c->ngy + 1);
        Arena a;
        const size_t n = (size_t)(d.nsp * d.maxnp);
        std::vector<GCP> sp(n);
        for (size_t k = 0; k < n; k++) {
            std::memset(&sp[k], 0, sizeof(GCP));
            sp[k].CellID = cellid[k];
        }
        std::vector<GPG> g = gpg(d, pnc, pnmc);
        GCP *ds = a.put(sp);
        GPG *dg = a.put(g);
        int *dsi = a.put(sidx, (size_t)ns);
        int *darr = a.alloc<int>((size_t)d.nsp * d.G);
        std::vector<long long> h(8, 0);
        h[6] = 1ll << 40;
        h[7] = -(1ll << 40);
        long long *dout = a.put(h);
        k_sort_probe<<<blocks((long long)d.nsp * d.G, 256), 256>>>(d.G, c->ngy, d.nsp, d.mpnc, ns, dsi, ds, dg, darr, dout);
        sync("sort probe");
        get(h, dout);
        std::memcpy(out, h.data(), 8 * sizeof(long long));
        cudaFuncAttributes fa;
        ck(cudaFuncGetAttributes(&fa, SortBoundary_Basic), "attributes");
        regs_local[0] = fa.numRegs;
        regs_local[1] = (int)fa.localSizeBytes;
    });
}

/* Deposit_Basic's kernels (src/cuda_Deposit.cu:3-104,277-325):
 * DepositInitDensity, DepositAtom, DepositBoundary, SumSource.  face,
 * boundary, cond_id, area [G]; sigma_in [nsp*G] the dielectric surface
 * charge (NULL: 0).  Out: den [nsp*G] (GPG.den), source [G], sigma_out [G]
 * (Sigma where SumSource sets it, else the value of sigma_node_in [G] or 0). */
int rk_deposit(const rk_case *c, const int *face, const int *boundary, const int *cond_id, const float *area,
               const int *pnc, const float *x, const float *y, const float *sigma_in, const float *sigma_node_in,
               float *den, float *source, float *sigma_out) {
    return guarded([&] {
        const Dims d = dims(c);
        check_counts(c, d, pnc, d.mpnc);
        Arena a;
        std::vector<Species> info = species(c, d);
        const size_t n = (size_t)(d.nsp * d.maxnp);
        std::vector<GCP> sp(n);
        for (size_t k = 0; k < n; k++) {
            std::memset(&sp[k], 0, sizeof(GCP));
            sp[k].x = x[k];
            sp[k].y = y[k];
        }
        std::vector<GPG> g = gpg(d, pnc, nullptr);
        if (sigma_in)
            for (size_t k = 0; k < g.size(); k++) g[k].sigma = sigma_in[k];
        std::vector<GGA> v((size_t)d.G);
        for (int k = 0; k < d.G; k++) {
            std::memset(&v[(size_t)k], 0, sizeof(GGA));
            v[(size_t)k].Boundary = boundary[k];
            v[(size_t)k].Face = face[k];
            v[(size_t)k].CondID = cond_id[k];
            v[(size_t)k].Area = area[k];
        }
        std::vector<float> sig((size_t)d.G, 0.f);
        if (sigma_node_in) std::memcpy(sig.data(), sigma_node_in, sig.size() * sizeof(float));
        Species *di = a.put(info);
        GCP *ds = a.put(sp);
        GPG *dg = a.put(g);
        GGA *dv = a.put(v);
        float *dsig = a.put(sig);
        float *dsrc = a.alloc<float>((size_t)d.G);
        if (g_reps > 0) { // DEPOSIT_GRID/DEPOSIT_BLOCK: DepositAtom's shape for all four kernels
            const GPG *dg0 = snapshot(a, dg, g.size());
            const float *dsig0 = snapshot(a, dsig, sig.size());
            const long long nt = (long long)d.nsp * d.G;
            const int b = ref_block(DepositAtom, nt);
            const unsigned gb = blocks(nt, b);
            Timed t(4);
            for (int r = 0; r < g_reps; r++) {
                restore(dg, dg0, g.size());
                restore(dsig, dsig0, sig.size());
                t.mark(0);
                DepositInitDensity<<<gb, b>>>(d.G, di, dg);
                t.mark(1);
                DepositAtom<<<gb, b>>>(d.G, c->ngy, di, ds, dg);
                t.mark(2);
                DepositBoundary<<<gb, b>>>(d.G, c->ngy, d.nsp, dv, dg);
                t.mark(3);
                SumSource<<<gb, b>>>(d.nsp, d.G, c->ngx, c->ngy, di, dv, dg, dsig, dsrc);
                t.mark(4);
                t.add();
            }
            sync("Deposit (timed)");
            restore(dg, dg0, g.size());
            restore(dsig, dsig0, sig.size());
        }
        const unsigned nb = blocks((long long)d.nsp * d.G, 256);
        DepositInitDensity<<<nb, 256>>>(d.G, di, dg);
        DepositAtom<<<nb, 256>>>(d.G, c->ngy, di, ds, dg);
        DepositBoundary<<<nb, 256>>>(d.G, c->ngy, d.nsp, dv, dg);
        SumSource<<<blocks(d.G, 256), 256>>>(d.nsp, d.G, c->ngx, c->ngy, di, dv, dg, dsig, dsrc);
        sync("Deposit");
        get(g, dg);
        for (size_t k = 0; k < g.size(); k++) den[k] = g[k].den;
        std::vector<float> hs((size_t)d.G);
        get(hs, dsrc);
        std::memcpy(source, hs.data(), hs.size() * sizeof(float));
        get(sig, dsig);
        if (sigma_out) std::memcpy(sigma_out, sig.data(), sig.size() * sizeof(float));
    });
}

/* Cond_Sigma then VtoEfield (src/cuda_Field.cu:500-558,698-846), as
 * Efield_cuda_Basic runs them: geom = {dx, dy, hdx, hdy, idx, idy, idxy};
 * eps [(ngx-1)*(ngy-1)] (GCA.eps); den [nsp*G] (GPG.den, for Cond_Sigma's
 * charge term); sigma [G] in: Sigma before the call, out: after Cond_Sigma;
 * phi [G]; out ex, ey [G]. */
int rk_efield(const rk_case *c, const float *geom, const int *face, const int *boundary, const float *eps,
              const float *den, float *sigma, const float *phi, float *ex, float *ey) {
    return guarded([&] {
        const Dims d = dims(c);
        Arena a;
        std::vector<Species> info = species(c, d);
        const int C = (c->ngx - 1) * (c->ngy - 1);
        std::vector<GCA> vc((size_t)C);
        for (int k = 0; k < C; k++) {
            std::memset(&vc[(size_t)k], 0, sizeof(GCA));
            vc[(size_t)k].eps = eps[k];
        }
        std::vector<GGA> v((size_t)d.G);
        for (int k = 0; k < d.G; k++) {
            std::memset(&v[(size_t)k], 0, sizeof(GGA));
            v[(size_t)k].Boundary = boundary[k];
            v[(size_t)k].Face = face[k];
        }
        std::vector<GPG> g = gpg(d, nullptr, nullptr);
        for (size_t k = 0; k < g.size(); k++) g[k].den = den[k];
        Species *di = a.put(info);
        GCA *dc = a.put(vc);
        GGA *dv = a.put(v);
        GPG *dg = a.put(g);
        float *dsig = a.put(sigma, (size_t)d.G);
        float *dphi = a.put(phi, (size_t)d.G);
        const unsigned nb = blocks(d.G, 256);
        Cond_Sigma<<<nb, 256>>>(c->ngx, c->ngy, geom[2], geom[3], geom[6], 1.0f, dv, dc, di, dg, dphi, dsig);
        VtoEfield<<<nb, 256>>>(c->ngx, c->ngy, geom[0], geom[1], geom[2], geom[3], geom[4], geom[5], dsig, dphi, dg, dc, dv);
        sync("Efield");
        get(v, dv);
        for (int k = 0; k < d.G; k++) {
            ex[k] = v[(size_t)k].Ex;
            ey[k] = v[(size_t)k].Ey;
        }
        std::vector<float> hs((size_t)d.G);
        get(hs, dsig);
        std::memcpy(sigma, hs.data(), hs.size() * sizeof(float));
    });
}

/* PCG_float (src/cuda_Field.cu:942-1072).  With nblocks = 0 it is launched
 * as PCG_SOLVER launches it (src/cuda_Field.cu:133-142, src/cuda_Init.cu:
 * 17-26): cooperative, 512 threads per block, as many blocks as fit on the
 * GPU at once.  Otherwise nblocks x nthreads (at most 512).  ai[n+1], aj[nnz]
 * are 1-based CSR (src/load.c:121-246), m the Jacobi preconditioner, b the
 * right-hand side, x the warm start in and the solution out.  The solve stops
 * when r'z <= tol2 (absolute) or after the kernel's own bound of 100000
 * iterations; *iters receives its counter and *ms the kernel time.
 *
 * The kernel updates the search direction (A_x_Y_p_X at the end of an
 * iteration) and reads other rows of it in the next iteration's product
 * with no grid synchronisation in between, so threads of other blocks, or
 * other warps of one block, can read a stale direction.  A launch of one
 * block of 32 threads runs every row on one warp, which executes the update
 * loop before the product loop. */
int rk_pcg(int n, int nnz, const int *ai, const int *aj, const float *val, const float *m, const float *b, float *x,
           float tol2, int nblocks, int nthreads, int *iters, float *ms) {
    return guarded([&] {
        need(n > 0 && nnz > 0 && ai[0] == 1 && ai[n] == nnz + 1, "bad CSR");
        for (int k = 0; k < nnz; k++) need(aj[k] >= 1 && aj[k] <= n, "CSR column out of range");
        for (int r = 0; r < n; r++) need(ai[r + 1] >= ai[r], "CSR rows must not decrease");
        Arena a;
        int *dI = a.put(ai, (size_t)n + 1);
        int *dJ = a.put(aj, (size_t)nnz);
        float *dA = a.put(val, (size_t)nnz);
        float *dX = a.put(x, (size_t)n);
        float *dM = a.put(m, (size_t)n);
        float *dAP = a.alloc<float>((size_t)n);
        float *dP = a.alloc<float>((size_t)n);
        float *dR = a.put(b, (size_t)n);
        float *dZ = a.alloc<float>((size_t)n);
        int *dIter = a.alloc<int>(1);
        float *dDot = a.alloc<float>(200004);
        int dev = 0, sms = 0, per_sm = 0;
        ck(cudaGetDevice(&dev), "device");
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
        const size_t smem = sizeof(float) * THREADS_PER_BLOCK;
        ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, PCG_float, THREADS_PER_BLOCK, smem), "occupancy");
        need(per_sm >= 1, "PCG_float does not fit on an SM");
        dim3 grid(sms * per_sm), block(THREADS_PER_BLOCK);
        if (nblocks > 0) {
            need(nthreads >= 32 && nthreads <= THREADS_PER_BLOCK && nthreads % 32 == 0, "bad block size");
            int fit = 0;
            ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, PCG_float, nthreads, smem), "occupancy");
            need((long long)nblocks <= (long long)fit * sms, "more blocks than fit on the GPU at once");
            grid = dim3(nblocks);
            block = dim3(nthreads);
        }
        int nn = n, nz = nnz;
        float t2 = tol2;
        void *args[] = {&dI, &dJ, &dA, &dX, &dM, &dAP, &dP, &dR, &dZ, &nn, &nz, &t2, &dIter, &dDot};
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        ck(cudaEventRecord(e0), "event");
        ck(cudaLaunchCooperativeKernel((void *)PCG_float, grid, block, args, smem, nullptr), "PCG_float launch");
        ck(cudaEventRecord(e1), "event");
        sync("PCG_float");
        float t = 0.f;
        ck(cudaEventElapsedTime(&t, e0, e1), "event");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms) *ms = t;
        ck(cudaMemcpy(x, dX, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost), "x");
        ck(cudaMemcpy(iters, dIter, sizeof(int), cudaMemcpyDeviceToHost), "iters");
    });
}

/* The MCC's cross-section lookups (Argon_CrossSection, O2_CrossSection,
 * ArO2_CrossSection: src/cuda_mccAr.cu:707-776, src/cuda_mccO2.cu:978-,
 * src/cuda_mccArO2.cu:2461-3018) for gas 0 Ar, 1 O2, 2 Ar/O2: channel ch at
 * energies engy[n] > 0; tab is the table in the reference's row layout
 * (xe, xee, cx_0 ...), n_logx rows of `width` floats. */
int rk_xsec(int gas, int ch, int n_logx, float idlogx, const float *tab, int width, const float *engy, float *out,
            int n) {
    return guarded([&] {
        need(gas >= 0 && gas <= 2 && width == table_width(gas), "table width differs from the reference's struct");
        need(ch >= 0 && ch < width - 2 && n_logx >= 2, "bad channel or table");
        for (int k = 0; k < n; k++) need(engy[k] > 0.f && engy[k] < 1e30f, "energies must be positive and finite");
        Arena a;
        std::vector<float> t = padded_table(tab, n_logx, width);
        float *dt = a.put(t);
        float *de = a.put(engy, (size_t)n);
        float *dout = a.alloc<float>((size_t)n);
        k_xsec<<<blocks(n, 128), 128>>>(gas, ch, n_logx, idlogx, dt, de, dout, n);
        sync("cross sections");
        ck(cudaMemcpy(out, dout, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost), "xsec");
    });
}

/* The scattering kinematics (src/cuda_mcc.cu:139-201) with given uniforms,
 * same in/out layouts as the oracle's or_kinematics: kind 0 dev_anewvel
 * (e_flag 0, as every reference call passes), 1 dev_newvel_IONSC, 2
 * dev_maxwellv. */
int rk_kinematics(int kind, const float *in, float *out, int n) {
    return guarded([&] {
        need(kind >= 0 && kind <= 2, "bad kind");
        const int w = kind == 0 ? 7 : kind == 1 ? 6 : 4;
        Arena a;
        float *din = a.put(in, (size_t)n * w);
        float *dout = a.alloc<float>((size_t)n * 3);
        k_kin<<<blocks(n, 128), 128>>>(kind, din, dout, n);
        sync("kinematics");
        ck(cudaMemcpy(out, dout, (size_t)n * 3 * sizeof(float), cudaMemcpyDeviceToHost), "kinematics");
    });
}

/* MCC_Ar_Basic (src/cuda_mcc.cu:97-106 -> Direct_Argon_ArIon,
 * Direct_Argon_Electron, src/cuda_mccAr.cu:41-232): one thread per node
 * draws from its own scripted list (start[G+1], key = node ID).  mcc =
 * {dt, dtm} and imcc = {MCCn, nvel, n_logx, tnrct}; idlogx; vsave[nvel];
 * xsec (ArCollD rows); sigv[>=3]; collf (CollF rows, 4 floats each,
 * tnrct of them); back_den1, back_vel1, fluid_n [G].  Particles and pnc are
 * updated in place (created pairs appended); mccr [G*tnrct] receives the
 * reaction tallies; *overrun the draws asked for beyond a list. */
int rk_mcc_ar(const rk_case *c, const float *mcc, const int *imcc, float idlogx, const float *vsave, const float *xsec,
              const float *sigv, const float *collf, const float *back_den1, const float *back_vel1, const float *fluid_n,
              const float *u, const long long *start, int *pnc, float *x, float *y, float *vx, float *vy, float *vz,
              float *mccr, long long *overrun) {
    return guarded([&] {
        const Dims d = dims(c);
        need(d.nsp == 2, "the Ar set has two species");
        const int mccn = imcc[0], nvel = imcc[1], n_logx = imcc[2], tnrct = imcc[3];
        need(mccn >= 1 && nvel >= 2 && n_logx >= 2 && tnrct >= 7, "bad MCC constants");
        // every particle can add one electron and one ion
        int most = 0;
        for (int k = 0; k < d.nsp * d.G; k++) most = std::max(most, pnc[k]);
        need(2LL * most + 1 <= d.mpnc, "slots per node too few for the created pairs");
        check_counts(c, d, pnc, d.mpnc);
        Arena a;
        set_script(a, u, start, d.G);
        std::vector<Species> info = species(c, d);
        std::vector<GCP> sp = pack(d, x, y, vx, vy, vz, nullptr);
        std::vector<GPG> g = gpg(d, pnc, nullptr);
        std::vector<GGA> bg((size_t)d.G);
        std::vector<GFG> fl((size_t)d.G);
        for (int k = 0; k < d.G; k++) {
            std::memset(&bg[(size_t)k], 0, sizeof(GGA));
            bg[(size_t)k].BackDen1 = back_den1[k];
            bg[(size_t)k].BackVel1 = back_vel1[k];
            fl[(size_t)k].n = fluid_n[k];
        }
        std::vector<float> tab = padded_table(xsec, n_logx, table_width(0));
        Species *di = a.put(info);
        GCP *ds = a.put(sp);
        GPG *dg = a.put(g);
        GGA *dbg = a.put(bg);
        GFG *dfl = a.put(fl);
        float *dvs = a.put(vsave, (size_t)nvel);
        float *dtab = a.put(tab);
        MCC_sigmav *dsv = (MCC_sigmav *)a.put(sigv, 3);
        CollF *dcf = (CollF *)a.put(collf, (size_t)tnrct * 4);
        float *dmccr = a.alloc<float>((size_t)d.G * tnrct);
        float *dstack = a.alloc<float>((size_t)d.G * 5);
        Fluid *dinfo_f = a.alloc<Fluid>(1);
        curandState *dst = a.alloc<curandState>((size_t)d.G);
        const int Csize = (c->ngx - 1) * (c->ngy - 1);
        MCC_Ar_Basic<<<blocks(d.G, 256), 256>>>(d.G, Csize, c->ngy, d.nsp, mcc[0], mccn, mcc[1], 0.f, 0.f, nvel, dvs, dst,
                                                 n_logx, idlogx, dsv, dcf, (ArCollD *)dtab, tnrct, dmccr, dstack, dinfo_f,
                                                 dfl, dbg, di, dg, ds);
        sync("MCC_Ar_Basic");
        get(sp, ds);
        get(g, dg);
        unpack(sp, x, y, vx, vy, vz, nullptr);
        for (size_t k = 0; k < g.size(); k++) pnc[k] = g[k].PtNumInCell;
        std::vector<float> hm((size_t)d.G * tnrct);
        get(hm, dmccr);
        std::memcpy(mccr, hm.data(), hm.size() * sizeof(float));
        if (overrun) *overrun = script_overrun();
    });
}

/* One collision per thread through the oxygen sets' species handlers
 * (ArO2_Electron, ArO2_Ar_ion, ArO2_O2_ion, ArO2_O_ion, ArO2_O_negative:
 * src/cuda_mccArO2.cu:51-1129; O2_Electron, O2_O2_ion, O2_O_ion,
 * O2_O_negative: src/cuda_mccO2.cu:2-866), as MCC_ArO2_Basic / MCC_O2_Basic
 * call them after the collision check has tagged the collider with its
 * target (src/cuda_mccArO2.cu:1130-1265).  gas 1 O2 (4 species) or 2 Ar/O2
 * (5); n colliders of species isp, collider k with velocity v[3k..] and
 * target t[k], background speeds bv1[k], bv2[k], drawing from u[k*nu ..
 * (k+1)*nu).  imcc = {nvel, n_logx, tnrct}.  Out per collider k and species
 * s: cnt[k*nsp + s] particles, their velocities vout[((k*nsp + s)*4 + q)*3
 * ..] (at most 4 per species), and mccr[k*tnrct ..] the reaction tallies. */
int rk_oxy_collide(int gas, int isp, int n, const int *imcc, float idlogx, const float *escale, const float *vsave,
                   const float *xsec, const float *sigv, int nsigv, const float *collf, const float *v, const int *t,
                   const float *bv1, const float *bv2, const float *u, int nu, int *cnt, float *vout, float *mccr,
                   long long *overrun) {
    return guarded([&] {
        need(gas == 1 || gas == 2, "gas must be 1 (O2) or 2 (Ar/O2)");
        const int nsp = gas == 2 ? 5 : 4;
        need(isp >= 0 && isp < nsp && n >= 1 && nu >= 0, "bad species or count");
        const int nvel = imcc[0], n_logx = imcc[1], tnrct = imcc[2];
        need(nvel >= 2 && n_logx >= 2 && tnrct >= 1 && nsigv >= 1, "bad MCC constants");
        rk_case c;
        std::memset(&c, 0, sizeof(c));
        c.ngx = 2;
        c.ngy = n;
        c.nsp = nsp;
        c.mpnc = 8;
        for (int s = 0; s < nsp; s++) c.escale[s] = escale[s];
        Dims d;
        d.G = n;
        d.nsp = nsp;
        d.mpnc = c.mpnc;
        d.maxnp = (long long)c.mpnc * n;
        Arena a;
        std::vector<long long> start((size_t)n + 1);
        for (int k = 0; k <= n; k++) start[(size_t)k] = (long long)k * nu;
        set_script(a, u, start.data(), n);
        std::vector<Species> info = species(&c, d);
        std::vector<GCP> sp((size_t)(nsp * d.maxnp));
        for (auto &p : sp) std::memset(&p, 0, sizeof(GCP));
        std::vector<GPG> g = gpg(d, nullptr, nullptr);
        for (int k = 0; k < n; k++) {
            // the collider at the top slot of its node, tagged with its target
            GCP &p = sp[(size_t)(isp * d.maxnp + k + (long long)(c.mpnc - 1) * n)];
            p.CellID = t[k];
            p.x = 0.25f;
            p.y = 0.75f;
            p.vx = v[3 * (size_t)k];
            p.vy = v[3 * (size_t)k + 1];
            p.vz = v[3 * (size_t)k + 2];
            g[(size_t)isp * n + k].PtNumMCCInCell = 1;
        }
        std::vector<GGA> bg((size_t)n);
        for (int k = 0; k < n; k++) {
            std::memset(&bg[(size_t)k], 0, sizeof(GGA));
            bg[(size_t)k].BackVel1 = bv1[k];
            bg[(size_t)k].BackVel2 = bv2[k];
        }
        std::vector<float> tab = padded_table(xsec, n_logx, table_width(gas));
        Species *di = a.put(info);
        GCP *ds = a.put(sp);
        GPG *dg = a.put(g);
        GGA *dbg = a.put(bg);
        float *dvs = a.put(vsave, (size_t)nvel);
        float *dtab = a.put(tab);
        MCC_sigmav *dsv = (MCC_sigmav *)a.put(sigv, (size_t)nsigv);
        CollF *dcf = (CollF *)a.put(collf, (size_t)tnrct * 4);
        float *dmccr = a.alloc<float>((size_t)nsp * n * tnrct);
        curandState *dst = a.alloc<curandState>((size_t)nsp * n);
        k_oxy<<<blocks(n, 128), 128>>>(gas, isp, n, n, nvel, dvs, dst, di, dg, ds, n_logx, idlogx, dsv, dcf, dtab, tnrct,
                                       dmccr, dbg);
        sync("oxygen species handler");
        get(sp, ds);
        get(g, dg);
        std::vector<float> hm((size_t)nsp * n * tnrct);
        get(hm, dmccr);
        for (int k = 0; k < n; k++) {
            for (int ch = 0; ch < tnrct; ch++) {
                // electrons tally at TID * tnrct (TID = node), ions at ID * tnrct
                mccr[(size_t)k * tnrct + ch] = hm[(size_t)k * tnrct + ch];
            }
            for (int s = 0; s < nsp; s++) {
                const int m = g[(size_t)s * n + k].PtNumInCell;
                cnt[(size_t)k * nsp + s] = m;
                for (int q = 0; q < std::min(m, 4); q++) {
                    const GCP &p = sp[(size_t)(s * d.maxnp + k + (long long)q * n)];
                    float *o = vout + (((size_t)k * nsp + s) * 4 + q) * 3;
                    o[0] = p.vx;
                    o[1] = p.vy;
                    o[2] = p.vz;
                }
            }
        }
        if (overrun) *overrun = script_overrun();
    });
}


// The fluid sources of G nodes (Argon_Update_Source, Oxygen_Update_Source,
// ArO2_Update_Source): rates[G*tnrct] the averaged collision rates in (and
// the neutral reaction channels the kernel fills, out); ave_e[G] the averaged
// electron density; fden[nfsp*G]; bd1, bd2[G]; rr[tnrct]; src[nfsp*G] out.
int rk_fluid_source(int gas, int G, int ngy, int tnrct, int nfsp, float *rates, const float *rr, const float *ave_e,
                    const float *fden, const float *bd1, const float *bd2, float *src) {
    return guarded([&] {
        need(gas >= 0 && gas <= 2 && G > 0, "rk_fluid_source: bad gas or size");
        // channels and fluid species the kernel indexes
        need(tnrct >= (gas == 0 ? 10 : gas == 1 ? 67 : 88), "rk_fluid_source: too few channels");
        need(nfsp >= (gas == 0 ? 1 : gas == 1 ? 4 : 5), "rk_fluid_source: too few fluid species");
        Arena a;
        std::vector<CollF> cf((size_t)tnrct);
        for (int k = 0; k < tnrct; k++) {
            std::memset(&cf[(size_t)k], 0, sizeof(CollF));
            cf[(size_t)k].RR = rr[k];
        }
        std::vector<GPG> sp((size_t)G);
        std::vector<GGA> bg((size_t)G);
        for (int g = 0; g < G; g++) {
            std::memset(&sp[(size_t)g], 0, sizeof(GPG));
            std::memset(&bg[(size_t)g], 0, sizeof(GGA));
            sp[(size_t)g].ave_den = ave_e[g];
            bg[(size_t)g].BackDen1 = bd1[g];
            bg[(size_t)g].BackDen2 = bd2[g];
        }
        std::vector<GFG> fg((size_t)nfsp * G), fs((size_t)nfsp * G);
        for (size_t k = 0; k < fg.size(); k++) {
            std::memset(&fg[k], 0, sizeof(GFG));
            std::memset(&fs[k], 0, sizeof(GFG));
            fg[k].n = fden[k];
        }
        float *dr = a.put(rates, (size_t)G * tnrct);
        CollF *dc = a.put(cf);
        GPG *dsp = a.put(sp);
        GGA *dbg = a.put(bg);
        GFG *dfg = a.put(fg);
        GFG *dfs = a.put(fs);
        const unsigned nb = blocks(G, 256);
        if (gas == 0) Argon_Update_Source<<<nb, 256>>>(G, ngy, tnrct, dr, dc, dsp, dfg, dfs, dbg);
        else if (gas == 1) Oxygen_Update_Source<<<nb, 256>>>(G, tnrct, dr, dc, dsp, dfg, dfs, dbg);
        else ArO2_Update_Source<<<nb, 256>>>(G, ngy, tnrct, dr, dc, dsp, dfg, dfs, dbg);
        sync("Update_Source");
        std::vector<float> hr((size_t)G * tnrct);
        get(hr, dr);
        std::memcpy(rates, hr.data(), hr.size() * sizeof(float));
        get(fs, dfs);
        for (size_t k = 0; k < fs.size(); k++) src[k] = fs[k].n;
    });
}

} // extern "C"
