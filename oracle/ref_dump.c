/*
 * ref_dump.c -- test infrastructure (checker only; never linked into the product).
 *
 * Driver that runs the reference's OWN host-side setup code on a JSON deck and
 * writes every table the per-step hot path consumes to a directory of raw
 * little-endian arrays plus a small text header.  It is linked against the
 * reference's unmodified sources (src/start.c, src/load.c, src/PhysicsData.c,
 * src/Particle.c, src/Efield.c, src/parson.c, src/Fluid.c, src/Diagnostics.c,
 * src/Tecplot.c, src/Variables.cu), compiled in place by oracle/Makefile, and
 * its outputs pin this project's case builder bit-for-bit:
 *
 *   InputRead()          src/start.c:19-1430     deck parse, cross-section tables
 *   Geometry_setting()   src/start.c:1432-1642   GGA/GCA, faces, areas, StructureIndex
 *   Source_setting()     src/Efield.c:3-79       dt, conductor drive flags
 *   FieldSolverSetting() src/start.c:1911-1998   A_idx + CG_Matrix_Setting (src/load.c:121-246)
 *   GasSetting()         src/start.c:1999-2051   species scalars, particle load (src/Particle.c)
 *
 * The call order is the reference main()'s (src/main.c:43-49).  The random seed
 * that main() takes from getpid() (src/main.c:43) is a command-line argument here.
 *
 * usage: ref_dump <deck.json> <seed> <outdir> [<temps.bin> [<src.bin> <nsteps>]]
 *
 * With temps.bin (float[Gsize], the gas temperature of every node) the
 * reference's fluid set-up and continuity solve also run (rf_fluid in
 * ref_fluid.cu); with src.bin (float[nfsp*Csize]) the solve takes nsteps
 * steps with those sources.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "def.h"

/* reference globals (src/Variables.cu) */
extern char InputFile[80];
extern long int seed;
extern double t;
extern int tstep, cstep, DumpFlag;
extern int ngx, ngy, Gsize, ncx, ncy, Csize;
extern float dx, dy, zlength, xlength, ylength;
extern float idxy, idx, idy, hdx, hdy;
extern float dt, dt_dx, dt_dy;
extern int nsp, nfsp, nBG, MainGas;
extern Species *SP;
extern Fluid *FG;
extern BackG *BG;
extern int CondNUM, CondNUMR, SrcNUM, DielNUM;
extern int *SrcM_ID;
extern float *SrcDC, *SrcAC, *SrcFREQ, *SrcPHASE, *SrcRPHASE, *Src2piFREQ;
extern int *Efield_Flag;
extern int External_Flag;
extern float **CC_a;
extern int DT_PIC, DT_CONTI, N_ave;
extern GGA *vec_G;
extern GCA *vec_C;
extern int *vec_StructureIndex;
extern int **A_idx;
extern int A_size;
extern float *A_val, *TA_val, *MatM, **cond_b, *temp_b;
extern int *Ai, *Aj;
extern int TnRct;
extern CollF *Coll_Flag;
extern int N_LOGX;
extern float idLOGX, LOGX_MIN, LOGX_MAX;
extern ArCollD *Ar_Data;
extern O2CollD *O2_Data;
extern ArO2CollD *ArO2_Data;
extern int h_nvel;
extern float *vsave;
extern HCP *PtD;
extern float PCGtol, PCGtol2;

extern void InputRead();
extern void Geometry_setting();
extern void Source_setting();
extern void FieldSolverSetting();
extern void GasSetting();

static char g_out[512];

/* ref_fluid.cu */
int rf_fluid(const char *outdir, const float *temps, const float *src, int nsteps);

static float *read_floats(const char *path, size_t n) {
    FILE *f = fopen(path, "rb");
    if (!f) { perror(path); exit(2); }
    float *p = (float *)malloc(n * sizeof(float));
    if (fread(p, sizeof(float), n, f) != n) { fprintf(stderr, "%s: short file\n", path); exit(2); }
    fclose(f);
    return p;
}

static void wr(const char *name, const void *p, size_t bytes) {
    char path[700];
    snprintf(path, sizeof path, "%s/%s.bin", g_out, name);
    FILE *f = fopen(path, "wb");
    if (!f) { perror(path); exit(2); }
    if (bytes && fwrite(p, 1, bytes, f) != bytes) { perror(path); exit(2); }
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc != 4 && argc != 5 && argc != 7) {
        fprintf(stderr, "usage: %s deck.json seed outdir [temps.bin [src.bin nsteps]]\n", argv[0]);
        return 1;
    }
    strncpy(InputFile, argv[1], 79);
    seed = atol(argv[2]);
    strncpy(g_out, argv[3], sizeof g_out - 1);
    t = 0.0; tstep = 0; cstep = 0; DumpFlag = 0;

    InputRead();
    Geometry_setting();
    Source_setting();
    FieldSolverSetting();
    GasSetting();

    char path[700];
    snprintf(path, sizeof path, "%s/meta.txt", g_out);
    FILE *m = fopen(path, "w");
    if (!m) { perror(path); return 2; }
    fprintf(m, "ngx %d\nngy %d\nncx %d\nncy %d\nGsize %d\nCsize %d\n", ngx, ngy, ncx, ncy, Gsize, Csize);
    fprintf(m, "dx %.9g\ndy %.9g\nzlength %.9g\nxlength %.9g\nylength %.9g\n", dx, dy, zlength, xlength, ylength);
    fprintf(m, "idx %.9g\nidy %.9g\nhdx %.9g\nhdy %.9g\nidxy %.9g\n", idx, idy, hdx, hdy, idxy);
    fprintf(m, "dt %.9g\ndt_dx %.9g\ndt_dy %.9g\nDT_PIC %d\n", dt, dt_dx, dt_dy, DT_PIC);
    fprintf(m, "DT_CONTI %d\nN_ave %d\n", DT_CONTI, N_ave);
    fprintf(m, "nsp %d\nnfsp %d\nnBG %d\nMainGas %d\n", nsp, nfsp, nBG, MainGas);
    fprintf(m, "CondNUM %d\nCondNUMR %d\nSrcNUM %d\nDielNUM %d\nA_size %d\n", CondNUM, CondNUMR, SrcNUM, DielNUM, A_size);
    fprintf(m, "TnRct %d\nN_LOGX %d\nidLOGX %.9g\nh_nvel %d\nPCGtol %.9g\n", TnRct, N_LOGX, idLOGX, h_nvel, PCGtol);
    for (int s = 0; s < nsp; s++) {
        fprintf(m, "sp%d_np %d\nsp%d_np2c %.9g\nsp%d_mass %.9g\nsp%d_q %.9g\nsp%d_q_density %.9g\n",
                s, SP[s].np, s, SP[s].np2c, s, SP[s].mass, s, SP[s].q, s, SP[s].q_density);
        fprintf(m, "sp%d_vti %.9g\nsp%d_qm %.9g\nsp%d_Escale %.9g\nsp%d_Ascale %.9g\nsp%d_Denscale %.9g\nsp%d_MCCscale %.9g\n",
                s, SP[s].vti, s, SP[s].qm, s, SP[s].Escale, s, SP[s].Ascale, s, SP[s].Denscale, s, SP[s].MCCscale);
        fprintf(m, "sp%d_MAXNP %d\nsp%d_Temp %.9g\nsp%d_InitDens %.9g\n", s, SP[s].MAXNP, s, SP[s].Temp, s, SP[s].InitDens);
    }
    for (int b = 0; b < nBG; b++)
        fprintf(m, "bg%d_Pres %.9g\nbg%d_Temp %.9g\nbg%d_mass %.9g\nbg%d_InitDens %.9g\n",
                b, BG[b].Pres, b, BG[b].Temp, b, BG[b].mass, b, BG[b].InitDens);
    for (int f = 0; f < nfsp; f++)
        fprintf(m, "fg%d_InitDens %.9g\nfg%d_Temp %.9g\nfg%d_mass %.9g\n", f, FG[f].InitDens, f, FG[f].Temp, f, FG[f].mass);
    for (int k = 0; k < SrcNUM; k++)
        fprintf(m, "src%d_MID %d\nsrc%d_DC %.9g\nsrc%d_AC %.9g\nsrc%d_FREQ %.9g\nsrc%d_RPHASE %.9g\n",
                k, SrcM_ID[k], k, SrcDC[k], k, SrcAC[k], k, SrcFREQ[k], k, SrcRPHASE[k]);
    for (int k = 0; k < CondNUMR; k++) fprintf(m, "efield_flag%d %d\n", k, Efield_Flag[k]);
    fclose(m);

    if (External_Flag) { /* external circuit coefficients (src/Efield.c:70-78), CondNUMR rows of 5 */
        float *a = (float *)malloc((size_t)CondNUMR * 5 * sizeof(float));
        for (int k = 0; k < CondNUMR; k++) memcpy(a + (size_t)k * 5, CC_a[k], 5 * sizeof(float));
        wr("cc_a", a, (size_t)CondNUMR * 5 * sizeof(float));
        free(a);
    }
    wr("gga", vec_G, (size_t)Gsize * sizeof(GGA));
    wr("gca", vec_C, (size_t)Csize * sizeof(GCA));
    wr("sidx", vec_StructureIndex, (size_t)(ncx + 2) * (ncy + 2) * sizeof(int));
    {
        int *a = (int *)malloc((size_t)Gsize * sizeof(int));
        for (int i = 0; i < ngx; i++)
            for (int j = 0; j < ngy; j++) a[i * ngy + j] = A_idx[i][j];
        wr("aidx", a, (size_t)Gsize * sizeof(int));
        free(a);
    }
    int nnz = Ai[A_size] - 1;
    wr("a_val", A_val, (size_t)nnz * sizeof(float));
    wr("ta_val", TA_val, (size_t)nnz * sizeof(float));
    wr("ai", Ai, (size_t)(A_size + 1) * sizeof(int));
    wr("aj", Aj, (size_t)nnz * sizeof(int));
    wr("matm", MatM, (size_t)A_size * sizeof(float));
    wr("temp_b", temp_b, (size_t)A_size * sizeof(float));
    {
        float *cb = (float *)malloc((size_t)CondNUMR * A_size * sizeof(float));
        for (int k = 0; k < CondNUMR; k++) memcpy(cb + (size_t)k * A_size, cond_b[k], (size_t)A_size * sizeof(float));
        wr("cond_b", cb, (size_t)CondNUMR * A_size * sizeof(float));
        free(cb);
    }
    wr("collf", Coll_Flag, (size_t)TnRct * sizeof(CollF));
    if (MainGas == ARGON) wr("xsec", Ar_Data, (size_t)N_LOGX * sizeof(ArCollD));
    else if (MainGas == OXYGEN) wr("xsec", O2_Data, (size_t)N_LOGX * sizeof(O2CollD));
    else wr("xsec", ArO2_Data, (size_t)N_LOGX * sizeof(ArO2CollD));
    if (vsave) wr("vsave", vsave, (size_t)h_nvel * sizeof(float));
    for (int s = 0; s < nsp; s++) {
        char nm[64];
        int np = SP[s].np;
        snprintf(nm, sizeof nm, "p%d_cell", s); wr(nm, PtD[s].CellID, (size_t)np * sizeof(int));
        snprintf(nm, sizeof nm, "p%d_x", s); wr(nm, PtD[s].x, (size_t)np * sizeof(float));
        snprintf(nm, sizeof nm, "p%d_y", s); wr(nm, PtD[s].y, (size_t)np * sizeof(float));
        snprintf(nm, sizeof nm, "p%d_vx", s); wr(nm, PtD[s].vx, (size_t)np * sizeof(float));
        snprintf(nm, sizeof nm, "p%d_vy", s); wr(nm, PtD[s].vy, (size_t)np * sizeof(float));
        snprintf(nm, sizeof nm, "p%d_vz", s); wr(nm, PtD[s].vz, (size_t)np * sizeof(float));
    }
    if (argc >= 5) {
        float *temps = read_floats(argv[4], (size_t)Gsize);
        float *src = argc == 7 ? read_floats(argv[5], (size_t)nfsp * Csize) : NULL;
        rf_fluid(g_out, temps, src, argc == 7 ? atoi(argv[6]) : 0);
        free(temps);
        free(src);
    }
    return 0;
}
