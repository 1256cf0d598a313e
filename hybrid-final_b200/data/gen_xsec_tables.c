/*
 * gen_xsec_tables.c -- development tool that regenerates the committed
 * cross-section tables (xsec_ar.txt, xsec_o2.txt, xsec_aro2.txt).
 *
 * The reference resamples its tabulated and fitted cross sections onto an
 * 81-point log10 energy grid (1e-4 .. 1e4 eV) in Argon_CrossSectionSET,
 * Oxygen_CrossSectionSET and ArO2_CrossSectionSET (src/PhysicsData.c:1579-3275),
 * multiplying every channel by its on/off flag from the deck.  This driver
 * links the reference's own src/PhysicsData.c, calls each setter with every
 * flag at 1.0, and prints the tables plus the per-channel threshold energies
 * (CollF.Th_e) and rate constants (CollF.RR).  The library multiplies the
 * tables by the deck's flags when it builds a case.  Built and run by
 * gen_xsec_tables.sh; needs the reference tree, which the GPU box does not
 * have (the generated .txt files are what ships).
 */
#include <stdio.h>
#include <stdlib.h>
#include "def.h"

extern int TnRct;
extern CollF *Coll_Flag;
extern int N_LOGX;
extern float idLOGX, LOGX_MIN, LOGX_MAX, dLOGX;
extern ArCollD *Ar_Data;
extern O2CollD *O2_Data;
extern ArO2CollD *ArO2_Data;
extern void Argon_CrossSectionSET(CollF *CF);
extern void Oxygen_CrossSectionSET(CollF *CF);
extern void ArO2_CrossSectionSET(CollF *CF);

/* allocation helpers the reference's setters call (defined in src/start.c,
 * which this tool does not link) */
float *VFMalloc(int size) { return (float *)calloc((size_t)(size > 0 ? size : 1), sizeof(float)); }
void VFInit(float *V, float C, int size) { for (int i = 0; i < size; i++) V[i] = C; }

static void dump(const char *path, const char *gas, int ncx, const float *tab, int stride_floats) {
    FILE *f = fopen(path, "w");
    if (!f) { perror(path); exit(1); }
    fprintf(f, "# %s cross sections, generated from the reference's src/PhysicsData.c with all channel flags 1\n", gas);
    fprintf(f, "# line 2: N_LOGX n_cx_channels TnRct idLOGX\n");
    fprintf(f, "%d %d %d %.9g\n", N_LOGX, ncx, TnRct, idLOGX);
    fprintf(f, "# Th_e[TnRct]\n");
    for (int i = 0; i < TnRct; i++) fprintf(f, "%.9g%c", Coll_Flag[i].Th_e, i + 1 == TnRct ? '\n' : ' ');
    fprintf(f, "# RR[TnRct]\n");
    for (int i = 0; i < TnRct; i++) fprintf(f, "%.9g%c", Coll_Flag[i].RR, i + 1 == TnRct ? '\n' : ' ');
    fprintf(f, "# rows: xe xee cx_0 .. cx_%d\n", ncx - 1);
    for (int r = 0; r < N_LOGX; r++) {
        const float *row = tab + (size_t)r * stride_floats;
        for (int k = 0; k < 2 + ncx; k++) fprintf(f, "%.9g%c", row[k], k + 1 == 2 + ncx ? '\n' : ' ');
    }
    fclose(f);
}

static void setup(int n) {
    TnRct = n;
    Coll_Flag = (CollF *)calloc((size_t)n, sizeof(CollF));
    for (int i = 0; i < n; i++) Coll_Flag[i].Flag = 1.0f;
}

int main(int argc, char **argv) {
    if (argc != 2) { fprintf(stderr, "usage: %s outdir\n", argv[0]); return 1; }
    char p[600];
    setup(10);
    Argon_CrossSectionSET(Coll_Flag);
    snprintf(p, sizeof p, "%s/xsec_ar.txt", argv[1]);
    dump(p, "Ar", 7, (const float *)Ar_Data, (int)(sizeof(ArCollD) / sizeof(float)));
    setup(67);
    Oxygen_CrossSectionSET(Coll_Flag);
    snprintf(p, sizeof p, "%s/xsec_o2.txt", argv[1]);
    dump(p, "O2", 58, (const float *)O2_Data, (int)(sizeof(O2CollD) / sizeof(float)));
    setup(88);
    ArO2_CrossSectionSET(Coll_Flag);
    snprintf(p, sizeof p, "%s/xsec_aro2.txt", argv[1]);
    dump(p, "Ar/O2", 68, (const float *)ArO2_Data, (int)(sizeof(ArO2CollD) / sizeof(float)));
    return 0;
}
