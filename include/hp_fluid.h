/*
 * hp_fluid.h -- the source terms of the fluid (metastable and radical)
 * species, shared by the CUDA kernels and the CPU checker so that both
 * evaluate the same float operations in the same order.
 *
 * Every AverageIter + 1 steps the reference averages the collision tallies
 * into rates per node and reaction channel and turns them into a source per
 * fluid species: Argon_Update_Source, Oxygen_Update_Source and
 * ArO2_Update_Source (src/cuda_Diagnostic.cu:634-743).  Those kernels first
 * fill the rates of the reactions among neutral species, RR x density x
 * density, then sum gains and losses.  The sums are written here term by term
 * in the reference's order (float additions left to right).
 *
 * R[TnRct]   in: the averaged rates of the collision channels at the node;
 *            out: also the neutral reaction channels filled here
 * n[5]       the fluid densities at the node (Ar: Ar*; O2: O2A, O2B, OP, OD;
 *            Ar/O2: Ar*, O2A, O2B, OP, OD)
 * bd1, bd2   the background gas densities at the node (BackDen1, BackDen2)
 * eden       0.25 x the averaged electron density at the node
 * rr[TnRct]  CollF.RR of every channel
 * S[5]       out: the source of each fluid species (m^-3 s^-1)
 */
#ifndef HP_FLUID_H
#define HP_FLUID_H

#if defined(__CUDACC__)
#define HP_FL __host__ __device__ __forceinline__
#else
#define HP_FL static inline
#endif

HP_FL void hp_fluid_sources(int gas, float *R, const float *n, float bd1, float bd2, float eden, const float *rr,
                            float *S) {
    if (gas == 0) { /* Argon_Update_Source (src/cuda_Diagnostic.cu:634-642) */
        R[7] = rr[7] * eden * n[0];
        R[9] = rr[9] * bd1 * n[0];
        S[0] = R[2] - R[4] - R[7] - 2.0f * R[8] - R[9];
        return;
    }
    if (gas == 1) { /* Oxygen_Update_Source (src/cuda_Diagnostic.cu:643-683) */
        R[59] = rr[59] * n[2] * n[3];
        R[60] = rr[60] * n[3] * bd1;
        R[61] = rr[61] * n[3] * bd1;
        R[62] = rr[62] * n[3] * bd1;
        R[63] = rr[63] * n[0] * n[2];
        R[64] = rr[64] * n[0] * bd1;
        R[65] = rr[65] * n[0] * n[0];
        R[66] = rr[66] * n[1] * bd1;
        const float sa = R[3] + R[61];
        const float da = R[14] + R[15] + R[16] + R[17] + R[18] + R[19] + R[20] + R[21] + R[46] + R[51] + R[56] + R[63] +
                         R[64] + 2.0f * R[65];
        const float sb = R[4] + R[62];
        const float db = R[22] + R[23] + R[24] + R[25] + R[26] + R[27] + R[28] + R[29] + R[52] + R[57] + R[58] + R[66];
        const float sp = R[6] + 2.0f * R[7] + R[8] + R[11] + R[13] + R[15] + 2.0f * R[18] + R[19] + R[21] + R[23] +
                         2.0f * R[26] + R[27] + R[29] + R[30] + R[31] + R[40] + R[42] + R[44] + 2.0f * R[45] + R[46] +
                         R[50] + R[53] + R[56] + R[57] + R[58] + R[59] + R[60] + R[61] + R[62];
        const float dp = R[33] + R[34] + R[35] + R[36] + R[37] + R[38] + R[43] + R[47];
        const float sd = R[8] + 2.0f * R[9] + R[19] + 2.0f * R[20] + R[27] + 2.0f * R[28] + R[31] + R[33];
        const float dd = R[39] + R[40] + R[59] + R[60] + R[61] + R[62];
        S[0] = sa - da;
        S[1] = sb - db;
        S[2] = sp - dp;
        S[3] = sd - dd;
        return;
    }
    /* ArO2_Update_Source (src/cuda_Diagnostic.cu:684-743) */
    const float N1 = n[0], N2 = n[1], N4 = n[3], N5 = n[4];
    R[68] = rr[68] * eden * N1;
    R[71] = rr[71] * N4 * N5;
    R[72] = rr[72] * N5 * bd2;
    R[73] = rr[73] * N5 * bd2;
    R[74] = rr[74] * N5 * bd2;
    R[75] = rr[75] * N2 * N4;
    R[76] = rr[76] * N2 * bd2;
    R[77] = rr[77] * N2 * N2;
    R[78] = rr[78] * n[2] * bd2;
    R[82] = rr[82] * N1 * bd1;
    R[83] = rr[83] * N1 * N4;
    R[84] = rr[84] * N1 * N4;
    R[85] = rr[85] * N1 * bd2;
    R[86] = rr[86] * N1 * bd2;
    R[87] = rr[87] * N1 * bd2;
    const float s_arm = R[2];
    const float d_arm = R[4] + R[68] + 2.0f * R[81] + R[82] + R[83] + R[84] + R[85] + R[86] + R[87];
    const float s_o2a = R[8] + R[73];
    const float d_o2a = R[19] + R[20] + R[21] + R[22] + R[23] + R[24] + R[25] + R[26] + R[51] + R[56] + R[30] + R[75] +
                        R[76] + 2.0f * R[77];
    const float s_o2b = R[9] + R[74];
    const float d_o2b = R[27] + R[28] + R[29] + R[30] + R[31] + R[32] + R[33] + R[34] + R[57] + R[64] + R[70] + R[78];
    const float s_op = R[11] + 2.0f * R[12] + R[13] + R[16] + R[18] + R[20] + 2.0f * R[23] + R[24] + R[26] + R[28] +
                       2.0f * R[31] + R[32] + R[34] + R[35] + R[36] + R[45] + R[47] + R[49] + 2.0f * R[50] + R[51] +
                       R[55] + R[60] + R[63] + R[64] + R[70] + R[71] + R[72] + R[73] + R[74] + R[69] + 2.0f * R[85] +
                       R[86];
    const float d_op = R[38] + R[39] + R[40] + R[41] + R[42] + R[43] + R[48] + R[52] + R[79] + R[83];
    const float s_od = R[13] + 2.0f * R[14] + R[24] + 2.0f * R[25] + R[32] + 2.0f * R[33] + R[36] + R[38] + R[83] + R[86];
    const float d_od = R[44] + R[45] + R[71] + R[72] + R[73] + R[74];
    S[0] = s_arm - d_arm;
    S[1] = s_o2a - d_o2a;
    S[2] = s_o2b - d_o2b;
    S[3] = s_op - d_op;
    S[4] = s_od - d_od;
}

#endif /* HP_FLUID_H */
