/*
 * hp_circuit.h -- the external circuit of the reference's Efield_cuda
 * (src/cuda_Field.cu:43-103), shared by the CUDA kernel and the CPU checker
 * so that both evaluate the same float operations in the same order.
 *
 * Every conductor i is driven through a series R-L-C (the ConductorSpec's
 * R(Ohm), L(H), C(F)).  With the second-order backward difference of the
 * charge q_i that flowed through the circuit, the reference's coefficients
 * cc[i][0..4] (src/Efield.c:70-78) give
 *
 *   K_t   = (cc1 q(t-1) + cc2 q(t-2) + cc3 q(t-3) + cc4 q(t-4)) / cc0
 *   b_i   = (V_i(t) - K_t) / cc0 - q_i(t-1) - q_conv,i + S_i(t-1) - P_i(t)
 *   A_ij  = L_ji + (i == j) / cc0_i
 *   phi   = A^-1 b       (conductor potentials of this step)
 *   q_i(t) = (V_i - phi_i) / cc0_i - K_t
 *
 * with V_i the conductor's source voltage, q_conv,i = -sum_s qd_s N_s,i the
 * charge of the particles it absorbed in the last step, S_i the surface
 * charge on it at the end of the last step, P_i that of this step's Poisson
 * part of the potential (conductors at 0 V) and L_ji that of the Laplace
 * basis with conductor j at 1 V.  The inverse is the reference's cofactor
 * expansion (src/cuda_Field.cu:847-941: determinants by first-row Laplace
 * expansion, the adjugate divided by the determinant), in float.
 *
 * Three things in the reference keep this from being a charge balance
 * (mode 0 reproduces them):
 *  - b_i subtracts K_t, a charge, from the voltage before dividing by cc0:
 *    (V - K_t) / cc0 where the balance needs V / cc0 - K_t, so the circuit's
 *    history enters b_i scaled by 1 / cc0;
 *  - the charge update of every conductor uses the K_t of the LAST conductor
 *    (K_t is one variable overwritten in the first loop and read in the
 *    second, src/cuda_Field.cu:57-80), so only the last conductor keeps its
 *    circuit history;
 *  - S_i is the Diagnostic's surface charge, Cond_Sigma of the Poisson part
 *    only (src/cuda_Field.cu:97-98, src/cuda_Diagnostic.cu:136-176), so the
 *    charge the conductor held through its own potential (the Laplace part)
 *    is not carried from one step to the next.
 * Mode 1 uses V / cc0 - K_t, gives each conductor its own K_t and takes S_i
 * as the conductor's whole charge after the last step,
 * sum_j L_ji phi_j(t-1) + P_i(t-1), so that the charge on a conductor
 * changes by the circuit's charge and the absorbed particles' charge only:
 * with no plasma an R-C-L driven electrode then follows its source through
 * the circuit as the network equations say.
 *
 * HP_CIRCUIT_MAX conductors at most (the expansion grows as n!).
 */
#ifndef HP_CIRCUIT_H
#define HP_CIRCUIT_H

#if defined(__CUDACC__)
#define HP_CI __host__ __device__ __forceinline__
#else
#define HP_CI static inline
#endif

#define HP_CIRCUIT_MAX 4

/* the reference's determinant (src/cuda_Field.cu:868-905), written out by
 * size (device code has no recursion): size 1 is the entry, else
 * det = 0, then det = det + s * (m[0][c] * det(minor of row 0, column c))
 * for c = 0.., s = 1, -1, ...  ld is the row stride of m. */
HP_CI float hp_ci_det2(const float *m, int ld) {
    float det = 0.0f;
    det = det + 1.0f * (m[0] * m[ld + 1]);
    det = det + -1.0f * (m[1] * m[ld]);
    return det;
}
HP_CI float hp_ci_det3(const float *m, int ld) {
    float det = 0.0f, s = 1.0f;
    for (int c = 0; c < 3; c++) {
        float mm[4];
        int k = 0;
        for (int i = 1; i < 3; i++)
            for (int j = 0; j < 3; j++)
                if (j != c) mm[k++] = m[i * ld + j];
        det = det + s * (m[c] * hp_ci_det2(mm, 2));
        s = -1.0f * s;
    }
    return det;
}
HP_CI float hp_ci_det4(const float *m, int ld) {
    float det = 0.0f, s = 1.0f;
    for (int c = 0; c < 4; c++) {
        float mm[9];
        int k = 0;
        for (int i = 1; i < 4; i++)
            for (int j = 0; j < 4; j++)
                if (j != c) mm[k++] = m[i * ld + j];
        det = det + s * (m[c] * hp_ci_det3(mm, 3));
        s = -1.0f * s;
    }
    return det;
}
HP_CI float hp_ci_det(const float *m, int ld, int n) {
    return n == 1 ? m[0] : n == 2 ? hp_ci_det2(m, ld) : n == 3 ? hp_ci_det3(m, ld) : hp_ci_det4(m, ld);
}

/* the reference's cofactor + transpose (src/cuda_Field.cu:847-867,906-941):
 * inv = adj(m) / det(m), in place, n >= 2 */
HP_CI void hp_ci_inverse(float *m, int n) {
    float cof[HP_CIRCUIT_MAX * HP_CIRCUIT_MAX];
    for (int q = 0; q < n; q++)
        for (int p = 0; p < n; p++) {
            float mm[HP_CIRCUIT_MAX * HP_CIRCUIT_MAX];
            int r = 0, k = 0;
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++)
                    if (i != q && j != p) {
                        mm[r * HP_CIRCUIT_MAX + k] = m[i * HP_CIRCUIT_MAX + j];
                        if (k < n - 2) k++;
                        else { k = 0; r++; }
                    }
            const float dm = hp_ci_det(mm, HP_CIRCUIT_MAX, n - 1);
            /* pow(-1, q + p) * det: an exact sign change */
            cof[q * HP_CIRCUIT_MAX + p] = ((q + p) & 1) ? -dm : dm;
        }
    const float d = hp_ci_det(m, HP_CIRCUIT_MAX, n);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) m[i * HP_CIRCUIT_MAX + j] = cof[j * HP_CIRCUIT_MAX + i] / d;
}

/* One step of the circuit (src/cuda_Field.cu:49-80).
 * nc conductors; cc[i*5 + 0..4] the coefficients; lap[j*HP_CIRCUIT_MAX + i]
 * the charge on conductor i of the Laplace basis of conductor j; vt, qconv,
 * surf per conductor as above, pois_new the P_i of this step; q[4*MAX] the
 * charge history (q(t-1), q(t-2), q(t-3), q(t-4) rows), phi[MAX] and
 * pois[MAX] those of the last step: all three updated.  mode as above. */
HP_CI void hp_circuit_step(int nc, const float *cc, const float *lap, const float *vt, const float *qconv,
                           const float *surf, const float *pois_new, float *q, float *phi, float *pois, int mode) {
    float A[HP_CIRCUIT_MAX * HP_CIRCUIT_MAX], b[HP_CIRCUIT_MAX], Kc[HP_CIRCUIT_MAX], S[HP_CIRCUIT_MAX];
    for (int i = 0; i < nc; i++) {
        if (mode == 1) {
            float s = 0.0f;
            for (int j = 0; j < nc; j++) s += lap[j * HP_CIRCUIT_MAX + i] * phi[j];
            S[i] = s + pois[i];
        } else {
            S[i] = surf[i];
        }
    }
    float K_t = 0.0f;
    for (int i = 0; i < nc; i++) {
        const float *a = cc + 5 * i;
        K_t = (a[1] * q[i] + a[2] * q[HP_CIRCUIT_MAX + i] + a[3] * q[2 * HP_CIRCUIT_MAX + i] +
               a[4] * q[3 * HP_CIRCUIT_MAX + i]) / a[0];
        Kc[i] = K_t;
        b[i] = (mode == 1 ? vt[i] / a[0] - K_t : (vt[i] - K_t) / a[0]) - q[i] - qconv[i] + S[i] - pois_new[i];
        for (int j = 0; j < nc; j++)
            A[i * HP_CIRCUIT_MAX + j] = i == j ? lap[j * HP_CIRCUIT_MAX + i] + 1 / a[0] : lap[j * HP_CIRCUIT_MAX + i];
    }
    hp_ci_inverse(A, nc);
    for (int i = 0; i < nc; i++) {
        float p = 0.0f;
        for (int j = 0; j < nc; j++) p += A[i * HP_CIRCUIT_MAX + j] * b[j];
        phi[i] = p;
        q[3 * HP_CIRCUIT_MAX + i] = q[2 * HP_CIRCUIT_MAX + i];
        q[2 * HP_CIRCUIT_MAX + i] = q[HP_CIRCUIT_MAX + i];
        q[HP_CIRCUIT_MAX + i] = q[i];
        q[i] = (vt[i] - p) / cc[5 * i] - (mode == 1 ? Kc[i] : K_t);
        pois[i] = pois_new[i];
    }
}

#endif /* HP_CIRCUIT_H */
