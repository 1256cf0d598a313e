// fastsolve.cpp -- separable inverse of the field operator, for the inner
// solve of the FP64 refinement (field_mode 2).
//
// The symmetrised operator S = D^-1 A (A from CG_Matrix_Setting,
// src/load.c:121-246; D the Neumann-edge doubling) is, for a rectangle of
// unknowns with uniform permittivity, a Kronecker sum
//     S = Tx (x) My + Mx (x) Ty
// with tridiagonal Tx, Ty and diagonal Mx, My.  Then
//     S^-1 = (V (x) W) (Lambda (x) I + I (x) Theta)^-1 (V^T (x) W^T)
// where Tx V = Mx V Lambda, V^T Mx V = I and Ty W = My W Theta, W^T My W = I.
// On a matrix of unknowns X[j][i] this is E = W ((W^T X V) ./ (lambda_i +
// theta_j)) V^T: four dense matrix products, which the GPU runs as GEMMs.
// The decomposition is detected from the stencil itself; any row that does
// not fit (a conductor or dielectric inside the domain) disables the path.
#include "fastsolve.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace hp {

namespace {

// Eigen-decomposition of a symmetric tridiagonal matrix (diagonal d, off
// diagonal e[0..n-2]) by the implicit QL algorithm with Wilkinson shifts
// (Golub & Van Loan, Matrix Computations, 4th ed., sec. 8.3).  On return d
// holds the eigenvalues and z (n x n, row-major, z[row*n + col]) the
// orthonormal eigenvectors as columns.
void tridiag_eigen(std::vector<double> &d, std::vector<double> e, std::vector<double> &z, int n) {
    z.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) z[(size_t)i * n + i] = 1.0;
    e.resize(n, 0.0);
    e[n - 1] = 0.0;
    for (int l = 0; l < n; l++) {
        int iter = 0;
        for (;;) {
            int m = l;
            for (; m < n - 1; m++) {
                double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= 1e-300 + 2.2e-16 * dd) break;
            }
            if (m == l) break;
            if (++iter > 200) throw std::runtime_error("tridiagonal eigensolver did not converge");
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
            double s = 1.0, c = 1.0, p = 0.0;
            int i = m - 1;
            for (; i >= l; i--) {
                double f = s * e[i], b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                for (int k = 0; k < n; k++) {
                    double zk1 = z[(size_t)k * n + i + 1], zk = z[(size_t)k * n + i];
                    z[(size_t)k * n + i + 1] = s * zk + c * zk1;
                    z[(size_t)k * n + i] = c * zk - s * zk1;
                }
            }
            if (r == 0.0 && i >= l) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
}

// Generalised problem T v = lambda M v with M diagonal positive: returns
// lambda and V (row-major n x n, columns = eigenvectors) with V^T M V = I.
void gen_eigen(const std::vector<double> &tdiag, const std::vector<double> &toff, const std::vector<double> &m,
               std::vector<double> &lambda, std::vector<double> &V) {
    const int n = (int)tdiag.size();
    std::vector<double> d(n), e(std::max(n - 1, 0));
    for (int i = 0; i < n; i++) d[i] = tdiag[i] / m[i];
    for (int i = 0; i + 1 < n; i++) e[i] = toff[i] / std::sqrt(m[i] * m[i + 1]);
    std::vector<double> z;
    tridiag_eigen(d, e, z, n);
    lambda = d;
    V.assign((size_t)n * n, 0.0);
    for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++) V[(size_t)r * n + c] = z[(size_t)r * n + c] / std::sqrt(m[r]);
}

} // namespace

bool build_fast_solver(const Setup &s, FastSolver &fs) {
    fs = FastSolver();
    const int ngy = s.ngy;
    // the unknowns must fill a rectangle of nodes
    int i0 = s.ngx, i1 = -1, j0 = s.ngy, j1 = -1;
    for (int n : s.unk_node) {
        int i = n / ngy, j = n % ngy;
        i0 = std::min(i0, i); i1 = std::max(i1, i);
        j0 = std::min(j0, j); j1 = std::max(j1, j);
    }
    if (i1 < 0) return false;
    const int nx = i1 - i0 + 1, ny = j1 - j0 + 1;
    if ((long long)nx * ny != (long long)s.n_unknowns || nx < 2 || ny < 2) return false;
    // symmetrised stencil of unknown (i, j)
    std::vector<int> pos(s.Gsize, -1);
    for (int u = 0; u < s.n_unknowns; u++) pos[s.unk_node[u]] = u;
    auto row = [&](int i, int j, int k) -> double {
        int u = pos[(i0 + i) * ngy + (j0 + j)];
        int gi = i0 + i, gj = j0 + j;
        double dsc = ((gi == 0 || gi == s.ncx) ? 2.0 : 1.0) * ((gj == 0 || gj == s.ncy) ? 2.0 : 1.0);
        return (double)s.stencil[(size_t)5 * u + k] / dsc;
    };
    // reference column/row in the interior of the rectangle
    const int ic = nx / 2, jc = ny / 2;
    if (ic + 1 >= nx || jc + 1 >= ny) return false;
    // x couplings -> My (normalised at jc) and Tx off-diagonals
    std::vector<double> My(ny), Mx(nx), tx_off(nx - 1), ty_off(ny - 1), tx_d(nx), ty_d(ny);
    const double ex = -row(ic, jc, 4), ny_ = -row(ic, jc, 3);
    if (!(ex > 0) || !(ny_ > 0)) return false;
    for (int j = 0; j < ny; j++) My[j] = -row(ic, j, 4) / ex;
    for (int i = 0; i + 1 < nx; i++) tx_off[i] = row(i, jc, 4) / My[jc];
    for (int i = 0; i < nx; i++) Mx[i] = -row(i, jc, 3) / ny_;
    for (int j = 0; j + 1 < ny; j++) ty_off[j] = row(ic, j, 3) / Mx[ic];
    for (int k = 0; k < nx; k++)
        if (!(Mx[k] > 0)) return false;
    for (int k = 0; k < ny; k++)
        if (!(My[k] > 0)) return false;
    // split the diagonal: Tx_ii = -(sum of its couplings) at the reference column
    tx_d[ic] = -(tx_off[ic - 1 >= 0 ? ic - 1 : 0] + tx_off[ic]);
    double ty_c = row(ic, jc, 2) - tx_d[ic] * My[jc];
    for (int j = 0; j < ny; j++) ty_d[j] = (row(ic, j, 2) - tx_d[ic] * My[j]) / Mx[ic];
    for (int i = 0; i < nx; i++) tx_d[i] = (row(i, jc, 2) - Mx[i] * ty_d[jc]) / My[jc];
    (void)ty_c;
    // verify every row of the operator
    double maxrel = 0.0;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            double w = i > 0 ? tx_off[i - 1] * My[j] : 0.0;
            double e = i + 1 < nx ? tx_off[i] * My[j] : 0.0;
            double sd = j > 0 ? Mx[i] * ty_off[j - 1] : 0.0;
            double no = j + 1 < ny ? Mx[i] * ty_off[j] : 0.0;
            double cc = tx_d[i] * My[j] + Mx[i] * ty_d[j];
            double want[5] = {w, sd, cc, no, e};
            for (int k = 0; k < 5; k++) {
                double got = row(i, j, k);
                double sc = std::fabs(row(i, j, 2));
                double rel = std::fabs(got - want[k]) / (sc > 0 ? sc : 1.0);
                maxrel = std::max(maxrel, rel);
            }
        }
    if (maxrel > 1e-5) return false;
    std::vector<double> lam, th, V, W;
    gen_eigen(tx_d, tx_off, Mx, lam, V);
    gen_eigen(ty_d, ty_off, My, th, W);
    fs.ok = true;
    fs.i0 = i0; fs.j0 = j0; fs.nx = nx; fs.ny = ny;
    fs.V.resize((size_t)nx * nx); fs.Vt.resize((size_t)nx * nx);
    fs.W.resize((size_t)ny * ny); fs.Wt.resize((size_t)ny * ny);
    for (int r = 0; r < nx; r++)
        for (int c = 0; c < nx; c++) {
            fs.V[(size_t)r * nx + c] = (float)V[(size_t)r * nx + c];
            fs.Vt[(size_t)c * nx + r] = (float)V[(size_t)r * nx + c];
        }
    for (int r = 0; r < ny; r++)
        for (int c = 0; c < ny; c++) {
            fs.W[(size_t)r * ny + c] = (float)W[(size_t)r * ny + c];
            fs.Wt[(size_t)c * ny + r] = (float)W[(size_t)r * ny + c];
        }
    fs.inv_eig.resize((size_t)nx * ny);
    double mineig = 1e300;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            double ev = lam[i] + th[j];
            mineig = std::min(mineig, ev);
            fs.inv_eig[(size_t)j * nx + i] = (float)(1.0 / ev);
        }
    if (!(mineig > 0)) {
        fs = FastSolver();
        return false;
    }
    fs.fit_error = maxrel;
    return true;
}

} // namespace hp
