// fastsolve.hpp -- separable inverse of the field operator (fastsolve.cpp).
#pragma once
#include <vector>

#include "setup.hpp"

namespace hp {

struct FastSolver {
    bool ok = false;
    int i0 = 0, j0 = 0, nx = 0, ny = 0;   // rectangle of unknowns (node indices)
    std::vector<float> V, Vt, W, Wt;      // row-major eigenvector matrices and transposes
    std::vector<float> inv_eig;           // [ny][nx] 1 / (lambda_i + theta_j)
    double fit_error = 0.0;               // largest relative misfit of the Kronecker form
};

// Detects the Kronecker-sum structure of the symmetrised operator and builds
// its eigen-decomposition; returns false (fs.ok = false) when the operator
// does not have that structure.
bool build_fast_solver(const Setup &s, FastSolver &fs);

} // namespace hp
