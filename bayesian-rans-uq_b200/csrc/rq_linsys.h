// Host set-up of standalone LDU linear systems for the device solvers
// (rq_linsolve.cu): validation with the reference's rules, the level-0
// operator in the reference's matvec order, and the AMG hierarchy built from
// the matrix values (greedy strength-0.25 aggregation, Galerkin coarse
// matrices, the dense inverse of the coarsest level).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace rq {

// a system outside what the device solvers handle (not an invalid system)
struct LinUnsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};

struct LinLevelHost {
    int n = 0, nc = 0;                 // rows; rows of the next level (0 on the coarsest)
    std::vector<int> ptr, col;         // CSR
    std::vector<double> val, rdg;      // values; 1/diag (1 where |diag| <= 1e-30)
    std::vector<int> agg;              // row -> next-level row
    std::vector<int> childPtr, childIdx; // next-level row -> rows, ascending
};

struct LinSysHost {
    int n = 0, nf = 0;
    std::vector<LinLevelHost> lev; // lev[0]: per row the diagonal, then each face's entry in face order
    std::vector<double> inv;       // dense inverse of the coarsest level (AMG only), row major
    int m = 0;                     // its rows
};

// Throws std::invalid_argument on the reference's admission failures
// (LinearSystem::validate / validateSolve, core/include/LinearSolver.hpp:63-92).
void validateLdu(int n, int nf, const double *diag, const double *upper, const double *lower,
                 const double *source, const int32_t *own, const int32_t *nbr);

// withAmg: build the hierarchy (coarsening to <= minCoarse rows); without it only
// level 0 is built (Jacobi PCG and BiCGSTAB). Throws LinUnsupported when the
// coarsest level exceeds maxCoarse rows or its pivots vanish.
LinSysHost buildLinSys(int n, int nf, const double *diag, const double *upper,
                       const double *lower, const int32_t *own, const int32_t *nbr, bool withAmg,
                       int minCoarse = 32, int maxLevels = 16, int maxCoarse = 128);

} // namespace rq
