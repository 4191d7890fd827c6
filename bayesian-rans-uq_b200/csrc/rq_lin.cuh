// Device-side layout of the standalone batched linear solves (rq_linsolve.cu):
// one DevLinSys per LDU system, its matrices and hierarchy in HBM, its vectors
// in the workspace slot of the CTA that solves it.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace rq {

constexpr int kLinMaxLevels = 16;
constexpr int kLinThreads = 512;
enum LinKind : int32_t { kLinAmg = 0, kLinPcg = 1, kLinBicgstab = 2 };

// SolverResult (core/include/LinearSolver.hpp:137-143); the layout of rq_solver_result
struct LinOut {
    int32_t iterations, converged;
    double finalRes, initialRes;
};

struct DevLinLevel {
    int32_t n, nc;                   // rows; rows of the next level (0 on the coarsest)
    int64_t vecOff;                  // b, x, r of this level in the level-vector area (levels >= 1)
    const int32_t *ptr, *col;        // CSR (level 0: diagonal, then faces in face order)
    const double *val, *rdg;         // values, 1/diag
    const float *val32, *rdg32;      // FP32 copies (mixed form)
    const int32_t *agg;              // row -> next-level row
    const int32_t *childPtr, *childIdx; // next-level row -> rows, ascending
};

struct DevLinSys {
    int32_t n, nlev, kind, precision, maxIter, m; // m: rows of the coarsest level
    double tol;
    int64_t lvOff;    // doubles: FP64 level vectors (after 8n FP64 Krylov vectors)
    int64_t f32Off;   // doubles: start of the FP32 area (mixed form)
    int64_t lvOff32;  // floats from f32Off: FP32 level vectors (after 6n FP32 vectors)
    const double *b;
    double *x;        // initial guess in, solution out
    const double *inv;
    const float *inv32;
    LinOut *out;
    DevLinLevel lev[kLinMaxLevels];
};

// Persistent CTAs of kLinThreads threads; *next zeroed by the caller; ws: grid
// slots of wsStride doubles.
cudaError_t launchLinear(const DevLinSys *systems, int nsys, int *next, double *ws, long wsStride,
                         int grid, cudaStream_t stream);
int linBlocksPerSM();

} // namespace rq
