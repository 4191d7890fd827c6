// Device-side data layout of the B200 forward model. One mesh class (mesh,
// boundary conditions, viscosity, settings, probes, AMG pattern) lives in HBM
// once; every coefficient draw is a job that one CTA runs from cold start to
// its verdict without leaving the GPU (see rq_solver.cu).
#pragma once
#include <cstddef>
#include <cstdint>

namespace rq {

constexpr int kMaxLevels = 12;    // AMG levels (the reference allows 20; meshes here need <= 8)
constexpr int kMaxCoarse = 128;   // rows of the dense coarsest AMG level
constexpr int kMaxProbes = 64;    // observations per problem
constexpr int kWindowCap = 64;    // 2 * convergenceWindow samples kept per estimator

enum Precision : int32_t { kFP64 = 0, kMixed = 1 };
enum PSolver : int32_t { kPAmg = 0, kPPcg = 1, kPBicgstab = 2 };

// SolverSettings subset of the hot path (rans-uq FlowFields.hpp:70-241).
struct DevSettings {
    int32_t maxIter, innerIter, window, monitorInterval;
    int32_t turbStart, turbInterval, floorIters, pSolver;
    int32_t precision, pad;
    double tol, innerTol, divLimit;
    double aU, aP, aK, aW;
    double fx, fy;
    double kMin, kMax, wMin;
};

// Levels >= 1 are stored in ELL form: value slot k*n + i holds the k-th entry of
// row i in column order (a warp reading slot k of 32 consecutive rows touches
// consecutive addresses); shorter rows are padded with column -1. The transfer
// operators between level l and level l+1 (nc rows) are ELL too: the prolongation
// P (slot k*n + i: the k-th coarse row of fine row i and its weight) and the
// restriction P^T (slot k*nc + I: the k-th fine row of coarse row I and its
// weight), padded with -1.
struct DevAmgLevel {
    int32_t n, nnz;             // rows; value slots (levels >= 1: width x n)
    int32_t valOff, vecOff;     // per-solve value / vector offsets (levels >= 1)
    int32_t width, pad;         // ELL width (levels >= 1)
    int32_t pw, rw;             // prolongation / restriction ELL widths (all but the last level)
    const int32_t *ecol, *diagPos;       // ELL columns (-1: padding); slot of the diagonal
    const int32_t *pcol, *rcol;          // prolongation / restriction ELL columns
    const double *pval, *rval;           // and weights
    const int32_t *gPtr, *gSrc;          // next-level value slot -> entries of this level
    const double *gW;                    // each entry's weight P_iI P_jJ in the Galerkin sum
};

struct DevClass {
    int32_t nx, ny, n, nfy;
    int32_t balance, nobs, nlev, obsComp;
    double nu, beta1Init;      // beta1 of the initial wall-omega face value (applyAllBCs default)
    double init[6];            // U xyz, p, k, omega
    DevSettings st;
    // cells
    const double *cx, *cy, *vol, *wd;
    // east faces (n)
    const double *xa, *xnx, *xny, *xw, *xdl, *xdx, *xdy, *xsh;
    // y faces (n + nx)
    const double *ya, *ynx, *yny, *yw, *ydl, *ydx, *ydy;
    // planar singular omega balance
    const double *sing, *slap, *sgx, *sgy;
    // probes: 4 neighbour slots each
    const int32_t *pcell, *pnnb, *pnb;
    const double *pox, *poy, *paxx, *paxy, *payy, *pdet, *pdx, *pdy, *pwt;
    const double *obsVal, *obsVar, *obsFloor;
    DevAmgLevel lev[kMaxLevels];
    double amgW, amgAlpha;     // V-cycle smoother weight, coarse-correction scale
    int32_t amgVals, amgVecs;  // per-solve doubles for coarse values / vectors
    int32_t amgSweeps, pad4;   // damped-Jacobi sweeps before and after each coarse correction
    int64_t wsDoubles;         // per-solve workspace
    // InferenceParameterSet: active indices, the coefficients filling the rest,
    // and the admission bounds (core/include/InferenceParameters.hpp:67-77, 127-165)
    int32_t nActive, pad2;
    int32_t active[11], pad3;
    double base[11], lo[11], hi[11];
};

// Outcome of one draw; the status values and order follow EvaluationStatus
// (core/include/EvaluationTypes.hpp:6).
struct RowOut {
    int32_t status, iterations, stalled, converged;
    double loglik, finalWorst, contractionRate;
};

struct DevJob {
    const DevClass *cls;
    const double *theta; // nActive values of this draw (device)
    RowOut *row;
    double *pred;      // nobs
    double *fields;    // optional 11 x n
    double *hist;      // optional hist_cap x 11
    long long *clock;  // optional, 12 per row: global-timer ns at start and end, inner
                       // Krylov iterations, inner pressure iterations, 8 stage cycle counts
    int32_t histCap;
    int32_t pad;
    // Warm start (optional): a converged state in the fields layout (11 x n: Ux Uy Uz p k
    // omega nuT F1 F2 Pk CDkw) copied in place of the uniform initial state, and the beta1
    // its wall-face omega was last set with (the cached solve's own coefficient).
    const double *warm;
    double warmBeta;
    // Snapshot (optional, written with the fields): the n + nfy face fluxes in the
    // device face layout (x faces, then y faces), the beta1 of the final wall-face omega,
    // and the turbulence-established marker (0 or 1).
    double *snap;
    // Solve workspace of this job (the serving loop's pool region of the job's class),
    // or null: the CTA's own per-slot workspace.
    double *ws;
};

// Request queue of the serving loop. The host appends requests (jobs[i], with
// theta, row and prediction slots) to host-mapped memory and then raises
// *published; CTAs claim them in order through *head (device memory) and raise
// done[i] when request i's results are in place.
struct ServeQueue {
    const DevJob *jobs;      // host-mapped, capacity entries
    const int *published;    // host-mapped: requests published so far
    const int *closed;       // host-mapped: 1 = no more requests (drain), 2 = cancel the rest
    int *done;               // host-mapped: one flag per request
    int *head;               // device: next request to claim
    int *exits;              // device: CTAs that have left (idle, drained or cancelled)
    int capacity, pad;
    long long idleNs;
};

} // namespace rq
