// The B200 forward model: one CTA runs one SIMPLE + k-omega SST solve, every
// outer iteration of it, from cold start to its verdict, with all state in
// HBM/L2 and the CTA's shared memory. Persistent CTAs pull draws from a job
// queue (atomic counter), so a batch of mixed mesh classes keeps every SM busy
// until the longest solve ends; a serving loop launches the same kernel per
// admitted request on its own stream.
//
// The loop restates SIMPLESolver::solve (rans-uq/src/SIMPLESolver.cpp:1193-1716)
// on the structured periodic layout of rq_setup.h. Every face sum is gathered
// per cell in the reference's face order; dot products are block reductions
// (warp shuffles, then a fixed-order sum of the warp partials that every
// thread evaluates identically, so control flow stays uniform in the CTA).
//
// Inner solvers (core/include/LinearSolver.hpp): right-Jacobi BiCGSTAB
// (:251-345) for momentum, k and omega; for the pressure correction PCG
// (:184-246) with Jacobi or with the AMG V-cycle of this project (fixed
// aggregation from rq_setup.cpp, damped-Jacobi smoothing, Galerkin values
// refreshed per solve, dense coarsest inverse), or BiCGSTAB.
#include "rq_device.cuh"
#include "rq_kernels.h"

#include <cuda_runtime.h>
#include <math.h>


#include <type_traits>

namespace rq {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kRedSlots = 8;             // values per block reduction

struct Work {
    double *Ux, *Uy, *p, *k, *w, *nuT, *F1, *F2, *Pk, *CD, *S;
    double *gUxx, *gUxy, *gUyx, *gUyy, *gKx, *gKy, *gWx, *gWy, *gPx, *gPy;
    double *phi, *phiOld, *phiPred, *pCoeff; // x faces [0,n) then y faces [n, n+nfy)
    double *fScr;                            // face scratch of the transport assemblies
    double *d, *aW, *aE, *aS, *aN, *b, *aP, *aPraw;
    double *Uxp, *Uyp, *kOld, *wOld, *pp;
    double *r, *rh, *pv, *v, *s, *t, *ph, *sh;
    double *z, *xa, *xb, *rr;                // PCG / level-0 V-cycle
    double *rd;                              // reciprocal diagonal of the system being solved
    double *amgVal, *amgVec, *dense0, *dense1;
};

// Krylov / AMG storage of one value type (see "inner linear solvers").
template <typename T> struct KW {
    T *d, *aW, *aE, *aS, *aN, *rd;        // matrix and reciprocal diagonal
    T *r, *rh, *pv, *v, *s, *t, *ph, *sh; // BiCGSTAB
    T *z, *xa, *xb, *rr;                  // PCG / level-0 V-cycle (share BiCGSTAB-only storage)
    T *x;                                 // FP32 correction of the mixed form
    T *amgVal, *amgVec;                   // coarse levels: values; b, xa, xb, r, 1/diag
};

struct LinRes {
    int iterations;
    double finalRes, initialRes;
    bool converged;
    bool breakdown = false; // stopped on the |p.Ap| < 1e-30 guard (a round-off right-hand side)
};

// The outer loop's scalars. Every thread derives them identically from the same
// block reductions and writes the same value, so they can live here rather than in
// registers: a phase call then has no live loop state to save and restore around it
// (those saves were local-memory traffic that missed L1 at large meshes).
struct LoopState {
    double lastK, lastW, worst, fluxRef, n0x, n0y, n0p, rateU;
    double momRes, momScale, contScaled, fluxScale, uChange;
    LinRes resU[2], resP, resK, resW;
    int amgNeed, amgAfter, status, finalIter;
    bool established, converged, diverged;
};

struct Shared {
    DevClass C;
    Work W;
    KW<double> K64;
    KW<float> K32;
    double coeff[11];
    double red[2][kRedSlots][32];
    double ring[4][kWindowCap];  // U, k, omega, Q change samples
    int cnt[4];
    double q[kMaxProbes], qPrev[kMaxProbes];
    int haveQPrev;
    int job;
    DevJob jd; // the request being served (a copy out of host-mapped memory)
    int admitted;
    long long innerKrylov, innerPressure; // inner iterations of the solve (work accounting)
    long long stage[8];                   // clock64 cycles per stage (thread 0)
    long long tmark;
    double wallBeta;  // beta1 the wall-face omega was last set with (applyAllBCs' default
                      // on a cold start, the cached solve's on a warm one, then b1)
    double coarse[32 * 32];               // in-place inverse of a coarsest level of <= 32 rows
    LoopState L;                          // the outer loop's scalars (runSolve)
};

// stage timers, as the reference's momentum / pressure / turbulence timers
// (rans-uq/include/SIMPLESolver.hpp:293-305): 0 set-up, 1 closure, 2 momentum,
// 3 pressure assembly, 4 pressure solve, 5 AMG refresh, 6 turbulence, 7 bookkeeping
__device__ __forceinline__ void mark(Shared &S, int k) {
    if (threadIdx.x == 0) {
        const long long t = clock64();
        S.stage[k] += t - S.tmark;
        S.tmark = t;
    }
}

// ---------------------------------------------------------------- reductions
template <int K> struct Red {
    double v[K];
};

// Block reductions. Each warp tree-reduces its lanes (lane 0 holds the sum),
// lane 0 parks it in shared memory, and after one barrier EVERY warp
// tree-reduces the same partials in the same order and broadcasts lane 0's
// result -- so all threads of the CTA hold bit-identical values and branch alike.
template <int K>
__device__ __forceinline__ void blockSum(double (&v)[K], Shared &S, int &rp) {
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1)
            v[k] += __shfl_down_sync(FULL, v[k], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k)
            S.red[rp][k][warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = lane < nw ? S.red[rp][k][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1)
            s += __shfl_down_sync(FULL, s, o);
        v[k] = __shfl_sync(FULL, s, 0);
    }
    rp ^= 1;
}

template <int K>
__device__ __forceinline__ void blockMax(double (&v)[K], Shared &S, int &rp) {
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1)
            v[k] = fmax(v[k], __shfl_xor_sync(FULL, v[k], o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k)
            S.red[rp][k][warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = lane < nw ? S.red[rp][k][lane] : S.red[rp][k][0];
        for (int o = 16; o > 0; o >>= 1)
            s = fmax(s, __shfl_xor_sync(FULL, s, o));
        v[k] = s;
    }
    rp ^= 1;
}

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

// ---------------------------------------------------------------- geometry helpers
struct Cell {
    int c, i, j, W, E;
    bool south, north; // internal south / north faces
    bool xEfirst;      // east before west in face order (first column)
    bool yNfirst;      // north before south (bottom row of a multi-row mesh)
};

// row of a cell or y face index (idx / nx), without an integer division: exact while
// (idx + 0.5) / nx stays clear of an integer by more than the FP32 rounding, i.e. for
// any index below 2^21
__device__ __forceinline__ int rowOf(const DevClass &C, int idx) {
    return __float2int_rd((static_cast<float>(idx) + 0.5f) * __frcp_rn(static_cast<float>(C.nx)));
}
// the east neighbour of the cell owning x face f (periodic in x)
__device__ __forceinline__ int eastOf(const DevClass &C, int f) {
    return (f - rowOf(C, f) * C.nx == C.nx - 1) ? f - C.nx + 1 : f + 1;
}

__device__ __forceinline__ Cell cellOf(const DevClass &C, int c) {
    Cell q;
    q.c = c;
    q.j = rowOf(C, c);
    q.i = c - q.j * C.nx;
    q.W = q.i == 0 ? c + C.nx - 1 : c - 1;
    q.E = q.i == C.nx - 1 ? c - C.nx + 1 : c + 1;
    q.south = q.j > 0;
    q.north = q.j < C.ny - 1;
    q.xEfirst = q.i == 0;
    q.yNfirst = q.j == 0 && C.ny > 1;
    return q;
}

// sum four face terms in the reference's face-index order
__device__ __forceinline__ double order4(const Cell &q, double tW, double tE, double tS, double tN) {
    const double x1 = q.xEfirst ? tE : tW, x2 = q.xEfirst ? tW : tE;
    const double y1 = q.yNfirst ? tN : tS, y2 = q.yNfirst ? tS : tN;
    return ((x1 + x2) + y1) + y2;
}
// accumulate onto a running value in face order
__device__ __forceinline__ double accum4(const Cell &q, double acc, double tW, double tE, double tS,
                                         double tN) {
    const double x1 = q.xEfirst ? tE : tW, x2 = q.xEfirst ? tW : tE;
    const double y1 = q.yNfirst ? tN : tS, y2 = q.yNfirst ? tS : tN;
    return (((acc + x1) + x2) + y1) + y2;
}

// the wall face of a wall cell; a cell touching both walls keeps the last (top) one
__device__ __forceinline__ int wallFaceOf(const DevClass &C, int c) {
    const int j = rowOf(C, c);
    return (j == C.ny - 1 ? C.ny : 0) * C.nx + (c - j * C.nx);
}
__device__ __forceinline__ bool isWallCell(const DevClass &C, int c) {
    return c < C.nx || c >= C.n - C.nx;
}

__device__ __forceinline__ double wallOmega(const DevClass &C, double b1, double y) {
    const double coefficient = C.balance ? 6.0 : 60.0; // resolvedWallOmega, SIMPLESolver.cpp:155-161
    return coefficient * C.nu / (b1 * y * y);
}
// wall face value of omega (applyOmegaBC, BoundaryCondition.hpp:361-384)
__device__ __forceinline__ double wallFaceOmega(const DevClass &C, double b1, int f) {
    const double y1 = dmax(C.ydl[f], 1e-20);
    return 60.0 * C.nu / (b1 * y1 * y1);
}

// Green-Gauss gradient of one cell (Field.hpp:178-212); bS / bN are the wall
// face values used where the cell touches the bottom / top wall.
__device__ __forceinline__ void ggCell(const DevClass &C, const Cell &q, const double *phi,
                                       double bS, double bN, double &gx, double &gy) {
    const int c = q.c;
    const double pc = phi[c];
    // east (owner c)
    const double wE = __ldg(C.xw + (c));
    const double fE = pc * wE + phi[q.E] * (1.0 - wE);
    const double sxE = __ldg(C.xnx + (c)) * __ldg(C.xa + (c)), syE = __ldg(C.xny + (c)) * __ldg(C.xa + (c));
    // west (owner W, neighbour c)
    const double wWf = __ldg(C.xw + (q.W));
    const double fW = phi[q.W] * wWf + pc * (1.0 - wWf);
    const double sxW = __ldg(C.xnx + (q.W)) * __ldg(C.xa + (q.W)), syW = __ldg(C.xny + (q.W)) * __ldg(C.xa + (q.W));
    // north: internal (owner c) or top wall (owner c)
    const int fn = c + C.nx;
    double fN;
    if (q.north) {
        const double w = __ldg(C.yw + (fn));
        fN = pc * w + phi[c + C.nx] * (1.0 - w);
    } else {
        fN = bN;
    }
    const double sxN = __ldg(C.ynx + (fn)) * __ldg(C.ya + (fn)), syN = __ldg(C.yny + (fn)) * __ldg(C.ya + (fn));
    // south: internal (owner c - nx, neighbour c) or bottom wall (owner c)
    const int fs = c;
    double fS;
    if (q.south) {
        const double w = __ldg(C.yw + (fs));
        fS = phi[c - C.nx] * w + pc * (1.0 - w);
    } else {
        fS = bS;
    }
    const double sxS = __ldg(C.ynx + (fs)) * __ldg(C.ya + (fs)), syS = __ldg(C.yny + (fs)) * __ldg(C.ya + (fs));
    const double sgnS = q.south ? -1.0 : 1.0;
    gx = order4(q, -(sxW * fW), sxE * fE, sgnS * (sxS * fS), sxN * fN);
    gy = order4(q, -(syW * fW), syE * fE, sgnS * (syS * fS), syN * fN);
    const double V = __ldg(C.vol + (c));
    if (V > 1e-30) {
        gx = gx / V;
        gy = gy / V;
    }
}

// matrix row times x in the reference's matvec order (diagonal first, then faces)
__device__ __forceinline__ double rowDot(const Cell &q, const double *d, const double *aW,
                                         const double *aE, const double *aS, const double *aN,
                                         const double *x, int nx) {
    const int c = q.c;
    const double tW = aW[c] * x[q.W], tE = aE[c] * x[q.E];
    const double tS = q.south ? aS[c] * x[c - nx] : 0.0;
    const double tN = q.north ? aN[c] * x[c + nx] : 0.0;
    return accum4(q, d[c] * x[c], tW, tE, tS, tN);
}

__device__ __forceinline__ double jac(double r, double d) {
    return (fabs(d) > 1e-30) ? r / d : r; // jacobiPrecond, LinearSolver.hpp:173-177
}

// The cells a thread owns in every per-cell sweep: c = thread, thread + threads, ...
// (a warp's loads of one sweep cover whole cache lines; contiguous blocks of cells per
// thread measured 12 % slower per outer iteration at 1536 cells). Every per-cell
// loop of a solve uses this one assignment, so a thread may read its own writes of
// an earlier loop without a barrier.
#define FOR_OWN(c, count) for (int c = threadIdx.x; c < (count); c += blockDim.x)
#define FOR_CELLS(c) FOR_OWN(c, n)

// ---------------------------------------------------------------- inner linear solvers
// The Krylov and AMG routines are templated on the value type T of their
// vectors and matrices: T = double for the plain FP64 form, where they work
// directly on the arrays the assembly wrote; T = float for the mixed form,
// which solves for an FP32 correction inside an FP64 residual-refinement loop
// (mixedSolve below). Scalar coefficients and every reduction stay FP64.

// the five coefficient arrays of a 5-point system, held by value in registers
template <typename T> struct Mat {
    const T *d, *aW, *aE, *aS, *aN;
};
template <typename T> __device__ __forceinline__ Mat<T> matOf(const KW<T> &K) {
    return Mat<T>{K.d, K.aW, K.aE, K.aS, K.aN};
}

// row of a 5-point system times x, diagonal first then faces in the reference's
// matvec order (LinearSystem::matvec, LinearSolver.hpp:99-108)
template <typename T>
__device__ __forceinline__ T rowDotT(const Cell &q, const Mat<T> &M, const T *x, int nx) {
    const int c = q.c;
    const T tW = M.aW[c] * x[q.W], tE = M.aE[c] * x[q.E];
    const T tS = q.south ? M.aS[c] * x[c - nx] : T(0);
    const T tN = q.north ? M.aN[c] * x[c + nx] : T(0);
    const T x1 = q.xEfirst ? tE : tW, x2 = q.xEfirst ? tW : tE;
    const T y1 = q.yNfirst ? tN : tS, y2 = q.yNfirst ? tS : tN;
    return (((M.d[c] * x[c] + x1) + x2) + y1) + y2;
}

// Right-Jacobi BiCGSTAB (LinearSolver.hpp:251-345). K.r holds b - A x0 on entry and
// r0n its norm; x is updated in place.
template <typename T>
__device__ __noinline__ LinRes bicgstabT(Shared &S, int &rp, const KW<T> &K, T *x, double r0n,
                                         int maxIter, double tol) {
    const DevClass &C = S.C;
    const int n = C.n, nx = C.nx;
    LinRes res{0, 0.0, r0n, false};
    if (r0n < 1e-30) {
        res.converged = true;
        return res;
    }
    T *r = K.r, *rh = K.rh, *p = K.pv, *v = K.v, *s = K.s, *t = K.t, *ph = K.ph, *sh = K.sh,
      *rd = K.rd;
    const Mat<T> M = matOf(K);
    double acc[1] = {0.0};
    FOR_CELLS(c) {
        rh[c] = r[c];
        p[c] = T(0);
        v[c] = T(0);
        const T dc = M.d[c];
        rd[c] = (fabs(double(dc)) > 1e-30) ? T(1) / dc : T(1); // jacobiPrecond as a product
        acc[0] += double(r[c]) * double(r[c]);
    }
    blockSum<1>(acc, S, rp);
    double rhoN = acc[0], rho = 1, alpha = 1, omega = 1;
    for (int it = 0; it < maxIter; ++it) {
        if (fabs(rhoN) < 1e-30)
            break;
        const double beta = (rhoN / (rho + 1e-30)) * (alpha / (omega + 1e-30));
        FOR_CELLS(c) {
            const T pc = r[c] + T(beta) * (p[c] - T(omega) * v[c]);
            p[c] = pc;
            ph[c] = pc * rd[c];
        }
        __syncthreads();
        double a1[1] = {0.0};
        FOR_CELLS(c) {
            const Cell q = cellOf(C, c);
            const T vc = rowDotT(q, M, ph, nx);
            v[c] = vc;
            a1[0] += double(rh[c]) * double(vc);
        }
        blockSum<1>(a1, S, rp);
        const double rv = a1[0];
        if (fabs(rv) < 1e-30)
            break;
        alpha = rhoN / rv;
        double a2[1] = {0.0};
        FOR_CELLS(c) {
            const T sc = r[c] - T(alpha) * v[c];
            s[c] = sc;
            sh[c] = sc * rd[c];
            a2[0] += double(sc) * double(sc);
        }
        blockSum<1>(a2, S, rp);
        const double sn = sqrt(a2[0]);
        if (sn / r0n < tol) {
            FOR_CELLS(c) x[c] += T(alpha) * ph[c];
            __syncthreads();
            res.iterations = it + 1;
            res.finalRes = sn / r0n;
            res.converged = true;
            return res;
        }
        double a3[2] = {0.0, 0.0};
        FOR_CELLS(c) {
            const Cell q = cellOf(C, c);
            const T tc = rowDotT(q, M, sh, nx);
            t[c] = tc;
            a3[0] += double(tc) * double(tc);
            a3[1] += double(tc) * double(s[c]);
        }
        blockSum<2>(a3, S, rp);
        const double tt = a3[0];
        omega = (tt > 1e-30) ? a3[1] / tt : 0.0;
        double a4[2] = {0.0, 0.0};
        FOR_CELLS(c) {
            x[c] += T(alpha) * ph[c] + T(omega) * sh[c];
            const T rc = s[c] - T(omega) * t[c];
            r[c] = rc;
            a4[0] += double(rc) * double(rc);
            a4[1] += double(rh[c]) * double(rc);
        }
        blockSum<2>(a4, S, rp);
        const double rn = sqrt(a4[0]);
        res.iterations = it + 1;
        res.finalRes = rn / r0n;
        if (res.finalRes < tol) {
            res.converged = true;
            return res;
        }
        if (fabs(omega) < 1e-30)
            break;
        rho = rhoN;
        rhoN = a4[1];
    }
    __syncthreads();
    return res;
}

// ---------------------------------------------------------------- AMG V-cycle
template <typename T> __device__ __forceinline__ T level0EntryT(const KW<T> &K, int n, int e) {
    const int slot = e / n, c = e - slot * n;
    const T *a = slot == 0 ? K.d : slot == 1 ? K.aW : slot == 2 ? K.aE : slot == 3 ? K.aS : K.aN;
    return a[c];
}

// Galerkin values of every coarse level from the current pressure system, the
// reciprocal diagonals of the smoothed levels, then the inverse of the coarsest
// level (Gauss-Jordan, SPD: no pivoting): in place by one warp, one row per lane,
// when it has at most 32 rows; above that (up to 128) by the whole CTA, one
// barrier per pivot, ping-ponging [A | I] between two workspace buffers. (One warp
// with two rows per lane was measured 17 % slower per outer iteration at 1536
// cells: 128 dependent updates per lane and pivot against 16 per thread.) The
// inverse is FP64 in both forms.
template <typename T> __device__ __noinline__ void amgRefreshT(Shared &S, const KW<T> &K) {
    const DevClass &C = S.C;
    const Work &W = S.W;
    const int L = C.nlev;
    for (int l = 0; l + 1 < L; ++l) {
        const DevAmgLevel &F = C.lev[l];
        const DevAmgLevel &Q = C.lev[l + 1];
        T *cv = K.amgVal + Q.valOff;
        const T *fv = K.amgVal + F.valOff;
        // the first Galerkin sums cancel strongly (diagonal against off-diagonals of
        // one aggregate), so they are always formed from the FP64 finest matrix
        for (int e = threadIdx.x; e < Q.nnz; e += blockDim.x) {
            double s = 0.0;
            for (int k = __ldg(F.gPtr + e); k < __ldg(F.gPtr + e + 1); ++k) {
                const double v = (l == 0) ? level0EntryT(S.K64, C.n, __ldg(F.gSrc + k))
                                          : double(fv[__ldg(F.gSrc + k)]);
                s += __ldg(F.gW + k) * v;
            }
            cv[e] = T(s);
        }
        __syncthreads();
    }
    for (int l = 1; l + 1 < L; ++l) {
        const DevAmgLevel &Lv = C.lev[l];
        const T *val = K.amgVal + Lv.valOff;
        T *rdl = K.amgVec + Lv.vecOff + 4 * Lv.n;
        for (int i = threadIdx.x; i < Lv.n; i += blockDim.x)
            rdl[i] = T(1) / val[__ldg(Lv.diagPos + i)];
    }
    const DevAmgLevel &Q = C.lev[L - 1];
    const int m = Q.n; // at most kMaxCoarse = 128 rows (the set-up rejects more)
    const T *qv = K.amgVal + Q.valOff;
    if (m <= 32) {
        double *a = S.coarse;
        for (int e = threadIdx.x; e < m * m; e += blockDim.x)
            a[e] = 0.0;
        __syncthreads();
        if (L == 1) {
            for (int r = threadIdx.x; r < m; r += blockDim.x) {
                const Cell q = cellOf(C, r);
                a[r * m + r] += double(K.d[r]);
                a[r * m + q.W] += double(K.aW[r]);
                a[r * m + q.E] += double(K.aE[r]);
                if (q.south)
                    a[r * m + r - C.nx] += double(K.aS[r]);
                if (q.north)
                    a[r * m + r + C.nx] += double(K.aN[r]);
            }
        } else {
            for (int r = threadIdx.x; r < m; r += blockDim.x)
                for (int k = 0; k < Q.width; ++k) {
                    const int c = __ldg(Q.ecol + k * m + r);
                    if (c >= 0)
                        a[r * m + c] = double(qv[k * m + r]);
                }
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            const int r = threadIdx.x;
            for (int k = 0; k < m; ++k) {
                const double p = 1.0 / a[k * m + k];
                const double f = (r < m) ? a[r * m + k] : 0.0;
                __syncwarp();
                if (r < m && r != k) {
                    for (int j = 0; j < m; ++j)
                        if (j != k)
                            a[r * m + j] -= f * a[k * m + j] * p;
                    a[r * m + k] = -f * p;
                }
                __syncwarp();
                if (r == k) {
                    for (int j = 0; j < m; ++j)
                        if (j != k)
                            a[k * m + j] *= p;
                    a[k * m + k] = p;
                }
                __syncwarp();
            }
        }
        __syncthreads();
        return;
    }
    // m x 2m [A | I], row-major; the inverse ends in the right half of dense0
    const int m2 = 2 * m;
    double *A0 = W.dense0, *A1 = W.dense1;
    for (int e = threadIdx.x; e < m * m2; e += blockDim.x)
        A0[e] = ((e % m2) == m + e / m2) ? 1.0 : 0.0;
    __syncthreads();
    if (L == 1) {
        for (int r = threadIdx.x; r < m; r += blockDim.x) {
            const Cell q = cellOf(C, r);
            A0[r * m2 + r] += double(K.d[r]);
            A0[r * m2 + q.W] += double(K.aW[r]);
            A0[r * m2 + q.E] += double(K.aE[r]);
            if (q.south)
                A0[r * m2 + r - C.nx] += double(K.aS[r]);
            if (q.north)
                A0[r * m2 + r + C.nx] += double(K.aN[r]);
        }
    } else {
        for (int r = threadIdx.x; r < m; r += blockDim.x)
            for (int k = 0; k < Q.width; ++k) {
                const int c = __ldg(Q.ecol + k * m + r);
                if (c >= 0)
                    A0[r * m2 + c] = double(qv[k * m + r]);
            }
    }
    __syncthreads();
    // the (row, column) of a thread's entries advance by the CTA width without a division
    const int dq = static_cast<int>(blockDim.x) / m2, dr = static_cast<int>(blockDim.x) - dq * m2;
    const int r0 = static_cast<int>(threadIdx.x) / m2, c0 = static_cast<int>(threadIdx.x) - r0 * m2;
    for (int piv = 0; piv < m; ++piv) {
        const double inv = 1.0 / A0[piv * m2 + piv];
        int r = r0, col = c0;
        for (int e = threadIdx.x; e < m * m2; e += blockDim.x) {
            const double pr = A0[piv * m2 + col] * inv;
            A1[e] = (r == piv) ? pr : A0[e] - A0[r * m2 + piv] * pr;
            r += dq;
            col += dr;
            if (col >= m2) {
                col -= m2;
                ++r;
            }
        }
        __syncthreads();
        double *tmp = A0;
        A0 = A1;
        A1 = tmp;
    }
    if (A0 != W.dense0) { // keep the inverse in dense0
        for (int e = threadIdx.x; e < m * m2; e += blockDim.x)
            W.dense0[e] = A0[e];
        __syncthreads();
    }
}

// Sum over the slots k = first, first + step, ... (< width) of one ELL row of
// coef(k) * vec(col(k)) for columns >= 0, k ascending. The loads of four slots are
// issued before their products are added (padding slots load entry 0 and add
// nothing), so a wide row costs a few load latencies, not one per slot.
template <typename T, typename C, typename V>
__device__ __forceinline__ T ellDot(const int32_t *cols, const C *coef, const V *vec, int width,
                                    int stride, int row, int first = 0, int step = 1) {
    T s = T(0);
    int k = first;
    for (; k + 3 * step < width; k += 4 * step) {
        int c[4];
        T v[4], x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            c[u] = __ldg(cols + (k + u * step) * stride + row);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            v[u] = T(coef[(k + u * step) * stride + row]);
            x[u] = T(vec[c[u] < 0 ? 0 : c[u]]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (c[u] >= 0)
                s += v[u] * x[u];
    }
    if (k + step < width) {
        const int c0 = __ldg(cols + k * stride + row), c1 = __ldg(cols + (k + step) * stride + row);
        const T v0 = T(coef[k * stride + row]), v1 = T(coef[(k + step) * stride + row]);
        const T x0 = T(vec[c0 < 0 ? 0 : c0]), x1 = T(vec[c1 < 0 ? 0 : c1]);
        if (c0 >= 0)
            s += v0 * x0;
        if (c1 >= 0)
            s += v1 * x1;
        k += 2 * step;
    }
    if (k < width) {
        const int c = __ldg(cols + k * stride + row);
        if (c >= 0)
            s += T(coef[k * stride + row]) * T(vec[c]);
    }
    return s;
}

// Threads per row of a pass over n rows: the largest power of two up to 32 for which
// one pass of the CTA still covers every row (1 when there are more rows than half
// the CTA's threads).
__device__ __forceinline__ int segOf(int n) {
    int seg = 1;
    while (seg < 32 && 2 * seg * n <= static_cast<int>(blockDim.x))
        seg *= 2;
    return seg;
}

// A pass over the rows of a small level with several threads per row: lane j of a
// row's segment computes part(i, j, seg), the partial sum of the row's terms j,
// j + seg, ...; the partials are added by shuffles within the segment (a tree) and
// the segment's first lane calls use(i, total). Every thread of the CTA takes part
// (the shuffles need whole warps), so calls must be uniform across the CTA. With one
// thread per row this is the plain row loop.
template <typename T, typename Part, typename Use>
__device__ __forceinline__ void segPass(int n, Part part, Use use) {
    const int seg = segOf(n), per = static_cast<int>(blockDim.x) / seg;
    const int r = threadIdx.x / seg, j = threadIdx.x - r * seg;
    for (int base = 0; base < n; base += per) {
        const int i = base + r;
        T s = i < n ? part(i, j, seg) : T(0);
        for (int o = seg >> 1; o > 0; o >>= 1)
            s += __shfl_xor_sync(FULL, s, o);
        if (j == 0 && i < n)
            use(i, s);
    }
}

// row i of an ELL level times x, entries in column order
template <typename T>
__device__ __forceinline__ T csrRowT(const DevAmgLevel &L, const T *val, const T *x, int i) {
    return ellDot<T>(L.ecol, val, x, L.width, L.n, i);
}

// z = M^-1 b at level 0 (b = K.r, z -> K.z): on every level above the coarsest,
// C.amgSweeps damped-Jacobi sweeps from zero, the residual, restriction by P^T (fused
// into the next level's first sweep), and after the coarse correction x + alpha P x_c
// (fused into the first post sweep) the same number of sweeps again (symmetric);
// a dense inverse on the coarsest level. Returns (r, z), reduced in the last phase.
// With one sweep a level costs three barrier-separated phases (two down, one up);
// with two, five. (Running the small coarse levels in one warp with warp barriers
// measured 15 % slower per outer iteration: one warp exposes the latency of its
// dependent loads that a CTA's many warps hide.)
template <typename T> __device__ __noinline__ double vcycleT(Shared &S, int &rp, const KW<T> &K) {
    const DevClass &C = S.C;
    const Work &W = S.W;
    const int L = C.nlev, n0 = C.n, nx = C.nx;
    const bool two = C.amgSweeps >= 2;
    const T om = T(C.amgW), al = T(C.amgAlpha);
    const Mat<T> M = matOf(K);
    T *const Krd = K.rd, *const Kr = K.r, *const Kz = K.z, *const Kxa = K.xa, *const Kxb = K.xb,
             *const Krr = K.rr, *const amgVec = K.amgVec, *const amgVal = K.amgVal;
    auto vb = [&](int l) { return amgVec + C.lev[l].vecOff; }; // b, xa, xb, r, 1/diag
    auto sync = [] { __syncthreads(); };
    const int t0 = threadIdx.x, ts = blockDim.x;
    // residual of level l-1 restricted to row I of level l: sum_k R_Ik r_k (lane j of
    // the row's segment: the terms j, j + seg, ...)
    auto restrictPart = [&](int l, int I, int j, int seg) {
        const DevAmgLevel &F = C.lev[l - 1];
        const T *fr = (l == 1) ? Krr : vb(l - 1) + 3 * F.n;
        return ellDot<T>(F.rcol, F.rval, fr, F.rw, C.lev[l].n, I, j, seg);
    };
    // the prolongated coarse correction at row i of level l: sum_k P_ik x_c
    auto prolong = [&](int l, int i) {
        const DevAmgLevel &Lv = C.lev[l];
        const T *xc = vb(l + 1) + 2 * C.lev[l + 1].n;
        return ellDot<T>(Lv.pcol, Lv.pval, xc, Lv.pw, Lv.n, i);
    };
    // one level of the down sweep; the pre-smoothed iterate ends in xa (one sweep) or
    // xb (two sweeps), the residual in rr. Coarse levels run several threads per row.
    auto down = [&](int l) {
        const DevAmgLevel &Lv = C.lev[l];
        const int n = Lv.n;
        if (l == 0) {
            FOR_OWN(i, n)
                Kxa[i] = om * Kr[i] * Krd[i];
            sync();
            const T *xs = Kxa;
            if (two) {
                FOR_OWN(i, n) {
                    const T ax = rowDotT(cellOf(C, i), M, Kxa, nx);
                    Kxb[i] = Kxa[i] + om * (Kr[i] - ax) * Krd[i];
                }
                sync();
                xs = Kxb;
            }
            FOR_OWN(i, n)
                Krr[i] = Kr[i] - rowDotT(cellOf(C, i), M, xs, nx);
            sync();
            return;
        }
        T *b = vb(l), *xa = b + n, *xb = b + 2 * n, *rr = b + 3 * n;
        const T *rd = b + 4 * n;
        const T *val = amgVal + Lv.valOff;
        segPass<T>(n, [&](int i, int j, int seg) { return restrictPart(l, i, j, seg); },
                   [&](int i, T bi) {
                       b[i] = bi;
                       xa[i] = om * bi * rd[i];
                   });
        sync();
        const T *xs = xa;
        if (two) {
            segPass<T>(n,
                       [&](int i, int j, int seg) {
                           return ellDot<T>(Lv.ecol, val, xa, Lv.width, n, i, j, seg);
                       },
                       [&](int i, T ax) { xb[i] = xa[i] + om * (b[i] - ax) * rd[i]; });
            sync();
            xs = xb;
        }
        segPass<T>(n,
                   [&](int i, int j, int seg) {
                       return ellDot<T>(Lv.ecol, val, xs, Lv.width, n, i, j, seg);
                   },
                   [&](int i, T ax) { rr[i] = b[i] - ax; });
        sync();
    };
    // the coarsest level: restriction of the level above, then the dense inverse
    auto coarsest = [&]() {
        const int l = L - 1;
        const int m = C.lev[l].n, m2 = 2 * m;
        T *b = vb(l), *xb = b + 2 * m;
        if (L == 1) {
            FOR_OWN(i, m)
                b[i] = Kr[i];
        } else {
            segPass<T>(m, [&](int i, int j, int seg) { return restrictPart(l, i, j, seg); },
                       [&](int i, T bi) { b[i] = bi; });
        }
        sync();
        // the coarsest solve stays FP64 in both forms: the coarsest level of the
        // pinned all-Neumann pressure system is nearly singular, and an FP32
        // copy of its inverse loses the coarse correction
        const double *inv = (m <= 32) ? S.coarse : W.dense0 + m;
        const int ld = (m <= 32) ? m : m2;
        segPass<double>(m,
                        [&](int i, int j, int seg) {
                            const double *row = inv + i * ld;
                            double s = 0.0;
                            for (int k = j; k < m; k += seg)
                                s += row[k] * double(b[k]);
                            return s;
                        },
                        [&](int i, double s) { xb[i] = T(s); });
        sync();
    };
    // one level of the up sweep (levels >= 1; level 0 ends in the reduction below):
    // x = x_pre + alpha P x_c, then the post sweeps; the result ends in xb. With a
    // piecewise-constant P (one coarse row per fine row) x is formed inside the first
    // sweep; with a smoothed P it is formed in a phase of its own (into the level's
    // residual slot, free by then), so that the sweep over a wide coarse row loads
    // each neighbour's x once instead of re-forming it from P.
    auto up = [&](int l) {
        const DevAmgLevel &Lv = C.lev[l];
        const int n = Lv.n;
        T *b = vb(l), *xa = b + n, *xb = b + 2 * n, *xi = b + 3 * n;
        const T *rd = b + 4 * n;
        const T *xpre = two ? xb : xa;
        T *out = two ? xa : xb;
        const T *val = amgVal + Lv.valOff;
        if (Lv.pw > 1) {
            for (int i = t0; i < n; i += ts)
                xi[i] = xpre[i] + al * prolong(l, i);
            sync();
            segPass<T>(n,
                       [&](int i, int j, int seg) {
                           return ellDot<T>(Lv.ecol, val, xi, Lv.width, n, i, j, seg);
                       },
                       [&](int i, T ax) { out[i] = xi[i] + om * (b[i] - ax) * rd[i]; });
        } else {
            for (int i = t0; i < n; i += ts) {
                const T x0 = xpre[i] + al * prolong(l, i);
                T ax = T(0);
                for (int k = 0; k < Lv.width; ++k) {
                    const int jj = __ldg(Lv.ecol + k * n + i);
                    if (jj >= 0)
                        ax += val[k * n + i] * (xpre[jj] + al * prolong(l, jj));
                }
                out[i] = x0 + om * (b[i] - ax) * rd[i];
            }
        }
        sync();
        if (two) {
            segPass<T>(n,
                       [&](int i, int j, int seg) {
                           return ellDot<T>(Lv.ecol, val, xa, Lv.width, n, i, j, seg);
                       },
                       [&](int i, T ax) { xb[i] = xa[i] + om * (b[i] - ax) * rd[i]; });
            sync();
        }
    };
    for (int l = 0; l + 1 < L; ++l)
        down(l);
    coarsest();
    for (int l = L - 2; l >= 1; --l)
        up(l);
    const int tid = t0, nt = ts;
    double rz = 0.0;
    if (L > 1 && C.lev[0].pw > 1) { // level 0, smoothed P: x = x_pre + alpha P x_c in a
        // sweep of its own (into rr, free since the restriction to level 1), then the
        // post sweep(s) read it (each x once, not re-formed at every neighbour)
        const int n = C.lev[0].n;
        const T *xprev = two ? Kxb : Kxa;
        T *out = two ? Kxa : Kz;
        FOR_OWN(i, n)
            Krr[i] = xprev[i] + al * prolong(0, i);
        __syncthreads();
        double part = 0.0;
        FOR_OWN(i, n) {
            const T ax = rowDotT(cellOf(C, i), M, Krr, nx);
            const T zi = Krr[i] + om * (Kr[i] - ax) * Krd[i];
            out[i] = zi;
            if (!two)
                part += double(Kr[i]) * double(zi);
        }
        if (two) {
            __syncthreads();
            FOR_OWN(i, n) {
                const T ax = rowDotT(cellOf(C, i), M, Kxa, nx);
                const T zi = Kxa[i] + om * (Kr[i] - ax) * Krd[i];
                Kz[i] = zi;
                part += double(Kr[i]) * double(zi);
            }
        }
        double a[1] = {part};
        blockSum<1>(a, S, rp);
        rz = a[0];
    } else if (L > 1) { // level 0, piecewise-constant P: prolongation fused into the
        // first post sweep (then the second)
        const int n = C.lev[0].n;
        const T *xprev = two ? Kxb : Kxa;
        T *out = two ? Kxa : Kz;
        double part = 0.0;
        FOR_OWN(i, n) {
            const T xi = xprev[i] + al * prolong(0, i);
            const Cell q = cellOf(C, i);
            const int c = i;
            auto X = [&](int jj) { return xprev[jj] + al * prolong(0, jj); };
            const T tW = M.aW[c] * X(q.W), tE = M.aE[c] * X(q.E);
            const T tS = q.south ? M.aS[c] * X(c - nx) : T(0);
            const T tN = q.north ? M.aN[c] * X(c + nx) : T(0);
            const T x1 = q.xEfirst ? tE : tW, x2 = q.xEfirst ? tW : tE;
            const T y1 = q.yNfirst ? tN : tS, y2 = q.yNfirst ? tS : tN;
            const T ax = (((M.d[c] * xi + x1) + x2) + y1) + y2;
            const T zi = xi + om * (Kr[i] - ax) * Krd[c];
            out[i] = zi;
            if (!two)
                part += double(Kr[i]) * double(zi);
        }
        if (two) {
            __syncthreads();
            FOR_OWN(i, n) {
                const T ax = rowDotT(cellOf(C, i), M, Kxa, nx);
                const T zi = Kxa[i] + om * (Kr[i] - ax) * Krd[i];
                Kz[i] = zi;
                part += double(Kr[i]) * double(zi);
            }
        }
        double a[1] = {part};
        blockSum<1>(a, S, rp);
        rz = a[0];
    } else {
        const T *xb = vb(0) + 2 * C.lev[0].n;
        double part = 0.0;
        FOR_OWN(i, n0) {
            Kz[i] = xb[i];
            part += double(Kr[i]) * double(xb[i]);
        }
        double a[1] = {part};
        blockSum<1>(a, S, rp);
        rz = a[0];
    }
    return rz;
}

// The sweeps of one PCG iteration as functions of their own, so that the PCG loop
// itself keeps only a few scalars live across the V-cycle call (every value live
// across a call is saved to and reloaded from local memory around it).
// Ap = A p; returns (p, Ap).
template <typename T> __device__ __noinline__ double pcgMatvec(Shared &S, int &rp, const KW<T> &K) {
    const DevClass &C = S.C;
    const int n = C.n, nx = C.nx;
    const Mat<T> M = matOf(K);
    const T *p = K.pv;
    T *Ap = K.v;
    double a[1] = {0.0};
    FOR_CELLS(c) {
        const T v = rowDotT(cellOf(C, c), M, p, nx);
        Ap[c] = v;
        a[0] += double(p[c]) * double(v);
    }
    blockSum<1>(a, S, rp);
    return a[0];
}
// x += alpha p, r -= alpha Ap; returns (r, r)
template <typename T>
__device__ __noinline__ double pcgUpdate(Shared &S, int &rp, const KW<T> &K, T *x, double alpha) {
    const int n = S.C.n;
    const T *p = K.pv, *Ap = K.v;
    T *r = K.r;
    double a[1] = {0.0};
    FOR_CELLS(c) {
        x[c] += T(alpha) * p[c];
        const T rc = r[c] - T(alpha) * Ap[c];
        r[c] = rc;
        a[0] += double(rc) * double(rc);
    }
    blockSum<1>(a, S, rp);
    return a[0];
}
// z = r / diag; returns (r, z)
template <typename T> __device__ __noinline__ double pcgJacobi(Shared &S, int &rp, const KW<T> &K) {
    const int n = S.C.n;
    const T *r = K.r, *rdv = K.rd;
    T *z = K.z;
    double a[1] = {0.0};
    FOR_CELLS(c) {
        z[c] = r[c] * rdv[c];
        a[0] += double(r[c]) * double(z[c]);
    }
    blockSum<1>(a, S, rp);
    return a[0];
}
// p = z + beta p (beta 0: p = z), then a barrier
template <typename T> __device__ __noinline__ void pcgDirection(Shared &S, const KW<T> &K, double beta) {
    const int n = S.C.n;
    const T *z = K.z;
    T *p = K.pv;
    if (beta == 0.0) {
        FOR_CELLS(c) p[c] = z[c];
    } else {
        FOR_CELLS(c) p[c] = z[c] + T(beta) * p[c];
    }
    __syncthreads();
}
// x += alpha p, r -= alpha Ap; returns (r, r) and the sum of r (the mixed form's
// deflation of the constant vector needs it)
struct Two {
    double a, b;
};
template <typename T>
__device__ __noinline__ Two pcgUpdateSum(Shared &S, int &rp, const KW<T> &K, T *x, double alpha) {
    const int n = S.C.n;
    const T *p = K.pv, *Ap = K.v;
    T *r = K.r;
    double a[2] = {0.0, 0.0};
    FOR_CELLS(c) {
        x[c] += T(alpha) * p[c];
        const T rc = r[c] - T(alpha) * Ap[c];
        r[c] = rc;
        a[0] += double(rc) * double(rc);
        a[1] += double(rc);
    }
    blockSum<2>(a, S, rp);
    return Two{a[0], a[1]};
}
// the sum of r (the first residual of a solve)
template <typename T> __device__ __noinline__ double sumOf(Shared &S, int &rp, const T *r) {
    const int n = S.C.n;
    double a[1] = {0.0};
    FOR_CELLS(c) a[0] += double(r[c]);
    blockSum<1>(a, S, rp);
    return a[0];
}

// z = M^-1 r of the mixed form: the FP32 V-cycle of S.K32 with the constant vector 1
// deflated in FP64. The pressure system is all-Neumann but for the pin of cell 0, so
// A 1 = rowsum0 e_0 and 1 spans its near-null space; FP32 coarse values round each
// coarse row sum (zero in exact arithmetic) by about 1e-7 of its diagonal, which is
// comparable to that mode's eigenvalue and spoils its coarse correction. So the
// constant mode is solved exactly in FP64 and the V-cycle sees only the rest
// (balancing: M^-1 = Q + (I - Q A) V (I - A Q), Q = 1 (1' A 1)^-1 1', SPD when V is):
//   r~ = r - (1'r) e_0,  y = V r~,  z = y + ((1'r) / rowsum0 - y_0) 1.
// sumR = 1'r; returns (r, z) and (r, z_previous) in FP64 (the latter for the flexible
// direction update: an FP32 V-cycle is symmetric only to its rounding).
template <typename T>
__device__ __noinline__ Two pcgPrecondF32(Shared &S, int &rp, const KW<T> &K, double sumR,
                                          double rowsum0) {
    const int n = S.C.n;
    {
        const KW<float> &F = S.K32;
        const T *r = K.r;
        FOR_CELLS(c) F.r[c] = float(c == 0 ? double(r[c]) - sumR : double(r[c]));
    }
    vcycleT<float>(S, rp, S.K32); // ends with a block reduction: F.z is complete
    const KW<float> &F = S.K32;
    const double shift = sumR / rowsum0 - double(F.z[0]);
    const T *r = K.r;
    T *z = K.z;
    double a[2] = {0.0, 0.0};
    FOR_CELLS(c) {
        const T zc = T(double(F.z[c]) + shift);
        a[1] += double(r[c]) * double(z[c]);
        z[c] = zc;
        a[0] += double(r[c]) * double(zc);
    }
    blockSum<2>(a, S, rp);
    return Two{a[0], a[1]};
}

// PCG (LinearSolver.hpp:184-246 / :908-982) from x = 0 with the Jacobi or the AMG
// preconditioner; K.r holds b and r0n its norm, x receives the solution.
// With F32Precond the AMG V-cycle runs on the FP32 copies (S.K32) while PCG itself
// stays in T = double: the mixed form of the pressure solve.
template <typename T, bool F32Precond>
__device__ __noinline__ LinRes pcgT(Shared &S, int &rp, const KW<T> &K, T *x, double r0n,
                                    int maxIter, double tol, bool amg, bool refresh) {
    LinRes res{0, 0.0, r0n, false};
    if (r0n < 1e-30) {
        res.converged = true;
        return res;
    }
    {
        const int n = S.C.n;
        const T *d = K.d;
        T *rdv = K.rd;
        FOR_CELLS(c) {
            const T dc = d[c];
            rdv[c] = (fabs(double(dc)) > 1e-30) ? T(1) / dc : T(1);
            x[c] = T(0);
        }
        if constexpr (F32Precond) {
            if (amg) { // FP32 copy of the finest level for the FP32 V-cycle
                const KW<float> &F = S.K32;
                const Mat<T> M = matOf(K);
                FOR_CELLS(c) {
                    F.d[c] = float(M.d[c]);
                    F.aW[c] = float(M.aW[c]);
                    F.aE[c] = float(M.aE[c]);
                    F.aS[c] = float(M.aS[c]);
                    F.aN[c] = float(M.aN[c]);
                    F.rd[c] = (fabs(double(F.d[c])) > 1e-30) ? 1.0f / F.d[c] : 1.0f;
                }
                __syncthreads();
            }
        }
    }
    if (amg && refresh) {
        mark(S, 4);
        if constexpr (F32Precond)
            amgRefreshT<float>(S, S.K32);
        else
            amgRefreshT(S, K); // begins with a barrier-separated phase
        mark(S, 5);
    } else {
        __syncthreads();
    }
    // the mixed form deflates the constant vector (pcgPrecondF32): the row sum of the
    // pinned row and the running sum of r
    double rowsum0 = 0.0, sumR = 0.0;
    if constexpr (F32Precond) {
        if (amg) {
            rowsum0 = double(K.d[0]) + double(K.aW[0]) + double(K.aE[0]) + double(K.aS[0]) +
                      double(K.aN[0]);
            sumR = sumOf(S, rp, K.r);
        }
    }
    // (r, z) of the new preconditioned residual; rzPrev receives (r, z_previous) where
    // the flexible update applies (the FP32 V-cycle), else 0
    double rzPrev = 0.0;
    auto precond = [&]() {
        if (!amg)
            return pcgJacobi(S, rp, K);
        if constexpr (F32Precond) {
            const Two u = pcgPrecondF32(S, rp, K, sumR, rowsum0);
            rzPrev = u.b;
            return u.a;
        } else {
            return vcycleT(S, rp, K);
        }
    };
    if constexpr (F32Precond) { // z_previous of the first direction: zero
        const int n = S.C.n;
        FOR_CELLS(c) K.z[c] = T(0);
    }
    double rz = precond();
    pcgDirection(S, K, 0.0);
    for (int it = 0; it < maxIter; ++it) {
        const double pAp = pcgMatvec(S, rp, K);
        if (fabs(pAp) < 1e-30) {
            res.breakdown = true;
            break;
        }
        double rr2;
        if constexpr (F32Precond) {
            const Two u = pcgUpdateSum(S, rp, K, x, rz / pAp);
            rr2 = u.a;
            sumR = u.b;
        } else {
            rr2 = pcgUpdate(S, rp, K, x, rz / pAp);
        }
        const double rn = sqrt(rr2);
        res.iterations = it + 1;
        res.finalRes = rn / r0n;
        if (res.finalRes < tol) {
            res.converged = true;
            return res;
        }
        const double rzNew = precond();
        // Fletcher-Reeves as the reference; Polak-Ribiere (flexible CG) around the
        // FP32 V-cycle
        pcgDirection(S, K, (rzNew - rzPrev) / (rz + 1e-30));
        rz = rzNew;
    }
    return res;
}

// Mixed form of one linear solve: FP32 Krylov (and AMG) iterations for a
// correction of the FP64 solution, with the residual of the FP64 system
// recomputed after each correction (iterative refinement) until it has dropped
// by tol relative to the initial residual or the iteration budget is spent.
// On entry W.b and W.r hold the FP64 right-hand side and b - A x (x = x64) and
// r0n its norm; initialRes is that FP64 norm, as in the plain form.
__device__ __noinline__ LinRes mixedSolve(Shared &S, int &rp, double *x64, double r0n, int maxIter,
                                          double tol, int kind, bool refresh) {
    const DevClass &C = S.C;
    const Work &W = S.W;
    const KW<float> &K = S.K32;
    const int n = C.n, nx = C.nx;
    LinRes out{0, 0.0, r0n, false};
    if (r0n < 1e-30) {
        out.converged = true;
        return out;
    }
    FOR_CELLS(c) {
        K.d[c] = float(W.d[c]);
        K.aW[c] = float(W.aW[c]);
        K.aE[c] = float(W.aE[c]);
        K.aS[c] = float(W.aS[c]);
        K.aN[c] = float(W.aN[c]);
        K.r[c] = float(W.r[c]);
    }
    __syncthreads();
    double rn = r0n;
    bool refreshNow = refresh;
    for (int round = 0; round < 8 && out.iterations < maxIter; ++round) {
        // the FP32 solve targets the remaining reduction of the FP64 residual
        const double innerTol = tol * r0n / rn;
        double an[1] = {0.0};
        FOR_CELLS(c) an[0] += double(K.r[c]) * double(K.r[c]);
        blockSum<1>(an, S, rp);
        const double r32n = sqrt(an[0]);
        LinRes in;
        FOR_CELLS(c) K.x[c] = 0.0f;
        __syncthreads();
        in = bicgstabT<float>(S, rp, K, K.x, r32n, maxIter - out.iterations, innerTol);
        (void)refreshNow;
        out.iterations += in.iterations;
        FOR_CELLS(c) x64[c] += double(K.x[c]);
        __syncthreads();
        double a[1] = {0.0};
        FOR_CELLS(c) {
            const Cell q = cellOf(C, c);
            const double rc = W.b[c] - rowDot(q, W.d, W.aW, W.aE, W.aS, W.aN, x64, nx);
            W.r[c] = rc;
            K.r[c] = float(rc);
            a[0] += rc * rc;
        }
        blockSum<1>(a, S, rp);
        rn = sqrt(a[0]);
        if (rn / r0n < tol) {
            out.converged = true;
            break;
        }
        if (in.iterations == 0 || !isfinite(rn))
            break;
    }
    out.finalRes = rn / r0n;
    return out;
}

// Linear-solve dispatch for the precision of the class.
__device__ __forceinline__ LinRes solveBicg(Shared &S, int &rp, double *x, double r0n, int maxIter,
                                            double tol) {
    if (S.C.st.precision == kMixed)
        return mixedSolve(S, rp, x, r0n, maxIter, tol, kPBicgstab, false);
    return bicgstabT<double>(S, rp, S.K64, x, r0n, maxIter, tol);
}

// The AMG coarse values (Galerkin products and the coarsest inverse) are refreshed
// when the previous pressure solve degraded: more than 1.5x (+2) the PCG iterations
// of the solve right after the last refresh, or stopped short of its tolerance
// other than on the |p.Ap| < 1e-30 guard. That is the rule AMGSolver applies to its
// aggregation (LinearSolver.hpp:924-941), except that a guard exit does not count:
// late in a solve the p' right-hand side is round-off (|b| ~ 1e-15), PCG stops on the
// guard whatever the preconditioner, and fresh coarse values would not change that.
// The stale coarse operator stays SPD, so PCG remains valid; the finest level
// always uses the current matrix.
__device__ __forceinline__ LinRes solvePressure(Shared &S, int &rp, double *x, double r0n,
                                                int maxIter, double tol, int kind,
                                                int &needRefresh, int &itersAfterRefresh) {
    const bool amg = kind == kPAmg;
    const bool refresh = amg && needRefresh;
    LinRes res;
    const bool mixed = S.C.st.precision == kMixed;
    if (kind == kPBicgstab)
        res = mixed ? mixedSolve(S, rp, x, r0n, maxIter, tol, kind, refresh)
                    : bicgstabT<double>(S, rp, S.K64, x, r0n, maxIter, tol);
    else if (mixed) // FP64 PCG, FP32 AMG V-cycle
        res = pcgT<double, true>(S, rp, S.K64, x, r0n, maxIter, tol, amg, refresh);
    else
        res = pcgT<double, false>(S, rp, S.K64, x, r0n, maxIter, tol, amg, refresh);
    if (amg && r0n >= 1e-30) {
        if (refresh) {
            needRefresh = 0;
            itersAfterRefresh = res.iterations;
        } else if (itersAfterRefresh <= 0) {
            itersAfterRefresh = res.iterations;
        } else if ((!res.converged && !res.breakdown) ||
                   res.iterations > 1.5 * itersAfterRefresh + 2) {
            needRefresh = 1;
        }
    }
    return res;
}

// ---------------------------------------------------------------- contraction estimate
// ContractionEstimate (SIMPLESolver.cpp:32-74) over a shared ring of samples;
// every warp evaluates the window maxima with shuffles (max is exact).
struct Est {
    double rate, remaining;
};
__device__ __forceinline__ Est estimate(const Shared &S, int e, int window, double negligible) {
    const int m = window < 2 ? 2 : window;
    const int cnt = S.cnt[e];
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    if (cnt < 2 * m)
        return {__longlong_as_double(0x7ff8000000000000LL), inf};
    const int lane = threadIdx.x & 31;
    double dNew = 0.0, dOld = 0.0;
    for (int l = lane; l < m; l += 32) {
        dNew = dmax(dNew, S.ring[e][(cnt - m + l) % kWindowCap]);
        dOld = dmax(dOld, S.ring[e][(cnt - 2 * m + l) % kWindowCap]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        dNew = dmax(dNew, __shfl_xor_sync(FULL, dNew, o));
        dOld = dmax(dOld, __shfl_xor_sync(FULL, dOld, o));
    }
    double rate;
    if (dOld <= 0.0)
        rate = dNew > 0.0 ? inf : 0.0;
    else
        rate = pow(dNew / dOld, 1.0 / m);
    double remaining;
    if (dNew <= negligible)
        remaining = dNew;
    else if (!(rate < 1.0))
        remaining = inf;
    else
        remaining = dNew * rate / (1.0 - rate);
    return {rate, remaining};
}

__device__ __forceinline__ void pushSample(Shared &S, int e, double v) {
    __syncthreads(); // everyone finished reading the ring
    if (threadIdx.x == 0) {
        S.ring[e][S.cnt[e] % kWindowCap] = v;
        S.cnt[e] += 1;
    }
    __syncthreads();
}

// ---------------------------------------------------------------- the solve
// Workspace placement: arrays in priority order go to the shared-memory arena
// while it has room (the hot Krylov/AMG vectors and the matrix first), the rest
// to this CTA's global workspace, which has a slot for every array.
__device__ void carve(Shared &S, double *ws, double *arena, long arenaDoubles) {
    const DevClass &C = S.C;
    const long n = C.n, nf = C.n + C.nfy;
    Work &W = S.W;
    double *g = ws;
    long used = 0;
    auto take = [&](long cnt) {
        const long sz = (cnt + 31) / 32 * 32;
        double *gp = g;
        g += sz;
        if (used + sz <= arenaDoubles) {
            double *sp = arena + used;
            used += sz;
            return sp;
        }
        return gp;
    };
    auto takeF = [&](long cnt) { return reinterpret_cast<float *>(take((cnt + 1) / 2)); };
    const int m = C.lev[C.nlev - 1].n;
    const bool mixed = C.st.precision == kMixed;
    KW<float> &F = S.K32;
    if (mixed) { // the FP32 inner-solver storage is the hot set of the mixed form
        F.d = takeF(n);
        F.aW = takeF(n);
        F.aE = takeF(n);
        F.aS = takeF(n);
        F.aN = takeF(n);
        F.rd = takeF(n);
        F.r = takeF(n);
        F.pv = takeF(n);
        F.v = takeF(n);
        F.ph = takeF(n);
        F.s = takeF(n);
        F.sh = takeF(n);
        F.t = takeF(n);
        F.rh = takeF(n);
        F.x = takeF(n);
        F.amgVec = takeF(C.amgVecs);
        F.amgVal = takeF(C.amgVals);
        F.z = F.s;
        F.xa = F.t;
        F.xb = F.sh;
        F.rr = F.rh;
    }
    // tier 1: matrix and Krylov vectors
    W.d = take(n);
    W.aW = take(n);
    W.aE = take(n);
    W.aS = take(n);
    W.aN = take(n);
    W.r = take(n);
    if (mixed) { // the mixed form keeps only the FP64 vectors of the pressure PCG
        W.pv = take(n);
        W.v = take(n);
        W.z = take(n);
        W.rd = take(n);
    } else {
        W.pv = take(n);
        W.v = take(n);
        W.ph = take(n);
        W.s = take(n);
        W.sh = take(n);
        W.t = take(n);
        W.rh = take(n);
        W.rd = take(n);
        // the pressure PCG / V-cycle vectors share storage with the BiCGSTAB-only
        // vectors: the two solvers never run at the same time
        W.z = W.s;
        W.xa = W.t;
        W.xb = W.sh;
        W.rr = W.rh;
        W.amgVec = take(C.amgVecs); // tier 2: AMG (vectors first: touched more often)
        W.amgVal = take(C.amgVals);
    }
    // tier 3: solved fields and assembly inputs
    W.pp = take(n);
    W.Ux = take(n);
    W.Uy = take(n);
    W.k = take(n);
    W.w = take(n);
    W.b = take(n);
    W.aP = take(n);
    W.nuT = take(n);
    W.F1 = take(n);
    W.phi = take(nf);
    W.phiPred = take(nf);
    W.pCoeff = take(nf);
    W.fScr = take(nf);
    W.gPx = take(n);
    W.gPy = take(n);
    W.gUxx = take(n);
    W.gUxy = take(n);
    W.gUyx = take(n);
    W.gUyy = take(n);
    W.gKx = take(n);
    W.gKy = take(n);
    W.gWx = take(n);
    W.gWy = take(n);
    // tier 4
    W.p = take(n);
    W.F2 = take(n);
    W.Pk = take(n);
    W.CD = take(n);
    W.S = take(n);
    W.phiOld = take(nf);
    W.aPraw = take(n);
    W.Uxp = take(n);
    W.Uyp = take(n);
    W.kOld = take(n);
    W.wOld = take(n);
    W.dense0 = take(2L * m * m); // [A | I] ping-pong of a coarsest level above 32 rows
    W.dense1 = take(2L * m * m);
    if (mixed) {
        W.ph = W.s = W.sh = W.t = W.rh = nullptr;
        W.xa = W.xb = W.rr = W.amgVec = W.amgVal = nullptr;
    }
    KW<double> &K = S.K64;
    K.d = W.d;
    K.aW = W.aW;
    K.aE = W.aE;
    K.aS = W.aS;
    K.aN = W.aN;
    K.rd = W.rd;
    K.r = W.r;
    K.rh = W.rh;
    K.pv = W.pv;
    K.v = W.v;
    K.s = W.s;
    K.t = W.t;
    K.ph = W.ph;
    K.sh = W.sh;
    K.z = W.z;
    K.xa = W.xa;
    K.xb = W.xb;
    K.rr = W.rr;
    K.x = nullptr;
    K.amgVal = W.amgVal;
    K.amgVec = W.amgVec;
}

// Locals shared by the phase functions (read from the CTA's shared state).
#define RQ_PRELUDE                                                                              \
    const DevClass &C = S.C;                                                                    \
    const Work &W = S.W;                                                                        \
    const DevSettings &st = C.st;                                                               \
    const int n = C.n, nx = C.nx, ny = C.ny, nfy = C.nfy;                                       \
    const double nu = C.nu;                                                                     \
    const double sk1 = S.coeff[0], sw1 = S.coeff[1], b1 = S.coeff[2], al1 = S.coeff[3];         \
    const double sk2 = S.coeff[4], sw2 = S.coeff[5], b2 = S.coeff[6], al2 = S.coeff[7];         \
    const double bs = S.coeff[8], a1 = S.coeff[9];                                              \
    auto blend = [](double p1, double p2, double F1) { return F1 * p1 + (1.0 - F1) * p2; };    \
    auto bwOf = [&](int f) { return wallFaceOmega(C, S.wallBeta, f); };                        \
    (void)st; (void)n; (void)nx; (void)ny; (void)nfy; (void)nu; (void)sk1; (void)sw1;          \
    (void)b1; (void)al1; (void)sk2; (void)sw2; (void)b2; (void)al2; (void)bs; (void)a1;         \
    (void)blend; (void)bwOf;

// ---------------------------------------------------------------- phases
// Each phase is a barrier-free sweep over cells or faces; the caller places
// the barriers and reductions. Phases are separate (non-inlined) functions so
// every sweep gets its own register allocation.
__device__ __noinline__ void phInitCells(Shared &S) {
    RQ_PRELUDE
    const double U0 = C.init[0], U1 = C.init[1], P0 = C.init[3], K0 = C.init[4], W0 = C.init[5];
    FOR_CELLS(c) {
        W.Ux[c] = U0;
        W.Uy[c] = U1;
        W.p[c] = P0;
        W.k[c] = K0;
        const double om = dmax(wallOmega(C, b1, dmax(C.wd[c], 1e-20)), W0);
        W.w[c] = om;
        W.F1[c] = 1.0;
        W.F2[c] = 1.0;
        W.Pk[c] = 0.0;
        W.CD[c] = 0.0;
        W.nuT[c] = a1 * K0 / dmax(a1 * om, 1e-20);
        W.S[c] = 0.0;
    }
}

// A cached converged state (fields layout, 11 x n) in place of the uniform one; the
// strain starts from zero as in solve() (SIMPLESolver.cpp:1205).
__device__ __noinline__ void phInitWarm(Shared &S, const double *wf) {
    RQ_PRELUDE
    FOR_CELLS(c) {
        W.Ux[c] = wf[c];
        W.Uy[c] = wf[n + c];
        W.p[c] = wf[3 * n + c];
        W.k[c] = wf[4 * n + c];
        W.w[c] = wf[5 * n + c];
        W.nuT[c] = wf[6 * n + c];
        W.F1[c] = wf[7 * n + c];
        W.F2[c] = wf[8 * n + c];
        W.Pk[c] = wf[9 * n + c];
        W.CD[c] = wf[10 * n + c];
        W.S[c] = 0.0;
    }
}

__device__ __noinline__ void phInitFlux(Shared &S) {
    RQ_PRELUDE
    for (int f = threadIdx.x; f < n + nfy; f += blockDim.x) {
        double v = 0.0;
        if (f < n) {
            const int q = eastOf(C, f);
            const double w = C.xw[f];
            const double ux = W.Ux[f] * w + W.Ux[q] * (1.0 - w), uy = W.Uy[f] * w + W.Uy[q] * (1.0 - w);
            v = (ux * C.xnx[f] + uy * C.xny[f]) * C.xa[f];
        } else {
            const int g = f - n, jf = rowOf(C, g);
            if (jf > 0 && jf < ny) {
                const int o = g - nx;
                const double w = C.yw[g];
                const double ux = W.Ux[o] * w + W.Ux[g] * (1.0 - w), uy = W.Uy[o] * w + W.Uy[g] * (1.0 - w);
                v = (ux * C.ynx[g] + uy * C.yny[g]) * C.ya[g];
            } else {
                v = (0.0 * C.ynx[g] + 0.0 * C.yny[g]) * C.ya[g];
            }
        }
        W.phi[f] = v;
    }
}

__device__ __noinline__ void phStart(Shared &S, bool turbUpdate) {
    RQ_PRELUDE
        for (int f = threadIdx.x; f < n + nfy; f += blockDim.x) {
            double v = 0.0;
            if (f < n) {
                const int q = eastOf(C, f);
                const double w = C.xw[f];
                const double ux = W.Ux[f] * w + W.Ux[q] * (1.0 - w), uy = W.Uy[f] * w + W.Uy[q] * (1.0 - w);
                v = (ux * C.xnx[f] + uy * C.xny[f]) * C.xa[f];
            } else {
                const int g = f - n, jf = rowOf(C, g);
                if (jf > 0 && jf < ny) {
                    const int o = g - nx;
                    const double w = C.yw[g];
                    const double ux = W.Ux[o] * w + W.Ux[g] * (1.0 - w), uy = W.Uy[o] * w + W.Uy[g] * (1.0 - w);
                    v = (ux * C.ynx[g] + uy * C.yny[g]) * C.ya[g];
                } else {
                    v = (0.0 * C.ynx[g] + 0.0 * C.yny[g]) * C.ya[g];
                }
            }
            W.phiOld[f] = v;
        }
        FOR_CELLS(c) {
            const Cell q = cellOf(C, c);
            W.Uxp[c] = W.Ux[c];
            W.Uyp[c] = W.Uy[c];
            double gx, gy;
            ggCell(C, q, W.Ux, 0.0, 0.0, gx, gy);
            W.gUxx[c] = gx;
            W.gUxy[c] = gy;
            ggCell(C, q, W.Uy, 0.0, 0.0, gx, gy);
            W.gUyx[c] = gx;
            W.gUyy[c] = gy;
            // pressure faces carry the owner value (Neumann walls)
            ggCell(C, q, W.p, W.p[c], W.p[c], gx, gy);
            W.gPx[c] = gx;
            W.gPy[c] = gy;
            if (turbUpdate) {
                ggCell(C, q, W.k, 0.0, 0.0, gx, gy);
                W.gKx[c] = gx;
                W.gKy[c] = gy;
                ggCell(C, q, W.w, bwOf(q.i), bwOf(C.ny * nx + q.i), gx, gy);
                W.gWx[c] = gx;
                W.gWy[c] = gy;
            }
        }
}

__device__ __noinline__ void phClosure(Shared &S, double floorV) {
    RQ_PRELUDE
            FOR_CELLS(c) {
                const double s11 = W.gUxx[c], s22 = W.gUyy[c];
                const double s12 = 0.5 * (W.gUxy[c] + W.gUyx[c]);
                const double Sc = sqrt(2.0 * (s11 * s11 + s22 * s22 + 0.0 + 2.0 * (s12 * s12 + 0.0 + 0.0)));
                W.S[c] = Sc;
                const double kc = dmax(W.k[c], 0.0), wc = dmax(W.w[c], 1e-20);
                const double y = dmax(C.wd[c], 1e-20);
                const double cd = 2.0 * sw2 / dmax(wc, 1e-20) * (W.gKx[c] * W.gWx[c] + W.gKy[c] * W.gWy[c]);
                W.CD[c] = cd;
                const double sqk = sqrt(dmax(kc, 0.0)), ws = dmax(wc, 1e-20);
                const double ys = dmax(y, 1e-20), y2 = ys * ys;
                const double t1 = sqk / (bs * ws * ys);
                const double t2 = 500.0 * nu / (y2 * ws);
                const double t3 = 4.0 * sw2 * dmax(kc, 0.0) / (dmax(cd, 1e-10) * y2);
                const double arg1 = dmin(dmax(t1, t2), t3);
                const double F1 = tanh(arg1 * arg1 * arg1 * arg1);
                W.F1[c] = F1;
                const double u1 = 2.0 * sqk / (bs * ws * ys);
                const double arg2 = dmax(u1, t2);
                const double F2 = tanh(arg2 * arg2);
                W.F2[c] = F2;
                double den = dmax(a1 * wc, Sc * F2);
                den = dmax(den, 1e-20);
                const double nut = a1 * dmax(kc, 0.0) / den;
                const double raw = nut * Sc * Sc;
                const double lim = 10.0 * bs * dmax(kc, 0.0) * dmax(wc, 1e-20);
                W.Pk[c] = dmin(raw, lim);
                W.nuT[c] = dmax(nut, floorV);
            }
}

// gradient of the solved Ux for the y assembly (Uy, and so its gradient from
// phStart, is unchanged until the y solve)
__device__ __noinline__ void phGradU(Shared &S) {
    RQ_PRELUDE
                FOR_CELLS(c) {
                    const Cell q = cellOf(C, c);
                    double gx, gy;
                    ggCell(C, q, W.Ux, 0.0, 0.0, gx, gy);
                    W.gUxx[c] = gx;
                    W.gUxy[c] = gy;
                }
}

// The internal faces of the momentum assembly, each once (assembleMomentum
// :303-482): the diffusion coefficient D = nu_f A / delta (both components: stored
// by the x pass in pCoeff, free until the p' assembly), the transpose-stress flux of
// this component (phiPred, free likewise) and its limitedLinearUpwind deferred
// correction F (phi_f - phi_up) (fScr, :495-532). Wall faces belong to one cell and
// are formed by the cell sweep.
__device__ __noinline__ void phMomentumFaces(Shared &S, int comp) {
    RQ_PRELUDE
            const double *U = comp == 0 ? W.Ux : W.Uy;
            const double *gUc_x = comp == 0 ? W.gUxx : W.gUyx; // grad of this component
            const double *gUc_y = comp == 0 ? W.gUxy : W.gUyy;
            const double *colX = comp == 0 ? W.gUxx : W.gUxy;  // dUx/dx_comp
            const double *colY = comp == 0 ? W.gUyx : W.gUyy;  // dUy/dx_comp
            for (int f = threadIdx.x; f < n + nfy; f += blockDim.x) {
                int fi, o, qn;
                const double *A, *NX, *NY, *WT, *DL;
                double sh = 0.0;
                if (f < n) {
                    fi = f;
                    o = f;
                    qn = eastOf(C, f);
                    A = C.xa; NX = C.xnx; NY = C.xny; WT = C.xw; DL = C.xdl;
                    sh = C.xsh[fi];
                } else {
                    fi = f - n;
                    const int jf = rowOf(C, fi);
                    if (jf == 0 || jf == ny)
                        continue;
                    o = fi - nx;
                    qn = fi;
                    A = C.ya; NX = C.ynx; NY = C.yny; WT = C.yw; DL = C.ydl;
                }
                const double delta = dmax(DL[fi], 1e-20);
                const double F = W.phi[f];
                const double w = WT[fi];
                if (comp == 0) {
                    const double nuO = nu + W.nuT[o], nuN = nu + W.nuT[qn];
                    const double nuF = w * nuO + (1.0 - w) * nuN;
                    W.pCoeff[f] = nuF * A[fi] / delta;
                }
                const double cf = w * W.nuT[o] + (1.0 - w) * W.nuT[qn];
                const double gxf = colX[o] * w + colX[qn] * (1.0 - w);
                const double gyf = colY[o] * w + colY[qn] * (1.0 - w);
                W.phiPred[f] = cf * (gxf * NX[fi] + gyf * NY[fi]) * A[fi];
                double corr = 0.0;
                if (F != 0.0) {
                    const bool ownerUp = F > 0.0;
                    const int up = ownerUp ? o : qn, dn = ownerUp ? qn : o;
                    const double xUx = C.cx[up], xUy = C.cy[up];
                    const double xDx = ownerUp ? C.cx[qn] + sh : C.cx[o] - sh;
                    const double xDy = ownerUp ? C.cy[qn] + 0.0 : C.cy[o] - 0.0;
                    const double dphi = U[dn] - U[up];
                    double psi = 0.0;
                    if (fabs(dphi) > 1e-300) {
                        const double rr = 2.0 * (gUc_x[up] * (xDx - xUx) + gUc_y[up] * (xDy - xUy)) / dphi - 1.0;
                        psi = rr > 0.0 ? (rr * rr + rr) / (rr * rr + 1.0) : 0.0;
                    }
                    const double pf = U[up] + 0.5 * psi * dphi;
                    corr = F * (pf - U[up]);
                }
                W.fScr[f] = corr;
            }
}

// The momentum rows of one component from the face values of phMomentumFaces
// (the wall faces here), summed in the reference's face order; the row's residual.
__device__ __noinline__ void phMomentum(Shared &S, int comp, double (&acc)[3]) {
    RQ_PRELUDE
            double *U = comp == 0 ? W.Ux : W.Uy;
            const double *colX = comp == 0 ? W.gUxx : W.gUxy;  // dUx/dx_comp
            const double *colY = comp == 0 ? W.gUyx : W.gUyy;  // dUy/dx_comp
            const double fb = comp == 0 ? st.fx : st.fy;
            FOR_CELLS(c) {
                const Cell q = cellOf(C, c);
                const int i = q.i, j = q.j;
                // faces: 0 W 1 E 2 S 3 N
                double dT[4], aT[4], tsT[4], ccT[4];
                const bool isWall[4] = {false, false, !q.south, !q.north};
                for (int k = 0; k < 4; ++k) {
                    dT[k] = 0.0;
                    aT[k] = 0.0;
                    tsT[k] = 0.0;
                    ccT[k] = 0.0;
                }
                for (int k = 0; k < 4; ++k) {
                    bool own;
                    int f, fi;
                    const double *A, *DL;
                    if (k < 2) {
                        fi = (k == 0) ? q.W : c;
                        own = (k == 1);
                        A = C.xa; DL = C.xdl;
                        f = fi;
                    } else {
                        fi = (k == 2) ? c : c + nx;
                        own = (k == 3) || isWall[k];
                        A = C.ya; DL = C.ydl;
                        f = n + fi;
                    }
                    const double F = W.phi[f];
                    if (isWall[k]) { // resolved wall: molecular viscosity, U_b = 0
                        const double delta = dmax(DL[fi], 1e-20);
                        const double Db = nu * A[fi] / delta;
                        const double Ub = 0.0;
                        if (F >= 0) {
                            dT[k] = F + Db;
                            tsT[k] = Db * Ub; // boundary source
                        } else {
                            dT[k] = Db;
                            tsT[k] = (Db - F) * Ub;
                        }
                        continue;
                    }
                    const double D = W.pCoeff[f];
                    const double cp = dmax(F, 0.0), cn = dmax(-F, 0.0);
                    dT[k] = own ? D + cp : D + cn;
                    aT[k] = own ? -(D + cn) : -(D + cp);
                    // transpose stress flux through this face (StressOperators.hpp:31-81)
                    const double fl = W.phiPred[f];
                    tsT[k] = own ? fl : -fl;
                    if (F != 0.0) {
                        const double corr = W.fScr[f];
                        ccT[k] = own ? -corr : corr;
                    }
                }
                (void)i;
                (void)j;
                // internal faces first in face order, then the wall (boundary faces come last)
                double dsum = 0.0, bsrc = 0.0, ts = 0.0, bcc;
                {
                    const double x1 = q.xEfirst ? dT[1] : dT[0], x2 = q.xEfirst ? dT[0] : dT[1];
                    dsum = dsum + x1;
                    dsum = dsum + x2;
                    const int y1 = q.yNfirst ? 3 : 2, y2 = q.yNfirst ? 2 : 3;
                    // walls come after internal faces: j == 0 puts S (wall) last via yNfirst
                    if (!isWall[y1])
                        dsum = dsum + dT[y1];
                    if (!isWall[y2])
                        dsum = dsum + dT[y2];
                    if (isWall[y1]) {
                        dsum = dsum + dT[y1];
                        bsrc = bsrc + tsT[y1];
                    }
                    if (isWall[y2]) {
                        dsum = dsum + dT[y2];
                        bsrc = bsrc + tsT[y2];
                    }
                    // transpose stress: internal faces in order, then the zero-coefficient wall
                    const double t1 = q.xEfirst ? tsT[1] : tsT[0], t2 = q.xEfirst ? tsT[0] : tsT[1];
                    ts = ts + t1;
                    ts = ts + t2;
                    if (!isWall[y1])
                        ts = ts + tsT[y1];
                    if (!isWall[y2])
                        ts = ts + tsT[y2];
                    for (int k = 2; k < 4; ++k)
                        if (isWall[k]) {
                            const double gcx = colX[c], gcy = colY[c];
                            const int fi = (k == 2) ? c : c + nx;
                            ts = ts + 0.0 * (gcx * C.ynx[fi] + gcy * C.yny[fi]) * C.ya[fi];
                        }
                    // deferred correction in face order (internal faces only)
                    bcc = 0.0;
                    (void)bcc;
                }
                double bsum = bsrc;
                bsum -= (comp == 0 ? W.gPx[c] : W.gPy[c]) * C.vol[c];
                if (fb != 0.0)
                    bsum += fb * C.vol[c];
                bsum += ts;
                {
                    const double x1 = q.xEfirst ? ccT[1] : ccT[0], x2 = q.xEfirst ? ccT[0] : ccT[1];
                    bsum += x1;
                    bsum += x2;
                    const int y1 = q.yNfirst ? 3 : 2, y2 = q.yNfirst ? 2 : 3;
                    if (!isWall[y1])
                        bsum += ccT[y1];
                    if (!isWall[y2])
                        bsum += ccT[y2];
                }
                const double aU = st.aU;
                const double draw = dsum;
                bsum += (1.0 - aU) / aU * draw * U[c];
                const double dd = draw / aU;
                W.aPraw[c] = draw;
                if (comp == 0)
                    W.aP[c] = dd;
                W.d[c] = dd;
                W.aW[c] = aT[0];
                W.aE[c] = aT[1];
                W.aS[c] = aT[2];
                W.aN[c] = aT[3];
                W.b[c] = bsum;
                // residual b - A U of this row (relaxation cancels at U)
                const double tW = aT[0] * U[q.W], tE = aT[1] * U[q.E];
                const double tS = q.south ? aT[2] * U[c - nx] : 0.0;
                const double tN = q.north ? aT[3] * U[c + nx] : 0.0;
                const double rc = bsum - accum4(q, dd * U[c], tW, tE, tS, tN);
                W.r[c] = rc;
                acc[0] += fabs(rc);
                acc[1] += rc * rc;
                if (comp == 0) {
                    const double un = sqrt(W.Ux[c] * W.Ux[c] + W.Uy[c] * W.Uy[c] + 0.0);
                    const double contribution = draw * un;
                    acc[2] += contribution;
                }
            }
}

__device__ __noinline__ void phPressureFaces(Shared &S, double (&fs)[1]) {
    RQ_PRELUDE
        const double relaxCorr = 1.0 - st.aU;
        for (int f = threadIdx.x; f < n + nfy; f += blockDim.x) {
            int o, q;
            const double *A, *NX, *NY, *WT, *DL, *DX, *DY;
            int fi;
            bool wall = false;
            if (f < n) {
                fi = f;
                o = f;
                q = eastOf(C, f);
                A = C.xa; NX = C.xnx; NY = C.xny; WT = C.xw; DL = C.xdl; DX = C.xdx; DY = C.xdy;
            } else {
                fi = f - n;
                const int jf = rowOf(C, fi);
                wall = (jf == 0 || jf == ny);
                o = fi - nx;
                q = fi;
                A = C.ya; NX = C.ynx; NY = C.yny; WT = C.yw; DL = C.ydl; DX = C.ydx; DY = C.ydy;
            }
            double ph, pc = 0.0;
            if (wall) {
                ph = (0.0 * NX[fi] + 0.0 * NY[fi]) * A[fi];
            } else {
                const double w = WT[fi];
                const double ux = W.Ux[o] * w + W.Ux[q] * (1.0 - w), uy = W.Uy[o] * w + W.Uy[q] * (1.0 - w);
                ph = (ux * NX[fi] + uy * NY[fi]) * A[fi];
                const double delta = dmax(DL[fi], 1e-20);
                const double dO = (fabs(W.aP[o]) > 1e-30) ? C.vol[o] / W.aP[o] : 0.0;
                const double dN = (fabs(W.aP[q]) > 1e-30) ? C.vol[q] / W.aP[q] : 0.0;
                const double dF = w * dO + (1.0 - w) * dN;
                const double dl = dmax(DL[fi], 1e-30);
                const double ex = DX[fi] / dl, ey = DY[fi] / dl;
                const double gbx = W.gPx[o] * w + W.gPx[q] * (1.0 - w);
                const double gby = W.gPy[o] * w + W.gPy[q] * (1.0 - w);
                ph += -dF * A[fi] * ((W.p[q] - W.p[o]) / delta - (gbx * ex + gby * ey));
                ph += relaxCorr * (W.phi[f] - W.phiOld[f]);
                pc = dF * A[fi] / delta;
            }
            W.phiPred[f] = ph;
            W.pCoeff[f] = pc;
            fs[0] += fabs(ph);
        }
}

__device__ __noinline__ void phPressureCells(Shared &S, double (&pacc)[3]) {
    RQ_PRELUDE
        FOR_CELLS(c) {
            const Cell q = cellOf(C, c);
            const int fE = c, fW = q.W, fN = n + c + nx, fS = n + c;
            // diagonal: coefficients of internal faces in order
            const double cW = W.pCoeff[fW], cE = W.pCoeff[fE];
            const double cS = q.south ? W.pCoeff[fS] : 0.0, cN = q.north ? W.pCoeff[fN] : 0.0;
            double dsum = 0.0;
            {
                const double x1 = q.xEfirst ? cE : cW, x2 = q.xEfirst ? cW : cE;
                dsum = dsum + x1;
                dsum = dsum + x2;
                if (q.yNfirst) {
                    if (q.north)
                        dsum = dsum + cN;
                } else {
                    if (q.south)
                        dsum = dsum + cS;
                    if (q.north)
                        dsum = dsum + cN;
                }
            }
            // source: -(owner fluxes) + (neighbour fluxes), walls last
            const double tW = W.phiPred[fW], tE = -W.phiPred[fE];
            double bsum = 0.0;
            {
                const double x1 = q.xEfirst ? tE : tW, x2 = q.xEfirst ? tW : tE;
                bsum += x1;
                bsum += x2;
                if (q.yNfirst) {
                    bsum += -W.phiPred[fN];
                    bsum += -W.phiPred[fS]; // bottom wall
                } else {
                    bsum += q.south ? W.phiPred[fS] : -W.phiPred[fS];
                    bsum += -W.phiPred[fN];
                }
            }
            if (c == 0)
                dsum += fabs(dsum) > 1e-30 ? dsum : 1.0; // pin of the outlet-free system
            W.d[c] = dsum;
            W.aW[c] = -cW;
            W.aE[c] = -cE;
            W.aS[c] = -cS;
            W.aN[c] = -cN;
            W.b[c] = bsum;
            W.r[c] = bsum;
            W.pp[c] = 0.0;
            pacc[0] += fabs(bsum);
            pacc[1] += bsum * bsum;
        }
}

// Pressure-velocity corrections (:916-940, :1443-1467): U -= grad p' V / aP with
// owner-valued wall faces for grad p', p += alpha_p p', the face fluxes from p'; on a
// turbulence update also the k and omega values the change norms compare against.
// The k and omega gradients of the transport equations are the ones phStart formed:
// k and omega do not change between the start of the iteration and their solves.
__device__ __noinline__ void phCorrect(Shared &S, bool turbUpdate) {
    RQ_PRELUDE
        FOR_CELLS(c) {
            const Cell q = cellOf(C, c);
            double gx, gy;
            ggCell(C, q, W.pp, W.pp[c], W.pp[c], gx, gy);
            const double rA = (fabs(W.aP[c]) > 1e-30) ? 1.0 / W.aP[c] : 0.0;
            W.Ux[c] -= rA * gx * C.vol[c];
            W.Uy[c] -= rA * gy * C.vol[c];
            W.p[c] += st.aP * W.pp[c];
            if (turbUpdate) {
                W.kOld[c] = W.k[c];
                W.wOld[c] = W.w[c];
            }
        }
        for (int f = threadIdx.x; f < n + nfy; f += blockDim.x) {
            double v;
            if (f < n) {
                const int q = eastOf(C, f);
                v = W.phiPred[f] - W.pCoeff[f] * (W.pp[q] - W.pp[f]);
            } else {
                const int g = f - n, jf = rowOf(C, g);
                if (jf > 0 && jf < ny)
                    v = W.phiPred[f] - W.pCoeff[f] * (W.pp[g] - W.pp[g - nx]);
                else
                    v = W.phiPred[f] + W.pCoeff[f] * W.pp[jf == 0 ? g : g - nx];
            }
            W.phi[f] = v;
        }
}

// bounds of the solved k and omega (:1489, :1505-1513); a wall cell of omega takes its wall
// value
__device__ __forceinline__ void clampK(const Shared &S, int c) {
    const DevSettings &st = S.C.st;
    S.W.k[c] = dmax(st.kMin, dmin(st.kMax, S.W.k[c]));
}
__device__ __forceinline__ void clampW(const Shared &S, int c) {
    const DevClass &C = S.C;
    const Cell q = cellOf(C, c);
    double v = dmax(C.st.wMin, dmin(1e15, S.W.w[c]));
    if (!q.south || !q.north)
        v = wallOmega(C, S.coeff[2], dmax(C.ydl[wallFaceOf(C, c)], 1e-20));
    S.W.w[c] = v;
}

// The internal faces of the k or omega assembly, each once (assembleKEquation
// :947-1028, assembleOmegaEquation :1030-1171): the diffusion coefficient
// (nu + sigma(F1_f) nuT)_f A / delta (pCoeff), the deferred correction of the
// limitedLinearUpwind face value (fScr, addConvectionCorrection :495-552) and, for
// omega with the near-wall balance, its face term (phiPred, :1073-1087). Wall faces
// are formed by the cell sweep.
__device__ __noinline__ void phTurbFaces(Shared &S, int eq) {
    RQ_PRELUDE
    const double *X = eq == 0 ? W.k : W.w;
    const double *gX = eq == 0 ? W.gKx : W.gWx, *gY = eq == 0 ? W.gKy : W.gWy;
            for (int f = threadIdx.x; f < n + nfy; f += blockDim.x) {
                int fi, o, qn;
                const double *A, *WT, *DL;
                double sh = 0.0;
                const bool xFace = f < n;
                if (xFace) {
                    fi = f;
                    o = f;
                    qn = eastOf(C, f);
                    A = C.xa; WT = C.xw; DL = C.xdl;
                    sh = C.xsh[fi];
                } else {
                    fi = f - n;
                    const int jf = rowOf(C, fi);
                    if (jf == 0 || jf == ny)
                        continue;
                    o = fi - nx;
                    qn = fi;
                    A = C.ya; WT = C.yw; DL = C.ydl;
                }
                const double delta = dmax(DL[fi], 1e-20);
                const double F = W.phi[f];
                const double w = WT[fi];
                const double F1f = w * W.F1[o] + (1.0 - w) * W.F1[qn];
                const double sg = eq == 0 ? blend(sk1, sk2, F1f) : blend(sw1, sw2, F1f);
                const double eO = nu + sg * W.nuT[o], eN = nu + sg * W.nuT[qn];
                const double ef = w * eO + (1.0 - w) * eN;
                W.pCoeff[f] = ef * A[fi] / delta;
                if (eq == 1 && C.balance) { // singular near-wall balance (:1073-1087)
                    const double amp = 6 * nu / b1;
                    const double diff = (C.sing[qn] - C.sing[o]) / delta;
                    const double sgd = xFace ? C.sgx[fi] : C.sgy[fi];
                    W.phiPred[f] = amp * A[fi] * ((ef - nu) * sgd - ef * diff);
                }
                double corr = 0.0;
                if (F != 0.0) {
                    const bool ownerUp = F > 0.0;
                    const int up = ownerUp ? o : qn, dn = ownerUp ? qn : o;
                    const double xDx = ownerUp ? C.cx[qn] + sh : C.cx[o] - sh;
                    const double xDy = ownerUp ? C.cy[qn] + 0.0 : C.cy[o] - 0.0;
                    const double dphi = X[dn] - X[up];
                    double psi = 0.0;
                    if (fabs(dphi) > 1e-300) {
                        const double rr = 2.0 * (gX[up] * (xDx - C.cx[up]) + gY[up] * (xDy - C.cy[up])) / dphi - 1.0;
                        psi = rr > 0.0 ? (rr * rr + rr) / (rr * rr + 1.0) : 0.0;
                    }
                    const double pf = X[up] + 0.5 * psi * dphi;
                    corr = F * (pf - X[up]);
                }
                W.fScr[f] = corr;
            }
}

// The k or omega rows from the face values of phTurbFaces (the wall faces here),
// sources, relaxation and the omega wall constraint, summed in face order.
__device__ __noinline__ void phTurbAssemble(Shared &S, int eq) {
    RQ_PRELUDE
    double *X = eq == 0 ? W.k : W.w;
                FOR_CELLS(c) {
                    if (eq == 1) // the bounds of the k just solved (read below at this cell only)
                        clampK(S, c);
                    const Cell q = cellOf(C, c);
                    const bool isWall[4] = {false, false, !q.south, !q.north};
                    double dT[4] = {0, 0, 0, 0}, aT[4] = {0, 0, 0, 0}, ccT[4] = {0, 0, 0, 0};
                    double bT[4] = {0, 0, 0, 0}, balT[4] = {0, 0, 0, 0};
                    for (int k = 0; k < 4; ++k) {
                        bool own;
                        int fi, f;
                        const double *A, *DL;
                        if (k < 2) {
                            fi = (k == 0) ? q.W : c;
                            own = (k == 1);
                            A = C.xa; DL = C.xdl;
                            f = fi;
                        } else {
                            fi = (k == 2) ? c : c + nx;
                            own = (k == 3) || isWall[k];
                            A = C.ya; DL = C.ydl;
                            f = n + fi;
                        }
                        const double F = W.phi[f];
                        if (isWall[k]) {
                            const double delta = dmax(DL[fi], 1e-20);
                            const double sg = eq == 0 ? blend(sk1, sk2, W.F1[c]) : blend(sw1, sw2, W.F1[c]);
                            const double Db = (nu + sg * W.nuT[c]) * A[fi] / delta;
                            const double xb = eq == 0 ? 0.0 : bwOf(fi);
                            if (F >= 0) {
                                dT[k] = F + Db;
                                bT[k] = Db * xb;
                            } else {
                                dT[k] = Db;
                                bT[k] = (Db - F) * xb;
                            }
                            continue;
                        }
                        const double D = W.pCoeff[f];
                        const double cp = dmax(F, 0.0), cn = dmax(-F, 0.0);
                        dT[k] = own ? D + cp : D + cn;
                        aT[k] = own ? -(D + cn) : -(D + cp);
                        if (eq == 1 && C.balance) {
                            const double corr = W.phiPred[f];
                            balT[k] = own ? corr : -corr;
                        }
                        if (F != 0.0) {
                            const double corr = W.fScr[f];
                            ccT[k] = own ? -corr : corr;
                        }
                    }
                    // face-order sums: internal faces, then the wall face
                    const int y1 = q.yNfirst ? 3 : 2, y2 = q.yNfirst ? 2 : 3;
                    const int x1 = q.xEfirst ? 1 : 0, x2 = q.xEfirst ? 0 : 1;
                    const int ord[4] = {x1, x2, y1, y2};
                    double dsum = 0.0, bsum = 0.0, bal = 0.0;
                    for (int t = 0; t < 4; ++t)
                        if (!isWall[ord[t]]) {
                            dsum = dsum + dT[ord[t]];
                            bal = bal + balT[ord[t]];
                        }
                    for (int t = 0; t < 4; ++t)
                        if (isWall[ord[t]]) {
                            dsum = dsum + dT[ord[t]];
                            bsum = bsum + bT[ord[t]];
                        }
                    const double V = C.vol[c], F1 = W.F1[c];
                    if (eq == 0) {
                        bsum += W.Pk[c] * V;
                        dsum += bs * dmax(W.w[c], 1e-20) * V;
                    } else {
                        const double wc = dmax(W.w[c], 1e-20);
                        const double Sv = W.S[c];
                        const double S2 = Sv * Sv;
                        const double lim = 10.0 * bs * dmax(W.k[c], 0.0) * dmax(W.w[c], 1e-20) / dmax(W.nuT[c], 1e-30);
                        const double prod = dmin(S2, lim);
                        bsum += blend(al1, al2, F1) * prod * V;
                        dsum += blend(b1, b2, F1) * wc * V;
                        bsum += (1.0 - F1) * W.CD[c] * V;
                        if (C.balance) {
                            const double corr = bal + nu * (6 * nu / b1) * C.slap[c] * V;
                            if (corr < 0)
                                dsum -= corr / wc;
                            else
                                bsum += corr;
                        }
                    }
                    for (int t = 0; t < 4; ++t)
                        if (!isWall[ord[t]])
                            bsum += ccT[ord[t]];
                    const double al = eq == 0 ? st.aK : st.aW;
                    bsum += (1.0 - al) / al * dsum * X[c];
                    dsum /= al;
                    // omega: eliminate constrained wall cells (constrainOmega :687-704)
                    double x0 = X[c];
                    if (eq == 1) {
                        const int nbc[4] = {q.W, q.E, c - nx, c + nx};
                        const bool selfW = !q.south || !q.north;
                        for (int t = 0; t < 4; ++t) {
                            const int k = ord[t];
                            if (isWall[k])
                                continue;
                            const int qq = nbc[k];
                            const bool nbW = qq < nx || qq >= n - nx; // first or last row
                            const bool own = (k == 1 || k == 3);
                            if (own) {
                                if (selfW) {
                                    aT[k] = 0.0;
                                } else if (nbW) {
                                    bsum -= aT[k] * wallOmega(C, b1, dmax(C.ydl[wallFaceOf(C, qq)], 1e-20));
                                    aT[k] = 0.0;
                                }
                            } else {
                                if (nbW) {
                                    bsum -= aT[k] * wallOmega(C, b1, dmax(C.ydl[wallFaceOf(C, qq)], 1e-20));
                                    aT[k] = 0.0;
                                } else if (selfW) {
                                    aT[k] = 0.0;
                                }
                            }
                        }
                        if (selfW) {
                            const double val = wallOmega(C, b1, dmax(C.ydl[wallFaceOf(C, c)], 1e-20));
                            bsum = dsum * val;
                            x0 = val;
                        }
                    }
                    W.d[c] = dsum;
                    W.aW[c] = aT[0];
                    W.aE[c] = aT[1];
                    W.aS[c] = aT[2];
                    W.aN[c] = aT[3];
                    W.b[c] = bsum;
                    (void)x0;
                }
}

__device__ __noinline__ void phTurbResidual(Shared &S, int eq, double (&acc)[1]) {
    RQ_PRELUDE
    double *X = eq == 0 ? W.k : W.w;
    const double *gX = eq == 0 ? W.gKx : W.gWx, *gY = eq == 0 ? W.gKy : W.gWy;
    (void)gX; (void)gY;
                FOR_CELLS(c) {
                    const Cell q = cellOf(C, c);
                    auto x0 = [&](int cc) {
                        return (eq == 1 && isWallCell(C, cc))
                                   ? wallOmega(C, b1, dmax(C.ydl[wallFaceOf(C, cc)], 1e-20))
                                   : X[cc];
                    };
                    const double tW = W.aW[c] * x0(q.W), tE = W.aE[c] * x0(q.E);
                    const double tS = q.south ? W.aS[c] * x0(c - nx) : 0.0;
                    const double tN = q.north ? W.aN[c] * x0(c + nx) : 0.0;
                    const double xc = x0(c);
                    const double rc = W.b[c] - accum4(q, W.d[c] * xc, tW, tE, tS, tN);
                    W.r[c] = rc;
                    acc[0] += rc * rc;
                    if (eq == 1)
                        X[c] = xc;
                }
}

__device__ __noinline__ void phNorms(Shared &S, bool turbUpdate, double (&mx)[6]) {
    RQ_PRELUDE
        if (turbUpdate && threadIdx.x == 0)
            S.wallBeta = b1;
        FOR_CELLS(c) {
            if (turbUpdate) {
                clampW(S, c);
                mx[0] = dmax(mx[0], fabs(W.k[c]));
                mx[1] = dmax(mx[1], fabs(W.w[c]));
                mx[2] = dmax(mx[2], fabs(W.k[c] - W.kOld[c]));
                mx[3] = dmax(mx[3], fabs(W.w[c] - W.wOld[c]));
            }
            mx[4] = dmax(mx[4], sqrt(W.Ux[c] * W.Ux[c] + W.Uy[c] * W.Uy[c] + 0.0));
            const double ax = W.Ux[c] - W.Uxp[c], ay = W.Uy[c] - W.Uyp[c];
            mx[5] = dmax(mx[5], sqrt(ax * ax + ay * ay + 0.0));
        }
}

__device__ __noinline__ void phProbes(Shared &S) {
    RQ_PRELUDE
            if (threadIdx.x < C.nobs) { // PreparedObservation::evaluate (:678-772)
                const int t = threadIdx.x;
                const int cell = C.pcell[t];
                const double *X = C.obsComp == 0 ? W.Ux : W.Uy;
                const double center = X[cell];
                double bx = 0, by = 0;
                for (int k = 0; k < C.pnnb[t]; ++k) {
                    const int nb = C.pnb[4 * t + k];
                    const double diff = (nb < 0 ? 0.0 : X[nb]) - center;
                    bx += C.pwt[4 * t + k] * C.pdx[4 * t + k] * diff;
                    by += C.pwt[4 * t + k] * C.pdy[4 * t + k] * diff;
                }
                double gx = 0.0, gy = 0.0;
                if (fabs(C.pdet[t]) > 1e-14 * (C.paxx[t] * C.payy[t] + 1e-300)) {
                    gx = (C.payy[t] * bx - C.paxy[t] * by) / C.pdet[t];
                    gy = (C.paxx[t] * by - C.paxy[t] * bx) / C.pdet[t];
                }
                S.q[t] = center + gx * C.pox[t] + gy * C.poy[t];
            }
}

__device__ void runSolve(Shared &S, const DevJob &job) {
    const DevClass &C = S.C;
    const Work &W = S.W;
    const DevSettings &st = C.st;
    const int n = C.n, nx = C.nx, ny = C.ny, nfy = C.nfy;
    const double nu = C.nu;
    int rp = 0;
    // coefficients (InferenceParameterSet order) and their blends (SSTModel.hpp:12-61)
    const double sk1 = S.coeff[0], sw1 = S.coeff[1], b1 = S.coeff[2], al1 = S.coeff[3];
    const double sk2 = S.coeff[4], sw2 = S.coeff[5], b2 = S.coeff[6], al2 = S.coeff[7];
    const double bs = S.coeff[8], a1 = S.coeff[9];
    auto blend = [](double p1, double p2, double F1) { return F1 * p1 + (1.0 - F1) * p2; };
    const double inf = __longlong_as_double(0x7ff0000000000000LL);

    // ---- initUniform (SIMPLESolver.cpp:267-298) and applyAllBCs, or the cached state of
    // a warm start (ForwardModel.cpp:79-82), whose turbulence is established
    if (job.warm)
        phInitWarm(S, job.warm);
    else
        phInitCells(S);
    if (threadIdx.x < 4)
        S.cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0)
        S.wallBeta = job.warm ? job.warmBeta : C.beta1Init;
    if (threadIdx.x == 0) {
        S.haveQPrev = 0;
        S.innerKrylov = 0;
        S.innerPressure = 0;
        for (int t = 0; t < 8; ++t)
            S.stage[t] = 0;
        S.tmark = clock64();
    }
    __syncthreads();
    // phi = interpolated fluxes of the initial state (wall faces carry U_b = 0)
    phInitFlux(S);
    __syncthreads();

    // the loop state lives in shared memory (LoopState); every thread writes the same
    // values, and reads after its own writes
    LoopState &Ls = S.L;
    bool &established = Ls.established, &converged = Ls.converged, &diverged = Ls.diverged;
    int &amgNeed = Ls.amgNeed, &amgAfter = Ls.amgAfter; // AMG coarse-value refresh state
    double &lastK = Ls.lastK, &lastW = Ls.lastW;
    double &worst = Ls.worst, &fluxRef = Ls.fluxRef, &n0x = Ls.n0x, &n0y = Ls.n0y, &n0p = Ls.n0p;
    int &status = Ls.status, &finalIter = Ls.finalIter;
    double &rateU = Ls.rateU;
    established = job.warm != nullptr;
    amgNeed = 1;
    amgAfter = -1;
    lastK = 1.0;
    lastW = 1.0;
    worst = inf;
    fluxRef = 0.0;
    n0x = n0y = n0p = 1.0;
    status = 1;
    finalIter = st.maxIter;
    converged = diverged = false;
    rateU = __longlong_as_double(0x7ff8000000000000LL);


    for (int iter = 0; iter < st.maxIter; ++iter) {
        const bool turbActive = iter >= st.turbStart;
        const bool turbUpdate = turbActive && ((iter - st.turbStart) % st.turbInterval == 0);
        // ---- phase: save U, interpolated old flux, gradients of U and p
        phStart(S, turbUpdate);
        __syncthreads();

        mark(S, 7);
        // ---- SST closure (SSTModel.cpp:157-241) and the startup nuT floor (:1322-1337)
        if (turbUpdate) {
            if (!established && iter >= st.turbStart + st.floorIters)
                established = true;
            const double floorV = established ? 0.0 : 0.1 * nu;
            phClosure(S, floorV);
            __syncthreads();
        }

        mark(S, 1);
        // ---- momentum x then y (assembleMomentum :303-482)
        LinRes *resU = Ls.resU;
        double &momRes = Ls.momRes, &momScale = Ls.momScale;
        for (int comp = 0; comp < 2; ++comp) {
            if (comp == 1) { // gradients of the updated Ux for the y assembly
                phGradU(S);
                __syncthreads();
            }
            double *U = comp == 0 ? W.Ux : W.Uy;
            double acc[3] = {0.0, 0.0, 0.0};
            phMomentumFaces(S, comp);
            __syncthreads();
            phMomentum(S, comp, acc);
            blockSum<3>(acc, S, rp);
            momRes = comp == 0 ? acc[0] : dmax(momRes, acc[0]);
            if (comp == 0)
                momScale = acc[2];
            resU[comp] = solveBicg(S, rp, U, sqrt(acc[1]), st.innerIter, st.innerTol);
            if (threadIdx.x == 0)
                S.innerKrylov += resU[comp].iterations;
            __syncthreads();
        }

        mark(S, 2);
        // ---- predicted flux (stored Rhie-Chow, :1401-1419) and p' assembly (:717-830)
        double fs[1] = {0.0};
        phPressureFaces(S, fs);
        __syncthreads();
        double pacc[3] = {0.0, 0.0, fs[0]};
        phPressureCells(S, pacc);
        blockSum<3>(pacc, S, rp);
        Ls.contScaled = pacc[0] / dmax(pacc[2], 1e-300);
        Ls.fluxScale = pacc[2];
        mark(S, 3);
        LinRes &resP = Ls.resP;
        resP = solvePressure(S, rp, W.pp, sqrt(pacc[1]), st.innerIter, st.innerTol, st.pSolver,
                             amgNeed, amgAfter);
        if (threadIdx.x == 0)
            S.innerPressure += resP.iterations;
        __syncthreads();

        mark(S, 4);
        // ---- corrections (:916-940, :1443-1467)
        phCorrect(S, turbUpdate);
        __syncthreads();

        // ---- turbulence (:1476-1538)
        LinRes &resK = Ls.resK, &resW = Ls.resW;
        resK = LinRes{0, 0, 0, true};
        resW = LinRes{0, 0, 0, true};
        if (turbUpdate) {
            // the clamp of k runs inside the omega assembly and the clamp of omega
            // inside the change norms (each reads only its own cell's value)
            for (int eq = 0; eq < 2; ++eq) { // 0: k, 1: omega
                double *X = eq == 0 ? W.k : W.w;
                double acc[1] = {0.0};
                phTurbFaces(S, eq);
                __syncthreads();
                phTurbAssemble(S, eq);
                __syncthreads();
                // initial residual with the (constrained) initial guess: wall cells of
                // omega start from their wall value (read through x0, never from X,
                // so the in-place update below cannot race with a neighbour's read)
                phTurbResidual(S, eq, acc);
                blockSum<1>(acc, S, rp);
                LinRes rr = solveBicg(S, rp, X, sqrt(acc[0]), st.innerIter, st.innerTol);
                if (eq == 0)
                    resK = rr;
                else
                    resW = rr;
                if (threadIdx.x == 0)
                    S.innerKrylov += rr.iterations;
                __syncthreads();
            }
        }

        mark(S, 6);
        // ---- change norms and bookkeeping (:1520-1715)
        double mx[6] = {1e-30, 1e-30, 0.0, 0.0, 1e-300, 0.0};
        phNorms(S, turbUpdate, mx);
        blockMax<6>(mx, S, rp);
        if (turbUpdate) {
            lastK = mx[2] / mx[0];
            lastW = mx[3] / mx[1];
        }
        Ls.uChange = mx[5] / mx[4];
        // one barrier pair for every sample of this iteration (U, k, omega, monitor)
        __syncthreads();
        if (threadIdx.x == 0) {
            S.ring[0][S.cnt[0] % kWindowCap] = Ls.uChange;
            S.cnt[0] += 1;
            if (turbUpdate) {
                S.ring[1][S.cnt[1] % kWindowCap] = lastK;
                S.cnt[1] += 1;
                S.ring[2][S.cnt[2] % kWindowCap] = lastW;
                S.cnt[2] += 1;
            }
        }
        __syncthreads();
        const bool haveMonitor = C.nobs > 0;
        if (haveMonitor && iter % (st.monitorInterval > 1 ? st.monitorInterval : 1) == 0) {
            phProbes(S);
            __syncthreads();
            bool finite = true;
            for (int t = 0; t < C.nobs; ++t)
                finite = finite && isfinite(S.q[t]);
            if (!finite) { // the reference throws here: the row becomes Unknown
                status = 4;
                finalIter = iter;
                break;
            }
            if (S.haveQPrev) {
                double qMax = 0.0, dq = 0.0;
                for (int t = 0; t < C.nobs; ++t)
                    qMax = dmax(qMax, fabs(S.q[t]));
                for (int t = 0; t < C.nobs; ++t) {
                    const double fl = C.obsFloor[t];
                    dq = dmax(dq, fabs(S.q[t] - S.qPrev[t]) / dmax(dmax(fabs(S.q[t]), fl), 1e-300));
                }
                pushSample(S, 3, dq);
            }
            __syncthreads();
            if (threadIdx.x < C.nobs)
                S.qPrev[threadIdx.x] = S.q[threadIdx.x];
            if (threadIdx.x == 0)
                S.haveQPrev = 1;
            __syncthreads();
        }
        // the history entry of this iteration (ResidualEntry order); no phase call follows
        const double tol = st.tol, negligible = 0.01 * tol;
        double e[11];
        e[0] = iter;
        e[1] = resU[0].initialRes;
        e[2] = resU[1].initialRes;
        e[3] = 0.0;
        e[4] = resP.initialRes;
        e[5] = turbActive ? lastK : 0.0;
        e[6] = turbActive ? lastW : 0.0;
        e[7] = momRes / dmax(momScale, 1e-300);
        e[8] = Ls.contScaled;
        e[9] = Ls.uChange;
        e[10] = inf;
        if (iter == 0) {
            n0x = dmax(e[1], 1e-30);
            n0y = dmax(e[2], 1e-30);
            n0p = dmax(e[4], 1e-30);
            fluxRef = Ls.fluxScale;
        } else if (iter < 50) {
            n0p = dmax(n0p, e[4]);
            fluxRef = dmax(fluxRef, Ls.fluxScale);
        }
        auto safe = [](double v, double ref) { return ref < 1e-20 ? 0.0 : v / ref; };
        const double nm = dmax(n0x, n0y);
        const double nUx = safe(e[1], nm), nUy = safe(e[2], nm);
        const double nP = safe(e[4], dmax(n0p, fluxRef));
        double maxRes = dmax(dmax(nUx, nUy), nP);
        if (turbActive)
            maxRes = dmax(dmax(maxRes, lastK), lastW);
        bool bad = !isfinite(lastK) || !isfinite(lastW);
        for (int t = 1; t <= 9; ++t)
            bad = bad || !isfinite(e[t]);
        if (bad)
            maxRes = inf;
        // The contraction estimates only change the verdict when every directly
        // measured quantity already passes, so they are evaluated then, on the
        // last iteration, on a divergence exit and for recorded history.
        const double qLast = (haveMonitor && S.cnt[3] > 0) ? S.ring[3][(S.cnt[3] - 1) % kWindowCap] : inf;
        double cheap = dmax(dmax(e[7], e[8]), e[9]);
        if (turbActive)
            cheap = dmax(dmax(cheap, lastK), lastW);
        if (haveMonitor)
            cheap = dmax(cheap, qLast);
        const bool divergingNow = isnan(maxRes) || isinf(maxRes) || maxRes > st.divLimit;
        const bool needEst = cheap < tol || iter == st.maxIter - 1 || divergingNow ||
                             (job.hist && iter < job.histCap);
        double w;
        if (needEst) {
            const Est eU = estimate(S, 0, st.window, negligible);
            e[10] = eU.remaining;
            rateU = eU.rate;
            double wv = e[7];
            wv = dmax(wv, e[8]);
            wv = dmax(wv, e[9]);
            wv = dmax(wv, e[10]);
            if (turbActive) {
                const Est eK = estimate(S, 1, st.window, negligible);
                const Est eW = estimate(S, 2, st.window, negligible);
                wv = dmax(wv, lastK);
                wv = dmax(wv, eK.remaining);
                wv = dmax(wv, lastW);
                wv = dmax(wv, eW.remaining);
            }
            if (haveMonitor) {
                const Est eQ = estimate(S, 3, st.window, negligible);
                wv = dmax(wv, qLast);
                wv = dmax(wv, eQ.remaining);
            }
            w = isfinite(wv) ? wv : inf;
        } else {
            w = cheap; // >= tol: not a verdict iteration
        }
        if (job.hist && iter < job.histCap && threadIdx.x == 0)
            for (int t = 0; t < 11; ++t)
                job.hist[11L * iter + t] = e[t];
        if (bad)
            w = inf;
        worst = w;
        const bool turbScheduled = st.turbStart < st.maxIter;
        if (w < tol && iter > 0 && (!turbScheduled || (turbActive && established))) {
            converged = true;
            finalIter = iter;
            status = 0;
            break;
        }
        if (isnan(maxRes) || isinf(maxRes) || maxRes > st.divLimit) {
            diverged = true;
            finalIter = iter;
            status = 2;
            break;
        }
    }
    __syncthreads();
    const bool stalled = !converged && !diverged && status == 1 && isfinite(rateU) && rateU >= 1.0;

    // ---- outputs: verdict, probe predictions, log-likelihood (ObservationOperator.hpp:592-609)
    if (status == 0 || status == 1) {
        phProbes(S);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        RowOut o;
        o.iterations = finalIter;
        o.stalled = stalled;
        o.converged = converged;
        o.finalWorst = worst;
        o.contractionRate = rateU;
        o.status = status;
        o.loglik = status == 2 ? -1e6 : (status == 4 ? -1e6 : 0.0);
        if (status == 0 || status == 1) {
            double ll = 0.0;
            bool ok = true;
            for (int t = 0; t < C.nobs; ++t) {
                const double v = S.q[t];
                job.pred[t] = v;
                ok = ok && isfinite(v);
                const double diff = v - C.obsVal[t];
                ll += -0.5 * diff * diff / C.obsVar[t];
            }
            if (!ok || !isfinite(ll)) {
                o.status = 4;
                o.loglik = -1e6;
            } else {
                o.loglik = ll;
            }
        }
        if (o.status != 0 && o.status != 1)
            for (int t = 0; t < C.nobs; ++t)
                job.pred[t] = __longlong_as_double(0x7ff8000000000000LL);
        *job.row = o;
    }
    if (job.fields && status != 2) {
        const double *src[11] = {W.Ux, W.Uy, nullptr, W.p, W.k, W.w, W.nuT, W.F1, W.F2, W.Pk, W.CD};
        for (int b = 0; b < 11; ++b)
            FOR_CELLS(c) job.fields[(long)b * n + c] = src[b] ? src[b][c] : 0.0;
    } else if (job.fields) { // a diverged solve leaves no valid state (ForwardModel.cpp:88-96)
        for (long e = threadIdx.x; e < 11L * n; e += blockDim.x)
            job.fields[e] = __longlong_as_double(0x7ff8000000000000LL);
    }
    if (job.snap && status != 2) {
        for (int f = threadIdx.x; f < n + nfy; f += blockDim.x)
            job.snap[f] = W.phi[f];
        if (threadIdx.x == 0) {
            job.snap[n + nfy] = S.wallBeta;
            job.snap[n + nfy + 1] = established ? 1.0 : 0.0;
        }
    }
    __syncthreads();
}

} // namespace

// One job on this CTA: class descriptor into shared memory, admission and unpack
// of theta (InferenceParameterSet::inBounds / unpack), the solve or the
// InvalidParameters row, then the per-row timing record.
__device__ void runJob(Shared &S, const DevJob &job, double *ws, double *arena, int arenaDoubles) {
    long long t0 = 0;
    if (threadIdx.x == 0)
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    {
        const int words = sizeof(DevClass) / 4;
        const int *src = reinterpret_cast<const int *>(job.cls);
        int *dst = reinterpret_cast<int *>(&S.C);
        for (int t = threadIdx.x; t < words; t += blockDim.x)
            dst[t] = src[t];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        bool ok = true;
        for (int i = 0; i < 11; ++i)
            S.coeff[i] = S.C.base[i];
        for (int a = 0; a < S.C.nActive; ++a) {
            const int idx = S.C.active[a];
            const double v = job.theta[a];
            if (v < S.C.lo[idx] || v > S.C.hi[idx] || isnan(v) || isinf(v))
                ok = false;
            S.coeff[idx] = v;
        }
        S.admitted = ok;
        if (ok)
            carve(S, ws, arena, arenaDoubles);
    }
    __syncthreads();
    if (S.admitted) {
        runSolve(S, job);
    } else {
        if (threadIdx.x == 0) {
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
            RowOut o{3, 0, 0, 0, -1e30, nan, nan};
            *job.row = o;
        }
        for (int t = threadIdx.x; t < S.C.nobs; t += blockDim.x)
            job.pred[t] = __longlong_as_double(0x7ff8000000000000LL);
        if (job.fields)
            for (long e = threadIdx.x; e < 11L * S.C.n; e += blockDim.x)
                job.fields[e] = __longlong_as_double(0x7ff8000000000000LL);
    }
    __syncthreads();
    if (threadIdx.x == 0 && job.clock) {
        long long t1;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
        job.clock[0] = t0;
        job.clock[1] = t1;
        job.clock[2] = S.admitted ? S.innerKrylov : 0;
        job.clock[3] = S.admitted ? S.innerPressure : 0;
        for (int t = 0; t < 8; ++t)
            job.clock[4 + t] = S.admitted ? S.stage[t] : 0;
    }
}

__device__ __forceinline__ long long globalNs() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// One kernel body, instantiated per CTA size so each gets its full register budget.
template <int NT>
__global__ void __launch_bounds__(NT) solveKernel(const DevJob *jobs, int njobs, int *nextJob,
                                                  double *wsBase, long wsStride, int arenaDoubles) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    Shared &S = *reinterpret_cast<Shared *>(smemRaw);
    double *arena = reinterpret_cast<double *>(smemRaw + ((sizeof(Shared) + 15) / 16) * 16);
    double *ws = wsBase + wsStride * blockIdx.x;
    for (;;) {
        if (threadIdx.x == 0)
            S.job = atomicAdd(nextJob, 1);
        __syncthreads();
        const int j = S.job;
        if (j >= njobs)
            break;
        runJob(S, jobs[j], ws, arena, arenaDoubles);
    }
}

// The serving loop: persistent CTAs claim requests as the host publishes them.
// Requests live in host-mapped memory (ServeQueue); a CTA claims request h only
// once h < published, by a compare-and-swap on the device-side head, so no
// ticket is ever held for an unpublished request. A CTA leaves when the host
// closes the queue and nothing is left, or after idleNs without work (the host
// launches more CTAs when requests wait and fewer than the slots run); closed = 2
// cancels the requests not yet claimed (solves in flight still finish). A request
// solves in its own pool region when it carries one (DevJob::ws), else in the CTA's
// slot workspace. Results go straight to host-mapped rows; the request's done flag
// is raised after a system-scope fence; every CTA counts its exit.
template <int NT>
__global__ void __launch_bounds__(NT) serveKernel(ServeQueue q, double *wsBase, long wsStride,
                                                  int arenaDoubles) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    Shared &S = *reinterpret_cast<Shared *>(smemRaw);
    double *arena = reinterpret_cast<double *>(smemRaw + ((sizeof(Shared) + 15) / 16) * 16);
    double *ws = wsBase + wsStride * blockIdx.x;
    for (;;) {
        if (threadIdx.x == 0) {
            int got = -1;
            const long long idleFrom = globalNs();
            for (;;) {
                int closed, pub;
                asm volatile("ld.acquire.sys.global.s32 %0, [%1];" : "=r"(closed) : "l"(q.closed) : "memory");
                if (closed >= 2) // cancelled: leave unclaimed requests alone
                    break;
                asm volatile("ld.acquire.sys.global.s32 %0, [%1];" : "=r"(pub) : "l"(q.published) : "memory");
                pub = min(pub, q.capacity);
                const int h = atomicAdd(q.head, 0);
                if (h < pub) {
                    if (atomicCAS(q.head, h, h + 1) == h) {
                        got = h;
                        break;
                    }
                    continue;
                }
                if (closed) // closed and drained
                    break;
                if (globalNs() - idleFrom > q.idleNs) // idle: leave (the host tops up)
                    break;
                __nanosleep(4000);
            }
            S.job = got;
            if (got >= 0)
                S.jd = q.jobs[got];
        }
        __syncthreads();
        const int j = S.job;
        if (j < 0)
            break;
        runJob(S, S.jd, S.jd.ws ? S.jd.ws : ws, arena, arenaDoubles);
        __threadfence_system();
        __syncthreads();
        if (threadIdx.x == 0)
            asm volatile("st.release.sys.global.s32 [%0], %1;" ::"l"(q.done + j), "r"(1) : "memory");
        __syncthreads();
    }
    if (threadIdx.x == 0) // counted so the host can tell how many CTAs still run
        atomicAdd(q.exits, 1);
}

// ---------------------------------------------------------------- allocation-free single solve
// Workspace of rq_evaluate_noalloc: one solve's scratch in a fixed device array
// that the module owns, so that the call itself needs no device allocation. It
// lives on every GPU that loads this library until the process exits.
constexpr long kNoAllocScratchDoubles = 1L << 20; // 8 MiB
static __device__ __align__(256) double g_noallocScratch[kNoAllocScratchDoubles];

// One job passed by value (no job array, no queue counter), solved by one CTA in
// the scratch array.
template <int NT>
__global__ void __launch_bounds__(NT) solveOneKernel(DevJob job, double *ws, int arenaDoubles) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    Shared &S = *reinterpret_cast<Shared *>(smemRaw);
    double *arena = reinterpret_cast<double *>(smemRaw + ((sizeof(Shared) + 15) / 16) * 16);
    if (threadIdx.x == 0)
        S.jd = job;
    __syncthreads();
    runJob(S, S.jd, ws, arena, arenaDoubles);
}

size_t solveSharedBytes() { return ((sizeof(Shared) + 15) / 16) * 16; }

namespace {
template <int NT> void *kernelFor() { return reinterpret_cast<void *>(&solveKernel<NT>); }
template <int NT> void *serveFor() { return reinterpret_cast<void *>(&serveKernel<NT>); }
void *pick(int block) {
    switch (block) {
    case 64: return kernelFor<64>();
    case 128: return kernelFor<128>();
    case 256: return kernelFor<256>();
    case 512: return kernelFor<512>();
    case 768: return kernelFor<768>();
    case 1024: return kernelFor<1024>();
    default: return nullptr;
    }
}
void *pickServe(int block) {
    switch (block) {
    case 256: return serveFor<256>();
    case 512: return serveFor<512>();
    case 768: return serveFor<768>();
    case 1024: return serveFor<1024>();
    default: return nullptr;
    }
}
} // namespace

bool launchVariantExists(int block) { return pick(block) != nullptr; }

int normalizeBlock(int block) {
    return block <= 64 ? 64 : block <= 128 ? 128 : block <= 256 ? 256 : block <= 512 ? 512
         : block <= 768 ? 768 : 1024;
}

cudaError_t launchSolve(const DevJob *jobs, int njobs, int *nextJob, double *ws, long wsStride,
                        int grid, int block, int arenaDoubles, cudaStream_t stream) {
    const size_t smem = solveSharedBytes() + sizeof(double) * static_cast<size_t>(arenaDoubles);
    void *fn = pick(block);
    if (!fn)
        return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    void *args[] = {&jobs, &njobs, &nextJob, &ws, &wsStride, &arenaDoubles};
    e = cudaLaunchKernel(fn, dim3(grid), dim3(block), args, smem, stream);
    if (e != cudaSuccess)
        return e;
    return cudaGetLastError();
}

int solveBlocksPerSM(int block, int arenaDoubles) {
    const size_t smem = solveSharedBytes() + sizeof(double) * static_cast<size_t>(arenaDoubles);
    void *fn = pick(block);
    if (!fn)
        return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
        cudaSuccess)
        return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, block, smem) != cudaSuccess)
        return 0;
    return blocks;
}

cudaError_t launchServe(const ServeQueue &q, double *ws, long wsStride, int grid, int block,
                        int arenaDoubles, cudaStream_t stream) {
    const size_t smem = solveSharedBytes() + sizeof(double) * static_cast<size_t>(arenaDoubles);
    void *fn = pickServe(block);
    if (!fn)
        return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    ServeQueue qq = q;
    void *args[] = {&qq, &ws, &wsStride, &arenaDoubles};
    e = cudaLaunchKernel(fn, dim3(grid), dim3(block), args, smem, stream);
    if (e != cudaSuccess)
        return e;
    return cudaGetLastError();
}

int serveBlocksPerSM(int block, int arenaDoubles) {
    const size_t smem = solveSharedBytes() + sizeof(double) * static_cast<size_t>(arenaDoubles);
    void *fn = pickServe(block);
    if (!fn)
        return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
        cudaSuccess)
        return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, block, smem) != cudaSuccess)
        return 0;
    return blocks;
}

long noAllocScratchDoubles() { return kNoAllocScratchDoubles; }

namespace {
template <int NT> void *oneFor() { return reinterpret_cast<void *>(&solveOneKernel<NT>); }
void *pickOne(int block) {
    switch (block) {
    case 64: return oneFor<64>();
    case 128: return oneFor<128>();
    case 256: return oneFor<256>();
    case 512: return oneFor<512>();
    case 768: return oneFor<768>();
    case 1024: return oneFor<1024>();
    default: return nullptr;
    }
}
} // namespace

// The device address of the scratch array on the current device. The host-side name
// of a __device__ array is only a stand-in, not an address a kernel may use, so it is
// looked up with cudaGetSymbolAddress (no allocation; the first lookup on a device
// loads the module there). Callers resolve it once per handle, when the handle is
// created, so that nothing stale survives a device reset.
cudaError_t noAllocScratch(double **out) {
    double *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noallocScratch);
    if (e != cudaSuccess)
        return e;
    *out = p;
    return cudaSuccess;
}

cudaError_t launchSolveNoAlloc(const DevJob &job, double *scratch, int block, int arenaDoubles,
                               cudaStream_t stream) {
    if (!scratch)
        return cudaErrorInvalidDevicePointer;
    double *ws = scratch;
    void *fn = pickOne(block);
    if (!fn)
        return cudaErrorInvalidConfiguration;
    const size_t smem = solveSharedBytes() + sizeof(double) * static_cast<size_t>(arenaDoubles);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    DevJob j = job;
    void *args[] = {&j, &ws, &arenaDoubles};
    e = cudaLaunchKernel(fn, dim3(1), dim3(block), args, smem, stream);
    if (e != cudaSuccess)
        return e;
    return cudaGetLastError();
}

} // namespace rq
