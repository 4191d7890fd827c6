// Standalone batched linear solves on the device: one CTA per LDU system,
// persistent CTAs pulling systems from a queue (largest first, as the host
// orders them). The solvers restate core/include/LinearSolver.hpp on CSR:
//   PCG (:184-246) with the Jacobi preconditioner or the AMG V-cycle of this
//   project (damped-Jacobi smoothing, aggregate-sum restriction, aggregate
//   broadcast prolongation scaled by an over-correction factor, dense coarsest
//   inverse), right-Jacobi BiCGSTAB
//   (:251-345), and a mixed form: FP32 PCG corrections inside an FP64
//   residual-refinement loop.
// Level 0 keeps the reference's matvec order per row (diagonal, then faces in
// increasing index); coarse levels are column-sorted CSR. Every dot product
// and norm is an FP64 block reduction whose result all threads share, so
// control flow is uniform and results do not depend on the launch shape.
#include "rq_lin.cuh"

#include <cuda_runtime.h>

namespace rq {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr double kOmega = 0.75; // damped-Jacobi weight of the V-cycle smoother
// Scale of the coarse-grid correction: piecewise-constant prolongation under-
// corrects smooth error, and over-correcting by 1.7 cuts the PCG iterations of
// the log-normal Poisson systems from 100 to 30 at 256 x 256 (CPU restatement).
constexpr double kAlpha = 1.7;
constexpr int kSweeps = 2;     // pre- and post-smoothing sweeps
constexpr int kMixedRounds = 12;
constexpr double kMixedInnerTol = 1e-4; // relative drop asked of each FP32 correction

template <int NT> struct LinShared {
    DevLinSys sys;
    double red[4][NT / 32];
    int job;
};

// Sum of K per-thread values over the CTA. Each warp reduces by shuffles, lane 0
// parks the partial, and every warp re-reduces all partials in the same order,
// so every thread returns the same bits.
template <int NT, int K> __device__ __forceinline__ void blockSum(double (&v)[K], LinShared<NT> &S) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1)
            v[k] += __shfl_xor_sync(FULL, v[k], o);
    __syncthreads(); // the previous reduction's readers are done with red
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k)
            S.red[k][warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = lane < NT / 32 ? S.red[k][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1)
            s += __shfl_xor_sync(FULL, s, o);
        v[k] = __shfl_sync(FULL, s, 0);
    }
}

// one level of the hierarchy in value type T (FP64, or the FP32 copies)
template <typename T> struct Lv {
    int n, nc;
    const int *ptr, *col;
    const T *val, *rdg;
    const int *agg, *childPtr, *childIdx;
    T *b, *x, *r; // workspace vectors (levels >= 1; level 0 uses the caller's)
};

template <typename T> __device__ __forceinline__ T rowTimes(const Lv<T> &A, int i, const T *x) {
    const int k0 = __ldg(A.ptr + i), k1 = __ldg(A.ptr + i + 1);
    T s = T(0);
    for (int k = k0; k < k1; ++k)
        s += __ldg(A.val + k) * x[__ldg(A.col + k)];
    return s;
}

template <typename T> __device__ __forceinline__ Lv<T> levelOf(const DevLinSys &S, int l, void *ws);

template <> __device__ __forceinline__ Lv<double> levelOf<double>(const DevLinSys &S, int l, void *ws) {
    const DevLinLevel &d = S.lev[l];
    double *w = static_cast<double *>(ws);
    return Lv<double>{d.n, d.nc, d.ptr, d.col, d.val, d.rdg, d.agg, d.childPtr, d.childIdx,
                      w + d.vecOff, w + d.vecOff + d.n, w + d.vecOff + 2L * d.n};
}
template <> __device__ __forceinline__ Lv<float> levelOf<float>(const DevLinSys &S, int l, void *ws) {
    const DevLinLevel &d = S.lev[l];
    float *w = static_cast<float *>(ws);
    return Lv<float>{d.n, d.nc, d.ptr, d.col, d.val32, d.rdg32, d.agg, d.childPtr, d.childIdx,
                     w + d.vecOff, w + d.vecOff + d.n, w + d.vecOff + 2L * d.n};
}

// z = M^-1 r by one V-cycle: damped Jacobi from zero, residual restricted by
// aggregate sums, the coarsest level by its dense inverse, the correction
// broadcast back and the same sweeps after it (a symmetric preconditioner).
// lvws: the level vectors of levels >= 1; t: a level-0 scratch vector.
template <int NT, typename T>
__device__ void vcycle(LinShared<NT> &S, const T *r, T *z, T *t, void *lvws, const T *inv) {
    const DevLinSys &sys = S.sys;
    const int L = sys.nlev;
    const T w = T(kOmega);
    if (L == 1) { // the whole system is the coarsest level
        const int m = sys.m;
        for (int i = threadIdx.x; i < m; i += NT) {
            T s = T(0);
            for (int j = 0; j < m; ++j)
                s += inv[i * m + j] * r[j];
            z[i] = s;
        }
        __syncthreads();
        return;
    }
    for (int l = 0; l + 1 < L; ++l) {
        Lv<T> A = levelOf<T>(sys, l, lvws);
        const T *b = l == 0 ? r : A.b;
        T *x = l == 0 ? z : A.x;
        T *res = l == 0 ? t : A.r;
        for (int i = threadIdx.x; i < A.n; i += NT)
            x[i] = w * b[i] * __ldg(A.rdg + i);
        __syncthreads();
        for (int s = 1; s < kSweeps; ++s) {
            for (int i = threadIdx.x; i < A.n; i += NT)
                res[i] = b[i] - rowTimes(A, i, x);
            __syncthreads();
            for (int i = threadIdx.x; i < A.n; i += NT)
                x[i] += w * res[i] * __ldg(A.rdg + i);
            __syncthreads();
        }
        for (int i = threadIdx.x; i < A.n; i += NT)
            res[i] = b[i] - rowTimes(A, i, x);
        __syncthreads();
        Lv<T> Cn = levelOf<T>(sys, l + 1, lvws);
        for (int I = threadIdx.x; I < A.nc; I += NT) {
            T s = T(0);
            for (int k = __ldg(A.childPtr + I); k < __ldg(A.childPtr + I + 1); ++k)
                s += res[__ldg(A.childIdx + k)];
            Cn.b[I] = s;
        }
        __syncthreads();
    }
    {
        Lv<T> Cl = levelOf<T>(sys, L - 1, lvws);
        const int m = Cl.n;
        for (int i = threadIdx.x; i < m; i += NT) {
            T s = T(0);
            for (int j = 0; j < m; ++j)
                s += inv[i * m + j] * Cl.b[j];
            Cl.x[i] = s;
        }
        __syncthreads();
    }
    for (int l = L - 2; l >= 0; --l) {
        Lv<T> A = levelOf<T>(sys, l, lvws);
        const Lv<T> Cn = levelOf<T>(sys, l + 1, lvws);
        const T *b = l == 0 ? r : A.b;
        T *x = l == 0 ? z : A.x;
        T *res = l == 0 ? t : A.r;
        for (int i = threadIdx.x; i < A.n; i += NT)
            x[i] += T(kAlpha) * Cn.x[__ldg(A.agg + i)];
        __syncthreads();
        for (int s = 0; s < kSweeps; ++s) {
            for (int i = threadIdx.x; i < A.n; i += NT)
                res[i] = b[i] - rowTimes(A, i, x);
            __syncthreads();
            for (int i = threadIdx.x; i < A.n; i += NT)
                x[i] += w * res[i] * __ldg(A.rdg + i);
            __syncthreads();
        }
    }
}

template <int NT, typename T>
__device__ __forceinline__ void precondition(LinShared<NT> &S, bool amg, const T *r, T *z, T *t,
                                             void *lvws, const T *inv, const T *rdg0) {
    if (amg) {
        vcycle<NT, T>(S, r, z, t, lvws, inv);
    } else {
        for (int i = threadIdx.x; i < S.sys.n; i += NT)
            z[i] = r[i] * __ldg(rdg0 + i);
        __syncthreads();
    }
}

struct PcgOut {
    int iterations;
    bool converged;
    double finalRes;
};

// PCG from x (in T) with r = b - A x already in r and r0n = ||r||; the
// reference's loop (LinearSolver.hpp:206-245). Vectors r, z, p, q, t: n each.
template <int NT, typename T>
__device__ PcgOut pcg(LinShared<NT> &S, const Lv<T> &A0, T *x, T *r, T *z, T *p, T *q, T *t,
                      void *lvws, const T *inv, double r0n, int maxIter, double tol, bool amg) {
    const int n = A0.n;
    PcgOut o{0, false, 0.0};
    precondition<NT, T>(S, amg, r, z, t, lvws, inv, A0.rdg);
    double a[1] = {0.0};
    for (int i = threadIdx.x; i < n; i += NT) {
        p[i] = z[i];
        a[0] += double(r[i]) * double(z[i]);
    }
    blockSum<NT, 1>(a, S);
    double rz = a[0];
    for (int it = 0; it < maxIter; ++it) {
        double b1[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            const T v = rowTimes(A0, i, p);
            q[i] = v;
            b1[0] += double(p[i]) * double(v);
        }
        blockSum<NT, 1>(b1, S);
        const double pAp = b1[0];
        if (fabs(pAp) < 1e-30)
            break;
        const double alpha = rz / pAp;
        double b2[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            x[i] += T(alpha) * p[i];
            const T ri = r[i] - T(alpha) * q[i];
            r[i] = ri;
            b2[0] += double(ri) * double(ri);
        }
        blockSum<NT, 1>(b2, S);
        o.iterations = it + 1;
        o.finalRes = sqrt(b2[0]) / r0n;
        if (o.finalRes < tol) {
            o.converged = true;
            return o;
        }
        precondition<NT, T>(S, amg, r, z, t, lvws, inv, A0.rdg);
        double b3[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += NT)
            b3[0] += double(r[i]) * double(z[i]);
        blockSum<NT, 1>(b3, S);
        const double beta = b3[0] / (rz + 1e-30);
        for (int i = threadIdx.x; i < n; i += NT)
            p[i] = z[i] + T(beta) * p[i];
        __syncthreads();
        rz = b3[0];
    }
    return o;
}

// Right-Jacobi BiCGSTAB (LinearSolver.hpp:251-345) in FP64; r holds b - A x.
template <int NT>
__device__ PcgOut bicgstab(LinShared<NT> &S, const Lv<double> &A0, double *x, double *ws,
                           double r0n, int maxIter, double tol) {
    const int n = A0.n;
    double *r = ws, *rh = ws + n, *p = ws + 2L * n, *v = ws + 3L * n, *s = ws + 4L * n,
           *t = ws + 5L * n, *ph = ws + 6L * n, *sh = ws + 7L * n;
    PcgOut o{0, false, 0.0};
    double a[1] = {0.0};
    for (int i = threadIdx.x; i < n; i += NT) {
        rh[i] = r[i];
        p[i] = 0.0;
        v[i] = 0.0;
        a[0] += r[i] * r[i];
    }
    blockSum<NT, 1>(a, S);
    double rhoN = a[0], rho = 1, alpha = 1, omega = 1;
    for (int it = 0; it < maxIter; ++it) {
        if (fabs(rhoN) < 1e-30)
            break;
        const double beta = (rhoN / (rho + 1e-30)) * (alpha / (omega + 1e-30));
        for (int i = threadIdx.x; i < n; i += NT) {
            const double pi = r[i] + beta * (p[i] - omega * v[i]);
            p[i] = pi;
            ph[i] = pi * __ldg(A0.rdg + i);
        }
        __syncthreads();
        double a1[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            const double vi = rowTimes(A0, i, ph);
            v[i] = vi;
            a1[0] += rh[i] * vi;
        }
        blockSum<NT, 1>(a1, S);
        if (fabs(a1[0]) < 1e-30)
            break;
        alpha = rhoN / a1[0];
        double a2[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            const double si = r[i] - alpha * v[i];
            s[i] = si;
            sh[i] = si * __ldg(A0.rdg + i);
            a2[0] += si * si;
        }
        blockSum<NT, 1>(a2, S);
        const double sn = sqrt(a2[0]);
        if (sn / r0n < tol) {
            for (int i = threadIdx.x; i < n; i += NT)
                x[i] += alpha * ph[i];
            __syncthreads();
            o.iterations = it + 1;
            o.finalRes = sn / r0n;
            o.converged = true;
            return o;
        }
        double a3[2] = {0.0, 0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            const double ti = rowTimes(A0, i, sh);
            t[i] = ti;
            a3[0] += ti * ti;
            a3[1] += ti * s[i];
        }
        blockSum<NT, 2>(a3, S);
        omega = a3[0] > 1e-30 ? a3[1] / a3[0] : 0.0;
        double a4[2] = {0.0, 0.0};
        for (int i = threadIdx.x; i < n; i += NT) {
            x[i] += alpha * ph[i] + omega * sh[i];
            const double ri = s[i] - omega * t[i];
            r[i] = ri;
            a4[0] += ri * ri;
            a4[1] += rh[i] * ri;
        }
        blockSum<NT, 2>(a4, S);
        o.iterations = it + 1;
        o.finalRes = sqrt(a4[0]) / r0n;
        if (o.finalRes < tol) {
            o.converged = true;
            return o;
        }
        if (fabs(omega) < 1e-30)
            break;
        rho = rhoN;
        rhoN = a4[1];
    }
    __syncthreads();
    return o;
}

// r = b - A x in FP64; returns ||r||
template <int NT>
__device__ double residual(LinShared<NT> &S, const Lv<double> &A0, const double *b,
                           const double *x, double *r) {
    double a[1] = {0.0};
    for (int i = threadIdx.x; i < A0.n; i += NT) {
        const double ri = b[i] - rowTimes(A0, i, x);
        r[i] = ri;
        a[0] += ri * ri;
    }
    blockSum<NT, 1>(a, S);
    return sqrt(a[0]);
}

template <int NT> __device__ void solveOne(LinShared<NT> &S, double *ws) {
    const DevLinSys &sys = S.sys;
    const int n = sys.n;
    const bool amg = sys.kind == kLinAmg;
    const Lv<double> A0 = levelOf<double>(sys, 0, ws + sys.lvOff);
    double *x = sys.x;
    double *r = ws;
    const double r0n = residual<NT>(S, A0, sys.b, x, r);
    LinOut out{0, 0, 0.0, r0n};
    if (r0n < 1e-30) {
        out.converged = 1;
    } else if (sys.kind == kLinBicgstab) {
        const PcgOut o = bicgstab<NT>(S, A0, x, ws, r0n, sys.maxIter, sys.tol);
        out.iterations = o.iterations;
        out.converged = o.converged;
        out.finalRes = o.finalRes;
    } else if (sys.precision == 0) {
        const PcgOut o = pcg<NT, double>(S, A0, x, r, ws + n, ws + 2L * n, ws + 3L * n,
                                         ws + 4L * n, ws + sys.lvOff, sys.inv, r0n, sys.maxIter,
                                         sys.tol, amg);
        out.iterations = o.iterations;
        out.converged = o.converged;
        out.finalRes = o.finalRes;
    } else {
        // mixed: FP32 PCG corrections d (A d = r) inside FP64 residual refinement
        float *f = reinterpret_cast<float *>(ws + sys.f32Off);
        float *fr = f, *fz = f + n, *fp = f + 2L * n, *fq = f + 3L * n, *ft = f + 4L * n,
              *fd = f + 5L * n;
        const Lv<float> F0 = levelOf<float>(sys, 0, f + sys.lvOff32);
        double rn = r0n;
        int total = 0;
        for (int round = 0; round < kMixedRounds && total < sys.maxIter; ++round) {
            for (int i = threadIdx.x; i < n; i += NT) {
                fr[i] = float(r[i]);
                fd[i] = 0.0f;
            }
            __syncthreads();
            const double innerTol = fmax(kMixedInnerTol, 0.5 * sys.tol * r0n / rn);
            const PcgOut o = pcg<NT, float>(S, F0, fd, fr, fz, fp, fq, ft, f + sys.lvOff32,
                                            sys.inv32, rn, sys.maxIter - total, innerTol, amg);
            total += o.iterations;
            for (int i = threadIdx.x; i < n; i += NT)
                x[i] += double(fd[i]);
            __syncthreads();
            rn = residual<NT>(S, A0, sys.b, x, r);
            out.finalRes = rn / r0n;
            if (out.finalRes < sys.tol) {
                out.converged = 1;
                break;
            }
            if (o.iterations == 0)
                break;
        }
        out.iterations = total;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        *sys.out = out;
}

template <int NT>
__global__ void __launch_bounds__(NT, 1) linKernel(const DevLinSys *systems, int nsys, int *next,
                                                double *wsBase, long wsStride) {
    __shared__ LinShared<NT> S;
    double *ws = wsBase + wsStride * blockIdx.x;
    for (;;) {
        if (threadIdx.x == 0)
            S.job = atomicAdd(next, 1);
        __syncthreads();
        const int j = S.job;
        if (j >= nsys)
            break;
        {
            const int words = sizeof(DevLinSys) / 4;
            const int *src = reinterpret_cast<const int *>(systems + j);
            int *dst = reinterpret_cast<int *>(&S.sys);
            for (int t = threadIdx.x; t < words; t += NT)
                dst[t] = src[t];
        }
        __syncthreads();
        solveOne<NT>(S, ws);
        __syncthreads();
    }
}

} // namespace

cudaError_t launchLinear(const DevLinSys *systems, int nsys, int *next, double *ws, long wsStride,
                         int grid, cudaStream_t stream) {
    linKernel<kLinThreads><<<grid, kLinThreads, 0, stream>>>(systems, nsys, next, ws, wsStride);
    return cudaGetLastError();
}

int linBlocksPerSM() {
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, linKernel<kLinThreads>, kLinThreads,
                                                      0) != cudaSuccess)
        return 0;
    return blocks;
}

} // namespace rq
