// Importance weights of a finite posterior on the device, in FP64:
//   w_i = exp(l_i - log q_i - m) / S,  m = max_j (l_j - log q_j),  S = sum_j exp(...)
// (cfdr.statistics.posterior_weights, rans-uq/python/cfdr/statistics.py:217-232,
// with the proposal density of the importance stage, docs/figures/calibration_coverage.py:165-180).
// The reference normalises by an exactly rounded sum (math.fsum); here every
// thread accumulates its terms with Neumaier's compensated summation and the
// (sum, compensation) pairs are combined by error-free TwoSum in a fixed order,
// which keeps the total within an ulp or two of the exact sum.
#include <cuda_runtime.h>

#include <cstdint>

namespace rq {
namespace {

constexpr int kT = 1024;
constexpr unsigned FULL = 0xffffffffu;

// exact s + t = hi + lo (Knuth's TwoSum)
__device__ __forceinline__ void twoSum(double a, double b, double &hi, double &lo) {
    hi = a + b;
    const double bb = hi - a;
    lo = (a - (hi - bb)) + (b - bb);
}

__device__ __forceinline__ void addCompensated(double &s, double &c, double x) {
    double hi, lo;
    twoSum(s, x, hi, lo);
    s = hi;
    c += lo;
}

__global__ void __launch_bounds__(kT) weightsKernel(const double *ll, const double *lq, int64_t n,
                                                    double *w, double *out /* m, S, bad */) {
    __shared__ double sm[kT / 32], sc[kT / 32];
    __shared__ int sb[kT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // pass 1: the maximum and the count of non-finite terms
    double m = -__longlong_as_double(0x7ff0000000000000LL);
    int bad = 0;
    for (int64_t i = threadIdx.x; i < n; i += kT) {
        const double v = ll[i] - (lq ? lq[i] : 0.0);
        if (!isfinite(ll[i]) || !isfinite(v))
            ++bad;
        else
            m = fmax(m, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_xor_sync(FULL, m, o));
        bad += __shfl_xor_sync(FULL, bad, o);
    }
    if (lane == 0) {
        sm[warp] = m;
        sb[warp] = bad;
    }
    __syncthreads();
    m = lane < kT / 32 ? sm[lane] : -__longlong_as_double(0x7ff0000000000000LL);
    bad = lane < kT / 32 ? sb[lane] : 0;
    for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_xor_sync(FULL, m, o));
        bad += __shfl_xor_sync(FULL, bad, o);
    }
    m = __shfl_sync(FULL, m, 0);
    bad = __shfl_sync(FULL, bad, 0);
    if (bad) {
        if (threadIdx.x == 0) {
            out[0] = m;
            out[1] = 0.0;
            out[2] = bad;
        }
        return;
    }
    // pass 2: compensated sum of exp(v - m)
    double s = 0.0, c = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += kT)
        addCompensated(s, c, exp(ll[i] - (lq ? lq[i] : 0.0) - m));
    for (int o = 16; o > 0; o >>= 1) {
        const double s2 = __shfl_xor_sync(FULL, s, o), c2 = __shfl_xor_sync(FULL, c, o);
        double hi, lo;
        twoSum(s, s2, hi, lo);
        s = hi;
        c = c + c2 + lo;
    }
    __syncthreads();
    if (lane == 0) {
        sm[warp] = s;
        sc[warp] = c;
    }
    __syncthreads();
    s = lane < kT / 32 ? sm[lane] : 0.0;
    c = lane < kT / 32 ? sc[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
        const double s2 = __shfl_xor_sync(FULL, s, o), c2 = __shfl_xor_sync(FULL, c, o);
        double hi, lo;
        twoSum(s, s2, hi, lo);
        s = hi;
        c = c + c2 + lo;
    }
    const double total = __shfl_sync(FULL, s + c, 0);
    // pass 3: the normalised weights
    for (int64_t i = threadIdx.x; i < n; i += kT)
        w[i] = exp(ll[i] - (lq ? lq[i] : 0.0) - m) / total;
    if (threadIdx.x == 0) {
        out[0] = m;
        out[1] = total;
        out[2] = 0.0;
    }
}

} // namespace

cudaError_t launchWeights(const double *ll, const double *lq, int64_t n, double *w, double *out,
                          cudaStream_t stream) {
    weightsKernel<<<1, kT, 0, stream>>>(ll, lq, n, w, out);
    return cudaGetLastError();
}

} // namespace rq
