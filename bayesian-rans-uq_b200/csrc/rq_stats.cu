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

// ---- resampling: numpy's Generator.choice(n, p=w) for one uniform per output
// (cdf = w.cumsum(); cdf /= cdf[-1]; index = cdf.searchsorted(u, side='right')).
// The cumulative sum runs in index order on one thread so that every partial sum
// rounds exactly as numpy's sequential cumsum does; the division is elementwise.
__global__ void __launch_bounds__(kT) cdfKernel(const double *w, int64_t n, double *cdf) {
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            s = __dadd_rn(s, w[i]);
            cdf[i] = s;
        }
    }
    __syncthreads();
    const double last = cdf[n - 1];
    __syncthreads();
    for (int64_t i = threadIdx.x; i < n; i += kT)
        cdf[i] = __ddiv_rn(cdf[i], last);
}

// number of cdf values <= u (searchsorted side='right'), one output per thread
__global__ void searchKernel(const double *cdf, int64_t n, const double *u, int64_t m,
                             int64_t *idx) {
    const int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (j >= m)
        return;
    const double v = u[j];
    int64_t lo = 0, hi = n; // first index with cdf > v lies in [lo, hi]
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] <= v)
            lo = mid + 1;
        else
            hi = mid;
    }
    idx[j] = lo;
}

// ---- column moments with numpy's summation order: x.mean(axis=0) and
// x.var(axis=0, ddof=0) of a C-ordered n x d matrix. numpy adds the rows in order
// when d >= 2 and uses its pairwise blocks (8 accumulators over blocks of at most 128,
// halves above) along a single column. Explicit round-to-nearest intrinsics keep
// products and sums from contracting into fused multiply-adds.
constexpr int kPairwiseDepth = 40; // blocks of <= 128 halve: enough below 2^38 rows

// one block of at most 128 terms: 8 accumulators, combined as a tree, then the tail;
// fewer than 8 terms are added in order
__device__ double pairwiseLeaf(const double *x, int64_t n, int64_t stride, double shift,
                               bool square) {
    auto term = [&](int64_t i) {
        const double v = x[i * stride];
        if (!square)
            return v;
        const double dv = __dsub_rn(v, shift);
        return __dmul_rn(dv, dv);
    };
    if (n < 8) {
        double r = -0.0;
        for (int64_t i = 0; i < n; ++i)
            r = __dadd_rn(r, term(i));
        return r;
    }
    double r[8];
    for (int j = 0; j < 8; ++j)
        r[j] = term(j);
    int64_t i = 8;
    for (; i < n - (n % 8); i += 8)
        for (int j = 0; j < 8; ++j)
            r[j] = __dadd_rn(r[j], term(i + j));
    double res = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                           __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
    for (; i < n; ++i)
        res = __dadd_rn(res, term(i));
    return res;
}

// numpy's pairwise sum of a strided column (a block above 128 terms splits at half its
// length rounded down to a multiple of 8), without recursion: each frame holds a block
// length, the sum of its left half once known and which half is pending; blocks are
// reached in index order, so a running position gives every leaf's offset.
__device__ double pairwiseColumn(const double *x, int64_t n, int64_t stride, double shift,
                                 bool square) {
    int64_t len[kPairwiseDepth];
    double left[kPairwiseDepth];
    unsigned char stage[kPairwiseDepth];
    int sp = 0;
    len[0] = n;
    stage[0] = 0;
    int64_t pos = 0;
    double ret = 0.0;
    while (sp >= 0) {
        if (stage[sp] == 0 && len[sp] <= 128) {
            ret = pairwiseLeaf(x + pos * stride, len[sp], stride, shift, square);
            pos += len[sp];
            --sp;
            continue;
        }
        int64_t h = len[sp] / 2;
        h -= h % 8;
        if (stage[sp] == 0) { // descend into the left half
            stage[sp] = 1;
            ++sp;
            len[sp] = h;
            stage[sp] = 0;
        } else if (stage[sp] == 1) { // left half done: descend into the right half
            left[sp] = ret;
            stage[sp] = 2;
            ++sp;
            len[sp] = len[sp - 1] - h;
            stage[sp] = 0;
        } else { // both halves done
            ret = __dadd_rn(left[sp], ret);
            --sp;
        }
    }
    return ret;
}

__global__ void momentsKernel(const double *x, int64_t n, int d, double *mean, double *var) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d)
        return;
    const double rn = static_cast<double>(n);
    double mu;
    if (d == 1) {
        mu = __ddiv_rn(pairwiseColumn(x, n, 1, 0.0, false), rn);
        var[0] = __ddiv_rn(pairwiseColumn(x, n, 1, mu, true), rn);
        mean[0] = mu;
        return;
    }
    double s = x[c];
    for (int64_t r = 1; r < n; ++r)
        s = __dadd_rn(s, x[r * d + c]);
    mu = __ddiv_rn(s, rn);
    const double d0 = __dsub_rn(x[c], mu);
    double q = __dmul_rn(d0, d0);
    for (int64_t r = 1; r < n; ++r) {
        const double dv = __dsub_rn(x[r * d + c], mu);
        q = __dadd_rn(q, __dmul_rn(dv, dv));
    }
    mean[c] = mu;
    var[c] = __ddiv_rn(q, rn);
}

// ---- order statistic: the k-th smallest (1-based) of n nonnegative doubles, exactly
// (np.partition(values, k-1)[k-1]). The bit patterns of nonnegative doubles order as
// the values do, so a most-significant-digit radix select (8 passes of 8 bits) finds
// the k-th key; -0.0 counts as +0.0.
__device__ __forceinline__ unsigned long long keyOf(double v) {
    return v == 0.0 ? 0ull : static_cast<unsigned long long>(__double_as_longlong(v));
}

__global__ void __launch_bounds__(kT) selectKernel(const double *v, int64_t n, int64_t k,
                                                   double *out) {
    __shared__ unsigned int hist[256];
    __shared__ unsigned long long prefix;
    __shared__ int64_t want;
    if (threadIdx.x == 0) {
        prefix = 0ull;
        want = k;
    }
    for (int pass = 0; pass < 8; ++pass) {
        const int shift = 56 - 8 * pass;
        const unsigned long long highMask = pass == 0 ? 0ull : (~0ull << (shift + 8));
        for (int b = threadIdx.x; b < 256; b += kT)
            hist[b] = 0u;
        __syncthreads();
        const unsigned long long pre = prefix;
        for (int64_t i = threadIdx.x; i < n; i += kT) {
            const unsigned long long key = keyOf(v[i]);
            if ((key & highMask) == pre)
                atomicAdd(&hist[(key >> shift) & 0xffu], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t acc = 0;
            int b = 0;
            for (; b < 255; ++b) {
                if (acc + hist[b] >= want)
                    break;
                acc += hist[b];
            }
            want -= acc;
            prefix = pre | (static_cast<unsigned long long>(b) << shift);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *out = __longlong_as_double(static_cast<long long>(prefix));
}

__global__ void absDiffKernel(const double *a, const double *b, int64_t n, double *out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        out[i] = fabs(__dsub_rn(a[i], b[i]));
}

__global__ void intervalKernel(const double *test, int64_t m, const double *radius, double *lo,
                               double *hi) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < m) {
        const double r = *radius;
        lo[i] = __dsub_rn(test[i], r);
        hi[i] = __dadd_rn(test[i], r);
    }
}

} // namespace

cudaError_t launchResample(const double *w, int64_t n, const double *u, int64_t m, int64_t *idx,
                           double *cdf, cudaStream_t stream) {
    cdfKernel<<<1, kT, 0, stream>>>(w, n, cdf);
    if (m > 0)
        searchKernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, stream>>>(cdf, n, u, m, idx);
    return cudaGetLastError();
}

cudaError_t launchMoments(const double *x, int64_t n, int d, double *mean, double *var,
                          cudaStream_t stream) {
    momentsKernel<<<(d + 127) / 128, 128, 0, stream>>>(x, n, d, mean, var);
    return cudaGetLastError();
}

cudaError_t launchSelect(const double *v, int64_t n, int64_t k, double *out, cudaStream_t stream) {
    selectKernel<<<1, kT, 0, stream>>>(v, n, k, out);
    return cudaGetLastError();
}

cudaError_t launchAbsDiff(const double *a, const double *b, int64_t n, double *out,
                          cudaStream_t stream) {
    absDiffKernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(a, b, n, out);
    return cudaGetLastError();
}

cudaError_t launchInterval(const double *test, int64_t m, const double *radius, double *lo,
                           double *hi, cudaStream_t stream) {
    intervalKernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, stream>>>(test, m, radius, lo,
                                                                            hi);
    return cudaGetLastError();
}

cudaError_t launchWeights(const double *ll, const double *lq, int64_t n, double *w, double *out,
                          cudaStream_t stream) {
    weightsKernel<<<1, kT, 0, stream>>>(ll, lq, n, w, out);
    return cudaGetLastError();
}

} // namespace rq
