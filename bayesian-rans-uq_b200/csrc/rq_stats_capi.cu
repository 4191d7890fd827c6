// C ABI: the statistics of a finished ensemble on the device (cfdr.statistics,
// rans-uq/python/cfdr/statistics.py:235-378), each reproducing numpy's rounding so
// the results are identical to the reference's: multinomial resampling indices,
// the latent mixture moments of the predictive summary, and split-conformal
// quantiles and intervals. Random draws stay on the host (they come from the
// reference's per-sample PCG64 streams); everything that scales with the ensemble
// runs here.
#include "rq_capi_common.h"

using namespace rqc;

namespace {

void copyIn(double *dst, const double *src, int64_t n, const char *what) {
    check(cudaMemcpy(dst, src, sizeof(double) * static_cast<size_t>(n), cudaMemcpyHostToDevice),
          what);
}

void copyOut(double *dst, const double *src, int64_t n, const char *what) {
    check(cudaMemcpy(dst, src, sizeof(double) * static_cast<size_t>(n), cudaMemcpyDeviceToHost),
          what);
}

// np.random.Generator.choice admits p only when every entry is nonnegative and the
// Kahan sum is within sqrt(machine epsilon) of 1
void checkProbabilities(const double *w, int64_t n) {
    double sum = 0.0, c = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (!(w[i] >= 0.0) || !std::isfinite(w[i]))
            throw std::invalid_argument("probabilities are not non-negative");
        const double y = w[i] - c, t = sum + y;
        c = (t - sum) - y;
        sum = t;
    }
    if (std::abs(sum - 1.0) > std::sqrt(std::numeric_limits<double>::epsilon()))
        throw std::invalid_argument("probabilities do not sum to 1");
}

void checkFinite(const double *v, int64_t n, const char *what) {
    if (n < 1)
        throw std::invalid_argument(std::string(what) + " must be a finite nonempty vector");
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i]))
            throw std::invalid_argument(std::string(what) + " must be a finite nonempty vector");
}

// k = ceil((n + 1)(1 - alpha)) as conformal_quantile computes it (statistics.py:349-355)
int64_t conformalRank(int64_t n, double alpha) {
    if (!std::isfinite(alpha) || !(alpha > 0.0 && alpha < 1.0))
        throw std::invalid_argument("alpha must lie in (0,1) and scores must be nonnegative");
    return static_cast<int64_t>(std::ceil(static_cast<double>(n + 1) * (1.0 - alpha)));
}

} // namespace

extern "C" {

int rq_resample_indices(const double *weights, int64_t n, const double *uniforms, int64_t m,
                        int64_t *indices) {
    return guarded([&] {
        if (!weights || (m > 0 && (!uniforms || !indices)) || n < 1 || m < 0)
            throw std::invalid_argument("null argument or empty weights");
        checkProbabilities(weights, n);
        for (int64_t j = 0; j < m; ++j)
            if (!(uniforms[j] >= 0.0 && uniforms[j] < 1.0))
                throw std::invalid_argument("uniforms must lie in [0, 1)");
        DevBuf d;
        d.ensure(sizeof(double) * static_cast<size_t>(2 * n + 2 * m + 1));
        double *dw = d.as<double>(), *dcdf = dw + n, *du = dcdf + n;
        int64_t *didx = reinterpret_cast<int64_t *>(du + m);
        copyIn(dw, weights, n, "weights");
        if (m > 0)
            copyIn(du, uniforms, m, "uniforms");
        check(rq::launchResample(dw, n, du, m, didx, dcdf, nullptr), "resample launch");
        if (m > 0)
            check(cudaMemcpy(indices, didx, sizeof(int64_t) * static_cast<size_t>(m),
                             cudaMemcpyDeviceToHost), "indices");
        check(cudaDeviceSynchronize(), "resample");
    });
}

int rq_predictive_moments(const double *latent, int64_t n, int32_t d, double *mean,
                          double *variance) {
    return guarded([&] {
        if (!latent || !mean || !variance)
            throw std::invalid_argument("null argument");
        if (n < 1 || d < 1)
            throw std::invalid_argument(
                "successful predictions must be finite equal-length nonempty vectors");
        if (n >= (int64_t(1) << 38))
            throw std::invalid_argument("at most 2^38 evaluations");
        checkFinite(latent, n * d, "successful predictions");
        DevBuf buf;
        buf.ensure(sizeof(double) * static_cast<size_t>(n * d + 2 * d));
        double *dx = buf.as<double>(), *dm = dx + n * d, *dv = dm + d;
        copyIn(dx, latent, n * d, "latent");
        check(rq::launchMoments(dx, n, d, dm, dv, nullptr), "moments launch");
        copyOut(mean, dm, d, "mean");
        copyOut(variance, dv, d, "variance");
    });
}

int rq_conformal_quantile(const double *scores, int64_t n, double alpha, double *quantile) {
    return guarded([&] {
        if (!scores || !quantile)
            throw std::invalid_argument("null argument");
        checkFinite(scores, n, "conformal scores");
        const int64_t k = conformalRank(n, alpha);
        for (int64_t i = 0; i < n; ++i)
            if (scores[i] < 0)
                throw std::invalid_argument(
                    "alpha must lie in (0,1) and scores must be nonnegative");
        if (k > n) {
            *quantile = std::numeric_limits<double>::infinity();
            return;
        }
        DevBuf buf;
        buf.ensure(sizeof(double) * static_cast<size_t>(n + 1));
        double *dv = buf.as<double>(), *dout = dv + n;
        copyIn(dv, scores, n, "scores");
        check(rq::launchSelect(dv, n, k, dout, nullptr), "select launch");
        copyOut(quantile, dout, 1, "quantile");
    });
}

int rq_split_conformal(const double *cal_y, const double *cal_pred, int64_t n,
                       const double *test_pred, int64_t m, double alpha, double *lower,
                       double *upper) {
    return guarded([&] {
        if (!cal_y || !cal_pred || !test_pred || !lower || !upper)
            throw std::invalid_argument("null argument");
        checkFinite(cal_y, n, "calibration targets");
        checkFinite(cal_pred, n, "calibration predictions");
        checkFinite(test_pred, m, "test predictions");
        const int64_t k = conformalRank(n, alpha);
        DevBuf buf;
        buf.ensure(sizeof(double) * static_cast<size_t>(3 * n + 3 * m + 1));
        double *dy = buf.as<double>(), *dp = dy + n, *dr = dp + n, *dt = dr + n, *dlo = dt + m,
               *dhi = dlo + m, *drad = dhi + m;
        copyIn(dy, cal_y, n, "calibration targets");
        copyIn(dp, cal_pred, n, "calibration predictions");
        copyIn(dt, test_pred, m, "test predictions");
        check(rq::launchAbsDiff(dy, dp, n, dr, nullptr), "residual launch");
        if (k > n) {
            const double inf = std::numeric_limits<double>::infinity();
            check(cudaMemcpy(drad, &inf, sizeof(double), cudaMemcpyHostToDevice), "radius");
        } else {
            check(rq::launchSelect(dr, n, k, drad, nullptr), "select launch");
        }
        check(rq::launchInterval(dt, m, drad, dlo, dhi, nullptr), "interval launch");
        copyOut(lower, dlo, m, "lower");
        copyOut(upper, dhi, m, "upper");
    });
}

} // extern "C"
