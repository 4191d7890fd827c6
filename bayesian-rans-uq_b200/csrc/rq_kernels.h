// Launch entry points of the device code (rq_solver.cu), used by rq_capi.cu.
#pragma once
#include <cuda_runtime.h>

#include "rq_device.cuh"

namespace rq {

size_t solveSharedBytes();
// Persistent CTAs: each pulls job indices from *nextJob (zeroed by the caller)
// until njobs are taken; ws is grid x wsStride doubles of per-CTA workspace.
// arenaDoubles: shared-memory arena per CTA for the hot arrays (0 = all global).
// block: a compiled CTA size (64, 128, 256, 512 or 1024).
cudaError_t launchSolve(const DevJob *jobs, int njobs, int *nextJob, double *ws, long wsStride,
                        int grid, int block, int arenaDoubles, cudaStream_t stream);
// CTAs of the variant with the given arena that fit on one SM at once (0: does not fit).
int solveBlocksPerSM(int block, int arenaDoubles);
bool launchVariantExists(int block);
// The serving loop (serveKernel): grid persistent CTAs of `block` threads (256, 512
// or 1024) serving q until it is closed and drained, or until q.idleNs passes
// without a request.
cudaError_t launchServe(const ServeQueue &q, double *ws, long wsStride, int grid, int block,
                        int arenaDoubles, cudaStream_t stream);
int serveBlocksPerSM(int block, int arenaDoubles);
int normalizeBlock(int block);
// One solve of one job in the module's fixed scratch array (no device allocation):
// capacity in doubles, the array's device address on the current device (looked up
// by cudaGetSymbolAddress at every call of noAllocScratch, which allocates nothing),
// and the launch (grid of one CTA of `block` threads) on that address.
long noAllocScratchDoubles();
cudaError_t noAllocScratch(double **out);
cudaError_t launchSolveNoAlloc(const DevJob &job, double *scratch, int block, int arenaDoubles,
                               cudaStream_t stream);
// Posterior weights (rq_stats.cu): one CTA; out = {max, sum of exp, non-finite count}.
cudaError_t launchWeights(const double *ll, const double *lq, int64_t n, double *w, double *out,
                          cudaStream_t stream);
// Statistics of an ensemble (rq_stats.cu), each with numpy's rounding: multinomial
// indices for given uniforms (cdf: n doubles of scratch), column mean / variance,
// the k-th smallest nonnegative value, |a - b|, and test -/+ radius.
cudaError_t launchResample(const double *w, int64_t n, const double *u, int64_t m, int64_t *idx,
                           double *cdf, cudaStream_t stream);
cudaError_t launchMoments(const double *x, int64_t n, int d, double *mean, double *var,
                          cudaStream_t stream);
cudaError_t launchSelect(const double *v, int64_t n, int64_t k, double *out, cudaStream_t stream);
cudaError_t launchAbsDiff(const double *a, const double *b, int64_t n, double *out,
                          cudaStream_t stream);
cudaError_t launchInterval(const double *test, int64_t m, const double *radius, double *lo,
                           double *hi, cudaStream_t stream);

} // namespace rq
