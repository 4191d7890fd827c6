// C ABI of the standalone linear solves (rq_linear_solve*, rq_linsys_*): host
// set-up of the LDU systems (rq_linsys.cpp), their packing into device buffers
// and the persistent linKernel launch (rq_linsolve.cu).
#include "rq_capi_common.h"

using namespace rqc;

// Standalone LDU systems resident on the device (rq_linsys_*).
struct rq_linsys {
    int nsys = 0, kind = 0, precision = 0, maxLevels = 0, grid = 1;
    long wsStride = 0;
    int64_t totalRows = 0, totalNnz = 0;
    std::vector<int> rows;
    std::vector<int64_t> xOff;
    std::vector<rq::DevLinSys> sys; // queue order (largest first), device pointers
    DevBuf dI, dD, dF, dB, dX, dSys, dOut, dWs, dNext;
    std::mutex mu;
};

namespace {

void checkSolveArgs(int maxIter, double tol) {
    if (maxIter < 0 || !std::isfinite(tol) || tol <= 0.)
        throw std::invalid_argument("linear solve requires matching x, nonnegative iteration "
                                    "cap and positive finite tolerance");
}

void buildLinsys(rq_linsys &L, const rq_ldu *systems, int n, int kind, int precision) {
    L.nsys = n;
    L.kind = kind;
    L.precision = precision;
    for (int s = 0; s < n; ++s) {
        const rq_ldu &A = systems[s];
        rq::validateLdu(A.n_cells, A.n_faces, A.diag, A.upper, A.lower, A.source, A.owner,
                        A.neighbour);
        if (A.n_cells < 1)
            throw std::invalid_argument("linear system needs at least one cell");
    }
    // host set-up of every system, on all host threads
    std::vector<rq::LinSysHost> H(n);
    std::vector<std::string> err(n);
    std::vector<int> unsupported(n, 0);
    {
        const int nt = std::max(1, std::min<int>(n, static_cast<int>(std::thread::hardware_concurrency())));
        std::atomic<int> next{0};
        auto work = [&] {
            for (int s = next++; s < n; s = next++) {
                const rq_ldu &A = systems[s];
                try {
                    H[s] = rq::buildLinSys(A.n_cells, A.n_faces, A.diag, A.upper, A.lower, A.owner,
                                           A.neighbour, kind == rq::kLinAmg);
                } catch (const rq::LinUnsupported &e) {
                    err[s] = e.what();
                    unsupported[s] = 1;
                } catch (const std::exception &e) {
                    err[s] = e.what();
                }
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t)
            pool.emplace_back(work);
        work();
        for (auto &t : pool)
            t.join();
    }
    for (int s = 0; s < n; ++s)
        if (!err[s].empty())
            throw RqError(unsupported[s] ? RQ_E_UNSUPPORTED : RQ_E_INVALID,
                          "system " + std::to_string(s) + ": " + err[s]);
    // Layout pass: every array of every system gets an offset in one of three
    // device buffers (int32, FP64, FP32); the copies then run on all host threads.
    enum { P_PTR, P_COL, P_VAL, P_RDG, P_VAL32, P_RDG32, P_AGG, P_CPTR, P_CIDX, P_INV, P_INV32 };
    struct Piece {
        int s, l, what;
        size_t off;
        const void *src; // std::vector<int> or std::vector<double> of the host set-up
    };
    std::vector<Piece> pieces;
    size_t nI = 0, nD = 0, nF = 0;
    auto addI = [&](int s, int l, int what, const std::vector<int> &v) {
        pieces.push_back({s, l, what, nI, &v});
        nI += (v.size() + 7) / 8 * 8;
    };
    auto addD = [&](int s, int l, int what, const std::vector<double> &v) {
        pieces.push_back({s, l, what, nD, &v});
        nD += (v.size() + 3) / 4 * 4;
    };
    auto addF = [&](int s, int l, int what, const std::vector<double> &v) {
        pieces.push_back({s, l, what, nF, &v});
        nF += (v.size() + 7) / 8 * 8;
    };
    const bool mixed = precision == RQ_PREC_MIXED;
    L.rows.resize(n);
    L.xOff.resize(n);
    std::vector<rq::DevLinSys> byIndex(n);
    long wsMax = 0;
    for (int s = 0; s < n; ++s) {
        const rq::LinSysHost &h = H[s];
        rq::DevLinSys &d = byIndex[s];
        std::memset(&d, 0, sizeof(d));
        const int nl = static_cast<int>(h.lev.size());
        if (nl > rq::kLinMaxLevels)
            throw RqError(RQ_E_UNSUPPORTED, "AMG hierarchy deeper than 16 levels");
        d.n = h.n;
        d.nlev = nl;
        d.kind = kind;
        d.precision = mixed && kind != rq::kLinBicgstab ? 1 : 0;
        d.m = h.m;
        long lvecs = 0;
        for (int l = 0; l < nl; ++l) {
            const rq::LinLevelHost &lv = h.lev[l];
            rq::DevLinLevel &dl = d.lev[l];
            dl.n = lv.n;
            dl.nc = lv.nc;
            dl.vecOff = l > 0 ? lvecs : 0;
            if (l > 0)
                lvecs += 3L * lv.n;
            addI(s, l, P_PTR, lv.ptr);
            addI(s, l, P_COL, lv.col);
            addD(s, l, P_VAL, lv.val);
            addD(s, l, P_RDG, lv.rdg);
            if (d.precision) {
                addF(s, l, P_VAL32, lv.val);
                addF(s, l, P_RDG32, lv.rdg);
            }
            if (l + 1 < nl) {
                addI(s, l, P_AGG, lv.agg);
                addI(s, l, P_CPTR, lv.childPtr);
                addI(s, l, P_CIDX, lv.childIdx);
            }
            L.totalNnz += static_cast<int64_t>(lv.col.size());
        }
        if (kind == rq::kLinAmg) {
            addD(s, 0, P_INV, h.inv);
            if (d.precision)
                addF(s, 0, P_INV32, h.inv);
        }
        const long nn = h.n;
        d.lvOff = pad32(8 * nn);
        d.f32Off = d.lvOff + pad32(lvecs);
        d.lvOff32 = 2 * pad32((6 * nn + 1) / 2);
        const long ws = d.f32Off + (d.precision ? (d.lvOff32 / 2 + pad32((lvecs + 1) / 2)) : 0);
        wsMax = std::max(wsMax, ws);
        L.rows[s] = h.n;
        L.xOff[s] = L.totalRows;
        L.totalRows += h.n;
        L.maxLevels = std::max(L.maxLevels, nl);
    }
    std::unique_ptr<int32_t[]> I(new int32_t[std::max<size_t>(nI, 1)]);
    std::unique_ptr<double[]> D(new double[std::max<size_t>(nD, 1)]);
    std::unique_ptr<float[]> F(new float[std::max<size_t>(nF, 1)]);
    std::unique_ptr<double[]> hb(new double[std::max<int64_t>(L.totalRows, 1)]);
    {
        const int nt = std::max(1, std::min<int>(static_cast<int>(pieces.size()),
                                                 static_cast<int>(std::thread::hardware_concurrency())));
        std::atomic<size_t> next{0};
        std::atomic<int> nextRhs{0};
        auto work = [&] {
            for (size_t k = next++; k < pieces.size(); k = next++) {
                const Piece &p = pieces[k];
                switch (p.what) {
                case P_PTR: case P_COL: case P_AGG: case P_CPTR: case P_CIDX: {
                    const auto &v = *static_cast<const std::vector<int> *>(p.src);
                    std::copy(v.begin(), v.end(), I.get() + p.off);
                    std::fill(I.get() + p.off + v.size(), I.get() + p.off + (v.size() + 7) / 8 * 8, 0);
                    break;
                }
                case P_VAL: case P_RDG: case P_INV: {
                    const auto &v = *static_cast<const std::vector<double> *>(p.src);
                    std::copy(v.begin(), v.end(), D.get() + p.off);
                    std::fill(D.get() + p.off + v.size(), D.get() + p.off + (v.size() + 3) / 4 * 4, 0.0);
                    break;
                }
                default: {
                    const auto &v = *static_cast<const std::vector<double> *>(p.src);
                    for (size_t e = 0; e < v.size(); ++e)
                        F[p.off + e] = static_cast<float>(v[e]);
                    std::fill(F.get() + p.off + v.size(), F.get() + p.off + (v.size() + 7) / 8 * 8, 0.0f);
                }
                }
            }
            for (int s = nextRhs++; s < n; s = nextRhs++)
                std::memcpy(hb.get() + L.xOff[s], systems[s].source, sizeof(double) * L.rows[s]);
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t)
            pool.emplace_back(work);
        work();
        for (auto &t : pool)
            t.join();
    }
    L.dI.ensure(std::max<size_t>(nI, 1) * sizeof(int32_t));
    L.dD.ensure(std::max<size_t>(nD, 1) * sizeof(double));
    L.dF.ensure(std::max<size_t>(nF, 1) * sizeof(float));
    check(cudaMemcpy(L.dI.p, I.get(), nI * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
    check(cudaMemcpy(L.dD.p, D.get(), nD * sizeof(double), cudaMemcpyHostToDevice), "upload");
    if (nF)
        check(cudaMemcpy(L.dF.p, F.get(), nF * sizeof(float), cudaMemcpyHostToDevice), "upload");
    for (const Piece &p : pieces) {
        rq::DevLinSys &d = byIndex[p.s];
        rq::DevLinLevel &dl = d.lev[p.l];
        const int32_t *ip = L.dI.as<int32_t>() + p.off;
        const double *dp = L.dD.as<double>() + p.off;
        const float *fp = L.dF.as<float>() + p.off;
        switch (p.what) {
        case P_PTR: dl.ptr = ip; break;
        case P_COL: dl.col = ip; break;
        case P_VAL: dl.val = dp; break;
        case P_RDG: dl.rdg = dp; break;
        case P_VAL32: dl.val32 = fp; break;
        case P_RDG32: dl.rdg32 = fp; break;
        case P_AGG: dl.agg = ip; break;
        case P_CPTR: dl.childPtr = ip; break;
        case P_CIDX: dl.childIdx = ip; break;
        case P_INV: d.inv = dp; break;
        case P_INV32: d.inv32 = fp; break;
        }
    }
    // right-hand sides (gathered above), solutions and results
    L.dB.ensure(sizeof(double) * L.totalRows);
    L.dX.ensure(sizeof(double) * L.totalRows);
    L.dOut.ensure(sizeof(rq::LinOut) * n);
    check(cudaMemcpy(L.dB.p, hb.get(), sizeof(double) * L.totalRows, cudaMemcpyHostToDevice), "rhs");
    for (int s = 0; s < n; ++s) {
        byIndex[s].b = L.dB.as<double>() + L.xOff[s];
        byIndex[s].x = L.dX.as<double>() + L.xOff[s];
        byIndex[s].out = L.dOut.as<rq::LinOut>() + s;
    }
    // queue order: largest systems first (longest-processing-time)
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return L.rows[a] > L.rows[b]; });
    L.sys.clear();
    for (int s : order)
        L.sys.push_back(byIndex[s]);
    int dev = 0, sms = 1;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
    const int perSM = std::max(1, rq::linBlocksPerSM());
    L.grid = std::max(1, std::min(n, sms * perSM));
    L.wsStride = wsMax;
    L.dWs.ensure(sizeof(double) * wsMax * L.grid);
    L.dSys.ensure(sizeof(rq::DevLinSys) * n);
    L.dNext.ensure(sizeof(int));
}

void launchLinsys(rq_linsys &L, int maxIter, double tol, cudaStream_t stream) {
    for (auto &d : L.sys) {
        d.maxIter = maxIter;
        d.tol = tol;
    }
    check(cudaMemcpyAsync(L.dSys.p, L.sys.data(), sizeof(rq::DevLinSys) * L.nsys,
                          cudaMemcpyHostToDevice, stream), "systems");
    check(cudaMemsetAsync(L.dNext.p, 0, sizeof(int), stream), "counter");
    check(rq::launchLinear(L.dSys.as<rq::DevLinSys>(), L.nsys, L.dNext.as<int>(),
                           L.dWs.as<double>(), L.wsStride, L.grid, stream), "linear solve launch");
}

void fetchLinsys(rq_linsys &L, double *const *x, rq_solver_result *results) {
    static_assert(sizeof(rq::LinOut) == sizeof(rq_solver_result), "result layout");
    if (results)
        check(cudaMemcpy(results, L.dOut.p, sizeof(rq::LinOut) * L.nsys, cudaMemcpyDeviceToHost),
              "results");
    if (x) {
        std::vector<double> hx(L.totalRows);
        check(cudaMemcpy(hx.data(), L.dX.p, sizeof(double) * hx.size(), cudaMemcpyDeviceToHost), "x");
        for (int s = 0; s < L.nsys; ++s)
            std::memcpy(x[s], hx.data() + L.xOff[s], sizeof(double) * L.rows[s]);
    }
}

} // namespace

extern "C" {
int rq_linsys_create(const rq_ldu *systems, int32_t n_systems, int32_t kind, int32_t precision,
                     rq_linsys **out) {
    return guarded([&] {
        if (!systems || n_systems < 1 || !out)
            throw std::invalid_argument("null argument");
        *out = nullptr;
        if (kind == 3)
            throw RqError(RQ_E_UNSUPPORTED, "the Gauss-Seidel solver is not on the GPU path");
        if (kind < 0 || kind > 2)
            throw std::invalid_argument("unknown linear solver kind");
        if (precision != RQ_PREC_FP64 && precision != RQ_PREC_MIXED)
            throw std::invalid_argument("unknown precision");
        auto L = std::make_unique<rq_linsys>();
        buildLinsys(*L, systems, n_systems, kind, precision);
        *out = L.release();
    });
}

int rq_linsys_solve(rq_linsys *L, int32_t max_iter, double tol, double *const *x,
                    rq_solver_result *results) {
    return guarded([&] {
        if (!L)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(L->mu);
        checkSolveArgs(max_iter, tol);
        if (x)
            for (int s = 0; s < L->nsys; ++s) {
                if (!x[s])
                    throw std::invalid_argument("null initial guess");
                for (int i = 0; i < L->rows[s]; ++i)
                    if (!std::isfinite(x[s][i]))
                        throw std::invalid_argument("linear solve initial values must be finite");
            }
        if (x) {
            std::vector<double> hx(L->totalRows);
            for (int s = 0; s < L->nsys; ++s)
                std::memcpy(hx.data() + L->xOff[s], x[s], sizeof(double) * L->rows[s]);
            check(cudaMemcpy(L->dX.p, hx.data(), sizeof(double) * hx.size(), cudaMemcpyHostToDevice), "x");
        } else {
            check(cudaMemset(L->dX.p, 0, sizeof(double) * L->totalRows), "x");
        }
        launchLinsys(*L, max_iter, tol, nullptr);
        check(cudaStreamSynchronize(nullptr), "linear solve");
        fetchLinsys(*L, x, results);
    });
}

int rq_linsys_solve_device(rq_linsys *L, int32_t max_iter, double tol, void *stream) {
    return guarded([&] {
        if (!L)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(L->mu);
        checkSolveArgs(max_iter, tol);
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        check(cudaMemsetAsync(L->dX.p, 0, sizeof(double) * L->totalRows, st), "x");
        launchLinsys(*L, max_iter, tol, st);
    });
}

int rq_linsys_results(rq_linsys *L, rq_solver_result *results, double *const *x) {
    return guarded([&] {
        if (!L)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(L->mu);
        check(cudaDeviceSynchronize(), "linear solve");
        fetchLinsys(*L, x, results);
    });
}

int rq_linsys_info(const rq_linsys *L, int32_t *n_systems, int64_t *total_rows, int64_t *total_nnz,
                   int32_t *max_levels) {
    return guarded([&] {
        if (!L)
            throw std::invalid_argument("null argument");
        if (n_systems)
            *n_systems = L->nsys;
        if (total_rows)
            *total_rows = L->totalRows;
        if (total_nnz)
            *total_nnz = L->totalNnz;
        if (max_levels)
            *max_levels = L->maxLevels;
    });
}

int rq_linsys_destroy(rq_linsys *L) {
    return guarded([&] { delete L; });
}

int rq_linear_solve_batch(const rq_ldu *systems, int32_t n_systems, double *const *x,
                          int32_t max_iter, double tol, int32_t kind, int32_t precision,
                          rq_solver_result *results) {
    rq_linsys *L = nullptr;
    int rc = rq_linsys_create(systems, n_systems, kind, precision, &L);
    if (rc != RQ_OK)
        return rc;
    rc = rq_linsys_solve(L, max_iter, tol, x, results);
    rq_linsys_destroy(L);
    return rc;
}

int rq_linear_solve(const rq_ldu *A, double *x, int32_t max_iter, double tol, int32_t kind,
                    rq_solver_result *result) {
    if (!x) {
        g_error = "null argument";
        return RQ_E_INVALID;
    }
    double *xs[1] = {x};
    return rq_linear_solve_batch(A, 1, xs, max_iter, tol, kind, RQ_PREC_FP64, result);
}

} // extern "C"
