// C ABI of the B200 forward model (include/rq_b200.h). Host work here is the
// per-mesh-class set-up (rq_setup.cpp), admission of inputs with the
// reference's rules, and the launch of persistent solve CTAs; all per-draw
// numerics run in rq_solver.cu.
#include "../../include/rq_b200.h"
#include "rq_device.cuh"
#include "rq_kernels.h"
#include "rq_lin.cuh"
#include "rq_linsys.h"
#include "rq_setup.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_error;

struct RqError : std::runtime_error {
    int code;
    RqError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void check(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        throw RqError(RQ_E_OOM, std::string(what) + ": " + cudaGetErrorString(e));
    if (e != cudaSuccess)
        throw RqError(RQ_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F> int guarded(F &&f) {
    try {
        f();
        return RQ_OK;
    } catch (const RqError &e) {
        g_error = e.what();
        return e.code;
    } catch (const std::invalid_argument &e) {
        g_error = e.what();
        return RQ_E_INVALID;
    } catch (const std::bad_alloc &e) {
        g_error = "host allocation failed";
        return RQ_E_OOM;
    } catch (const std::exception &e) {
        g_error = e.what();
        return RQ_E_CUDA;
    }
}

// device allocation that frees itself
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void ensure(size_t b) {
        if (b <= bytes)
            return;
        release();
        check(cudaMalloc(&p, b), "cudaMalloc");
        bytes = b;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// The reference's parameter bounds (core/include/InferenceParameters.hpp:147-165).
const double kLower[11] = {0.1, 0.1, 0.01, 0.1, 0.1, 0.1, 0.01, 0.1, 0.01, 0.1, 0.35};
const double kUpper[11] = {2.0, 2.0, 0.2, 1.5, 2.0, 2.0, 0.2, 1.5, 0.2, 0.8, 0.50};

long pad32(long n) { return (n + 31) / 32 * 32; }

} // namespace

struct rq_problem {
    rq::StructMesh mesh;
    rq::AmgHost amg;
    rq::DevClass cls{};      // host copy with device pointers
    DevBuf dCls, dDoubles, dInts;
    std::vector<int32_t> active;
    double base[11];
    int32_t nObs = 0;
    int block = 512; // CTA size of this class's launches
    int arenaKb = 0; // shared-memory arena per CTA, 0 = automatic
    cudaStream_t stream = nullptr; // for concurrent per-class launches of a multi-class batch
    cudaEvent_t done = nullptr;
    ~rq_problem() {
        if (done)
            cudaEventDestroy(done);
        if (stream)
            cudaStreamDestroy(stream);
    }
    // launch scratch, reused across calls
    DevBuf dWs, dJobs, dRows, dPred, dFields, dHist, dTheta, dCounter, dClock;
    std::mutex mu;
};

namespace {

void validateSettings(const rq_settings &s) {
    if (s.max_iterations < 0 || s.inner_iterations <= 0 || s.convergence_window < 2 ||
        s.monitor_interval <= 0 || s.turb_update_interval <= 0 || s.turb_start_iter < 0 ||
        s.nut_floor_iters < 0)
        throw std::invalid_argument("invalid SIMPLE iteration count or cadence");
    if (2 * s.convergence_window > rq::kWindowCap)
        throw RqError(RQ_E_UNSUPPORTED, "convergence_window above 32 is not supported on the GPU path");
    if (!std::isfinite(s.divergence_limit) || s.divergence_limit < 0)
        throw std::invalid_argument("SIMPLE divergence limit must be finite and nonnegative");
    if (!std::isfinite(s.convergence_tol) || s.convergence_tol < 0)
        throw std::invalid_argument("SIMPLE convergence tolerance must be finite and nonnegative");
    for (double v : {s.inner_tolerance, s.alpha_u, s.alpha_k, s.alpha_omega})
        if (!std::isfinite(v) || v <= 0)
            throw std::invalid_argument("SIMPLE tolerances and relaxation denominators must be finite and positive");
    if (!std::isfinite(s.alpha_p) || s.alpha_p < 0)
        throw std::invalid_argument("SIMPLE pressure/source relaxation must be finite and nonnegative");
    for (double v : s.body_force)
        if (!std::isfinite(v))
            throw std::invalid_argument("SIMPLE body force must be finite");
    if (s.body_force[2] != 0.0)
        throw RqError(RQ_E_UNSUPPORTED, "the 2-D GPU path takes no spanwise body force");
    for (double v : {s.k_min, s.k_max, s.omega_min})
        if (!std::isfinite(v) || v < 0)
            throw std::invalid_argument("SIMPLE turbulence limits must be finite and nonnegative");
    if (s.k_max < s.k_min)
        throw std::invalid_argument("SIMPLE kMax must be at least kMin");
    if (s.pressure_solver < 0 || s.pressure_solver > 2)
        throw std::invalid_argument("unknown pressure solver");
    if (s.precision != RQ_PREC_FP64 && s.precision != RQ_PREC_MIXED)
        throw std::invalid_argument("unknown precision");
    if (s.block_threads != 0 &&
        (s.block_threads < 64 || s.block_threads > 1024 || s.block_threads % 32 != 0))
        throw std::invalid_argument("block_threads must be 0 or a multiple of 32 in [64, 1024]");
}

rq::StructMesh buildMesh(const rq_mesh_desc &d) {
    if (d.kind == RQ_MESH_PERIODIC_CHANNEL) {
        if (d.nx < 3 || d.ny < 1)
            throw std::invalid_argument("periodic channel needs nx >= 3 and ny >= 1");
        return rq::makePeriodicChannel(d.nx, d.ny, d.lx, d.h, d.re_tau, d.yplus);
    }
    if (d.kind == RQ_MESH_CURVED_PERIODIC) {
        if (!d.x_nodes || !d.y_bottom || d.nx < 3)
            throw std::invalid_argument("curved mesh needs nx >= 3 and nx+1 node samples");
        std::vector<double> xn(d.x_nodes, d.x_nodes + d.nx + 1), yb(d.y_bottom, d.y_bottom + d.nx + 1);
        return rq::makeCurvedPeriodic(xn, yb, d.y_top, d.ny, d.re, d.yplus);
    }
    throw std::invalid_argument("unknown mesh kind");
}

// Upload the class arrays and fill the device descriptor.
void upload(rq_problem &P, const rq_obs_desc *obs, double nu, const rq_settings &s,
            const double init[6]) {
    const rq::StructMesh &m = P.mesh;
    const rq::AmgHost &h = P.amg;
    std::vector<double> D;
    std::vector<int32_t> I;
    std::vector<std::pair<const double **, size_t>> dptr;
    std::vector<std::pair<const int32_t **, size_t>> iptr;
    rq::DevClass &C = P.cls;
    auto addD = [&](const double **slot, const std::vector<double> &v) {
        dptr.push_back({slot, D.size()});
        D.insert(D.end(), v.begin(), v.end());
        while (D.size() % 4)
            D.push_back(0.0);
    };
    auto addI = [&](const int32_t **slot, const std::vector<int32_t> &v) {
        iptr.push_back({slot, I.size()});
        I.insert(I.end(), v.begin(), v.end());
        while (I.size() % 8)
            I.push_back(0);
    };
    C.nx = m.nx;
    C.ny = m.ny;
    C.n = m.n;
    C.nfy = m.nfy();
    C.balance = m.balance ? 1 : 0;
    C.nu = nu;
    C.beta1Init = 0.075; // applyAllBCs -> applyOmegaBC default (BoundaryCondition.hpp:361, 416-422)
    for (int i = 0; i < 6; ++i)
        C.init[i] = init[i];
    rq::DevSettings &st = C.st;
    st.maxIter = s.max_iterations;
    st.innerIter = s.inner_iterations;
    st.window = s.convergence_window;
    st.monitorInterval = s.monitor_interval;
    st.turbStart = s.turb_start_iter;
    st.turbInterval = s.turb_update_interval;
    st.floorIters = s.nut_floor_iters;
    st.pSolver = s.pressure_solver;
    st.precision = s.precision;
    st.tol = s.convergence_tol;
    st.innerTol = s.inner_tolerance;
    st.divLimit = s.divergence_limit;
    st.aU = s.alpha_u;
    st.aP = s.alpha_p;
    st.aK = s.alpha_k;
    st.aW = s.alpha_omega;
    st.fx = s.body_force[0];
    st.fy = s.body_force[1];
    st.kMin = s.k_min;
    st.kMax = s.k_max;
    st.wMin = s.omega_min;
    addD(&C.cx, m.cx);
    addD(&C.cy, m.cy);
    addD(&C.vol, m.vol);
    addD(&C.wd, m.wd);
    addD(&C.xa, m.xa);
    addD(&C.xnx, m.xnx);
    addD(&C.xny, m.xny);
    addD(&C.xw, m.xw);
    addD(&C.xdl, m.xdl);
    addD(&C.xdx, m.xdx);
    addD(&C.xdy, m.xdy);
    addD(&C.xsh, m.xsh);
    addD(&C.ya, m.ya);
    addD(&C.ynx, m.ynx);
    addD(&C.yny, m.yny);
    addD(&C.yw, m.yw);
    addD(&C.ydl, m.ydl);
    addD(&C.ydx, m.ydx);
    addD(&C.ydy, m.ydy);
    if (m.balance) {
        addD(&C.sing, m.sing);
        addD(&C.slap, m.slap);
        addD(&C.sgx, m.sgx);
        addD(&C.sgy, m.sgy);
    }
    // probes
    const int nobs = obs ? obs->n_obs : 0;
    if (nobs < 0 || nobs > rq::kMaxProbes)
        throw RqError(RQ_E_UNSUPPORTED, "at most 64 observations per problem on the GPU path");
    C.nobs = nobs;
    C.obsComp = obs ? obs->component : 0;
    if (nobs > 0) {
        if (C.obsComp < 0 || C.obsComp > 2)
            throw std::invalid_argument("velocity observation component must be in [0,2]");
        if (C.obsComp == 2)
            throw RqError(RQ_E_UNSUPPORTED, "the 2-D GPU path observes x or y velocity only");
        std::vector<int32_t> cell(nobs), nnb(nobs), nb(4 * nobs);
        std::vector<double> ox(nobs), oy(nobs), axx(nobs), axy(nobs), ayy(nobs), det(nobs),
            dx(4 * nobs), dy(4 * nobs), wt(4 * nobs), val(nobs), var(nobs), fl(nobs);
        for (int t = 0; t < nobs; ++t) {
            const double so = obs->sigma_obs[t], sm = obs->sigma_model ? obs->sigma_model[t] : 0.0;
            const double variance = so * so + sm * sm; // Measurement::totalVariance
            if (!std::isfinite(obs->observed[t]) || !std::isfinite(so) || so < 0 ||
                !std::isfinite(sm) || sm < 0 || !std::isfinite(variance) || variance <= 0)
                throw std::invalid_argument(
                    "Gaussian measurements require finite values, nonnegative uncertainties "
                    "and finite positive total variance");
            if (!std::isfinite(obs->x[t]) || !std::isfinite(obs->y[t]))
                throw std::invalid_argument("observation location must be finite");
            const rq::ProbeHost p = rq::prepareProbe(m, obs->x[t], obs->y[t]);
            cell[t] = p.cell;
            nnb[t] = p.nnb;
            ox[t] = p.ox;
            oy[t] = p.oy;
            axx[t] = p.axx;
            axy[t] = p.axy;
            ayy[t] = p.ayy;
            det[t] = p.det;
            for (int k = 0; k < 4; ++k) {
                nb[4 * t + k] = p.nb[k];
                dx[4 * t + k] = p.dx[k];
                dy[4 * t + k] = p.dy[k];
                wt[4 * t + k] = p.wt[k];
            }
            val[t] = obs->observed[t];
            var[t] = variance;
            fl[t] = std::sqrt(variance); // monitor floor sigma_i (ForwardModel.cpp:64-71)
        }
        addI(&C.pcell, cell);
        addI(&C.pnnb, nnb);
        addI(&C.pnb, nb);
        addD(&C.pox, ox);
        addD(&C.poy, oy);
        addD(&C.paxx, axx);
        addD(&C.paxy, axy);
        addD(&C.payy, ayy);
        addD(&C.pdet, det);
        addD(&C.pdx, dx);
        addD(&C.pdy, dy);
        addD(&C.pwt, wt);
        addD(&C.obsVal, val);
        addD(&C.obsVar, var);
        addD(&C.obsFloor, fl);
    }
    // AMG hierarchy
    const int L = static_cast<int>(h.lev.size());
    if (L > rq::kMaxLevels)
        throw RqError(RQ_E_UNSUPPORTED, "AMG hierarchy deeper than 12 levels");
    if (h.coarseN() > rq::kMaxCoarse)
        throw RqError(RQ_E_UNSUPPORTED, "coarsest AMG level above 64 rows");
    C.nlev = L;
    // ELL slots of levels >= 1: CSR entry k of row i -> (k - ptr[i]) * n + i
    std::vector<std::vector<int>> slotOf(L), entryOf(L);
    std::vector<int> width(L, 0);
    for (int l = 1; l < L; ++l) {
        const auto &Lv = h.lev[l];
        for (int i = 0; i < Lv.n; ++i)
            width[l] = std::max(width[l], Lv.ptr[i + 1] - Lv.ptr[i]);
        slotOf[l].resize(Lv.col.size());
        entryOf[l].assign(static_cast<size_t>(width[l]) * Lv.n, -1);
        for (int i = 0; i < Lv.n; ++i)
            for (int k = Lv.ptr[i]; k < Lv.ptr[i + 1]; ++k) {
                const int slot = (k - Lv.ptr[i]) * Lv.n + i;
                slotOf[l][k] = slot;
                entryOf[l][slot] = k;
            }
    }
    int valOff = 0, vecOff = 0;
    for (int l = 0; l < L; ++l) {
        const auto &Lv = h.lev[l];
        rq::DevAmgLevel &dl = C.lev[l];
        dl.n = Lv.n;
        dl.width = l > 0 ? width[l] : 0;
        dl.nnz = l > 0 ? width[l] * Lv.n : 0;
        dl.valOff = valOff;
        dl.vecOff = vecOff;
        if (l > 0) {
            valOff += static_cast<int>(pad32(dl.nnz));
            std::vector<int> ecol(dl.nnz, -1), dpos(Lv.n);
            for (int slot = 0; slot < dl.nnz; ++slot)
                if (entryOf[l][slot] >= 0)
                    ecol[slot] = Lv.col[entryOf[l][slot]];
            for (int i = 0; i < Lv.n; ++i)
                dpos[i] = slotOf[l][Lv.diagPos[i]];
            addI(&dl.ecol, ecol);
            addI(&dl.diagPos, dpos);
        }
        if (l > 0 || L == 1)
            vecOff += static_cast<int>(pad32(5L * Lv.n)); // b, xa, xb, r, 1/diag
        if (l + 1 < L) {
            addI(&dl.agg, Lv.agg);
            addI(&dl.childPtr, Lv.childPtr);
            addI(&dl.childIdx, Lv.childIdx);
            // gather lists in the next level's slot order; sources of level >= 1 as slots
            const int ns = width[l + 1] * h.lev[l + 1].n;
            std::vector<int> gp(ns + 1, 0), gs;
            for (int slot = 0; slot < ns; ++slot) {
                const int e = entryOf[l + 1][slot];
                if (e >= 0)
                    for (int k = Lv.gPtr[e]; k < Lv.gPtr[e + 1]; ++k)
                        gs.push_back(l == 0 ? Lv.gSrc[k] : slotOf[l][Lv.gSrc[k]]);
                gp[slot + 1] = static_cast<int>(gs.size());
            }
            addI(&dl.gPtr, gp);
            addI(&dl.gSrc, gs);
        }
    }
    C.amgW = h.w;
    C.amgAlpha = h.alpha;
    C.amgVals = valOff;
    C.amgVecs = vecOff;
    C.nActive = static_cast<int32_t>(P.active.size());
    for (int a = 0; a < 11; ++a) {
        C.active[a] = a < C.nActive ? P.active[a] : 0;
        C.base[a] = P.base[a];
        C.lo[a] = kLower[a];
        C.hi[a] = kUpper[a];
    }
    const long n = m.n, nf = m.n + m.nfy(), mc = h.coarseN();
    // FP64 arrays, FP32 inner-solver copies (mixed form), faces, AMG, dense coarse
    C.wsDoubles = 43 * pad32(n) + 15 * pad32((n + 1) / 2) + pad32((valOff + 1) / 2) +
                  pad32((vecOff + 1) / 2) +
                  4 * pad32(nf) + pad32(valOff) + pad32(vecOff) + 2 * pad32(2 * mc * mc);
    // upload and patch pointers
    P.dDoubles.ensure(std::max<size_t>(D.size(), 1) * sizeof(double));
    P.dInts.ensure(std::max<size_t>(I.size(), 1) * sizeof(int32_t));
    check(cudaMemcpy(P.dDoubles.p, D.data(), D.size() * sizeof(double), cudaMemcpyHostToDevice), "upload");
    check(cudaMemcpy(P.dInts.p, I.data(), I.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
    for (auto &e : dptr)
        *e.first = P.dDoubles.as<double>() + e.second;
    for (auto &e : iptr)
        *e.first = P.dInts.as<int32_t>() + e.second;
    P.dCls.ensure(sizeof(rq::DevClass));
    check(cudaMemcpy(P.dCls.p, &C, sizeof(rq::DevClass), cudaMemcpyHostToDevice), "upload");
}

// CTA size of a class: 512 threads measured fastest for 384-1536 cells (256 and
// 1024 were slower at every size).
constexpr int kDefaultBlock = 512;

int maxSmemOptin() {
    int dev = 0, v = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "attribute");
    return v;
}

// Shared-memory arena of a launch, in doubles. Classes of up to 768 cells run two
// CTAs per SM and place their whole hot set in half the SM's shared memory each.
// Larger classes run one CTA per SM and take no arena: their hot set does not fit
// (14 level-0 Krylov arrays plus the AMG coarse levels), and leaving the unified
// L1/shared storage to the L1 cache measured faster (1536 cells: 537 us per outer
// iteration without an arena against 656 us with the largest one).
int arenaDoublesFor(long wsDoubles, int knobKb, int nmax) {
    const long shared = static_cast<long>(rq::solveSharedBytes());
    const long optin = maxSmemOptin();
    long bytes;
    if (knobKb > 0)
        bytes = std::min<long>(knobKb * 1024L, optin - shared);
    else if (nmax <= 768)
        bytes = (optin / 2 - 1024) - shared; // two CTAs per SM
    else
        bytes = 0;
    bytes = std::max<long>(0, std::min(bytes, wsDoubles * 8));
    return static_cast<int>(bytes / 8 / 32 * 32);
}

int chooseArena(const std::vector<const rq_problem *> &probs) {
    long ws = 0;
    int knob = 0;
    int nmax = 0;
    for (const auto *p : probs) {
        ws = std::max(ws, static_cast<long>(p->cls.wsDoubles));
        knob = std::max(knob, p->arenaKb);
        nmax = std::max(nmax, p->mesh.n);
    }
    return arenaDoublesFor(ws, knob, nmax);
}

// One persistent launch of a single mesh class over its rows.
void launchClass(rq_problem &P, const std::vector<int> &rows, const double *thetaDev,
                 int thetaStride, rq::RowOut *rowsDev, double *predDev, int predStride,
                 double *fieldsDev, long fieldStride, double *histDev, int histCap,
                 long long *clockDev, cudaStream_t stream) {
    const int n = static_cast<int>(rows.size());
    std::vector<rq::DevJob> jobs(n);
    for (int k = 0; k < n; ++k) {
        const int r = rows[k];
        rq::DevJob &j = jobs[k];
        j.cls = P.dCls.as<rq::DevClass>();
        j.theta = thetaDev + static_cast<long>(r) * thetaStride;
        j.row = rowsDev + r;
        j.pred = predDev + static_cast<long>(r) * predStride;
        j.fields = fieldsDev ? fieldsDev + static_cast<long>(r) * fieldStride : nullptr;
        j.hist = histDev ? histDev + static_cast<long>(r) * histCap * 11 : nullptr;
        j.histCap = histCap;
        j.clock = clockDev ? clockDev + 12L * r : nullptr;
    }
    const long wsStride = P.cls.wsDoubles;
    const int arena = chooseArena({&P});
    int dev = 0, sms = 1;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
    const int perSM = rq::solveBlocksPerSM(P.block, arena);
    if (perSM < 1)
        throw RqError(RQ_E_CUDA, "solve kernel does not fit on an SM with this arena");
    const int grid = std::max(1, std::min(n, sms * perSM));
    P.dJobs.ensure(sizeof(rq::DevJob) * n);
    P.dWs.ensure(sizeof(double) * wsStride * grid);
    P.dCounter.ensure(sizeof(int));
    check(cudaMemcpyAsync(P.dJobs.p, jobs.data(), sizeof(rq::DevJob) * n, cudaMemcpyHostToDevice,
                          stream), "jobs");
    check(cudaMemsetAsync(P.dCounter.p, 0, sizeof(int), stream), "counter");
    check(rq::launchSolve(P.dJobs.as<rq::DevJob>(), n, P.dCounter.as<int>(), P.dWs.as<double>(),
                          wsStride, grid, P.block, arena, stream),
          "solve launch");
}

// Launches the rows (row r belongs to mesh class probOfRow[r]; theta rows live on the
// device at thetaDev + r * thetaStride; outputs are device buffers indexed by row).
// Each class is one persistent launch with its own kernel variant; several classes
// run concurrently on per-class streams (largest class first) joined back into `stream`.
void launchRows(rq_problem &owner, const std::vector<const rq_problem *> &probOfRow,
                const double *thetaDev, int thetaStride, rq::RowOut *rowsDev, double *predDev,
                int predStride, double *fieldsDev, long fieldStride, double *histDev, int histCap,
                long long *clockDev, cudaStream_t stream) {
    (void)owner;
    std::vector<rq_problem *> classes;
    std::vector<std::vector<int>> rowsOf;
    for (int r = 0; r < static_cast<int>(probOfRow.size()); ++r) {
        rq_problem *P = const_cast<rq_problem *>(probOfRow[r]);
        auto it = std::find(classes.begin(), classes.end(), P);
        if (it == classes.end()) {
            classes.push_back(P);
            rowsOf.push_back({r});
        } else {
            rowsOf[it - classes.begin()].push_back(r);
        }
    }
    if (classes.empty())
        return;
    std::vector<int> order(classes.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return classes[a]->mesh.n > classes[b]->mesh.n; });
    if (classes.size() == 1) {
        launchClass(*classes[0], rowsOf[0], thetaDev, thetaStride, rowsDev, predDev, predStride,
                    fieldsDev, fieldStride, histDev, histCap, clockDev, stream);
        return;
    }
    cudaEvent_t fork;
    check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
    check(cudaEventRecord(fork, stream), "event record");
    for (int g : order) {
        rq_problem &P = *classes[g];
        if (!P.stream)
            check(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking), "stream");
        if (!P.done)
            check(cudaEventCreateWithFlags(&P.done, cudaEventDisableTiming), "event");
        check(cudaStreamWaitEvent(P.stream, fork, 0), "stream wait");
        launchClass(P, rowsOf[g], thetaDev, thetaStride, rowsDev, predDev, predStride, fieldsDev,
                    fieldStride, histDev, histCap, clockDev, P.stream);
        check(cudaEventRecord(P.done, P.stream), "event record");
    }
    for (int g : order)
        check(cudaStreamWaitEvent(stream, classes[g]->done, 0), "stream wait");
    cudaEventDestroy(fork);
}

rq_row_out toRow(const rq::RowOut &o) {
    return rq_row_out{o.status, o.iterations, o.stalled, o.converged, o.loglik, o.finalWorst,
                      o.contractionRate};
}

// pinned, device-mapped host allocation that frees itself
struct MappedBuf {
    void *p = nullptr;
    MappedBuf() = default;
    MappedBuf(const MappedBuf &) = delete;
    MappedBuf &operator=(const MappedBuf &) = delete;
    ~MappedBuf() {
        if (p)
            cudaFreeHost(p);
    }
    void alloc(size_t b) {
        check(cudaHostAlloc(&p, b, cudaHostAllocMapped | cudaHostAllocPortable), "cudaHostAlloc");
        std::memset(p, 0, b);
    }
};

} // namespace

// The serving loop's host half: a request queue in host-mapped memory that a
// persistent kernel drains while the host keeps appending to it.
struct rq_server {
    std::vector<rq_problem *> problems;
    int capacity = 0, thetaStride = 1, predStride = 1, block = 512, grid = 1, arena = 0;
    long wsStride = 0;
    long long idleNs = 0;
    MappedBuf host; // jobs | theta | rows | predictions | clocks | done | published | closed
    rq::DevJob *jobs = nullptr;
    double *theta = nullptr, *pred = nullptr;
    rq::RowOut *rows = nullptr;
    long long *clock = nullptr;
    int *done = nullptr, *published = nullptr, *closed = nullptr;
    DevBuf dWs, dCtl; // per-slot workspace; head and idle-exit counters
    cudaStream_t stream = nullptr;
    int submitted = 0, launches = 0;
    std::mutex mu;
    ~rq_server() {
        if (closed)
            __atomic_store_n(closed, 2, __ATOMIC_RELEASE); // cancel what is not yet claimed
        if (stream) {
            cudaStreamSynchronize(stream); // in-flight solves finish first
            cudaStreamDestroy(stream);
        }
    }
    rq::ServeQueue queue() const {
        rq::ServeQueue q{};
        q.jobs = jobs;
        q.published = published;
        q.closed = closed;
        q.done = done;
        q.head = dCtl.as<int>();
        q.idleExits = dCtl.as<int>() + 1;
        q.capacity = capacity;
        q.idleNs = idleNs;
        return q;
    }
    void launch() {
        check(rq::launchServe(queue(), dWs.as<double>(), wsStride, grid, block, arena, stream),
              "serve launch");
        ++launches;
    }
    // The kernel's CTAs leave after idleNs without work; relaunch while requests
    // remain unclaimed (a relaunch never repeats a request: CTAs claim by head).
    void ensureRunning() {
        const cudaError_t e = cudaStreamQuery(stream);
        if (e == cudaErrorNotReady)
            return;
        check(e, "serve loop");
        for (int i = 0; i < submitted; ++i)
            if (!__atomic_load_n(done + i, __ATOMIC_ACQUIRE)) {
                launch();
                return;
            }
    }
};


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

const char *rq_last_error(void) { return g_error.c_str(); }
int rq_version(void) { return 100; }

int rq_default_settings(rq_settings *s) {
    return guarded([&] {
        if (!s)
            throw std::invalid_argument("null settings");
        std::memset(s, 0, sizeof(*s));
        s->max_iterations = 500;
        s->inner_iterations = 200;
        s->convergence_window = 25;
        s->monitor_interval = 10;
        s->turb_start_iter = 5;
        s->turb_update_interval = 1;
        s->nut_floor_iters = 500;
        s->pressure_solver = RQ_SOLVER_AMG;
        s->precision = RQ_PREC_FP64;
        s->block_threads = 0;
        s->convergence_tol = 1e-5;
        s->inner_tolerance = 1e-3;
        s->divergence_limit = 1e6;
        s->alpha_u = 0.7;
        s->alpha_p = 0.3;
        s->alpha_k = 0.5;
        s->alpha_omega = 0.5;
        s->k_min = 1e-10;
        s->k_max = 1e10;
        s->omega_min = 1e-6;
    });
}

int rq_problem_create(const rq_mesh_desc *mesh, const rq_bc_desc *bc, double nu,
                      const rq_settings *settings, const rq_obs_desc *obs, const double init[6],
                      const int32_t *active, int32_t n_active, const double base[11],
                      rq_problem **out) {
    return guarded([&] {
        if (!mesh || !bc || !settings || !init || !active || !base || !out)
            throw std::invalid_argument("null argument");
        *out = nullptr;
        // simple_admission::problem / initial (rans-uq/include/SIMPLEValidation.hpp:10-60)
        if (!std::isfinite(nu) || nu <= 0)
            throw std::invalid_argument("SIMPLE kinematic viscosity must be finite and positive");
        validateSettings(*settings);
        if (!std::isfinite(bc->u_in) || !std::isfinite(bc->k_in) || !std::isfinite(bc->omega_in))
            throw std::invalid_argument("active boundary values must be finite");
        for (int i = 0; i < 4; ++i)
            if (!std::isfinite(init[i]))
                throw std::invalid_argument("SIMPLE initial velocity and pressure must be finite");
        if (!std::isfinite(init[4]) || init[4] < 0)
            throw std::invalid_argument("SIMPLE initial k must be finite and nonnegative");
        if (!std::isfinite(init[5]) || init[5] <= 0)
            throw std::invalid_argument("SIMPLE initial omega must be finite and positive");
        if (init[2] != 0.0)
            throw RqError(RQ_E_UNSUPPORTED, "the 2-D GPU path starts from zero spanwise velocity");
        if (n_active < 1 || n_active > 11)
            throw std::invalid_argument("inference parameters require at least one active index");
        bool seen[11] = {};
        for (int a = 0; a < n_active; ++a) {
            if (active[a] < 0 || active[a] > 10)
                throw std::invalid_argument("inference parameter index must be in [0,10]");
            if (seen[active[a]])
                throw std::invalid_argument("inference parameter indices must be unique");
            seen[active[a]] = true;
        }
        for (int i = 0; i < 11; ++i)
            if (!std::isfinite(base[i]) || base[i] < 0)
                throw std::invalid_argument("SST coefficients must be finite and nonnegative");
        if (base[2] == 0 || base[8] == 0)
            throw std::invalid_argument("SST beta1 and betaStar must be positive");
        auto P = std::make_unique<rq_problem>();
        P->mesh = buildMesh(*mesh);
        P->amg = rq::buildAmg(P->mesh);
        P->active.assign(active, active + n_active);
        std::memcpy(P->base, base, sizeof(P->base));
        P->nObs = obs ? obs->n_obs : 0;
        P->block = settings->block_threads ? rq::normalizeBlock(settings->block_threads)
                                           : kDefaultBlock;
        upload(*P, obs, nu, *settings, init);
        *out = P.release();
    });
}

int rq_problem_destroy(rq_problem *p) {
    return guarded([&] { delete p; });
}

int rq_problem_info(const rq_problem *p, int32_t *n_cells, int32_t *n_obs, int32_t *n_active,
                    int32_t *amg_levels) {
    return guarded([&] {
        if (!p)
            throw std::invalid_argument("null problem");
        if (n_cells)
            *n_cells = p->mesh.n;
        if (n_obs)
            *n_obs = p->nObs;
        if (n_active)
            *n_active = static_cast<int32_t>(p->active.size());
        if (amg_levels)
            *amg_levels = static_cast<int32_t>(p->amg.lev.size());
    });
}

int rq_evaluate_multi(rq_problem *const *problems, int32_t n_problems,
                      const int32_t *problem_of_row, const double *theta, int32_t theta_stride,
                      int64_t n, rq_row_out *rows, double *predictions, int32_t pred_stride) {
    return guarded([&] {
        if (!problems || n_problems < 1 || (n > 0 && (!problem_of_row || !theta || !rows || !predictions)))
            throw std::invalid_argument("null argument");
        if (n < 0)
            throw std::invalid_argument("negative row count");
        if (n == 0)
            return;
        int maxActive = 0, maxObs = 0;
        for (int i = 0; i < n_problems; ++i) {
            if (!problems[i])
                throw std::invalid_argument("null problem");
            maxActive = std::max<int>(maxActive, static_cast<int>(problems[i]->active.size()));
            maxObs = std::max(maxObs, problems[i]->nObs);
        }
        if (theta_stride < maxActive || pred_stride < std::max(maxObs, 1))
            throw std::invalid_argument("theta/prediction stride below the problems' widths");
        std::vector<const rq_problem *> probOfRow(n);
        for (int64_t r = 0; r < n; ++r) {
            if (problem_of_row[r] < 0 || problem_of_row[r] >= n_problems)
                throw std::invalid_argument("problem index out of range");
            probOfRow[r] = problems[problem_of_row[r]];
        }
        rq_problem &owner = *problems[0];
        std::lock_guard<std::mutex> lock(owner.mu);
        owner.dTheta.ensure(sizeof(double) * n * theta_stride);
        owner.dRows.ensure(sizeof(rq::RowOut) * n);
        owner.dPred.ensure(sizeof(double) * n * pred_stride);
        check(cudaMemcpy(owner.dTheta.p, theta, sizeof(double) * n * theta_stride,
                         cudaMemcpyHostToDevice), "theta");
        launchRows(owner, probOfRow, owner.dTheta.as<double>(), theta_stride,
                   owner.dRows.as<rq::RowOut>(), owner.dPred.as<double>(), pred_stride, nullptr, 0,
                   nullptr, 0, nullptr, nullptr);
        std::vector<rq::RowOut> hr(n);
        std::vector<double> hp(static_cast<size_t>(n) * pred_stride);
        check(cudaMemcpy(hr.data(), owner.dRows.p, sizeof(rq::RowOut) * n, cudaMemcpyDeviceToHost), "rows");
        check(cudaMemcpy(hp.data(), owner.dPred.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost), "predictions");
        const double nan = std::nan("");
        for (int64_t r = 0; r < n; ++r) {
            rows[r] = toRow(hr[r]);
            const int no = probOfRow[r]->nObs;
            for (int t = 0; t < pred_stride; ++t)
                predictions[r * pred_stride + t] = t < no ? hp[r * pred_stride + t] : nan;
        }
    });
}

int rq_evaluate_multi_device(rq_problem *const *problems, int32_t n_problems,
                             const int32_t *problem_of_row_host, const double *theta_dev,
                             int32_t theta_stride, int64_t n, rq_row_out *rows_dev,
                             double *predictions_dev, int32_t pred_stride, void *stream,
                             int64_t *clock_ns_dev) {
    return guarded([&] {
        if (!problems || n_problems < 1 || (n > 0 && (!problem_of_row_host || !theta_dev || !rows_dev || !predictions_dev)))
            throw std::invalid_argument("null argument");
        if (n < 0)
            throw std::invalid_argument("negative row count");
        int maxActive = 0, maxObs = 0;
        for (int i = 0; i < n_problems; ++i) {
            if (!problems[i])
                throw std::invalid_argument("null problem");
            maxActive = std::max<int>(maxActive, static_cast<int>(problems[i]->active.size()));
            maxObs = std::max(maxObs, problems[i]->nObs);
        }
        if (theta_stride < maxActive || pred_stride < std::max(maxObs, 1))
            throw std::invalid_argument("theta/prediction stride below the problems' widths");
        static_assert(sizeof(rq::RowOut) == sizeof(rq_row_out), "row layout");
        std::vector<const rq_problem *> probOfRow(n);
        for (int64_t r = 0; r < n; ++r) {
            if (problem_of_row_host[r] < 0 || problem_of_row_host[r] >= n_problems)
                throw std::invalid_argument("problem index out of range");
            probOfRow[r] = problems[problem_of_row_host[r]];
        }
        rq_problem &owner = *problems[0];
        std::lock_guard<std::mutex> lock(owner.mu);
        launchRows(owner, probOfRow, theta_dev, theta_stride,
                   reinterpret_cast<rq::RowOut *>(rows_dev), predictions_dev, pred_stride, nullptr,
                   0, nullptr, 0, reinterpret_cast<long long *>(clock_ns_dev),
                   static_cast<cudaStream_t>(stream));
    });
}

int rq_evaluate_batch(rq_problem *p, const double *theta, int64_t n, rq_row_out *rows,
                      double *predictions, double *fields, double *history, int32_t hist_cap) {
    return guarded([&] {
        if (!p || (n > 0 && (!theta || !rows)))
            throw std::invalid_argument("null argument");
        if (n < 0 || hist_cap < 0)
            throw std::invalid_argument("negative size");
        if (n == 0)
            return;
        std::lock_guard<std::mutex> lock(p->mu);
        const int na = static_cast<int>(p->active.size());
        const int no = std::max(p->nObs, 1), nc = p->mesh.n;
        std::vector<const rq_problem *> probOfRow(n, p);
        p->dTheta.ensure(sizeof(double) * n * na);
        p->dRows.ensure(sizeof(rq::RowOut) * n);
        p->dPred.ensure(sizeof(double) * n * no);
        if (fields)
            p->dFields.ensure(sizeof(double) * n * 11L * nc);
        const bool wantHist = history && hist_cap > 0;
        if (wantHist)
            p->dHist.ensure(sizeof(double) * n * 11L * hist_cap);
        check(cudaMemcpy(p->dTheta.p, theta, sizeof(double) * n * na, cudaMemcpyHostToDevice), "theta");
        launchRows(*p, probOfRow, p->dTheta.as<double>(), na, p->dRows.as<rq::RowOut>(),
                   p->dPred.as<double>(), no, fields ? p->dFields.as<double>() : nullptr, 11L * nc,
                   wantHist ? p->dHist.as<double>() : nullptr, hist_cap, nullptr, nullptr);
        std::vector<rq::RowOut> hr(n);
        std::vector<double> hp(static_cast<size_t>(n) * no);
        check(cudaMemcpy(hr.data(), p->dRows.p, sizeof(rq::RowOut) * n, cudaMemcpyDeviceToHost), "rows");
        check(cudaMemcpy(hp.data(), p->dPred.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost), "predictions");
        if (fields)
            check(cudaMemcpy(fields, p->dFields.p, sizeof(double) * n * 11L * nc, cudaMemcpyDeviceToHost), "fields");
        if (wantHist)
            check(cudaMemcpy(history, p->dHist.p, sizeof(double) * n * 11L * hist_cap, cudaMemcpyDeviceToHost), "history");
        for (int64_t r = 0; r < n; ++r) {
            rows[r] = toRow(hr[r]);
            if (predictions)
                for (int t = 0; t < p->nObs; ++t)
                    predictions[r * p->nObs + t] = hp[r * no + t];
        }
    });
}

int rq_solve(rq_problem *p, const double coeffs[11], rq_row_out *row, double *predictions,
             double *fields, double *history, int32_t hist_cap) {
    return guarded([&] {
        if (!p || !coeffs || !row)
            throw std::invalid_argument("null argument");
        for (int i = 0; i < 11; ++i)
            if (!std::isfinite(coeffs[i]) || coeffs[i] < 0)
                throw std::invalid_argument("SST coefficients must be finite and nonnegative");
        if (coeffs[2] == 0 || coeffs[8] == 0)
            throw std::invalid_argument("SST beta1 and betaStar must be positive");
        // a one-off problem view whose parameter set activates all eleven coefficients
        std::lock_guard<std::mutex> lock(p->mu);
        rq::DevClass all = p->cls;
        all.nActive = 11;
        for (int a = 0; a < 11; ++a) {
            all.active[a] = a;
            all.lo[a] = -std::numeric_limits<double>::infinity();
            all.hi[a] = std::numeric_limits<double>::infinity();
        }
        DevBuf dAll;
        dAll.ensure(sizeof(rq::DevClass));
        check(cudaMemcpy(dAll.p, &all, sizeof(all), cudaMemcpyHostToDevice), "class");
        const int no = std::max(p->nObs, 1), nc = p->mesh.n;
        p->dTheta.ensure(sizeof(double) * 11);
        p->dRows.ensure(sizeof(rq::RowOut));
        p->dPred.ensure(sizeof(double) * no);
        if (fields)
            p->dFields.ensure(sizeof(double) * 11L * nc);
        const bool wantHist = history && hist_cap > 0;
        if (wantHist)
            p->dHist.ensure(sizeof(double) * 11L * hist_cap);
        check(cudaMemcpy(p->dTheta.p, coeffs, sizeof(double) * 11, cudaMemcpyHostToDevice), "coeffs");
        std::vector<const rq_problem *> probOfRow{p};
        // one job whose class descriptor is the all-eleven view
        std::vector<rq::DevJob> jobs(1);
        rq::DevJob &j = jobs[0];
        j.cls = dAll.as<rq::DevClass>();
        j.theta = p->dTheta.as<double>();
        j.row = p->dRows.as<rq::RowOut>();
        j.pred = p->dPred.as<double>();
        j.fields = fields ? p->dFields.as<double>() : nullptr;
        j.hist = wantHist ? p->dHist.as<double>() : nullptr;
        j.histCap = hist_cap;
        j.clock = nullptr;
        const int arena = chooseArena(probOfRow);
        p->dJobs.ensure(sizeof(rq::DevJob));
        p->dWs.ensure(sizeof(double) * p->cls.wsDoubles);
        p->dCounter.ensure(sizeof(int));
        check(cudaMemcpy(p->dJobs.p, jobs.data(), sizeof(rq::DevJob), cudaMemcpyHostToDevice), "jobs");
        check(cudaMemset(p->dCounter.p, 0, sizeof(int)), "counter");
        check(rq::launchSolve(p->dJobs.as<rq::DevJob>(), 1, p->dCounter.as<int>(),
                              p->dWs.as<double>(), p->cls.wsDoubles, 1, p->block, arena,
                              nullptr),
              "solve launch");
        rq::RowOut o;
        check(cudaMemcpy(&o, p->dRows.p, sizeof(o), cudaMemcpyDeviceToHost), "row");
        *row = toRow(o);
        if (predictions && p->nObs > 0)
            check(cudaMemcpy(predictions, p->dPred.p, sizeof(double) * p->nObs, cudaMemcpyDeviceToHost), "predictions");
        if (fields)
            check(cudaMemcpy(fields, p->dFields.p, sizeof(double) * 11 * nc, cudaMemcpyDeviceToHost), "fields");
        if (wantHist)
            check(cudaMemcpy(history, p->dHist.p, sizeof(double) * 11 * hist_cap, cudaMemcpyDeviceToHost), "history");
    });
}

int rq_mesh_geometry(const rq_mesh_desc *mesh, int32_t *n_cells, double *cells) {
    return guarded([&] {
        if (!mesh || !n_cells)
            throw std::invalid_argument("null argument");
        const rq::StructMesh m = buildMesh(*mesh);
        *n_cells = m.n;
        if (cells)
            for (int c = 0; c < m.n; ++c) {
                cells[4 * c] = m.cx[c];
                cells[4 * c + 1] = m.cy[c];
                cells[4 * c + 2] = m.vol[c];
                cells[4 * c + 3] = m.wd[c];
            }
    });
}

int rq_server_create(rq_problem *const *problems, int32_t n_problems, int32_t capacity,
                     double idle_timeout_s, int32_t max_slots, rq_server **out) {
    return guarded([&] {
        if (!problems || n_problems < 1 || !out)
            throw std::invalid_argument("null argument");
        *out = nullptr;
        if (capacity < 1)
            throw std::invalid_argument("server capacity must be positive");
        if (!std::isfinite(idle_timeout_s) || idle_timeout_s <= 0 || idle_timeout_s > 600)
            throw std::invalid_argument("idle timeout must be in (0, 600] seconds");
        if (max_slots < 0)
            throw std::invalid_argument("max_slots must be nonnegative");
        auto S = std::make_unique<rq_server>();
        std::vector<const rq_problem *> cp;
        long ws = 0;
        for (int i = 0; i < n_problems; ++i) {
            if (!problems[i])
                throw std::invalid_argument("null problem");
            S->problems.push_back(problems[i]);
            cp.push_back(problems[i]);
            S->thetaStride = std::max<int>(S->thetaStride, static_cast<int>(problems[i]->active.size()));
            S->predStride = std::max(S->predStride, problems[i]->nObs);
            ws = std::max(ws, static_cast<long>(problems[i]->cls.wsDoubles));
        }
        S->capacity = capacity;
        S->wsStride = ws;
        S->idleNs = static_cast<long long>(idle_timeout_s * 1e9);
        S->arena = chooseArena(cp);
        int dev = 0, sms = 1;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
        const int perSM = rq::serveBlocksPerSM(S->block, S->arena);
        if (perSM < 1)
            throw RqError(RQ_E_CUDA, "serve kernel does not fit on an SM with this arena");
        // admission by free HBM: as many solve slots as the SMs hold and free memory allows
        size_t freeB = 0, totalB = 0;
        check(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo");
        const long byMem = static_cast<long>(0.8 * static_cast<double>(freeB) / (8.0 * ws));
        long slots = std::min<long>(static_cast<long>(sms) * perSM, byMem);
        if (max_slots > 0)
            slots = std::min<long>(slots, max_slots);
        if (slots < 1)
            throw RqError(RQ_E_OOM, "free device memory holds no solve slot");
        S->grid = static_cast<int>(slots);
        S->dWs.ensure(sizeof(double) * ws * S->grid);
        S->dCtl.ensure(2 * sizeof(int));
        check(cudaMemset(S->dCtl.p, 0, 2 * sizeof(int)), "server counters");
        const size_t c = static_cast<size_t>(capacity);
        auto up = [](size_t b) { return (b + 255) / 256 * 256; };
        const size_t oJobs = 0, oTheta = oJobs + up(c * sizeof(rq::DevJob)),
                     oRows = oTheta + up(c * S->thetaStride * sizeof(double)),
                     oPred = oRows + up(c * sizeof(rq::RowOut)),
                     oClock = oPred + up(c * S->predStride * sizeof(double)),
                     oDone = oClock + up(c * 12 * sizeof(long long)),
                     oCtl = oDone + up(c * sizeof(int)), total = oCtl + 256;
        S->host.alloc(total);
        char *base = static_cast<char *>(S->host.p);
        S->jobs = reinterpret_cast<rq::DevJob *>(base + oJobs);
        S->theta = reinterpret_cast<double *>(base + oTheta);
        S->rows = reinterpret_cast<rq::RowOut *>(base + oRows);
        S->pred = reinterpret_cast<double *>(base + oPred);
        S->clock = reinterpret_cast<long long *>(base + oClock);
        S->done = reinterpret_cast<int *>(base + oDone);
        S->published = reinterpret_cast<int *>(base + oCtl);
        S->closed = S->published + 1;
        // unified addressing: the mapped host pointers are also the device pointers
        void *dp = nullptr;
        check(cudaHostGetDevicePointer(&dp, S->host.p, 0), "mapped pointer");
        if (dp != S->host.p)
            throw RqError(RQ_E_UNSUPPORTED, "serving needs unified virtual addressing");
        check(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking), "stream");
        check(cudaDeviceSynchronize(), "server set-up");
        S->launch();
        *out = S.release();
    });
}

int rq_server_submit(rq_server *s, int32_t problem, const double *theta, int64_t *ticket) {
    return guarded([&] {
        if (!s || !theta || !ticket)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(s->mu);
        if (__atomic_load_n(s->closed, __ATOMIC_ACQUIRE))
            throw std::invalid_argument("server is closed");
        if (problem < 0 || problem >= static_cast<int>(s->problems.size()))
            throw std::invalid_argument("problem index out of range");
        if (s->submitted >= s->capacity)
            throw std::invalid_argument("server capacity reached");
        const int t = s->submitted;
        const rq_problem &P = *s->problems[problem];
        double *th = s->theta + static_cast<long>(t) * s->thetaStride;
        for (size_t a = 0; a < P.active.size(); ++a)
            th[a] = theta[a];
        rq::DevJob &j = s->jobs[t];
        j.cls = P.dCls.as<rq::DevClass>();
        j.theta = th;
        j.row = s->rows + t;
        j.pred = s->pred + static_cast<long>(t) * s->predStride;
        j.fields = nullptr;
        j.hist = nullptr;
        j.clock = s->clock + 12L * t;
        j.histCap = 0;
        s->submitted = t + 1;
        __atomic_store_n(s->published, t + 1, __ATOMIC_RELEASE);
        s->ensureRunning();
        *ticket = t;
    });
}

int rq_server_poll(rq_server *s, int64_t ticket, int32_t *done, rq_row_out *row,
                   double *predictions, int64_t *clock12) {
    return guarded([&] {
        if (!s || !done)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(s->mu);
        if (ticket < 0 || ticket >= s->submitted)
            throw std::invalid_argument("unknown ticket");
        *done = __atomic_load_n(s->done + ticket, __ATOMIC_ACQUIRE) ? 1 : 0;
        if (!*done) {
            s->ensureRunning();
            return;
        }
        if (row)
            *row = toRow(s->rows[ticket]);
        if (predictions)
            std::memcpy(predictions, s->pred + ticket * s->predStride,
                        sizeof(double) * s->predStride);
        if (clock12)
            std::memcpy(clock12, s->clock + 12 * ticket, sizeof(long long) * 12);
    });
}

int rq_server_wait(rq_server *s, double timeout_s, int64_t *completed) {
    return guarded([&] {
        if (!s)
            throw std::invalid_argument("null argument");
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            {
                std::lock_guard<std::mutex> lock(s->mu);
                int64_t n = 0;
                for (int i = 0; i < s->submitted; ++i)
                    n += __atomic_load_n(s->done + i, __ATOMIC_ACQUIRE) ? 1 : 0;
                if (completed)
                    *completed = n;
                if (n == s->submitted)
                    return;
                s->ensureRunning();
            }
            const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (el >= timeout_s)
                return;
            std::this_thread::sleep_for(std::chrono::microseconds(200));
        }
    });
}

int rq_server_close(rq_server *s) {
    return guarded([&] {
        if (!s)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(s->mu);
        __atomic_store_n(s->closed, 1, __ATOMIC_RELEASE);
    });
}

int rq_server_info(rq_server *s, int32_t *slots, int64_t *submitted, int64_t *completed,
                   int32_t *launches) {
    return guarded([&] {
        if (!s)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(s->mu);
        if (slots)
            *slots = s->grid;
        if (submitted)
            *submitted = s->submitted;
        if (completed) {
            int64_t n = 0;
            for (int i = 0; i < s->submitted; ++i)
                n += __atomic_load_n(s->done + i, __ATOMIC_ACQUIRE) ? 1 : 0;
            *completed = n;
        }
        if (launches)
            *launches = s->launches;
    });
}

int rq_server_destroy(rq_server *s) {
    return guarded([&] { delete s; });
}

int rq_evaluate_noalloc(rq_problem *p, const double *theta_dev, rq_row_out *row_dev,
                        double *predictions_dev, void *stream) {
    return guarded([&] {
        if (!p || !theta_dev || !row_dev || (p->nObs > 0 && !predictions_dev))
            throw std::invalid_argument("null argument");
        const long need = static_cast<long>(p->cls.wsDoubles);
        if (need > rq::noAllocScratchDoubles())
            throw std::invalid_argument(
                "this mesh class needs " + std::to_string(need) +
                " doubles of solve scratch; the allocation-free entry point holds at most " +
                std::to_string(rq::noAllocScratchDoubles()) +
                " (8 MiB, about 17000 cells): use rq_evaluate_batch for larger meshes");
        rq::DevJob job{};
        job.cls = p->dCls.as<rq::DevClass>();
        job.theta = theta_dev;
        job.row = reinterpret_cast<rq::RowOut *>(row_dev);
        job.pred = predictions_dev;
        // shared-memory arena as the batch path sizes it for one class
        const int arena = arenaDoublesFor(need, p->arenaKb, p->mesh.n);
        check(rq::launchSolveNoAlloc(job, p->block, arena, static_cast<cudaStream_t>(stream)),
              "allocation-free solve launch");
    });
}

int rq_posterior_weights(const double *loglik, const double *log_q, int64_t n, double *weights,
                         double *log_evidence) {
    return guarded([&] {
        if (n < 1)
            throw std::invalid_argument("at least one evaluation is required");
        if (!loglik || !weights)
            throw std::invalid_argument("null argument");
        DevBuf d;
        const size_t b = sizeof(double) * static_cast<size_t>(n);
        d.ensure(3 * b + 4 * sizeof(double));
        double *dl = d.as<double>(), *dq = log_q ? dl + n : nullptr, *dw = dl + 2 * n,
               *dout = dl + 3 * n;
        check(cudaMemcpy(dl, loglik, b, cudaMemcpyHostToDevice), "loglik");
        if (log_q)
            check(cudaMemcpy(dq, log_q, b, cudaMemcpyHostToDevice), "log_q");
        check(rq::launchWeights(dl, dq, n, dw, dout, nullptr), "weights launch");
        double out[3];
        check(cudaMemcpy(out, dout, sizeof(out), cudaMemcpyDeviceToHost), "weights");
        if (out[2] != 0.0)
            throw std::invalid_argument("successful log likelihoods must be finite");
        check(cudaMemcpy(weights, dw, b, cudaMemcpyDeviceToHost), "weights");
        if (log_evidence)
            *log_evidence = out[0] + std::log(out[1]);
    });
}

int rq_posterior_weights_device(const double *loglik_dev, const double *log_q_dev, int64_t n,
                                double *weights_dev, double *out3_dev, void *stream) {
    return guarded([&] {
        if (n < 1 || !loglik_dev || !weights_dev || !out3_dev)
            throw std::invalid_argument("null argument or empty input");
        check(rq::launchWeights(loglik_dev, log_q_dev, n, weights_dev, out3_dev,
                                static_cast<cudaStream_t>(stream)), "weights launch");
    });
}

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
