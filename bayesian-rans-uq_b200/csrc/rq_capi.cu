// C ABI of the B200 forward model (include/rq_b200.h). Host work here is the
// per-mesh-class set-up (rq_setup.cpp), admission of inputs with the
// reference's rules, and the launch of persistent solve CTAs; all per-draw
// numerics run in rq_solver.cu.
#include "rq_capi_common.h"

#include <cstdio>

using namespace rqc;

namespace rqc {

thread_local std::string g_error;

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
    if (knobKb >= 0)
        bytes = std::min<long>(knobKb * 1024L, optin - shared);
    else if (nmax <= 768)
        bytes = (optin / 2 - 1024) - shared; // half the SM (the whole hot set fits)
    else
        bytes = 0;
    bytes = std::max<long>(0, std::min(bytes, wsDoubles * 8));
    return static_cast<int>(bytes / 8 / 32 * 32);
}

void runOneJob(rq_problem &p, const rq::DevJob &job) {
    const int arena = chooseArena({&p});
    p.dJobs.ensure(sizeof(rq::DevJob));
    p.dWs.ensure(sizeof(double) * p.cls.wsDoubles);
    p.dCounter.ensure(sizeof(int));
    check(cudaMemcpy(p.dJobs.p, &job, sizeof(rq::DevJob), cudaMemcpyHostToDevice), "job");
    check(cudaMemset(p.dCounter.p, 0, sizeof(int)), "counter");
    check(rq::launchSolve(p.dJobs.as<rq::DevJob>(), 1, p.dCounter.as<int>(), p.dWs.as<double>(),
                          p.cls.wsDoubles, 1, p.block, arena, nullptr),
          "solve launch");
}

int chooseArena(const std::vector<const rq_problem *> &probs) {
    long ws = 0;
    int knob = -1;
    int nmax = 0;
    for (const auto *p : probs) {
        ws = std::max(ws, static_cast<long>(p->cls.wsDoubles));
        knob = std::max(knob, p->arenaKb);
        nmax = std::max(nmax, p->mesh.n);
    }
    return arenaDoublesFor(ws, knob, nmax);
}

} // namespace rqc

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
    // cell and face rows are found without integer division (exact below 2^21)
    if (static_cast<long>(m.n) + m.nfy() >= (1L << 21))
        throw RqError(RQ_E_UNSUPPORTED, "meshes of 2^21 cells and faces or more are not supported on the GPU path");
    // AMG hierarchy
    const int L = static_cast<int>(h.lev.size());
    if (L > rq::kMaxLevels)
        throw RqError(RQ_E_UNSUPPORTED, "AMG hierarchy deeper than 12 levels");
    if (h.coarseN() > rq::kMaxCoarse)
        throw RqError(RQ_E_UNSUPPORTED, "coarsest AMG level above 128 rows");
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
            // transfer operators as ELL (slot k * rows + row, -1 padding)
            auto ell = [](const std::vector<int> &ptr, const std::vector<int> &col,
                          const std::vector<double> &val, int rows, int &w,
                          std::vector<int> &ec, std::vector<double> &ev) {
                w = 0;
                for (int r = 0; r < rows; ++r)
                    w = std::max(w, ptr[r + 1] - ptr[r]);
                ec.assign(static_cast<size_t>(w) * rows, -1);
                ev.assign(static_cast<size_t>(w) * rows, 0.0);
                for (int r = 0; r < rows; ++r)
                    for (int k = ptr[r]; k < ptr[r + 1]; ++k) {
                        ec[static_cast<size_t>(k - ptr[r]) * rows + r] = col[k];
                        ev[static_cast<size_t>(k - ptr[r]) * rows + r] = val[k];
                    }
            };
            const int nc = h.lev[l + 1].n;
            std::vector<int> pc, rc;
            std::vector<double> pv, rv;
            ell(Lv.pPtr, Lv.pCol, Lv.pVal, Lv.n, dl.pw, pc, pv);
            ell(Lv.rPtr, Lv.rCol, Lv.rVal, nc, dl.rw, rc, rv);
            addI(&dl.pcol, pc);
            addD(&dl.pval, pv);
            addI(&dl.rcol, rc);
            addD(&dl.rval, rv);
            // gather lists in the next level's slot order; sources of level >= 1 as slots
            const int ns = width[l + 1] * nc;
            std::vector<int> gp(ns + 1, 0), gs;
            std::vector<double> gw;
            for (int slot = 0; slot < ns; ++slot) {
                const int e = entryOf[l + 1][slot];
                if (e >= 0)
                    for (int k = Lv.gPtr[e]; k < Lv.gPtr[e + 1]; ++k) {
                        gs.push_back(l == 0 ? Lv.gSrc[k] : slotOf[l][Lv.gSrc[k]]);
                        gw.push_back(Lv.gW[k]);
                    }
                gp[slot + 1] = static_cast<int>(gs.size());
            }
            addI(&dl.gPtr, gp);
            addI(&dl.gSrc, gs);
            addD(&dl.gW, gw);
        }
    }
    C.amgW = h.w;
    C.amgAlpha = h.alpha;
    C.amgSweeps = h.sweeps;
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
                  5 * pad32(nf) + pad32(valOff) + pad32(vecOff) + 2 * pad32(2 * mc * mc);
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

// CTA size of a class, measured per outer iteration on a B200 (FP64): 512 threads
// for up to 1024 cells (384 cells: 153 us at 512, 182 us at 768; 768 cells: equal),
// 768 threads above (1536 cells: 431 us at 768, 465 us at 512, 567 us at 1024 --
// two cells per thread; 1024 threads cap registers at 64 and spill).
int defaultBlock(int nCells) { return nCells > 1024 ? 768 : 512; }




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

// weights of n host log-likelihoods (and optional log proposal densities) on the device:
// out = {m, sum of exp(. - m)}; the weights land in `weights` (host)
void weightsOnDevice(const double *loglik, const double *log_q, int64_t n, double *weights,
                     double out[2]) {
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
    double o3[3];
    check(cudaMemcpy(o3, dout, sizeof(o3), cudaMemcpyDeviceToHost), "weights");
    if (o3[2] != 0.0)
        throw std::invalid_argument("successful log likelihoods must be finite");
    check(cudaMemcpy(weights, dw, b, cudaMemcpyDeviceToHost), "weights");
    out[0] = o3[0];
    out[1] = o3[1];
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
        check(cudaGetDevice(&P->device), "cudaGetDevice");
        P->mesh = buildMesh(*mesh);
        P->amg = rq::buildAmg(P->mesh);
        P->active.assign(active, active + n_active);
        std::memcpy(P->base, base, sizeof(P->base));
        P->nObs = obs ? obs->n_obs : 0;
        P->block = settings->block_threads ? rq::normalizeBlock(settings->block_threads)
                                           : defaultBlock(P->mesh.n);
        upload(*P, obs, nu, *settings, init);
        // the device address of rq_evaluate_noalloc's fixed scratch array, resolved here
        // (this call allocates anyway) so that the allocation-free call itself only launches
        check(rq::noAllocScratch(&P->noallocScratch), "scratch address");
        *out = P.release();
    });
}

int rq_problem_destroy(rq_problem *p) {
    return guarded([&] {
        if (!p)
            return;
        DeviceScope on(p->device);
        delete p;
    });
}

int rq_problem_workspace_bytes(const rq_problem *p, uint64_t *bytes) {
    return guarded([&] {
        if (!p || !bytes)
            throw std::invalid_argument("null argument");
        *bytes = sizeof(double) * static_cast<uint64_t>(p->cls.wsDoubles);
    });
}

int rq_problem_set_launch(rq_problem *p, const rq_launch_shape *shape) {
    return guarded([&] {
        if (!p || !shape)
            throw std::invalid_argument("null argument");
        requireDevice(*p);
        if (!rq::launchVariantExists(shape->block_threads))
            throw std::invalid_argument("block_threads must be 64, 128, 256, 512, 768 or 1024");
        if (shape->arena_kb < -1)
            throw std::invalid_argument("arena_kb must be -1 (default rule), 0 or positive");
        std::lock_guard<std::mutex> lock(p->mu);
        const int arena = arenaDoublesFor(p->cls.wsDoubles, shape->arena_kb, p->mesh.n);
        if (rq::solveBlocksPerSM(shape->block_threads, arena) < 1)
            throw std::invalid_argument("this launch shape does not fit on an SM");
        p->block = shape->block_threads;
        p->arenaKb = shape->arena_kb;
    });
}

int rq_problem_get_launch(const rq_problem *p, rq_launch_shape *shape) {
    return guarded([&] {
        if (!p || !shape)
            throw std::invalid_argument("null argument");
        shape->block_threads = p->block;
        shape->arena_kb = p->arenaKb;
        shape->us_per_iteration = 0.0;
    });
}

int rq_problem_tune(rq_problem *p, const double *theta, int32_t iters,
                    const rq_launch_shape *candidates, int32_t n_candidates,
                    rq_launch_shape *measured, rq_launch_shape *chosen) {
    return guarded([&] {
        if (!p || !theta || !chosen)
            throw std::invalid_argument("null argument");
        if (iters < 1)
            throw std::invalid_argument("iters must be positive");
        if (candidates && n_candidates < 1)
            throw std::invalid_argument("need at least one candidate");
        requireDevice(*p);
        std::vector<rq_launch_shape> cand;
        if (candidates) {
            cand.assign(candidates, candidates + n_candidates);
        } else {
            const long ws = p->cls.wsDoubles;
            const int largest = static_cast<int>(
                std::min<long>(maxSmemOptin() - static_cast<long>(rq::solveSharedBytes()), ws * 8) /
                1024);
            for (int b : {256, 512, 768})
                for (int a : {0, -1, largest})
                    cand.push_back(rq_launch_shape{b, a, 0.0});
        }
        std::lock_guard<std::mutex> lock(p->mu);
        const int na = static_cast<int>(p->active.size());
        // the class with its outer-iteration cap set to `iters` and no convergence exit
        rq::DevClass capped = p->cls;
        capped.st.maxIter = iters;
        capped.st.tol = -1.0;
        DevBuf dCap, dTheta, dRow, dPred, dClock, dWs, dJob, dCounter;
        dCap.ensure(sizeof(rq::DevClass));
        dTheta.ensure(sizeof(double) * na);
        dRow.ensure(sizeof(rq::RowOut));
        dPred.ensure(sizeof(double) * std::max(p->nObs, 1));
        dClock.ensure(sizeof(long long) * 12);
        dWs.ensure(sizeof(double) * p->cls.wsDoubles);
        dJob.ensure(sizeof(rq::DevJob));
        dCounter.ensure(sizeof(int));
        check(cudaMemcpy(dCap.p, &capped, sizeof(capped), cudaMemcpyHostToDevice), "class");
        check(cudaMemcpy(dTheta.p, theta, sizeof(double) * na, cudaMemcpyHostToDevice), "theta");
        rq::DevJob job{};
        job.cls = dCap.as<rq::DevClass>();
        job.theta = dTheta.as<double>();
        job.row = dRow.as<rq::RowOut>();
        job.pred = dPred.as<double>();
        job.clock = dClock.as<long long>();
        check(cudaMemcpy(dJob.p, &job, sizeof(job), cudaMemcpyHostToDevice), "job");
        int best = -1;
        for (size_t k = 0; k < cand.size(); ++k) {
            rq_launch_shape &c = cand[k];
            c.us_per_iteration = -1.0;
            if (!rq::launchVariantExists(c.block_threads) || c.arena_kb < -1)
                continue;
            const int arena = arenaDoublesFor(p->cls.wsDoubles, c.arena_kb, p->mesh.n);
            if (rq::solveBlocksPerSM(c.block_threads, arena) < 1)
                continue;
            check(cudaMemset(dCounter.p, 0, sizeof(int)), "counter");
            check(rq::launchSolve(dJob.as<rq::DevJob>(), 1, dCounter.as<int>(), dWs.as<double>(),
                                  p->cls.wsDoubles, 1, c.block_threads, arena, nullptr),
                  "tuning launch");
            check(cudaDeviceSynchronize(), "tuning solve");
            long long clk[12];
            rq::RowOut row;
            check(cudaMemcpy(clk, dClock.p, sizeof(clk), cudaMemcpyDeviceToHost), "clock");
            check(cudaMemcpy(&row, dRow.p, sizeof(row), cudaMemcpyDeviceToHost), "row");
            if (row.status == 3) // InvalidParameters: theta outside the box
                throw std::invalid_argument("tuning theta is outside the parameter bounds");
            const int it = std::max(row.iterations, 1);
            c.us_per_iteration = static_cast<double>(clk[1] - clk[0]) / 1e3 / it;
            if (best < 0 || c.us_per_iteration < cand[best].us_per_iteration)
                best = static_cast<int>(k);
        }
        if (measured)
            for (size_t k = 0; k < cand.size(); ++k)
                measured[k] = cand[k];
        if (best < 0)
            throw std::invalid_argument("no candidate launch shape fits on an SM");
        p->block = cand[best].block_threads;
        p->arenaKb = cand[best].arena_kb;
        *chosen = cand[best];
    });
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
            requireDevice(*problems[i]);
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
            requireDevice(*problems[i]);
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
        requireDevice(*p);
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
        requireDevice(*p);
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
        // one job whose class descriptor is the all-eleven view
        rq::DevJob j{};
        j.cls = dAll.as<rq::DevClass>();
        j.theta = p->dTheta.as<double>();
        j.row = p->dRows.as<rq::RowOut>();
        j.pred = p->dPred.as<double>();
        j.fields = fields ? p->dFields.as<double>() : nullptr;
        j.hist = wantHist ? p->dHist.as<double>() : nullptr;
        j.histCap = hist_cap;
        runOneJob(*p, j);
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

int rq_mesh_save_binary(const rq_mesh_desc *mesh, const char *path) {
    return guarded([&] {
        if (!mesh || !path)
            throw std::invalid_argument("null argument");
        const std::vector<char> bytes = rq::meshBinary(buildMesh(*mesh));
        std::FILE *f = std::fopen(path, "wb");
        if (!f)
            throw std::runtime_error(std::string("Cannot open binary mesh for writing: ") + path);
        const size_t put = std::fwrite(bytes.data(), 1, bytes.size(), f);
        const bool closed = std::fclose(f) == 0;
        if (put != bytes.size() || !closed)
            throw std::runtime_error(std::string("Cannot write binary mesh: ") + path);
    });
}

int rq_evaluate_noalloc(rq_problem *p, const double *theta_dev, rq_row_out *row_dev,
                        double *predictions_dev, void *stream) {
    return guarded([&] {
        if (!p || !theta_dev || !row_dev || (p->nObs > 0 && !predictions_dev))
            throw std::invalid_argument("null argument");
        requireDevice(*p);
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
        check(rq::launchSolveNoAlloc(job, p->noallocScratch, p->block, arena,
                                     static_cast<cudaStream_t>(stream)),
              "allocation-free solve launch");
    });
}

int rq_posterior_weights(const double *loglik, const double *log_q, int64_t n, double *weights,
                         double *log_evidence) {
    return guarded([&] {
        double ms[2];
        weightsOnDevice(loglik, log_q, n, weights, ms);
        if (log_evidence)
            *log_evidence = ms[0] + std::log(ms[1]);
    });
}

int rq_posterior_weights_parts(const double *loglik, const double *log_q, int64_t n,
                               double *weights, double *max_out, double *sum_out) {
    return guarded([&] {
        if (!max_out || !sum_out)
            throw std::invalid_argument("null argument");
        double ms[2];
        weightsOnDevice(loglik, log_q, n, weights, ms);
        *max_out = ms[0];
        *sum_out = ms[1];
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

} // extern "C"
