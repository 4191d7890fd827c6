// Test infrastructure only. A C-ABI harness over the reference's OWN public
// C++ API (compiled from the reference sources by oracle/Makefile into
// oracle/_ref/). It adds no numerics: every number it returns is computed by
// the reference's ForwardModel / SIMPLESolver / LinearSolver code.
//
//   Mesh::makePeriodicChannel2D / makeCurvedChannelPeriodic2D  core/src/Mesh.cpp:490-521
//   ForwardModel::evaluateWithDiagnostics                       rans-uq/src/ForwardModel.cpp:35-137
//   makeSolver(name)->solve                                     core/include/LinearSolver.hpp:988-998
#include "ForwardModel.hpp"
#include "oracle_case.h"

#include <cstring>
#include <iostream>
#include <sstream>

namespace {

Mesh buildMesh(const orc_case &c) {
    if (c.curved) {
        std::vector<double> xn(c.x_nodes, c.x_nodes + c.nx + 1);
        std::vector<double> yb(c.y_bottom, c.y_bottom + c.nx + 1);
        return Mesh::makeCurvedChannelPeriodic2D(xn, yb, c.y_top, c.ny, c.re_mesh, c.yplus);
    }
    return Mesh::makePeriodicChannel2D(c.nx, c.ny, c.lx, c.h, c.re_tau, c.yplus);
}

SolverSettings buildSettings(const orc_case &c) {
    SolverSettings s;
    s.maxIterations = c.max_iter;
    s.innerIterations = c.inner_iter;
    s.convergenceWindow = c.conv_window;
    s.monitorInterval = c.monitor_interval;
    s.turbStartIter = c.turb_start;
    s.nuTFloorIters = c.nut_floor_iters;
    s.convergenceTol = c.tol;
    s.innerTolerance = c.inner_tol;
    s.alphaU = c.alpha_u;
    s.alphaP = c.alpha_p;
    s.alphaK = c.alpha_k;
    s.alphaOmega = c.alpha_w;
    s.bodyForce = Vec3(c.body_force[0], c.body_force[1], c.body_force[2]);
    s.divergenceLimit = c.div_limit;
    s.kMin = c.k_min;
    s.kMax = c.k_max;
    s.omegaMin = c.omega_min;
    s.verbose = false;
    s.pressureSolver = c.pressure_solver == ORC_P_PCG        ? "PCG"
                       : c.pressure_solver == ORC_P_BICGSTAB ? "BiCGSTAB"
                                                             : "AMG";
    return s;
}

void copyFields(const Mesh &m, const FlowFields &f, double *out) {
    const int n = m.nCells();
    for (int i = 0; i < n; ++i) {
        out[0 * n + i] = f.U[i].x;
        out[1 * n + i] = f.U[i].y;
        out[2 * n + i] = f.U[i].z;
        out[3 * n + i] = f.p[i];
        out[4 * n + i] = f.k[i];
        out[5 * n + i] = f.omega[i];
        out[6 * n + i] = f.nuT[i];
        out[7 * n + i] = f.F1[i];
        out[8 * n + i] = f.F2[i];
        out[9 * n + i] = f.Pk[i];
        out[10 * n + i] = f.CDkw[i];
    }
}

thread_local std::string lastError;

} // namespace

extern "C" {

const char *ref_last_error() { return lastError.c_str(); }

// Mesh geometry as the reference builds it. cells: nCells x 4 (cx, cy, volume,
// wall distance); faces: nFaces x 13 (owner, neighbour, cx, cy, nx, ny, area,
// delta, dx, dy, weight, shift_x, patch). Returns nCells*1e6+nFaces style
// counts through the two out pointers; arrays may be null to query sizes.
int ref_mesh(const orc_case *c, int32_t *n_cells, int32_t *n_faces, int32_t *n_internal,
             double *cells, double *faces) {
    try {
        std::streambuf *old = std::cout.rdbuf(nullptr);
        Mesh m = buildMesh(*c);
        std::cout.rdbuf(old);
        m.computeWallDistance();
        *n_cells = m.nCells();
        *n_faces = m.nFaces();
        *n_internal = m.nInternalFaces();
        if (cells) {
            const auto &wd = m.wallDistance();
            for (int i = 0; i < m.nCells(); ++i) {
                cells[4 * i + 0] = m.cell(i).center.x;
                cells[4 * i + 1] = m.cell(i).center.y;
                cells[4 * i + 2] = m.cell(i).volume;
                cells[4 * i + 3] = wd[i];
            }
        }
        if (faces) {
            for (int fi = 0; fi < m.nFaces(); ++fi) {
                const Face &f = m.face(fi);
                double *o = faces + 13 * fi;
                o[0] = f.owner;
                o[1] = f.neighbor;
                o[2] = f.center.x;
                o[3] = f.center.y;
                o[4] = f.normal.x;
                o[5] = f.normal.y;
                o[6] = f.area;
                o[7] = f.delta;
                o[8] = f.d.x;
                o[9] = f.d.y;
                o[10] = f.weight;
                o[11] = f.shift.x;
                o[12] = f.patchID;
            }
        }
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

// One cold ForwardModel evaluation (a1_betaStar parameter set whose base
// carries the other nine coefficients), returning the verdict, predictions,
// the retained fields and the residual history.
int ref_solve(const orc_case *c, orc_result *res, double *fields, double *predictions,
              double *history, int32_t hist_cap) {
    try {
        std::streambuf *old = std::cout.rdbuf(nullptr);
        Mesh mesh = buildMesh(*c);
        std::cout.rdbuf(old);
        mesh.computeWallDistance();
        auto bcs = FlowBoundaryConditions::channelDefaults(mesh, c->bc_u, c->bc_k, c->bc_w);
        ObservationOperator obs;
        for (int i = 0; i < c->n_obs; ++i)
            obs.addVelocityProfile(Vec3(c->obs_x[i], c->obs_y[i], 0.0), c->obs_component,
                                   c->obs_value[i], c->obs_sigma[i]);
        auto params = InferenceParameterSet::a1_betaStar();
        params.base = InferenceParameterSet::fromVector(std::vector<double>(c->coeffs, c->coeffs + 11));
        ForwardModel model(mesh, params, obs, bcs, c->nu, buildSettings(*c),
                           Vec3(c->init_u[0], c->init_u[1], c->init_u[2]), c->init_p, c->init_k,
                           c->init_w);
        std::vector<double> theta = {c->coeffs[9], c->coeffs[8]};
        auto ev = model.evaluateWithDiagnostics(theta);
        if (!ev.error.empty()) {
            lastError = ev.error;
        }
        res->status = static_cast<int32_t>(ev.result.status);
        res->iterations = ev.result.simpleIters;
        res->converged = ev.convergence.converged;
        res->diverged = ev.convergence.diverged;
        res->stalled = ev.convergence.stalled;
        res->loglik = ev.result.loglik;
        res->final_worst = ev.convergence.finalWorstMeasure;
        res->contraction_rate = ev.convergence.contractionRateU;
        const auto &h = ev.convergence.entries;
        res->n_hist = static_cast<int32_t>(h.size());
        if (history) {
            for (int i = 0; i < static_cast<int>(h.size()) && i < hist_cap; ++i) {
                double *o = history + ORC_NHIST * i;
                o[0] = h[i].iteration;
                o[1] = h[i].Ux;
                o[2] = h[i].Uy;
                o[3] = h[i].Uz;
                o[4] = h[i].p;
                o[5] = h[i].k;
                o[6] = h[i].omega;
                o[7] = h[i].momentumScaled;
                o[8] = h[i].continuityScaled;
                o[9] = h[i].changeU;
                o[10] = h[i].remainingU;
            }
        }
        if (predictions)
            for (size_t i = 0; i < ev.result.predictions.size(); ++i)
                predictions[i] = ev.result.predictions[i];
        if (fields && model.hasLastFields())
            copyFields(mesh, model.lastFields(), fields);
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

// A sequence of evaluateWithDiagnostics calls on ONE ForwardModel, whose warm-start
// cache (ForwardModel.hpp:21-157; the model builds it as cache_(50, 0.5),
// ForwardModel.cpp:14) seeds each call from the nearest converged state. Only the
// byte budget can be changed after construction (setByteBudget), so max_size and
// threshold must be the model's own 50 and 0.5.
int ref_solve_sequence(const orc_case *c, const double *thetas, int32_t m_calls, int32_t max_size,
                       double threshold, int64_t byte_budget, orc_result *res,
                       double *predictions, int32_t *used_warm, int64_t *retained) {
    try {
        if (max_size != 50 || threshold != 0.5)
            throw std::invalid_argument("the reference model's cache is (50, 0.5)");
        std::streambuf *old = std::cout.rdbuf(nullptr);
        Mesh mesh = buildMesh(*c);
        std::cout.rdbuf(old);
        mesh.computeWallDistance();
        auto bcs = FlowBoundaryConditions::channelDefaults(mesh, c->bc_u, c->bc_k, c->bc_w);
        ObservationOperator obs;
        for (int i = 0; i < c->n_obs; ++i)
            obs.addVelocityProfile(Vec3(c->obs_x[i], c->obs_y[i], 0.0), c->obs_component,
                                   c->obs_value[i], c->obs_sigma[i]);
        auto params = InferenceParameterSet::a1_betaStar();
        params.base = InferenceParameterSet::fromVector(std::vector<double>(c->coeffs, c->coeffs + 11));
        ForwardModel model(mesh, params, obs, bcs, c->nu, buildSettings(*c),
                           Vec3(c->init_u[0], c->init_u[1], c->init_u[2]), c->init_p, c->init_k,
                           c->init_w);
        model.cache().setByteBudget(static_cast<size_t>(byte_budget));
        for (int i = 0; i < m_calls; ++i) {
            std::vector<double> theta = {thetas[2 * i], thetas[2 * i + 1]};
            auto ev = model.evaluateWithDiagnostics(theta);
            if (!ev.error.empty())
                lastError = ev.error;
            orc_result &r = res[i];
            std::memset(&r, 0, sizeof(r));
            r.status = static_cast<int32_t>(ev.result.status);
            r.iterations = ev.result.simpleIters;
            r.converged = ev.convergence.converged;
            r.diverged = ev.convergence.diverged;
            r.stalled = ev.convergence.stalled;
            r.loglik = ev.result.loglik;
            r.final_worst = ev.convergence.finalWorstMeasure;
            r.contraction_rate = ev.convergence.contractionRateU;
            used_warm[i] = ev.usedWarmStart;
            if (predictions)
                for (size_t k = 0; k < ev.result.predictions.size(); ++k)
                    predictions[static_cast<size_t>(i) * c->n_obs + k] = ev.result.predictions[k];
            if (retained)
                retained[i] = static_cast<int64_t>(model.cache().retainedBytes());
        }
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

// One cold evaluateWithDiagnostics(theta, snapshot = true) (ForwardModel.cpp:118-119,
// OwnedFlowSnapshot ForwardModel.hpp:162-186): cells (11 x nC blocks Ux Uy Uz p k omega
// nuT F1 F2 Pk CDkw), boundary faces (the same 11 blocks over nB faces), the face fluxes
// (nF, owner-outward, the mesh's face order) and the turbulence marker. has_snapshot = 0
// when the reference returns none (a diverged or invalid evaluation).
int ref_solve_snapshot(const orc_case *c, orc_result *res, double *cells, double *boundary,
                       double *fluxes, int32_t *turb_established, int32_t *has_snapshot) {
    try {
        std::streambuf *old = std::cout.rdbuf(nullptr);
        Mesh mesh = buildMesh(*c);
        std::cout.rdbuf(old);
        mesh.computeWallDistance();
        auto bcs = FlowBoundaryConditions::channelDefaults(mesh, c->bc_u, c->bc_k, c->bc_w);
        ObservationOperator obs;
        for (int i = 0; i < c->n_obs; ++i)
            obs.addVelocityProfile(Vec3(c->obs_x[i], c->obs_y[i], 0.0), c->obs_component,
                                   c->obs_value[i], c->obs_sigma[i]);
        auto params = InferenceParameterSet::a1_betaStar();
        params.base = InferenceParameterSet::fromVector(std::vector<double>(c->coeffs, c->coeffs + 11));
        ForwardModel model(mesh, params, obs, bcs, c->nu, buildSettings(*c),
                           Vec3(c->init_u[0], c->init_u[1], c->init_u[2]), c->init_p, c->init_k,
                           c->init_w);
        std::vector<double> theta = {c->coeffs[9], c->coeffs[8]};
        auto ev = model.evaluateWithDiagnostics(theta, true);
        std::memset(res, 0, sizeof(*res));
        res->status = static_cast<int32_t>(ev.result.status);
        res->iterations = ev.result.simpleIters;
        res->loglik = ev.result.loglik;
        *has_snapshot = ev.snapshot.has_value();
        if (!ev.snapshot)
            return 0;
        const OwnedFlowSnapshot &s = *ev.snapshot;
        const size_t n = s.p.size(), nb = s.pBoundary.size();
        auto put = [](double *dst, size_t m, const std::vector<Vec3> &v,
                      const std::initializer_list<const std::vector<double> *> &scalars) {
            for (size_t i = 0; i < m; ++i) {
                dst[i] = v[i].x;
                dst[m + i] = v[i].y;
                dst[2 * m + i] = v[i].z;
            }
            size_t b = 3;
            for (const std::vector<double> *f : scalars) {
                for (size_t i = 0; i < m; ++i)
                    dst[b * m + i] = (*f)[i];
                ++b;
            }
        };
        put(cells, n, s.U, {&s.p, &s.k, &s.omega, &s.nuT, &s.F1, &s.F2, &s.Pk, &s.CDkw});
        put(boundary, nb, s.UBoundary,
            {&s.pBoundary, &s.kBoundary, &s.omegaBoundary, &s.nuTBoundary, &s.F1Boundary,
             &s.F2Boundary, &s.PkBoundary, &s.CDkwBoundary});
        for (size_t f = 0; f < s.faceFluxes.size(); ++f)
            fluxes[f] = s.faceFluxes[f];
        *turb_established = s.turbEstablished;
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

// Mesh::saveBinary (core/src/Mesh.cpp:751-811) of the case's generated mesh.
int ref_mesh_save_binary(const orc_case *c, const char *path) {
    try {
        std::streambuf *old = std::cout.rdbuf(nullptr);
        Mesh mesh = buildMesh(*c);
        std::cout.rdbuf(old);
        mesh.saveBinary(path);
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

// The reference linear solvers on one LDU system: kind 0 AMG, 1 PCG, 2 BiCGSTAB,
// 3 GaussSeidel. x is the initial guess on input and the solution on output.
int ref_linear_solve(int32_t kind, int32_t n, int32_t nif, const double *diag,
                     const double *upper, const double *lower, const double *source,
                     const int32_t *own, const int32_t *nbr, double *x, int32_t max_iter,
                     double tol, int32_t *iterations, double *final_res, double *initial_res,
                     int32_t *converged) {
    try {
        LinearSystem A(n, nif);
        std::memcpy(A.diag.data(), diag, sizeof(double) * n);
        std::memcpy(A.source.data(), source, sizeof(double) * n);
        std::memcpy(A.upper.data(), upper, sizeof(double) * nif);
        std::memcpy(A.lower.data(), lower, sizeof(double) * nif);
        for (int f = 0; f < nif; ++f) {
            A.own[f] = own[f];
            A.nbr[f] = nbr[f];
        }
        const char *names[] = {"AMG", "PCG", "BiCGSTAB", "GaussSeidel"};
        auto solver = makeSolver(names[kind]);
        std::vector<double> xv(x, x + n);
        SolverResult r = solver->solve(A, xv, max_iter, tol);
        std::memcpy(x, xv.data(), sizeof(double) * n);
        *iterations = r.iterations;
        *final_res = r.finalRes;
        *initial_res = r.initialRes;
        *converged = r.converged;
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

} // extern "C"
