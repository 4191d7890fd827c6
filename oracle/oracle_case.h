/*
 * Test infrastructure only: the plain-data case description shared by the two
 * CPU checkers under oracle/ (the compiled reference harness and the C++
 * restatement). Product code never includes this file.
 *
 * A case is one SIMPLE + k-omega SST solve on a streamwise-periodic 2-D mesh
 * built by the reference's periodic generator (core/src/Mesh.cpp:490-741),
 * driven exactly as ForwardModel::evaluateWithDiagnostics drives it
 * (rans-uq/src/ForwardModel.cpp:35-137) with channelDefaults boundary
 * conditions (core/include/BoundaryCondition.hpp:113-167) and velocity-profile
 * probes as the convergence monitor and likelihood (ObservationOperator.hpp).
 */
#ifndef RQ_ORACLE_CASE_H
#define RQ_ORACLE_CASE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_P_AMG = 0, ORC_P_PCG = 1, ORC_P_BICGSTAB = 2 };

typedef struct {
    /* mesh: curved == 0 -> makePeriodicChannel2D(nx, ny, lx, h, re_tau, yplus)
             curved == 1 -> makeCurvedChannelPeriodic2D(x_nodes, y_bottom, y_top, ny, re_mesh, yplus) */
    int32_t nx, ny, curved, pad0;
    double lx, h, re_tau, yplus;
    const double *x_nodes, *y_bottom;
    double y_top, re_mesh;
    /* physics */
    double nu;
    double bc_u, bc_k, bc_w;          /* channelDefaults(mesh, bc_u, bc_k, bc_w) */
    double init_u[3], init_p, init_k, init_w;
    /* SolverSettings (rans-uq FlowFields.hpp:70-241) */
    int32_t max_iter, inner_iter, conv_window, monitor_interval;
    int32_t turb_start, nut_floor_iters, pressure_solver, pad1;
    double tol, inner_tol, alpha_u, alpha_p, alpha_k, alpha_w;
    double body_force[3], div_limit, k_min, k_max, omega_min;
    /* the eleven SST coefficients, InferenceParameterSet order */
    double coeffs[11];
    /* velocity-profile probes of component obs_component */
    int32_t n_obs, obs_component;
    const double *obs_x, *obs_y, *obs_value, *obs_sigma;
} orc_case;

typedef struct {
    int32_t status;      /* EvaluationStatus: 0 Converged 1 Unconverged 2 Diverged 3 Invalid 4 Unknown */
    int32_t iterations;  /* ConvergenceHistory::finalIter */
    int32_t converged, diverged, stalled, n_hist;
    double loglik, final_worst, contraction_rate;
} orc_result;

/* fields layout written by both checkers: 11 blocks of nCells doubles
   Ux Uy Uz p k omega nuT F1 F2 Pk CDkw; history: 11 doubles per iteration
   (iteration Ux Uy Uz p k omega momentumScaled continuityScaled changeU remainingU) */
#define ORC_NFIELD 11
#define ORC_NHIST 11

#ifdef __cplusplus
}
#endif
#endif
