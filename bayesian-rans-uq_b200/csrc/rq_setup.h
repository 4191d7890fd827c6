// Host-side set-up of one mesh class for the device solver: the periodic
// terrain-following mesh in structured (i, j) form, its wall distance, the
// planar singular-omega balance, the fixed AMG hierarchy of the pressure
// correction and the velocity-probe stencils. Everything here runs once per
// mesh class; the per-draw work is on the GPU.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace rq {

// Structured periodic mesh. Cell c = j*nx + i. "x-face" c is the east face of
// cell c (owner c, neighbour (i+1) mod nx, the last column's being the
// periodic wrap face). "y-face" jf*nx + i lies below cell row jf: jf = 0 is the
// bottom wall (owner row 0), jf = ny the top wall (owner row ny-1) and the rest
// are internal with owner row jf-1 and neighbour row jf.
struct StructMesh {
    int nx = 0, ny = 0, n = 0;
    double lx = 0;
    std::vector<double> cx, cy, vol, wd;
    std::vector<double> xa, xnx, xny, xw, xdl, xdx, xdy, xsh, xfx, xfy; // n
    std::vector<double> ya, ynx, yny, yw, ydl, ydx, ydy, yfx, yfy;      // n + nx
    // planar singular omega balance (empty unless the mesh qualifies)
    bool balance = false;
    std::vector<double> sing, slap, sgx, sgy; // sgx per x-face, sgy per y-face
    // generator nodes (front plane: x of column i, y of node (i, j) at j * (nx + 1) + i)
    // and the wall patch names, for the binary mesh export
    std::vector<double> xNodes, yNodes;
    std::string bottomName = "bottom", topName = "top";
    int nfy() const { return n + nx; }
};

// Mesh generators (restating core/src/Mesh.cpp:490-741 and :431-463).
StructMesh buildPeriodic(const std::vector<double> &xNodes, const std::vector<double> &yBottom,
                         double yTop, int ny, double y1t);
StructMesh makePeriodicChannel(int nx, int ny, double lx, double h, double reTau, double yPlus);
StructMesh makeCurvedPeriodic(const std::vector<double> &xNodes,
                              const std::vector<double> &yBottom, double yTop, int ny, double re,
                              double yPlus);

// The reference's binary mesh file (MSH2, Mesh::saveBinary, core/src/Mesh.cpp:751-811):
// native byte order, int32 indices, IEEE binary64 geometry, the periodic shift after
// each face's weight. Byte-identical to the reference's file for the same generator call.
std::vector<char> meshBinary(const StructMesh &m);

// Planar singular-omega qualification and arrays (rans-uq/src/SIMPLESolver.cpp:92-153).
void preparePlanarBalance(StructMesh &m);

// Fixed AMG hierarchy of the pressure-correction pattern. Level 0 is the
// structured 5-point matrix (entry slot*n + cell, slots: 0 diag, 1 W, 2 E,
// 3 S, 4 N); coarser levels are CSR. Aggregation is the reference's greedy
// strength-0.25 rule (core/include/LinearSolver.hpp:535-575) applied to the
// geometric Laplacian area/delta with the cell-0 pin. On that hierarchy the
// prolongation is smoothed (smoothed aggregation: one damped-Jacobi step of the
// strength-filtered geometric matrix applied to the piecewise-constant
// prolongation); on the row-relative fallback it stays piecewise constant. Coarse
// values are the Galerkin products P^T A P of the current matrix, gathered per
// coarse entry as weighted fine entries in one fixed order.
struct AmgHost {
    struct Level {
        int n = 0;
        std::vector<int> ptr, col;            // CSR (levels >= 1)
        std::vector<int> diagPos;             // CSR position of (i,i)
        std::vector<int> pPtr, pCol;          // prolongation: row -> coarse rows (all but
        std::vector<double> pVal;             //   the last level), columns ascending
        std::vector<int> rPtr, rCol;          // restriction P^T: coarse row -> fine rows,
        std::vector<double> rVal;             //   ascending
        std::vector<int> gPtr, gSrc;          // coarse nnz -> fine entries summed into it,
        std::vector<double> gW;               //   each times its weight P_iI P_jJ
    };
    std::vector<Level> lev;
    // V-cycle smoother weight, coarse-correction scale and damped-Jacobi sweeps
    // before and after the coarse correction: 0.6, 1 and 1 on the smoothed-aggregation
    // hierarchy; 0.75, 1.7 and 2 on the row-relative fallback, whose piecewise-constant
    // prolongation under-corrects (bump-wall meshes: 29 -> 16 PCG iterations per outer
    // iteration on 200 x 100 cells)
    double w = 0.6, alpha = 1.0;
    int sweeps = 1;
    int coarseN() const { return lev.back().n; }
    size_t coarseNnz() const { return lev.size() > 1 ? lev.back().col.size() : 0; }
};
// Coarsening stops at <= 96 rows (the reference stops at 50): a dense inverse of up
// to 96 rows, applied with several threads per row, costs less per V-cycle than the
// level below it (each coarse level is two barrier-separated phases down and two up,
// about 14k cycles per V-cycle at 1536 cells).
AmgHost buildAmg(const StructMesh &m, int minCoarse = 96, int maxLevels = 20);
// Smoothing weight of the prolongation, as a fraction of 1 / rho(D_F^-1 F): 0.85
// (PCG on pressure systems taken from Re_tau 182-1000 channel solves needs 2-4
// iterations with it; 1.15 and above lose the coarse correction).
constexpr double kProlongWeight = 0.85;

// Velocity/pressure probe (PreparedObservation, core/include/ObservationOperator.hpp:630-670).
struct ProbeHost {
    int cell = -1;
    double ox = 0, oy = 0, axx = 0, axy = 0, ayy = 0, det = 0;
    int nnb = 0;
    int nb[4] = {-1, -1, -1, -1}; // neighbour cell, or -1 for a wall face
    double dx[4] = {0, 0, 0, 0}, dy[4] = {0, 0, 0, 0}, wt[4] = {0, 0, 0, 0};
};
ProbeHost prepareProbe(const StructMesh &m, double x, double y);

// The faces of cell c in the reference's face-index order (creation order of
// buildPeriodic2D): returned as codes 0 W, 1 E, 2 S, 3 N. Used where the
// order of a sum or of a search must follow the reference.
int cellFaceOrder(const StructMesh &m, int c, int out[4]);

} // namespace rq
