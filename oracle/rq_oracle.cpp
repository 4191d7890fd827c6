// Test infrastructure only (the oracle): a C++ restatement of the reference
// SIMPLE + k-omega SST forward model on streamwise-periodic 2-D meshes. It is
// the checker for the CUDA path, never part of it. Every routine cites the
// reference lines it restates (paths relative to the reference project).
//
// Arithmetic follows the reference's operation order (face loops accumulate
// into owner then neighbour, products associate left to right, no FMA under
// the -O2 x86-64 flags of oracle/Makefile), so with the same linear solvers the
// restatement reproduces the compiled reference to round-off. Linear solvers:
//   PCG (Jacobi)  LinearSolver.hpp:184-246      BiCGSTAB  LinearSolver.hpp:251-345
//   "AMG" here is the DEVICE-STYLE preconditioner of the GPU path: the
//   reference's greedy aggregation (LinearSolver.hpp:535-575) and Galerkin
//   product (:578-618) applied once to the geometric Laplacian of the mesh,
//   damped-Jacobi pre/post smoothing and an exact dense coarsest solve, inside
//   the reference's PCG loop (:908-982). The reference's own Gauss-Seidel AMG is
//   exercised through the compiled reference (oracle/_ref), not restated here.
#include "oracle_case.h"

#include <algorithm>
#include <array>
#include <initializer_list>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

using Vec = std::vector<double>;
static const double INF = std::numeric_limits<double>::infinity();

// ---------------------------------------------------------------- mesh
// Restates Mesh::buildPeriodic2D (core/src/Mesh.cpp:523-741) and the two
// periodic factories (:490-521); wall distance as computeWallDistance (:431-463).
struct Mesh {
    int nx = 0, ny = 0, nC = 0, nF = 0, nI = 0;
    Vec cx, cy, vol, wd;
    std::vector<int> own, nbr, patch;
    Vec fcx, fcy, fnx, fny, area, delta, ddx, ddy, w, shx;
    std::vector<std::vector<int>> cellFaces;
    int nB() const { return nF - nI; }
};

static Mesh buildPeriodic(const Vec &xN, const Vec &yB, double yTop, int ny, double y1t) {
    Mesh m;
    const int nx = static_cast<int>(xN.size()) - 1;
    if (nx < 3 || static_cast<int>(yB.size()) != nx + 1 || ny < 1)
        throw std::invalid_argument("periodic mesh needs nx >= 3 columns and ny >= 1 rows");
    m.nx = nx;
    m.ny = ny;
    const double Lx = xN.back() - xN.front();
    double meanH = 0.0;
    for (int i = 0; i <= nx; ++i)
        meanH += (yTop - yB[i]);
    meanH /= (nx + 1);
    // tanh stretch bisected for the first-cell height (Mesh.cpp:554-576)
    double stretch = 2.0;
    if (y1t > 0) {
        auto firstHeight = [&](double s) {
            return 0.5 * meanH * (1.0 + std::tanh(s * (2.0 / ny - 1.0)) / std::tanh(s));
        };
        if (y1t < meanH / ny) {
            double lo = 0.1, hi = 20.0;
            if (y1t < firstHeight(hi)) {
                stretch = hi;
            } else {
                for (int it = 0; it < 100; ++it) {
                    double mid = 0.5 * (lo + hi);
                    if (firstHeight(mid) > y1t)
                        lo = mid;
                    else
                        hi = mid;
                    if (hi - lo < 1e-10)
                        break;
                }
                stretch = 0.5 * (lo + hi);
            }
        }
    }
    Vec eta(ny + 1);
    for (int j = 0; j <= ny; ++j) {
        double e = static_cast<double>(j) / ny;
        eta[j] = 0.5 * (1.0 + std::tanh(stretch * (2.0 * e - 1.0)) / std::tanh(stretch));
    }
    auto yn = [&](int i, int j) { return yB[i] + (yTop - yB[i]) * eta[j]; };
    const int nC = nx * ny;
    m.nC = nC;
    m.cx.resize(nC);
    m.cy.resize(nC);
    m.vol.resize(nC);
    m.cellFaces.resize(nC);
    auto cid = [&](int i, int j) { return j * nx + i; };
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double px[4] = {xN[i], xN[i + 1], xN[i + 1], xN[i]};
            const double py[4] = {yn(i, j), yn(i + 1, j), yn(i + 1, j + 1), yn(i, j + 1)};
            double a2 = 0.0, sx = 0.0, sy = 0.0;
            for (int k = 0; k < 4; ++k) {
                const int kn = (k + 1) % 4;
                const double cr = px[k] * py[kn] - px[kn] * py[k];
                a2 += cr;
                sx += (px[k] + px[kn]) * cr;
                sy += (py[k] + py[kn]) * cr;
            }
            const double A = 0.5 * a2;
            m.cx[cid(i, j)] = sx / (6.0 * A);
            m.cy[cid(i, j)] = sy / (6.0 * A);
            m.vol[cid(i, j)] = std::abs(A) * 1.0;
        }
    const int nV = (nx - 1) * ny, nW = ny, nH = nx * (ny - 1);
    m.nI = nV + nW + nH;
    m.nF = m.nI + 2 * nx;
    const int nF = m.nF;
    for (Vec *v : {&m.fcx, &m.fcy, &m.fnx, &m.fny, &m.area, &m.delta, &m.ddx, &m.ddy, &m.shx})
        v->assign(nF, 0.0);
    m.w.assign(nF, 0.5);
    m.own.assign(nF, -1);
    m.nbr.assign(nF, -1);
    m.patch.assign(nF, -1);
    int f = 0;
    auto edge = [&](int fi, double x0, double y0, double x1, double y1, bool plusX) {
        const double ex = x1 - x0, ey = y1 - y0;
        const double len = std::sqrt(ex * ex + ey * ey);
        m.fcx[fi] = 0.5 * (x0 + x1);
        m.fcy[fi] = 0.5 * (y0 + y1);
        m.area[fi] = len * 1.0;
        if (plusX) {
            m.fnx[fi] = ey / len;
            m.fny[fi] = -ex / len;
        } else {
            m.fnx[fi] = -ey / len;
            m.fny[fi] = ex / len;
        }
    };
    auto distWeight = [&](int fi, double ox, double oy, double nxc, double nyc) {
        m.ddx[fi] = nxc - ox;
        m.ddy[fi] = nyc - oy;
        m.delta[fi] = std::max(std::sqrt(m.ddx[fi] * m.ddx[fi] + m.ddy[fi] * m.ddy[fi]), 1e-20);
        const double ax = m.fcx[fi] - ox, ay = m.fcy[fi] - oy;
        const double bx = m.fcx[fi] - nxc, by = m.fcy[fi] - nyc;
        const double dP = std::sqrt(ax * ax + ay * ay), dN = std::sqrt(bx * bx + by * by);
        const double s = dP + dN;
        m.w[fi] = (s > 1e-30) ? dN / s : 0.5;
    };
    auto link = [&](int fi) {
        m.cellFaces[m.own[fi]].push_back(fi);
        if (m.nbr[fi] >= 0)
            m.cellFaces[m.nbr[fi]].push_back(fi);
    };
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx - 1; ++i, ++f) {
            m.own[f] = cid(i, j);
            m.nbr[f] = cid(i + 1, j);
            edge(f, xN[i + 1], yn(i + 1, j), xN[i + 1], yn(i + 1, j + 1), true);
            distWeight(f, m.cx[m.own[f]], m.cy[m.own[f]], m.cx[m.nbr[f]], m.cy[m.nbr[f]]);
            link(f);
        }
    for (int j = 0; j < ny; ++j, ++f) {
        m.own[f] = cid(nx - 1, j);
        m.nbr[f] = cid(0, j);
        edge(f, xN[nx], yn(nx, j), xN[nx], yn(nx, j + 1), true);
        m.shx[f] = Lx;
        distWeight(f, m.cx[m.own[f]], m.cy[m.own[f]], m.cx[m.nbr[f]] + Lx, m.cy[m.nbr[f]] + 0.0);
        link(f);
    }
    for (int j = 0; j < ny - 1; ++j)
        for (int i = 0; i < nx; ++i, ++f) {
            m.own[f] = cid(i, j);
            m.nbr[f] = cid(i, j + 1);
            edge(f, xN[i], yn(i, j + 1), xN[i + 1], yn(i + 1, j + 1), false);
            distWeight(f, m.cx[m.own[f]], m.cy[m.own[f]], m.cx[m.nbr[f]], m.cy[m.nbr[f]]);
            link(f);
        }
    for (int side = 0; side < 2; ++side)
        for (int i = 0; i < nx; ++i, ++f) {
            const int j = side == 0 ? 0 : ny - 1, jn = side == 0 ? 0 : ny;
            m.own[f] = cid(i, j);
            m.patch[f] = side;
            edge(f, xN[i], yn(i, jn), xN[i + 1], yn(i + 1, jn), side == 0);
            m.ddx[f] = m.fcx[f] - m.cx[m.own[f]];
            m.ddy[f] = m.fcy[f] - m.cy[m.own[f]];
            m.delta[f] = std::max(std::sqrt(m.ddx[f] * m.ddx[f] + m.ddy[f] * m.ddy[f]), 1e-20);
            link(f);
        }
    // brute-force wall distance over every wall-face centre (both patches are walls)
    m.wd.assign(nC, 0.0);
    for (int c = 0; c < nC; ++c) {
        double best = std::numeric_limits<double>::max();
        for (int b = m.nI; b < nF; ++b) {
            const double dx = m.cx[c] - m.fcx[b], dy = m.cy[c] - m.fcy[b];
            const double d = std::sqrt(dx * dx + dy * dy);
            if (d < best)
                best = d;
        }
        m.wd[c] = best;
    }
    return m;
}

static Mesh buildMesh(const orc_case &c) {
    if (c.curved) {
        Vec xN(c.x_nodes, c.x_nodes + c.nx + 1), yB(c.y_bottom, c.y_bottom + c.nx + 1);
        double y1t = 0.0;
        if (c.re_mesh > 0) { // skin-friction sizing, Mesh.cpp:496-506
            double meanH = 0.0;
            for (double v : yB)
                meanH += (c.y_top - v);
            meanH /= static_cast<double>(yB.size());
            const double cf = 0.058 * std::pow(c.re_mesh, -0.2);
            const double uTau = std::sqrt(cf / 2.0);
            const double nu = meanH / c.re_mesh;
            y1t = c.yplus * nu / uTau;
        }
        return buildPeriodic(xN, yB, c.y_top, c.ny, y1t);
    }
    Vec xN(c.nx + 1), yB(c.nx + 1, 0.0);
    for (int i = 0; i <= c.nx; ++i)
        xN[i] = c.lx * i / c.nx;
    return buildPeriodic(xN, yB, 2.0 * c.h, c.ny, c.yplus * c.h / c.re_tau);
}

// ---------------------------------------------------------------- LDU system
// LinearSystem (core/include/LinearSolver.hpp:20-116)
struct Ldu {
    int n = 0, nf = 0;
    Vec d, up, lo, b;
    const std::vector<int> *own = nullptr, *nbr = nullptr;
    void init(const Mesh &m) {
        n = m.nC;
        nf = m.nI;
        d.assign(n, 0.0);
        b.assign(n, 0.0);
        up.assign(nf, 0.0);
        lo.assign(nf, 0.0);
        own = &m.own;
        nbr = &m.nbr;
    }
    void zero() {
        std::fill(d.begin(), d.end(), 0.0);
        std::fill(b.begin(), b.end(), 0.0);
        std::fill(up.begin(), up.end(), 0.0);
        std::fill(lo.begin(), lo.end(), 0.0);
    }
    void matvec(const Vec &x, Vec &y) const {
        for (int i = 0; i < n; ++i)
            y[i] = d[i] * x[i];
        for (int f = 0; f < nf; ++f) {
            const int o = (*own)[f], q = (*nbr)[f];
            y[o] += up[f] * x[q];
            y[q] += lo[f] * x[o];
        }
    }
    void residual(const Vec &x, Vec &r) const {
        matvec(x, r);
        for (int i = 0; i < n; ++i)
            r[i] = b[i] - r[i];
    }
};

static double dot(const Vec &a, const Vec &b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i)
        s += a[i] * b[i];
    return s;
}
static double norm2(const Vec &a) { return std::sqrt(dot(a, a)); }
static void jacobi(const Ldu &A, const Vec &r, Vec &z) {
    for (int i = 0; i < A.n; ++i)
        z[i] = (std::abs(A.d[i]) > 1e-30) ? r[i] / A.d[i] : r[i];
}

struct LinResult {
    int iterations = 0;
    double finalRes = 0.0, initialRes = 0.0;
    bool converged = false;
    bool breakdown = false; // PCG stopped on |p.Ap| < 1e-30
};

// Right-Jacobi BiCGSTAB (LinearSolver.hpp:251-345)
static LinResult bicgstab(const Ldu &A, Vec &x, int maxIter, double tol) {
    const int n = A.n;
    Vec r(n), rh(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
    LinResult res;
    A.residual(x, r);
    const double r0 = norm2(r);
    res.initialRes = r0;
    if (r0 < 1e-30) {
        res.converged = true;
        return res;
    }
    rh = r;
    double rho = 1, alpha = 1, omega = 1;
    for (int it = 0; it < maxIter; ++it) {
        const double rhoN = dot(rh, r);
        if (std::abs(rhoN) < 1e-30)
            break;
        const double beta = (rhoN / (rho + 1e-30)) * (alpha / (omega + 1e-30));
        for (int i = 0; i < n; ++i)
            p[i] = r[i] + beta * (p[i] - omega * v[i]);
        jacobi(A, p, ph);
        A.matvec(ph, v);
        const double rv = dot(rh, v);
        if (std::abs(rv) < 1e-30)
            break;
        alpha = rhoN / rv;
        for (int i = 0; i < n; ++i)
            s[i] = r[i] - alpha * v[i];
        const double sn = norm2(s);
        if (sn / r0 < tol) {
            for (int i = 0; i < n; ++i)
                x[i] += alpha * ph[i];
            res.iterations = it + 1;
            res.finalRes = sn / r0;
            res.converged = true;
            return res;
        }
        jacobi(A, s, sh);
        A.matvec(sh, t);
        const double tt = dot(t, t);
        omega = (tt > 1e-30) ? dot(t, s) / tt : 0.0;
        for (int i = 0; i < n; ++i)
            x[i] += alpha * ph[i] + omega * sh[i];
        for (int i = 0; i < n; ++i)
            r[i] = s[i] - omega * t[i];
        const double rn = norm2(r);
        res.iterations = it + 1;
        res.finalRes = rn / r0;
        if (res.finalRes < tol) {
            res.converged = true;
            return res;
        }
        if (std::abs(omega) < 1e-30)
            break;
        rho = rhoN;
    }
    return res;
}

// ---------------------------------------------------------------- device-style AMG
// Hierarchy fixed per mesh: greedy strength-0.25 aggregation (LinearSolver.hpp:535-575)
// of the geometric Laplacian area/delta with the cell-0 pin of the pressure system.
// The prolongation is smoothed (smoothed aggregation: P = (I - omega D_F^-1 F) P_tent,
// F the strength-filtered geometric matrix with weak entries lumped into its diagonal,
// omega = 0.85 / rho(D_F^-1 F)); the row-relative fallback and the standalone linear
// solves keep the piecewise-constant P_tent. Coarse values are Galerkin products
// P^T A P (:578-618 with P_tent) refreshed from the current level-0 values, damped
// Jacobi smoothing and an exact dense coarsest solve.
struct Csr {
    int n = 0;
    std::vector<int> ptr, col;
    Vec val, dg;
};

struct AmgLevel {
    Csr A;
    int nc = 0;
    std::vector<int> pPtr, pCol; // prolongation rows: fine row -> coarse rows ascending
    Vec pVal;
    // Galerkin terms in generation order: coarse nnz tC[t] += tW[t] * fine nnz tF[t]
    std::vector<int> tF, tC;
    Vec tW;
    std::vector<int> dpos;
};

struct Amg {
    std::vector<AmgLevel> lev;
    std::vector<int> upPos, loPos; // LDU face -> level-0 nnz
    Vec inv;                        // dense inverse of the coarsest level (row major)
    // coarse values are re-summed only when the previous solve degraded, the rule
    // AMGSolver applies to its aggregation (LinearSolver.hpp:924-941), a stop on the
    // |p.Ap| < 1e-30 guard not counting as degradation
    bool needRefresh = true;
    int itersAfterRefresh = -1;
    // smoother weight, coarse-correction scale and sweeps before / after the coarse
    // correction: the smoothed-aggregation pressure hierarchy uses 0.6, 1 and 1; the
    // fallback and the standalone linear solves 0.75, 1.7 and 2 (over-correction of
    // the piecewise-constant prolongation)
    double w = 0.6, alpha = 1.0;
    int sweeps = 1;
    int levels() const { return static_cast<int>(lev.size()); }
};

// coarsening stops at this many rows: the reference stops at 50 (LinearSolver.hpp:664);
// the pressure hierarchy at 96 (a dense inverse of up to 96 rows is cheaper than the
// level below it), the standalone linear solves at 32
static const int AMG_MIN_COARSE = 96;
static const int AMG_MIN_COARSE_LINEAR = 32;
static const int AMG_MAX_LEVELS = 20;  // :663
static const double AMG_PROLONG_WEIGHT = 0.85;

static Csr lduCsr(int n, const std::vector<int> &own, const std::vector<int> &nbr, int nf,
                  const Vec &d, const Vec &up, const Vec &lo, std::vector<int> *upPos,
                  std::vector<int> *loPos) {
    // rows sorted by column, diagonal included (LinearSolver.hpp:472-532)
    std::vector<std::vector<std::pair<int, int>>> rows(n); // (col, source id)
    for (int i = 0; i < n; ++i)
        rows[i].push_back({i, -1});
    for (int f = 0; f < nf; ++f) {
        rows[own[f]].push_back({nbr[f], 2 * f});
        rows[nbr[f]].push_back({own[f], 2 * f + 1});
    }
    Csr A;
    A.n = n;
    A.ptr.assign(n + 1, 0);
    A.dg.assign(n, 0.0);
    if (upPos) {
        upPos->assign(nf, -1);
        loPos->assign(nf, -1);
    }
    for (int i = 0; i < n; ++i) {
        std::stable_sort(rows[i].begin(), rows[i].end(),
                         [](auto &a, auto &b) { return a.first < b.first; });
        A.ptr[i + 1] = A.ptr[i] + static_cast<int>(rows[i].size());
        for (auto &e : rows[i]) {
            const int k = static_cast<int>(A.col.size());
            A.col.push_back(e.first);
            double v;
            if (e.second < 0) {
                v = d[i];
                A.dg[i] = v;
            } else if (e.second % 2 == 0) {
                v = up[e.second / 2];
                if (upPos)
                    (*upPos)[e.second / 2] = k;
            } else {
                v = lo[e.second / 2];
                if (loPos)
                    (*loPos)[e.second / 2] = k;
            }
            A.val.push_back(v);
        }
    }
    return A;
}

static int csrFind(const Csr &A, int r, int c) {
    for (int k = A.ptr[r]; k < A.ptr[r + 1]; ++k)
        if (A.col[k] == c)
            return k;
    return -1;
}

static void aggregate(const Csr &A, std::vector<int> &map, int &nc) {
    const int n = A.n;
    map.assign(n, -1);
    nc = 0;
    for (int i = 0; i < n; ++i) { // seeds claim unaggregated strong neighbours
        if (map[i] >= 0)
            continue;
        const int g = nc++;
        map[i] = g;
        const double aii = std::abs(A.dg[i]);
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int c = A.col[k];
            if (c == i || map[c] >= 0)
                continue;
            const double ajj = std::abs(A.dg[c]);
            if (std::abs(A.val[k]) / std::sqrt(aii * ajj + 1e-30) > 0.25)
                map[c] = g;
        }
    }
    for (int i = 0; i < n; ++i) { // orphans join the strongest aggregated neighbour
        if (map[i] >= 0)
            continue;
        double best = -1.0;
        int bestAgg = 0;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int c = A.col[k];
            if (c == i && map[c] < 0)
                continue;
            if (map[c] >= 0 && std::abs(A.val[k]) > best) {
                best = std::abs(A.val[k]);
                bestAgg = map[c];
            }
        }
        map[i] = bestAgg;
    }
}

// Aggregation of the standalone linear systems on the device (the product's
// rq_linsys.cpp): the reference's greedy pass (LinearSolver.hpp:535-575) with
// row-relative strength |a_ij| >= 0.25 max_k |a_ik|, singleton seeds merged
// into their strongest neighbour's aggregate, ids renumbered by first use.
static void aggregateLinear(const Csr &A, std::vector<int> &map, int &nc) {
    const int n = A.n;
    map.assign(n, -1);
    int groups = 0;
    for (int i = 0; i < n; ++i) {
        if (map[i] >= 0)
            continue;
        const int g = groups++;
        map[i] = g;
        double rowMax = 0.0;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (A.col[k] != i)
                rowMax = std::max(rowMax, std::abs(A.val[k]));
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int c = A.col[k];
            if (c != i && map[c] < 0 && rowMax > 0.0 && std::abs(A.val[k]) >= 0.25 * rowMax)
                map[c] = g;
        }
    }
    std::vector<int> count(groups, 0);
    for (int i = 0; i < n; ++i)
        ++count[map[i]];
    for (int i = 0; i < n; ++i) {
        if (count[map[i]] != 1)
            continue;
        double best = 0.0;
        int j = -1;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (A.col[k] != i && std::abs(A.val[k]) > best) {
                best = std::abs(A.val[k]);
                j = A.col[k];
            }
        if (j < 0)
            continue;
        --count[map[i]];
        map[i] = map[j];
        ++count[map[j]];
    }
    std::vector<int> id(groups, -1);
    nc = 0;
    for (int i = 0; i < n; ++i) {
        if (id[map[i]] < 0)
            id[map[i]] = nc++;
        map[i] = id[map[i]];
    }
}

// P of one level: smoothed (weight > 0) or piecewise constant (weight 0), rows with
// their coarse columns ascending and exact zeros dropped.
static void prolongation(const Csr &A, const std::vector<int> &agg, double weight,
                         AmgLevel &fine) {
    const int n = A.n;
    auto strongAt = [&](int i, int k) {
        const int c = A.col[k];
        return c != i &&
               std::abs(A.val[k]) / std::sqrt(std::abs(A.dg[i]) * std::abs(A.dg[c]) + 1e-30) > 0.25;
    };
    Vec fd(n);
    for (int i = 0; i < n; ++i) {
        double d = A.dg[i];
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (A.col[k] != i && !strongAt(i, k))
                d += A.val[k];
        fd[i] = d;
    }
    auto usable = [&](int i) { return std::abs(fd[i]) > 1e-12 * std::abs(A.dg[i]); };
    double omega = 0.0;
    if (weight > 0.0) { // rho(D_F^-1 F) by 100 power iterations from a fixed start
        Vec x(n), y(n);
        for (int i = 0; i < n; ++i)
            x[i] = 1.0 + 0.1 * (i % 7);
        double rho = 0.0;
        for (int it = 0; it < 100; ++it) {
            double ny = 0.0, nx = 0.0;
            for (int i = 0; i < n; ++i) {
                double v = 0.0;
                if (usable(i)) {
                    v = fd[i] * x[i];
                    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                        if (strongAt(i, k))
                            v += A.val[k] * x[A.col[k]];
                    v /= fd[i];
                }
                y[i] = v;
                ny += v * v;
                nx += x[i] * x[i];
            }
            rho = std::sqrt(ny / std::max(nx, 1e-300));
            const double inv = 1.0 / std::max(std::sqrt(ny), 1e-300);
            for (int i = 0; i < n; ++i)
                x[i] = y[i] * inv;
        }
        omega = rho > 0.0 ? weight / rho : 0.0;
    }
    fine.pPtr.assign(n + 1, 0);
    fine.pCol.clear();
    fine.pVal.clear();
    for (int i = 0; i < n; ++i) {
        std::map<int, double> row;
        row[agg[i]] += 1.0;
        if (omega > 0.0 && usable(i)) {
            const double sc = omega / fd[i];
            row[agg[i]] -= sc * fd[i];
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if (strongAt(i, k))
                    row[agg[A.col[k]]] -= sc * A.val[k];
        }
        for (auto &e : row)
            if (e.second != 0.0) {
                fine.pCol.push_back(e.first);
                fine.pVal.push_back(e.second);
            }
        fine.pPtr[i + 1] = static_cast<int>(fine.pCol.size());
    }
}

// The coarse level of `fine` under its P: the pattern of P^T A P and the Galerkin terms
// in generation order (fine rows ascending, each row's entries in column order, then
// P's entries of the row and of the column), then the values from the fine values.
static void galerkinLevel(AmgLevel &fine, AmgLevel &coarse) {
    const Csr &A = fine.A;
    const int nc = fine.nc;
    std::vector<std::map<int, int>> rows(nc);
    for (int i = 0; i < A.n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int j = A.col[k];
            for (int a = fine.pPtr[i]; a < fine.pPtr[i + 1]; ++a)
                for (int b = fine.pPtr[j]; b < fine.pPtr[j + 1]; ++b)
                    rows[fine.pCol[a]][fine.pCol[b]] = 0;
        }
    Csr &C = coarse.A;
    C = Csr{};
    C.n = nc;
    C.ptr.assign(nc + 1, 0);
    C.dg.assign(nc, 0.0);
    for (int I = 0; I < nc; ++I) {
        C.ptr[I + 1] = C.ptr[I] + static_cast<int>(rows[I].size());
        for (auto &e : rows[I]) {
            e.second = static_cast<int>(C.col.size());
            C.col.push_back(e.first);
            C.val.push_back(0.0);
        }
    }
    fine.tF.clear();
    fine.tC.clear();
    fine.tW.clear();
    for (int i = 0; i < A.n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int j = A.col[k];
            for (int a = fine.pPtr[i]; a < fine.pPtr[i + 1]; ++a)
                for (int b = fine.pPtr[j]; b < fine.pPtr[j + 1]; ++b) {
                    fine.tF.push_back(k);
                    fine.tC.push_back(rows[fine.pCol[a]][fine.pCol[b]]);
                    fine.tW.push_back(fine.pVal[a] * fine.pVal[b]);
                }
        }
    coarse.dpos.resize(nc);
    for (int I = 0; I < nc; ++I)
        coarse.dpos[I] = csrFind(C, I, I);
}

static void sumCoarse(const AmgLevel &fine, AmgLevel &coarse) {
    std::fill(coarse.A.val.begin(), coarse.A.val.end(), 0.0);
    for (size_t t = 0; t < fine.tF.size(); ++t)
        coarse.A.val[fine.tC[t]] += fine.tW[t] * fine.A.val[fine.tF[t]];
    for (int I = 0; I < coarse.A.n; ++I)
        coarse.A.dg[I] = coarse.A.val[coarse.dpos[I]];
}

// Exact inverse of the small SPD coarsest matrix by Gauss-Jordan elimination.
static void denseInverse(const Csr &A, Vec &inv) {
    const int n = A.n;
    Vec a(static_cast<size_t>(n) * n, 0.0);
    inv.assign(static_cast<size_t>(n) * n, 0.0);
    for (int i = 0; i < n; ++i) {
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            a[static_cast<size_t>(i) * n + A.col[k]] = A.val[k];
        inv[static_cast<size_t>(i) * n + i] = 1.0;
    }
    for (int k = 0; k < n; ++k) {
        const double piv = a[static_cast<size_t>(k) * n + k];
        const double rp = 1.0 / piv;
        for (int j = 0; j < n; ++j) {
            a[static_cast<size_t>(k) * n + j] *= rp;
            inv[static_cast<size_t>(k) * n + j] *= rp;
        }
        for (int i = 0; i < n; ++i) {
            if (i == k)
                continue;
            const double f = a[static_cast<size_t>(i) * n + k];
            if (f == 0.0)
                continue;
            for (int j = 0; j < n; ++j) {
                a[static_cast<size_t>(i) * n + j] -= f * a[static_cast<size_t>(k) * n + j];
                inv[static_cast<size_t>(i) * n + j] -= f * inv[static_cast<size_t>(k) * n + j];
            }
        }
    }
}

// Geometric hierarchy of one mesh (the GPU host setup restates the same steps).
static Amg buildAmg(const Mesh &m) {
    Amg h;
    Vec d(m.nC, 0.0), up(m.nI), lo(m.nI);
    for (int f = 0; f < m.nI; ++f) {
        const double c = m.area[f] / std::max(m.delta[f], 1e-20);
        d[m.own[f]] += c;
        d[m.nbr[f]] += c;
        up[f] = lo[f] = -c;
    }
    d[0] += d[0];
    // the reference's aggregation first; if it stalls above AMG_MIN_COARSE rows
    // (strongly varying aspect ratios), the row-relative rule of aggregateLinear
    for (int attempt = 0; attempt < 2; ++attempt) {
    h = Amg{};
    AmgLevel l0;
    l0.A = lduCsr(m.nC, m.own, m.nbr, m.nI, d, up, lo, &h.upPos, &h.loPos);
    l0.dpos.resize(m.nC);
    for (int i = 0; i < m.nC; ++i)
        l0.dpos[i] = csrFind(l0.A, i, i);
    h.lev.push_back(std::move(l0));
    for (int l = 0; l < AMG_MAX_LEVELS; ++l) {
        AmgLevel &fine = h.lev[l];
        if (fine.A.n <= AMG_MIN_COARSE)
            break;
        std::vector<int> map;
        int nc = 0;
        if (attempt == 0)
            aggregate(fine.A, map, nc);
        else
            aggregateLinear(fine.A, map, nc);
        if (nc == 0 || nc >= fine.A.n)
            break;
        AmgLevel coarse;
        fine.nc = nc;
        prolongation(fine.A, map, attempt == 0 ? AMG_PROLONG_WEIGHT : 0.0, fine);
        galerkinLevel(fine, coarse);
        sumCoarse(fine, coarse);
        h.lev.push_back(std::move(coarse));
    }
    if (attempt == 1) { // the fallback hierarchy over-corrects (as the linear solves)
        h.w = 0.75;
        h.alpha = 1.7;
        h.sweeps = 2;
    }
    if (h.lev.back().A.n <= AMG_MIN_COARSE)
        break;
    }
    return h;
}

static void amgLevel0(Amg &h, const Ldu &A) {
    AmgLevel &l0 = h.lev[0];
    for (int i = 0; i < A.n; ++i) {
        l0.A.val[l0.dpos[i]] = A.d[i];
        l0.A.dg[i] = A.d[i];
    }
    for (int f = 0; f < A.nf; ++f) {
        l0.A.val[h.upPos[f]] = A.up[f];
        l0.A.val[h.loPos[f]] = A.lo[f];
    }
}

static void amgCoarse(Amg &h) {
    for (int l = 0; l + 1 < h.levels(); ++l)
        sumCoarse(h.lev[l], h.lev[l + 1]);
    denseInverse(h.lev.back().A, h.inv);
}

static void csrResidual(const Csr &A, const Vec &x, const Vec &b, Vec &r) {
    for (int i = 0; i < A.n; ++i) {
        double s = 0.0;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            s += A.val[k] * x[A.col[k]];
        r[i] = b[i] - s;
    }
}

// One V-cycle z = M^-1 r: pre-smoothing from zero (h.sweeps damped-Jacobi sweeps),
// restriction by P^T, prolongation x + alpha P x_c, the same post-smoothing (symmetric).
static void vcycle(const Amg &h, int l, const Vec &b, Vec &x) {
    const Csr &A = h.lev[l].A;
    const int n = A.n;
    if (l == h.levels() - 1) {
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int j = 0; j < n; ++j)
                s += h.inv[static_cast<size_t>(i) * n + j] * b[j];
            x[i] = s;
        }
        return;
    }
    Vec r(n);
    for (int i = 0; i < n; ++i)
        x[i] = h.w * b[i] / A.dg[i];
    for (int s = 1; s < h.sweeps; ++s) {
        csrResidual(A, x, b, r);
        for (int i = 0; i < n; ++i)
            x[i] += h.w * r[i] / A.dg[i];
    }
    csrResidual(A, x, b, r);
    const AmgLevel &fl = h.lev[l];
    Vec bc(fl.nc, 0.0), xc(fl.nc, 0.0);
    for (int i = 0; i < n; ++i)
        for (int a = fl.pPtr[i]; a < fl.pPtr[i + 1]; ++a)
            bc[fl.pCol[a]] += fl.pVal[a] * r[i];
    vcycle(h, l + 1, bc, xc);
    for (int i = 0; i < n; ++i) {
        double pc = 0.0;
        for (int a = fl.pPtr[i]; a < fl.pPtr[i + 1]; ++a)
            pc += fl.pVal[a] * xc[fl.pCol[a]];
        x[i] += h.alpha * pc;
    }
    for (int s = 0; s < h.sweeps; ++s) {
        csrResidual(A, x, b, r);
        for (int i = 0; i < n; ++i)
            x[i] += h.w * r[i] / A.dg[i];
    }
}

// PCG with the Jacobi (amg == nullptr) or AMG preconditioner: the reference's
// PCG loop (LinearSolver.hpp:184-246 and :908-982 share it).
static LinResult pcgBody(const Ldu &A, Vec &x, int maxIter, double tol, Amg *amg);
static LinResult pcg(const Ldu &A, Vec &x, int maxIter, double tol, Amg *amg) {
    const int n = A.n;
    bool refreshed = false;
    if (amg) {
        amgLevel0(*amg, A);
        Vec r0(n);
        A.residual(x, r0);
        if (norm2(r0) < 1e-30) // solved at once: no preconditioner and no refresh bookkeeping
            return pcgBody(A, x, maxIter, tol, amg);
        if (amg->needRefresh) {
            amgCoarse(*amg);
            amg->needRefresh = false;
            refreshed = true;
        }
    }
    (void)n;
    LinResult res = pcgBody(A, x, maxIter, tol, amg);
    if (amg) {
        if (refreshed || amg->itersAfterRefresh <= 0)
            amg->itersAfterRefresh = res.iterations;
        else if ((!res.converged && !res.breakdown) ||
                 res.iterations > 1.5 * amg->itersAfterRefresh + 2)
            amg->needRefresh = true;
    }
    return res;
}

static LinResult pcgBody(const Ldu &A, Vec &x, int maxIter, double tol, Amg *amg) {
    const int n = A.n;
    Vec r(n), z(n), p(n), Ap(n);
    LinResult res;
    A.residual(x, r);
    const double r0 = norm2(r);
    res.initialRes = r0;
    if (r0 < 1e-30) {
        res.converged = true;
        return res;
    }
    auto precond = [&](const Vec &rr, Vec &zz) {
        if (amg)
            vcycle(*amg, 0, rr, zz);
        else
            jacobi(A, rr, zz);
    };
    precond(r, z);
    p = z;
    double rz = dot(r, z);
    for (int it = 0; it < maxIter; ++it) {
        A.matvec(p, Ap);
        const double pAp = dot(p, Ap);
        if (std::abs(pAp) < 1e-30) {
            res.breakdown = true;
            break;
        }
        const double alpha = rz / pAp;
        for (int i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
        }
        const double rn = norm2(r);
        res.iterations = it + 1;
        res.finalRes = rn / r0;
        if (res.finalRes < tol) {
            res.converged = true;
            return res;
        }
        precond(r, z);
        const double rzNew = dot(r, z);
        const double beta = rzNew / (rz + 1e-30);
        for (int i = 0; i < n; ++i)
            p[i] = z[i] + beta * p[i];
        rz = rzNew;
    }
    return res;
}

// ---------------------------------------------------------------- SST closure
// SSTCoefficients (core/include/SSTModel.hpp:12-61) in InferenceParameterSet order.
struct Coef {
    double sk1, sw1, b1, a1c, sk2, sw2, b2, a2c, bs, a1, kap;
    explicit Coef(const double *c)
        : sk1(c[0]), sw1(c[1]), b1(c[2]), a1c(c[3]), sk2(c[4]), sw2(c[5]), b2(c[6]), a2c(c[7]),
          bs(c[8]), a1(c[9]), kap(c[10]) {}
    static double blend(double p1, double p2, double F1) { return F1 * p1 + (1.0 - F1) * p2; }
    double sigK(double F1) const { return blend(sk1, sk2, F1); }
    double sigW(double F1) const { return blend(sw1, sw2, F1); }
    double beta(double F1) const { return blend(b1, b2, F1); }
    double alpha(double F1) const { return blend(a1c, a2c, F1); }
};

// Field state: cell values plus boundary-face values (Field.hpp:21-163).
struct State {
    Vec Ux, Uy, Uz, p, k, w, nuT, F1, F2, Pk, CD;
    Vec bUx, bUy, bp, bk, bw; // boundary faces (all walls on periodic meshes)
    bool established = false;
};

// Green-Gauss gradient (Field.hpp:178-212): x and y components (normals have no z).
static void ggrad(const Mesh &m, const Vec &phi, const Vec &bphi, Vec &gx, Vec &gy) {
    gx.assign(m.nC, 0.0);
    gy.assign(m.nC, 0.0);
    for (int f = 0; f < m.nI; ++f) {
        const int o = m.own[f], q = m.nbr[f];
        const double pf = phi[o] * m.w[f] + phi[q] * (1.0 - m.w[f]);
        const double sx = m.fnx[f] * m.area[f], sy = m.fny[f] * m.area[f];
        gx[o] = gx[o] + sx * pf;
        gy[o] = gy[o] + sy * pf;
        gx[q] = gx[q] - sx * pf;
        gy[q] = gy[q] - sy * pf;
    }
    for (int f = m.nI; f < m.nF; ++f) {
        const int o = m.own[f];
        const double sx = m.fnx[f] * m.area[f], sy = m.fny[f] * m.area[f];
        gx[o] = gx[o] + sx * bphi[f - m.nI];
        gy[o] = gy[o] + sy * bphi[f - m.nI];
    }
    for (int c = 0; c < m.nC; ++c)
        if (m.vol[c] > 1e-30) {
            gx[c] = gx[c] / m.vol[c];
            gy[c] = gy[c] / m.vol[c];
        }
}

// SSTModel::computeFields (core/src/SSTModel.cpp:157-241) with the pointwise
// F1 (:15-33), F2 (:37-52), cross diffusion (:55-59), eddy viscosity (:66-75)
// and production (:80-85). Returns |S| (Field.hpp:387-414) in S.
static void closure(const Mesh &m, const Coef &cf, double nu, State &s, Vec &S) {
    Vec uxx, uxy, uyx, uyy, kx, ky, wx, wy;
    ggrad(m, s.Ux, s.bUx, uxx, uxy);
    ggrad(m, s.Uy, s.bUy, uyx, uyy);
    ggrad(m, s.k, s.bk, kx, ky);
    ggrad(m, s.w, s.bw, wx, wy);
    S.assign(m.nC, 0.0);
    for (int c = 0; c < m.nC; ++c) {
        const double s11 = uxx[c], s22 = uyy[c], s33 = 0.0;
        const double s12 = 0.5 * (uxy[c] + uyx[c]), s13 = 0.5 * (0.0 + 0.0),
                     s23 = 0.5 * (0.0 + 0.0);
        S[c] = std::sqrt(2.0 * (s11 * s11 + s22 * s22 + s33 * s33 +
                                2.0 * (s12 * s12 + s13 * s13 + s23 * s23)));
    }
    for (int c = 0; c < m.nC; ++c) {
        const double kc = std::max(s.k[c], 0.0), wc = std::max(s.w[c], 1e-20);
        const double y = std::max(m.wd[c], 1e-20), Sc = S[c];
        const double cd = 2.0 * cf.sw2 / std::max(wc, 1e-20) * (kx[c] * wx[c] + ky[c] * wy[c]);
        s.CD[c] = cd;
        // F1
        {
            const double sqk = std::sqrt(std::max(kc, 0.0)), ws = std::max(wc, 1e-20);
            const double ys = std::max(y, 1e-20), y2 = ys * ys;
            const double t1 = sqk / (cf.bs * ws * ys);
            const double t2 = 500.0 * nu / (y2 * ws);
            const double cdp = std::max(cd, 1e-10);
            const double t3 = 4.0 * cf.sw2 * std::max(kc, 0.0) / (cdp * y2);
            const double a = std::min(std::max(t1, t2), t3);
            s.F1[c] = std::tanh(a * a * a * a);
        }
        // F2
        {
            const double sqk = std::sqrt(std::max(kc, 0.0)), ws = std::max(wc, 1e-20);
            const double ys = std::max(y, 1e-20), y2 = ys * ys;
            const double t1 = 2.0 * sqk / (cf.bs * ws * ys);
            const double t2 = 500.0 * nu / (y2 * ws);
            const double a = std::max(t1, t2);
            s.F2[c] = std::tanh(a * a);
        }
        double den = std::max(cf.a1 * wc, Sc * s.F2[c]);
        den = std::max(den, 1e-20);
        s.nuT[c] = cf.a1 * std::max(kc, 0.0) / den;
        const double raw = s.nuT[c] * Sc * Sc;
        const double lim = 10.0 * cf.bs * std::max(kc, 0.0) * std::max(wc, 1e-20);
        s.Pk[c] = std::min(raw, lim);
    }
}

// ---------------------------------------------------------------- solver
struct Settings {
    int maxIter, innerIter, window, monitorInterval, turbStart, floorIters, pSolver;
    double tol, innerTol, aU, aP, aK, aW, fx, fy, divLimit, kMin, kMax, wMin;
};

// Least-squares probe stencil of PreparedObservation (ObservationOperator.hpp:630-670)
// with the containing-cell walk (:290-323) and nearest cell (:272-284).
struct Probe {
    int cell = -1;
    double ox = 0, oy = 0, axx = 0, axy = 0, ayy = 0, det = 0;
    std::vector<int> nc, nf;
    Vec dx, dy, wt;
};

static int nearestCell(const Mesh &m, double x, double y) {
    int best = 0;
    double bd = 1e30;
    for (int c = 0; c < m.nC; ++c) {
        const double dx = m.cx[c] - x, dy = m.cy[c] - y;
        const double d = dx * dx + dy * dy;
        if (d < bd) {
            bd = d;
            best = c;
        }
    }
    return best;
}

static Probe prepareProbe(const Mesh &m, double x, double y) {
    int c = nearestCell(m, x, y);
    double lx = x, ly = y;
    const int maxSteps = 2 * m.nC + 10;
    bool inside = false;
    for (int step = 0; step < maxSteps && !inside; ++step) {
        double worst = 0.0;
        int cross = -1;
        for (int f : m.cellFaces[c]) {
            const bool ow = m.own[f] == c;
            const double nx = ow ? m.fnx[f] : m.fnx[f] * -1.0, ny = ow ? m.fny[f] : m.fny[f] * -1.0;
            const double cx = ow ? m.fcx[f] : m.fcx[f] - m.shx[f], cy = m.fcy[f];
            const double out = (lx - cx) * nx + (ly - cy) * ny;
            if (out > worst + 1e-12 * std::sqrt(m.area[f])) {
                worst = out;
                cross = f;
            }
        }
        if (cross < 0 || m.nbr[cross] < 0) {
            inside = true;
            break;
        }
        const bool ow = m.own[cross] == c;
        lx = ow ? lx - m.shx[cross] : lx + m.shx[cross];
        c = ow ? m.nbr[cross] : m.own[cross];
    }
    if (!inside) {
        c = nearestCell(m, x, y);
        lx = x;
        ly = y;
    }
    Probe p;
    p.cell = c;
    p.ox = lx - m.cx[c];
    p.oy = ly - m.cy[c];
    for (int f : m.cellFaces[c]) {
        double dx, dy;
        int nb = -1;
        if (m.nbr[f] < 0) {
            dx = m.fcx[f] - m.cx[c];
            dy = m.fcy[f] - m.cy[c];
        } else {
            const bool ow = m.own[f] == c;
            nb = ow ? m.nbr[f] : m.own[f];
            dx = ow ? m.cx[nb] + m.shx[f] - m.cx[c] : m.cx[nb] - m.shx[f] - m.cx[c];
            dy = m.cy[nb] - m.cy[c];
        }
        const double wt = 1.0 / std::max(dx * dx + dy * dy, 1e-300);
        p.axx += wt * dx * dx;
        p.axy += wt * dx * dy;
        p.ayy += wt * dy * dy;
        p.nc.push_back(nb);
        p.nf.push_back(f);
        p.dx.push_back(dx);
        p.dy.push_back(dy);
        p.wt.push_back(wt);
    }
    p.det = p.axx * p.ayy - p.axy * p.axy;
    return p;
}

static double evalProbe(const Mesh &m, const Probe &p, const Vec &v, const Vec &bv) {
    const double center = v[p.cell];
    double bx = 0, by = 0;
    for (size_t i = 0; i < p.nc.size(); ++i) {
        const double diff = (p.nc[i] < 0 ? bv[p.nf[i] - m.nI] : v[p.nc[i]]) - center;
        bx += p.wt[i] * p.dx[i] * diff;
        by += p.wt[i] * p.dy[i] * diff;
    }
    double gx = 0, gy = 0;
    if (std::abs(p.det) > 1e-14 * (p.axx * p.ayy + 1e-300)) {
        gx = (p.ayy * bx - p.axy * by) / p.det;
        gy = (p.axx * by - p.axy * bx) / p.det;
    }
    return center + gx * p.ox + gy * p.oy;
}

// ContractionEstimate (rans-uq/src/SIMPLESolver.cpp:32-74)
struct Contraction {
    int m;
    Vec h;
    explicit Contraction(int window) : m(std::max(window, 2)) {}
    void push(double d) { h.push_back(d); }
    double last() const { return h.empty() ? INF : h.back(); }
    double rate() const {
        const size_t n = h.size(), mm = static_cast<size_t>(m);
        if (n < 2 * mm)
            return std::numeric_limits<double>::quiet_NaN();
        double dn = 0.0, dd = 0.0;
        for (size_t i = n - mm; i < n; ++i)
            dn = std::max(dn, h[i]);
        for (size_t i = n - 2 * mm; i < n - mm; ++i)
            dd = std::max(dd, h[i]);
        if (dd <= 0.0)
            return dn > 0.0 ? INF : 0.0;
        return std::pow(dn / dd, 1.0 / m);
    }
    double remaining(double negligible) const {
        const size_t n = h.size(), mm = static_cast<size_t>(m);
        if (n < 2 * mm)
            return INF;
        double dn = 0.0;
        for (size_t i = n - mm; i < n; ++i)
            dn = std::max(dn, h[i]);
        if (dn <= negligible)
            return dn;
        const double r = rate();
        if (!(r < 1.0))
            return INF;
        return dn * r / (1.0 - r);
    }
};

struct History {
    bool converged = false, diverged = false, stalled = false;
    int finalIter = 0;
    double worst = 0, rate = 0;
    std::vector<std::array<double, ORC_NHIST>> entries;
};

class Solver {
  public:
    const Mesh &m;
    Coef cf;
    double nu;
    Settings st;
    std::vector<Probe> probes;
    Vec floors;
    Amg amg;
    bool useAmg = false;
    // planar singular omega balance (SIMPLESolver.cpp:92-153)
    Vec sing, sgrad, slap;

    Solver(const Mesh &mesh, const double *coeffs, double nu_, const Settings &s)
        : m(mesh), cf(coeffs), nu(nu_), st(s) {
        prepareBalance();
        if (st.pSolver == ORC_P_AMG) {
            amg = buildAmg(m);
            useAmg = true;
        }
    }

    void prepareBalance() {
        if (m.nF == m.nI)
            return;
        const int f0 = m.nI;
        const double ix = m.fnx[f0] * -1.0, iy = m.fny[f0] * -1.0;
        const double origin = m.fcx[f0] * ix + m.fcy[f0] * iy;
        double height = 0;
        bool periodic = false;
        for (int f = m.nI; f < m.nF; ++f) {
            if (std::abs(std::abs(m.fnx[f] * ix + m.fny[f] * iy) - 1.0) > 1e-12)
                return;
            height = std::max(height, m.fcx[f] * ix + m.fcy[f] * iy - origin);
        }
        if (!(height > 0))
            return;
        const double tolr = 1e-12 * height;
        for (int f = 0; f < m.nF; ++f) {
            const double ex = m.ddx[f] - m.fnx[f] * m.delta[f], ey = m.ddy[f] - m.fny[f] * m.delta[f];
            if (std::sqrt(ex * ex + ey * ey) > 1e-9 * m.delta[f] ||
                std::abs(m.shx[f] * ix) > tolr)
                return;
            periodic = periodic || m.shx[f] * m.shx[f] > 0;
            if (m.nbr[f] < 0) {
                const double y = m.fcx[f] * ix + m.fcy[f] * iy - origin;
                if (std::min(std::abs(y), std::abs(y - height)) > tolr)
                    return;
                if ((y < height / 2 ? -1.0 : 1.0) * (m.fnx[f] * ix + m.fny[f] * iy) < 1 - 1e-12)
                    return;
            }
        }
        if (!periodic)
            return;
        Vec s(m.nC), lap(m.nC), g(m.nI);
        for (int c = 0; c < m.nC; ++c) {
            const double y = m.cx[c] * ix + m.cy[c] * iy - origin;
            if (!(y > 0 && y < height))
                return;
            s[c] = 1 / (y * y) + 1 / ((height - y) * (height - y));
            lap[c] = 6 * (std::pow(y, -4) + std::pow(height - y, -4));
        }
        for (int f = 0; f < m.nI; ++f) {
            const double y = m.fcx[f] * ix + m.fcy[f] * iy - origin;
            if (!(y > 0 && y < height))
                return;
            g[f] = 2 * (std::pow(height - y, -3) - std::pow(y, -3)) * (m.fnx[f] * ix + m.fny[f] * iy);
        }
        sing = std::move(s);
        sgrad = std::move(g);
        slap = std::move(lap);
    }

    double wallOmega(double y) const { // resolvedWallOmega (:155-161)
        const double coefficient = sing.empty() ? 60.0 : 6.0;
        return coefficient * nu / (cf.b1 * y * y);
    }

    // BC applicators (BoundaryCondition.hpp:279-384): every boundary face is a
    // no-slip k-omega wall on the periodic meshes.
    void bcU(State &s) const {
        for (int f = m.nI; f < m.nF; ++f) {
            s.bUx[f - m.nI] = 0;
            s.bUy[f - m.nI] = 0;
        }
    }
    void bcP(State &s) const {
        for (int f = m.nI; f < m.nF; ++f)
            s.bp[f - m.nI] = s.p[m.own[f]];
    }
    void bcK(State &s) const {
        for (int f = m.nI; f < m.nF; ++f)
            s.bk[f - m.nI] = 0.0;
    }
    void bcW(State &s, double beta1) const {
        for (int f = m.nI; f < m.nF; ++f) {
            const double y1 = std::max(m.delta[f], 1e-20);
            s.bw[f - m.nI] = 60.0 * nu / (beta1 * y1 * y1);
        }
    }

    // initUniform (:267-298)
    void init(State &s, const double *U0, double p0, double k0, double w0) const {
        const int n = m.nC, nb = m.nB();
        s.Ux.assign(n, U0[0]);
        s.Uy.assign(n, U0[1]);
        s.Uz.assign(n, U0[2]);
        s.bUx.assign(nb, U0[0]);
        s.bUy.assign(nb, U0[1]);
        s.p.assign(n, p0);
        s.bp.assign(nb, p0);
        s.k.assign(n, k0);
        s.bk.assign(nb, k0);
        s.w.assign(n, w0);
        s.bw.assign(nb, w0);
        s.F1.assign(n, 1.0);
        s.F2.assign(n, 1.0);
        s.Pk.assign(n, 0.0);
        s.CD.assign(n, 0.0);
        s.nuT.assign(n, 0.0);
        s.established = false;
        for (int c = 0; c < n; ++c)
            s.w[c] = std::max(wallOmega(std::max(m.wd[c], 1e-20)), w0);
        for (int c = 0; c < n; ++c)
            s.nuT[c] = cf.a1 * k0 / std::max(cf.a1 * s.w[c], 1e-20);
        bcU(s);
        bcP(s);
        bcK(s);
        bcW(s, 0.075); // applyAllBCs uses applyOmegaBC's default beta1
    }

    // limitedLinearUpwind deferred correction (:495-532)
    void convectionCorrection(Ldu &A, const Vec &phiF, const Vec &v, const Vec &bv) const {
        Vec gx, gy;
        ggrad(m, v, bv, gx, gy);
        for (int f = 0; f < m.nI; ++f) {
            const double F = phiF[f];
            if (F == 0.0)
                continue;
            const int o = m.own[f], q = m.nbr[f];
            const bool ownerUp = F > 0.0;
            const int up = ownerUp ? o : q, dn = ownerUp ? q : o;
            const double xUx = m.cx[up], xUy = m.cy[up];
            const double xDx = ownerUp ? m.cx[q] + m.shx[f] : m.cx[o] - m.shx[f];
            const double xDy = ownerUp ? m.cy[q] + 0.0 : m.cy[o] - 0.0;
            const double dphi = v[dn] - v[up];
            double psi = 0.0;
            if (std::abs(dphi) > 1e-300) {
                const double r =
                    2.0 * (gx[up] * (xDx - xUx) + gy[up] * (xDy - xUy)) / dphi - 1.0;
                psi = r > 0.0 ? (r * r + r) / (r * r + 1.0) : 0.0;
            }
            const double pf = v[up] + 0.5 * psi * dphi;
            const double corr = F * (pf - v[up]);
            A.b[o] -= corr;
            A.b[q] += corr;
        }
    }

    // assembleMomentum (:303-482) with transposeStressSource (StressOperators.hpp:31-81)
    void momentum(Ldu &A, const State &s, const Vec &phiF, int comp, Vec &aP, Vec &aPraw) const {
        A.zero();
        for (int f = 0; f < m.nI; ++f) {
            const int o = m.own[f], q = m.nbr[f];
            const double delta = std::max(m.delta[f], 1e-20);
            const double nuO = nu + s.nuT[o], nuN = nu + s.nuT[q];
            const double nuF = m.w[f] * nuO + (1.0 - m.w[f]) * nuN;
            const double D = nuF * m.area[f] / delta;
            const double F = phiF[f];
            const double cp = std::max(F, 0.0), cn = std::max(-F, 0.0);
            A.d[o] += D + cp;
            A.d[q] += D + cn;
            A.up[f] = -(D + cn);
            A.lo[f] = -(D + cp);
        }
        const Vec &bU = comp == 0 ? s.bUx : s.bUy;
        for (int f = m.nI; f < m.nF; ++f) { // walls: molecular viscosity only
            const int o = m.own[f];
            const double delta = std::max(m.delta[f], 1e-20);
            const double D = nu * m.area[f] / delta;
            const double Ub = bU[f - m.nI];
            const double F = phiF[f];
            if (F >= 0) {
                A.d[o] += F + D;
                A.b[o] += D * Ub;
            } else {
                A.d[o] += D;
                A.b[o] += (D - F) * Ub;
            }
        }
        Vec gpx, gpy;
        ggrad(m, s.p, s.bp, gpx, gpy);
        for (int c = 0; c < m.nC; ++c)
            A.b[c] -= (comp == 0 ? gpx[c] : gpy[c]) * m.vol[c];
        const double fb = comp == 0 ? st.fx : st.fy;
        if (fb != 0.0)
            for (int c = 0; c < m.nC; ++c)
                A.b[c] += fb * m.vol[c];
        // transpose stress: column comp of grad U interpolated to faces, wall faces zero
        {
            Vec uxx, uxy, uyx, uyy;
            ggrad(m, s.Ux, s.bUx, uxx, uxy);
            ggrad(m, s.Uy, s.bUy, uyx, uyy);
            const Vec &cX = comp == 0 ? uxx : uxy; // dUx/dx_comp
            const Vec &cY = comp == 0 ? uyx : uyy; // dUy/dx_comp
            Vec src(m.nC, 0.0);
            for (int f = 0; f < m.nI; ++f) {
                const int o = m.own[f], q = m.nbr[f];
                const double w = m.w[f];
                const double c = w * s.nuT[o] + (1.0 - w) * s.nuT[q];
                const double gxf = cX[o] * w + cX[q] * (1.0 - w);
                const double gyf = cY[o] * w + cY[q] * (1.0 - w);
                const double fl = c * (gxf * m.fnx[f] + gyf * m.fny[f]) * m.area[f];
                src[o] += fl;
                src[q] -= fl;
            }
            for (int f = m.nI; f < m.nF; ++f) {
                const int o = m.own[f];
                const double fl = 0.0 * (cX[o] * m.fnx[f] + cY[o] * m.fny[f]) * m.area[f];
                src[o] += fl;
            }
            for (int c = 0; c < m.nC; ++c)
                A.b[c] += src[c];
        }
        convectionCorrection(A, phiF, comp == 0 ? s.Ux : s.Uy, bU);
        const double a = st.aU;
        const Vec &U = comp == 0 ? s.Ux : s.Uy;
        for (int c = 0; c < m.nC; ++c) {
            aPraw[c] = A.d[c];
            A.b[c] += (1.0 - a) / a * A.d[c] * U[c];
            A.d[c] /= a;
            aP[c] = A.d[c];
        }
    }

    void interpFlux(const State &s, Vec &phi) const { // interpolatedFluxes (:870-884)
        phi.resize(m.nF);
        for (int f = 0; f < m.nI; ++f) {
            const int o = m.own[f], q = m.nbr[f];
            const double ux = s.Ux[o] * m.w[f] + s.Ux[q] * (1.0 - m.w[f]);
            const double uy = s.Uy[o] * m.w[f] + s.Uy[q] * (1.0 - m.w[f]);
            phi[f] = (ux * m.fnx[f] + uy * m.fny[f]) * m.area[f];
        }
        for (int f = m.nI; f < m.nF; ++f)
            phi[f] = (s.bUx[f - m.nI] * m.fnx[f] + s.bUy[f - m.nI] * m.fny[f]) * m.area[f];
    }

    void rhieChow(const State &s, const Vec &aP, Vec &phi) const { // addRhieChow (:891-906)
        Vec gx, gy;
        ggrad(m, s.p, s.bp, gx, gy);
        for (int f = 0; f < m.nI; ++f) {
            const int o = m.own[f], q = m.nbr[f];
            const double delta = std::max(m.delta[f], 1e-20);
            const double dO = (std::abs(aP[o]) > 1e-30) ? m.vol[o] / aP[o] : 0.0;
            const double dN = (std::abs(aP[q]) > 1e-30) ? m.vol[q] / aP[q] : 0.0;
            const double dF = m.w[f] * dO + (1.0 - m.w[f]) * dN;
            const double dl = std::max(m.delta[f], 1e-30);
            const double ex = m.ddx[f] / dl, ey = m.ddy[f] / dl;
            const double gbx = gx[o] * m.w[f] + gx[q] * (1.0 - m.w[f]);
            const double gby = gy[o] * m.w[f] + gy[q] * (1.0 - m.w[f]);
            phi[f] += -dF * m.area[f] * ((s.p[q] - s.p[o]) / delta - (gbx * ex + gby * ey));
        }
    }

    // assemblePressureCorrection with predicted fluxes (:717-830); no outlets here
    void pressure(Ldu &A, const Vec &aP, const Vec &pred, Vec &pCoeff, double &fluxScale) const {
        A.zero();
        fluxScale = 0.0;
        pCoeff.assign(m.nF, 0.0);
        for (int f = 0; f < m.nI; ++f) {
            const int o = m.own[f], q = m.nbr[f];
            const double delta = std::max(m.delta[f], 1e-20);
            const double dO = (std::abs(aP[o]) > 1e-30) ? m.vol[o] / aP[o] : 0.0;
            const double dN = (std::abs(aP[q]) > 1e-30) ? m.vol[q] / aP[q] : 0.0;
            const double dF = m.w[f] * dO + (1.0 - m.w[f]) * dN;
            const double c = dF * m.area[f] / delta;
            pCoeff[f] = c;
            A.d[o] += c;
            A.d[q] += c;
            A.up[f] = -c;
            A.lo[f] = -c;
            A.b[o] -= pred[f];
            A.b[q] += pred[f];
            fluxScale += std::abs(pred[f]);
        }
        for (int f = m.nI; f < m.nF; ++f) { // patches: bottom then top, face order
            A.b[m.own[f]] -= pred[f];
            fluxScale += std::abs(pred[f]);
        }
        if (m.nC > 0)
            A.d[0] += std::abs(A.d[0]) > 1e-30 ? A.d[0] : 1.0;
    }

    // assembleKEquation (:947-1023)
    void kEq(Ldu &A, const State &s, const Vec &phiF) const {
        A.zero();
        for (int f = 0; f < m.nI; ++f) {
            const int o = m.own[f], q = m.nbr[f];
            const double delta = std::max(m.delta[f], 1e-20);
            const double F1f = m.w[f] * s.F1[o] + (1.0 - m.w[f]) * s.F1[q];
            const double sk = cf.sigK(F1f);
            const double eO = nu + sk * s.nuT[o], eN = nu + sk * s.nuT[q];
            const double ef = m.w[f] * eO + (1.0 - m.w[f]) * eN;
            const double D = ef * m.area[f] / delta;
            const double F = phiF[f];
            const double cp = std::max(F, 0.0), cn = std::max(-F, 0.0);
            A.d[o] += D + cp;
            A.d[q] += D + cn;
            A.up[f] = -(D + cn);
            A.lo[f] = -(D + cp);
        }
        for (int f = m.nI; f < m.nF; ++f) {
            const int o = m.own[f];
            const double delta = std::max(m.delta[f], 1e-20);
            const double sk = cf.sigK(s.F1[o]);
            const double D = (nu + sk * s.nuT[o]) * m.area[f] / delta;
            const double kb = s.bk[f - m.nI], F = phiF[f];
            if (F >= 0) {
                A.d[o] += F + D;
                A.b[o] += D * kb;
            } else {
                A.d[o] += D;
                A.b[o] += (D - F) * kb;
            }
        }
        for (int c = 0; c < m.nC; ++c) {
            A.b[c] += s.Pk[c] * m.vol[c];
            A.d[c] += cf.bs * std::max(s.w[c], 1e-20) * m.vol[c];
        }
        convectionCorrection(A, phiF, s.k, s.bk);
        const double a = st.aK;
        for (int c = 0; c < m.nC; ++c) {
            A.b[c] += (1.0 - a) / a * A.d[c] * s.k[c];
            A.d[c] /= a;
        }
    }

    // assembleOmegaEquation (:1030-1169), production by productionOmega (SSTModel.cpp:102-108)
    void wEq(Ldu &A, const State &s, const Vec &phiF, const Vec &S) const {
        A.zero();
        Vec bal;
        if (!sing.empty())
            bal.assign(m.nC, 0.0);
        for (int f = 0; f < m.nI; ++f) {
            const int o = m.own[f], q = m.nbr[f];
            const double delta = std::max(m.delta[f], 1e-20);
            const double F1f = m.w[f] * s.F1[o] + (1.0 - m.w[f]) * s.F1[q];
            const double sw = cf.sigW(F1f);
            const double eO = nu + sw * s.nuT[o], eN = nu + sw * s.nuT[q];
            const double ef = m.w[f] * eO + (1.0 - m.w[f]) * eN;
            const double D = ef * m.area[f] / delta;
            const double F = phiF[f];
            const double cp = std::max(F, 0.0), cn = std::max(-F, 0.0);
            A.d[o] += D + cp;
            A.d[q] += D + cn;
            A.up[f] = -(D + cn);
            A.lo[f] = -(D + cp);
            if (!sing.empty()) {
                const double amp = 6 * nu / cf.b1;
                const double diff = (sing[q] - sing[o]) / delta;
                const double corr = amp * m.area[f] * ((ef - nu) * sgrad[f] - ef * diff);
                bal[o] += corr;
                bal[q] -= corr;
            }
        }
        for (int f = m.nI; f < m.nF; ++f) {
            const int o = m.own[f];
            const double delta = std::max(m.delta[f], 1e-20);
            const double sw = cf.sigW(s.F1[o]);
            const double D = (nu + sw * s.nuT[o]) * m.area[f] / delta;
            const double wb = s.bw[f - m.nI], F = phiF[f];
            if (F >= 0) {
                A.d[o] += F + D;
                A.b[o] += D * wb;
            } else {
                A.d[o] += D;
                A.b[o] += (D - F) * wb;
            }
        }
        for (int c = 0; c < m.nC; ++c) {
            const double v = m.vol[c], F1 = s.F1[c], wc = std::max(s.w[c], 1e-20);
            const double S2 = S[c] * S[c];
            const double lim = 10.0 * cf.bs * std::max(s.k[c], 0.0) * std::max(s.w[c], 1e-20) /
                               std::max(s.nuT[c], 1e-30);
            const double prod = std::min(S2, lim);
            A.b[c] += cf.alpha(F1) * prod * v;
            A.d[c] += cf.beta(F1) * wc * v;
            A.b[c] += (1.0 - F1) * s.CD[c] * v;
            if (!bal.empty()) {
                const double corr = bal[c] + nu * (6 * nu / cf.b1) * slap[c] * v;
                if (corr < 0)
                    A.d[c] -= corr / wc;
                else
                    A.b[c] += corr;
            }
        }
        convectionCorrection(A, phiF, s.w, s.bw);
        const double a = st.aW;
        for (int c = 0; c < m.nC; ++c) {
            A.b[c] += (1.0 - a) / a * A.d[c] * s.w[c];
            A.d[c] /= a;
        }
    }

    // omegaWallValues (:665-685) and constrainOmega (:687-704)
    void wallValues(Vec &vals) const {
        vals.assign(m.nC, std::numeric_limits<double>::quiet_NaN());
        for (int f = m.nI; f < m.nF; ++f)
            vals[m.own[f]] = wallOmega(std::max(m.delta[f], 1e-20));
    }
    void constrain(Ldu &A, const Vec &vals) const {
        for (int f = 0; f < m.nI; ++f) {
            const int o = m.own[f], q = m.nbr[f];
            if (std::isfinite(vals[o])) {
                A.b[q] -= A.lo[f] * vals[o];
                A.up[f] = A.lo[f] = 0;
            } else if (std::isfinite(vals[q])) {
                A.b[o] -= A.up[f] * vals[q];
                A.up[f] = A.lo[f] = 0;
            }
        }
        for (int c = 0; c < m.nC; ++c)
            if (std::isfinite(vals[c]))
                A.b[c] = A.d[c] * vals[c];
    }

    Vec observe(const State &s) const {
        Vec q(probes.size());
        for (size_t i = 0; i < probes.size(); ++i)
            q[i] = evalProbe(m, probes[i], s.Ux, s.bUx);
        return q;
    }

    // SIMPLESolver::solve (:1193-1716)
    History solve(State &s, std::vector<std::array<double, ORC_NHIST>> *hist) {
        History H;
        const int n = m.nC;
        Ldu A;
        A.init(m);
        Vec aP(n, 0.0), aPraw(n, 0.0), aPstore(n), S(n, 0.0), x(n), r(n), pp(n, 0.0);
        Vec phi, phiOld, phiPred, pCoeff, kOld, wOld, wv, UxPrev(n), UyPrev(n), qPrev;
        double lastK = 1.0, lastW = 1.0;
        const double tol = st.tol, negl = 0.01 * tol;
        Contraction eU(st.window), eK(st.window), eW(st.window), eQ(st.window);
        double worst = INF, fluxRef = 0.0;
        double n0x = 1, n0y = 1, n0p = 1;
        auto l1 = [](const Vec &v) {
            double a = 0.0;
            for (double e : v)
                a += std::abs(e);
            return a;
        };
        interpFlux(s, phi);
        for (int iter = 0; iter < st.maxIter; ++iter) {
            UxPrev = s.Ux;
            UyPrev = s.Uy;
            double momRes = 0.0, momScale = 0.0;
            interpFlux(s, phiOld);
            const bool turbActive = iter >= st.turbStart;
            const bool turbUpdate = turbActive && ((iter - st.turbStart) % 1 == 0);
            if (turbUpdate) {
                closure(m, cf, nu, s, S);
                if (!s.established && iter >= st.turbStart + st.floorIters)
                    s.established = true;
                const double floor = s.established ? 0.0 : 0.1 * nu;
                for (int c = 0; c < n; ++c)
                    s.nuT[c] = std::max(s.nuT[c], floor);
            }
            LinResult rUx, rUy, rUz;
            // x momentum
            momentum(A, s, phi, 0, aP, aPraw);
            x = s.Ux;
            A.residual(x, r);
            momRes = l1(r);
            for (int c = 0; c < n; ++c) {
                const double un = std::sqrt(s.Ux[c] * s.Ux[c] + s.Uy[c] * s.Uy[c] + s.Uz[c] * s.Uz[c]);
                const double contribution = aPraw[c] * un;
                momScale += contribution;
            }
            rUx = bicgstab(A, x, st.innerIter, st.innerTol);
            s.Ux = x;
            aPstore = aP;
            // y momentum
            momentum(A, s, phi, 1, aP, aPraw);
            x = s.Uy;
            A.residual(x, r);
            momRes = std::max(momRes, l1(r));
            rUy = bicgstab(A, x, st.innerIter, st.innerTol);
            s.Uy = x;
            // z momentum: identically zero right-hand side on 2-D meshes (r0 = 0)
            rUz = LinResult{0, 0.0, 0.0, true};
            bcU(s);
            // pressure correction with stored Rhie-Chow fluxes
            interpFlux(s, phiPred);
            rhieChow(s, aPstore, phiPred);
            const double rc = 1.0 - st.aU;
            for (int f = 0; f < m.nI; ++f)
                phiPred[f] += rc * (phi[f] - phiOld[f]);
            double fluxScale = 0.0;
            pressure(A, aPstore, phiPred, pCoeff, fluxScale);
            const double contScaled = l1(A.b) / std::max(fluxScale, 1e-300);
            std::fill(x.begin(), x.end(), 0.0);
            LinResult rP;
            if (st.pSolver == ORC_P_BICGSTAB)
                rP = bicgstab(A, x, st.innerIter, st.innerTol);
            else
                rP = pcg(A, x, st.innerIter, st.innerTol, useAmg ? &amg : nullptr);
            pp = x;
            // correctVelocity / correctPressure (:916-940), p' Neumann faces = owner
            {
                Vec bpp(m.nB());
                for (int f = m.nI; f < m.nF; ++f)
                    bpp[f - m.nI] = pp[m.own[f]];
                Vec gx, gy;
                ggrad(m, pp, bpp, gx, gy);
                for (int c = 0; c < n; ++c) {
                    const double rA = (std::abs(aPstore[c]) > 1e-30) ? 1.0 / aPstore[c] : 0.0;
                    s.Ux[c] -= rA * gx[c] * m.vol[c];
                    s.Uy[c] -= rA * gy[c] * m.vol[c];
                    s.Uz[c] -= rA * 0.0 * m.vol[c];
                }
                bcU(s);
                for (int c = 0; c < n; ++c)
                    s.p[c] += st.aP * pp[c];
                bcP(s);
                for (int f = 0; f < m.nF; ++f)
                    phi[f] = m.nbr[f] < 0 ? phiPred[f] + pCoeff[f] * pp[m.own[f]]
                                          : phiPred[f] - pCoeff[f] * (pp[m.nbr[f]] - pp[m.own[f]]);
            }
            LinResult rK, rW;
            if (turbUpdate) {
                kOld = s.k;
                wOld = s.w;
                kEq(A, s, phi);
                x = s.k;
                rK = bicgstab(A, x, st.innerIter, st.innerTol);
                s.k = x;
                for (double &v : s.k)
                    v = std::max(st.kMin, std::min(st.kMax, v));
                for (double &v : s.bk)
                    v = std::max(st.kMin, std::min(st.kMax, v));
                bcK(s);
                wEq(A, s, phi, S);
                wallValues(wv);
                constrain(A, wv);
                x = s.w;
                for (int c = 0; c < n; ++c)
                    if (std::isfinite(wv[c]))
                        x[c] = wv[c];
                rW = bicgstab(A, x, st.innerIter, st.innerTol);
                s.w = x;
                for (double &v : s.w)
                    v = std::max(st.wMin, std::min(1e15, v));
                for (double &v : s.bw)
                    v = std::max(st.wMin, std::min(1e15, v));
                for (int c = 0; c < n; ++c)
                    if (std::isfinite(wv[c]))
                        s.w[c] = wv[c];
                bcW(s, cf.b1);
                double kMaxV = 1e-30, wMaxV = 1e-30, kD = 0.0, wD = 0.0;
                for (int c = 0; c < n; ++c) {
                    kMaxV = std::max(kMaxV, std::abs(s.k[c]));
                    wMaxV = std::max(wMaxV, std::abs(s.w[c]));
                    kD = std::max(kD, std::abs(s.k[c] - kOld[c]));
                    wD = std::max(wD, std::abs(s.w[c] - wOld[c]));
                }
                lastK = kD / kMaxV;
                lastW = wD / wMaxV;
                eK.push(lastK);
                eW.push(lastW);
            }
            std::array<double, ORC_NHIST> e{};
            e[0] = iter;
            e[1] = rUx.initialRes;
            e[2] = rUy.initialRes;
            e[3] = rUz.initialRes;
            e[4] = rP.initialRes;
            e[5] = turbActive ? lastK : 0.0;
            e[6] = turbActive ? lastW : 0.0;
            double uMax = 1e-300, duMax = 0.0;
            for (int c = 0; c < n; ++c) {
                uMax = std::max(uMax, std::sqrt(s.Ux[c] * s.Ux[c] + s.Uy[c] * s.Uy[c] + s.Uz[c] * s.Uz[c]));
                const double ax = s.Ux[c] - UxPrev[c], ay = s.Uy[c] - UyPrev[c], az = s.Uz[c] - 0.0;
                duMax = std::max(duMax, std::sqrt(ax * ax + ay * ay + az * az));
            }
            e[7] = momRes / std::max(momScale, 1e-300);
            e[8] = contScaled;
            e[9] = duMax / uMax;
            eU.push(e[9]);
            e[10] = eU.remaining(negl);
            const bool haveMonitor = !probes.empty();
            if (haveMonitor && iter % std::max(st.monitorInterval, 1) == 0) {
                Vec q = observe(s);
                for (double v : q)
                    if (!std::isfinite(v))
                        throw std::runtime_error("convergence monitor returned a nonfinite observation");
                if (qPrev.size() == q.size()) {
                    double qMax = 0.0, dq = 0.0;
                    for (double v : q)
                        qMax = std::max(qMax, std::abs(v));
                    for (size_t i = 0; i < q.size(); ++i) {
                        const double fl = i < floors.size() ? floors[i] : 1e-6 * qMax;
                        dq = std::max(dq, std::abs(q[i] - qPrev[i]) /
                                              std::max({std::abs(q[i]), fl, 1e-300}));
                    }
                    eQ.push(dq);
                }
                qPrev = std::move(q);
            }
            worst = std::max({e[7], e[8], e[9], e[10]});
            if (turbActive)
                worst = std::max({worst, lastK, eK.remaining(negl), lastW, eW.remaining(negl)});
            if (haveMonitor)
                worst = std::max({worst, eQ.last(), eQ.remaining(negl)});
            if (!std::isfinite(worst))
                worst = INF;
            if (iter == 0) {
                n0x = std::max(e[1], 1e-30);
                n0y = std::max(e[2], 1e-30);
                n0p = std::max(e[4], 1e-30);
                fluxRef = fluxScale;
            } else if (iter < 50) {
                n0p = std::max(n0p, e[4]);
                fluxRef = std::max(fluxRef, fluxScale);
            }
            auto safe = [](double v, double ref) { return ref < 1e-20 ? 0.0 : v / ref; };
            const double nm = std::max(n0x, n0y);
            const double nUx = safe(e[1], nm), nUy = safe(e[2], nm);
            const double nP = safe(e[4], std::max(n0p, fluxRef));
            if (hist)
                hist->push_back(e);
            double maxRes = std::max({nUx, nUy, nP});
            if (turbActive)
                maxRes = std::max({maxRes, lastK, lastW});
            bool bad = false;
            for (int i = 1; i <= 9; ++i)
                bad = bad || !std::isfinite(e[i]);
            bad = bad || !std::isfinite(lastK) || !std::isfinite(lastW);
            if (bad) {
                maxRes = INF;
                worst = INF;
            }
            const bool turbScheduled = st.turbStart < st.maxIter;
            H.worst = worst;
            H.rate = eU.rate();
            if (worst < tol && iter > 0 && (!turbScheduled || (turbActive && s.established))) {
                H.converged = true;
                H.finalIter = iter;
                return H;
            }
            if (std::isnan(maxRes) || std::isinf(maxRes) || maxRes > st.divLimit) {
                H.diverged = true;
                H.finalIter = iter;
                return H;
            }
        }
        H.finalIter = st.maxIter;
        H.stalled = std::isfinite(H.rate) && H.rate >= 1.0;
        return H;
    }
};

static thread_local std::string lastError;

} // namespace orc

using namespace orc;

extern "C" {

const char *orc_last_error() { return orc::lastError.c_str(); }

int orc_mesh(const orc_case *c, int32_t *n_cells, int32_t *n_faces, int32_t *n_internal,
             double *cells, double *faces) {
    try {
        Mesh m = buildMesh(*c);
        *n_cells = m.nC;
        *n_faces = m.nF;
        *n_internal = m.nI;
        if (cells)
            for (int i = 0; i < m.nC; ++i) {
                cells[4 * i] = m.cx[i];
                cells[4 * i + 1] = m.cy[i];
                cells[4 * i + 2] = m.vol[i];
                cells[4 * i + 3] = m.wd[i];
            }
        if (faces)
            for (int f = 0; f < m.nF; ++f) {
                double *o = faces + 13 * f;
                o[0] = m.own[f];
                o[1] = m.nbr[f];
                o[2] = m.fcx[f];
                o[3] = m.fcy[f];
                o[4] = m.fnx[f];
                o[5] = m.fny[f];
                o[6] = m.area[f];
                o[7] = m.delta[f];
                o[8] = m.ddx[f];
                o[9] = m.ddy[f];
                o[10] = m.w[f];
                o[11] = m.shx[f];
                o[12] = m.patch[f];
            }
        return 0;
    } catch (const std::exception &e) {
        orc::lastError = e.what();
        return -1;
    }
}

} // extern "C"

namespace orc {

// ForwardModel::evaluateWithDiagnostics (rans-uq/src/ForwardModel.cpp:35-137) for the
// a1_betaStar parameter set (InferenceParameters.hpp:103-156): bounds, cold or warm start,
// solve, classification, probe predictions and the Gaussian log-likelihood
// (ObservationOperator.hpp:592-609). theta = (a1, betaStar) replaces coeffs[9], coeffs[8].
// warm (optional) is a cached state copied in place of initUniform (ForwardModel.cpp:79-82);
// out (optional) receives the final state of a solve that ran.
static void evaluateOne(const orc_case *c, const double theta[2], const State *warm, State *out,
                        orc_result *res, double *fields, double *predictions, double *history,
                        int32_t hist_cap) {
    std::memset(res, 0, sizeof(*res));
    const double a1 = theta[0], bs = theta[1];
    auto outOf = [](double v, double lo, double hi) {
        return v < lo || v > hi || std::isnan(v) || std::isinf(v);
    };
    if (outOf(a1, 0.1, 0.8) || outOf(bs, 0.01, 0.2)) {
        res->status = 3;
        res->loglik = -1e30;
        return;
    }
    double coeffs[11];
    std::memcpy(coeffs, c->coeffs, sizeof(coeffs));
    coeffs[9] = a1;
    coeffs[8] = bs;
    Mesh m = buildMesh(*c);
    Settings st{c->max_iter, c->inner_iter, c->conv_window, c->monitor_interval,
                c->turb_start, c->nut_floor_iters, c->pressure_solver,
                c->tol, c->inner_tol, c->alpha_u, c->alpha_p, c->alpha_k, c->alpha_w,
                c->body_force[0], c->body_force[1], c->div_limit, c->k_min, c->k_max,
                c->omega_min};
    Solver sv(m, coeffs, c->nu, st);
    for (int i = 0; i < c->n_obs; ++i) {
        sv.probes.push_back(prepareProbe(m, c->obs_x[i], c->obs_y[i]));
        sv.floors.push_back(std::sqrt(c->obs_sigma[i] * c->obs_sigma[i] + 0.0 * 0.0));
    }
    State s;
    if (warm)
        s = *warm;
    else
        sv.init(s, c->init_u, c->init_p, c->init_k, c->init_w);
    std::vector<std::array<double, ORC_NHIST>> hist;
    History H = sv.solve(s, history ? &hist : nullptr);
    res->iterations = H.finalIter;
    res->converged = H.converged;
    res->diverged = H.diverged;
    res->stalled = H.stalled;
    res->final_worst = H.worst;
    res->contraction_rate = H.rate;
    res->n_hist = static_cast<int32_t>(hist.size());
    if (history)
        for (int i = 0; i < static_cast<int>(hist.size()) && i < hist_cap; ++i)
            std::memcpy(history + ORC_NHIST * i, hist[i].data(), sizeof(double) * ORC_NHIST);
    if (H.diverged) {
        res->status = 2;
        res->loglik = -1e6;
        return;
    }
    res->status = H.converged ? 0 : 1;
    Vec q = sv.observe(s);
    double ll = 0.0;
    for (int i = 0; i < c->n_obs; ++i) {
        if (predictions)
            predictions[i] = q[i];
        const double var = c->obs_sigma[i] * c->obs_sigma[i] + 0.0 * 0.0;
        const double diff = q[i] - c->obs_value[i];
        ll += -0.5 * diff * diff / var;
    }
    res->loglik = ll;
    if (fields) {
        const int n = m.nC;
        const Vec *src[ORC_NFIELD] = {&s.Ux, &s.Uy, &s.Uz, &s.p, &s.k, &s.w,
                                      &s.nuT, &s.F1, &s.F2, &s.Pk, &s.CD};
        for (int b = 0; b < ORC_NFIELD; ++b)
            std::memcpy(fields + static_cast<size_t>(b) * n, src[b]->data(), sizeof(double) * n);
    }
    if (out)
        *out = std::move(s);
}

// WarmStartCache (rans-uq/include/ForwardModel.hpp:21-157): converged states keyed by theta,
// FIFO eviction by count and by the payload byte count of entryBytes (:39-47): theta, the
// vector field and eight scalar fields, each over cells plus boundary faces.
struct WarmCache {
    struct Entry {
        std::array<double, 2> theta;
        State s;
        size_t bytes;
    };
    int maxSize;
    double threshold;
    size_t budget, retained = 0;
    std::vector<Entry> q; // front = oldest

    static size_t entryBytes(size_t cellsPlusBoundary) {
        return 2 * sizeof(double) + cellsPlusBoundary * (3 * sizeof(double)) +
               8 * cellsPlusBoundary * sizeof(double);
    }
    const Entry *nearest(const double theta[2]) const { // nearest (:132-144), strict <
        const Entry *best = nullptr;
        double bestDist = threshold;
        for (const Entry &e : q) {
            const double d0 = theta[0] - e.theta[0], d1 = theta[1] - e.theta[1];
            const double d = std::sqrt(d0 * d0 + d1 * d1);
            if (d < bestDist) {
                bestDist = d;
                best = &e;
            }
        }
        return best;
    }
    void store(const double theta[2], State &&s, size_t nCB) { // store (:70-92)
        if (!std::isfinite(theta[0]) || !std::isfinite(theta[1]))
            return;
        for (size_t i = 0; i < q.size(); ++i)
            if (q[i].theta[0] == theta[0] && q[i].theta[1] == theta[1]) {
                retained -= q[i].bytes;
                q.erase(q.begin() + static_cast<long>(i));
                break;
            }
        const size_t bytes = entryBytes(nCB);
        if (maxSize == 0 || bytes > budget)
            return;
        while (!q.empty() && (q.size() >= static_cast<size_t>(maxSize) || retained > budget - bytes)) {
            retained -= q.front().bytes;
            q.erase(q.begin());
        }
        q.push_back({{theta[0], theta[1]}, std::move(s), bytes});
        retained += bytes;
    }
};

} // namespace orc

extern "C" {

int orc_solve(const orc_case *c, orc_result *res, double *fields, double *predictions,
              double *history, int32_t hist_cap) {
    try {
        const double theta[2] = {c->coeffs[9], c->coeffs[8]};
        evaluateOne(c, theta, nullptr, nullptr, res, fields, predictions, history, hist_cap);
        return 0;
    } catch (const std::exception &e) {
        orc::lastError = e.what();
        res->status = 4;
        res->loglik = -1e6;
        return 0;
    }
}

// A sequence of ForwardModel::evaluateWithDiagnostics calls on one model, with its
// warm-start cache (ForwardModel.cpp:79-82 lookup, :116-117 store of converged solves):
// theta row i is (a1, betaStar); used_warm[i] = ForwardEvaluationResult::usedWarmStart.
// retained[i] (optional) = the cache's retained bytes after call i.
int orc_solve_sequence(const orc_case *c, const double *thetas, int32_t m_calls, int32_t max_size,
                       double threshold, int64_t byte_budget, orc_result *res,
                       double *predictions, int32_t *used_warm, int64_t *retained) {
    try {
        WarmCache cache{max_size, threshold, static_cast<size_t>(byte_budget)};
        Mesh mesh = buildMesh(*c);
        const size_t nCB = static_cast<size_t>(mesh.nF - mesh.nI) + mesh.nC;
        for (int i = 0; i < m_calls; ++i) {
            const double *th = thetas + 2 * i;
            orc_result &r = res[i];
            double *pred = predictions ? predictions + static_cast<size_t>(i) * c->n_obs : nullptr;
            const bool inBounds = !(th[0] < 0.1 || th[0] > 0.8 || th[1] < 0.01 || th[1] > 0.2 ||
                                    std::isnan(th[0]) || std::isnan(th[1]));
            const WarmCache::Entry *hit = inBounds ? cache.nearest(th) : nullptr;
            State warm, out;
            if (hit)
                warm = hit->s; // deep copy, as findNearest does
            used_warm[i] = hit != nullptr;
            try {
                evaluateOne(c, th, hit ? &warm : nullptr, &out, &r, nullptr, pred, nullptr, 0);
            } catch (const std::exception &e) {
                orc::lastError = e.what();
                std::memset(&r, 0, sizeof(r));
                r.status = 4;
                r.loglik = -1e6;
            }
            if (r.status == 0)
                cache.store(th, std::move(out), nCB);
            if (retained)
                retained[i] = static_cast<int64_t>(cache.retained);
        }
        return 0;
    } catch (const std::exception &e) {
        orc::lastError = e.what();
        return -1;
    }
}

// Linear solve on an LDU system: kind 1 PCG (Jacobi), 2 BiCGSTAB, 10 device-style AMG-PCG
// whose hierarchy is aggregated from the system's own values.
int orc_linear_solve(int32_t kind, int32_t n, int32_t nif, const double *diag,
                     const double *upper, const double *lower, const double *source,
                     const int32_t *own, const int32_t *nbr, double *x, int32_t max_iter,
                     double tol, int32_t *iterations, double *final_res, double *initial_res,
                     int32_t *converged) {
    try {
        std::vector<int> ow(own, own + nif), nb(nbr, nbr + nif);
        Ldu A;
        A.n = n;
        A.nf = nif;
        A.d.assign(diag, diag + n);
        A.b.assign(source, source + n);
        A.up.assign(upper, upper + nif);
        A.lo.assign(lower, lower + nif);
        A.own = &ow;
        A.nbr = &nb;
        Vec xv(x, x + n);
        LinResult r;
        if (kind == 2) {
            r = bicgstab(A, xv, max_iter, tol);
        } else if (kind == 10) {
            Amg h;
            h.w = 0.75;
            h.alpha = 1.7;
            h.sweeps = 2;
            AmgLevel l0;
            l0.A = lduCsr(n, ow, nb, nif, A.d, A.up, A.lo, &h.upPos, &h.loPos);
            l0.dpos.resize(n);
            for (int i = 0; i < n; ++i)
                l0.dpos[i] = csrFind(l0.A, i, i);
            h.lev.push_back(std::move(l0));
            for (int l = 0; l < AMG_MAX_LEVELS; ++l) {
                AmgLevel &fine = h.lev[l];
                if (fine.A.n <= AMG_MIN_COARSE_LINEAR)
                    break;
                std::vector<int> map;
                int nc = 0;
                aggregateLinear(fine.A, map, nc);
                if (nc == 0 || nc >= fine.A.n)
                    break;
                AmgLevel coarse;
                fine.nc = nc;
                prolongation(fine.A, map, 0.0, fine);
                galerkinLevel(fine, coarse);
                sumCoarse(fine, coarse);
                h.lev.push_back(std::move(coarse));
            }
            r = pcg(A, xv, max_iter, tol, &h);
        } else {
            r = pcg(A, xv, max_iter, tol, nullptr);
        }
        std::memcpy(x, xv.data(), sizeof(double) * n);
        *iterations = r.iterations;
        *final_res = r.finalRes;
        *initial_res = r.initialRes;
        *converged = r.converged;
        return 0;
    } catch (const std::exception &e) {
        orc::lastError = e.what();
        return -1;
    }
}

// Aggregation of the mesh's geometric pressure Laplacian, level by level:
// writes the level sizes into sizes[0..levels) and returns the level count;
// maps (if not null) receives the concatenated fine->coarse maps.
int orc_amg_hierarchy(const orc_case *c, int32_t *sizes, int32_t cap, int32_t *maps) {
    try {
        Mesh m = buildMesh(*c);
        Amg h = buildAmg(m);
        int off = 0;
        for (int l = 0; l < h.levels() && l < cap; ++l) {
            sizes[l] = h.lev[l].A.n;
            if (maps && l + 1 < h.levels())
                for (int i = 0; i < h.lev[l].A.n; ++i)
                    maps[off++] = h.lev[l].pCol[h.lev[l].pPtr[i]]; // first coarse row of P
        }
        return h.levels();
    } catch (const std::exception &e) {
        orc::lastError = e.what();
        return -1;
    }
}

} // extern "C"
