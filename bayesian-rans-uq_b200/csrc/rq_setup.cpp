// Host set-up of a mesh class: see rq_setup.h. Arithmetic of the generator
// follows the reference operation by operation so the geometry is bit-identical
// to core/src/Mesh.cpp:523-741 (the third coordinate is identically zero there
// and is dropped here).
#include "rq_setup.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <map>
#include <stdexcept>

namespace rq {

StructMesh buildPeriodic(const std::vector<double> &xN, const std::vector<double> &yB, double yTop,
                         int ny, double y1t) {
    const int nx = static_cast<int>(xN.size()) - 1;
    if (nx < 3 || static_cast<int>(yB.size()) != nx + 1)
        throw std::invalid_argument("periodic mesh needs nx >= 3 and nx+1 bottom samples");
    if (ny < 1)
        throw std::invalid_argument("periodic mesh needs ny >= 1");
    for (size_t i = 0; i < xN.size(); ++i) {
        if (!std::isfinite(xN[i]) || (i > 0 && xN[i] <= xN[i - 1]))
            throw std::invalid_argument("periodic x nodes must be finite and increasing");
        if (!(yTop - yB[i] > 0) || !std::isfinite(yTop - yB[i]))
            throw std::invalid_argument("periodic mesh local height must be positive");
    }
    if (std::abs(yB.front() - yB.back()) > 1e-12)
        throw std::invalid_argument("bottom profile must be periodic (first == last sample)");
    if (!std::isfinite(y1t) || y1t < 0)
        throw std::invalid_argument("first-cell height must be finite");
    StructMesh m;
    m.nx = nx;
    m.ny = ny;
    m.n = nx * ny;
    m.lx = xN.back() - xN.front();

    // shared wall-normal distribution from the mean height (Mesh.cpp:549-581)
    double meanH = 0.0;
    for (int i = 0; i <= nx; ++i)
        meanH += (yTop - yB[i]);
    meanH /= (nx + 1);
    double stretch = 2.0;
    if (y1t > 0 && y1t < meanH / ny) {
        auto h1 = [&](double s) {
            return 0.5 * meanH * (1.0 + std::tanh(s * (2.0 / ny - 1.0)) / std::tanh(s));
        };
        double lo = 0.1, hi = 20.0;
        if (y1t < h1(hi)) {
            stretch = hi;
        } else {
            for (int it = 0; it < 100; ++it) {
                const double mid = 0.5 * (lo + hi);
                (h1(mid) > y1t ? lo : hi) = mid;
                if (hi - lo < 1e-10)
                    break;
            }
            stretch = 0.5 * (lo + hi);
        }
    }
    std::vector<double> eta(ny + 1);
    for (int j = 0; j <= ny; ++j) {
        const double e = static_cast<double>(j) / ny;
        eta[j] = 0.5 * (1.0 + std::tanh(stretch * (2.0 * e - 1.0)) / std::tanh(stretch));
    }
    auto Y = [&](int i, int j) { return yB[i] + (yTop - yB[i]) * eta[j]; };
    m.xNodes = xN;
    m.yNodes.resize(static_cast<size_t>(nx + 1) * (ny + 1));
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i <= nx; ++i)
            m.yNodes[static_cast<size_t>(j) * (nx + 1) + i] = Y(i, j);

    const int n = m.n;
    m.cx.resize(n);
    m.cy.resize(n);
    m.vol.resize(n);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) { // shoelace centroid and area of the quad
            const double px[4] = {xN[i], xN[i + 1], xN[i + 1], xN[i]};
            const double py[4] = {Y(i, j), Y(i + 1, j), Y(i + 1, j + 1), Y(i, j + 1)};
            double twiceA = 0.0, mx = 0.0, my = 0.0;
            for (int k = 0; k < 4; ++k) {
                const int k1 = (k + 1) % 4;
                const double cr = px[k] * py[k1] - px[k1] * py[k];
                twiceA += cr;
                mx += (px[k] + px[k1]) * cr;
                my += (py[k] + py[k1]) * cr;
            }
            const double A = 0.5 * twiceA;
            const int c = j * nx + i;
            m.cx[c] = mx / (6.0 * A);
            m.cy[c] = my / (6.0 * A);
            m.vol[c] = std::abs(A) * 1.0;
        }

    // edge geometry: centre, area (unit depth) and in-plane unit normal
    struct Edge {
        double fx, fy, a, nxv, nyv;
    };
    auto edge = [](double x0, double y0, double x1, double y1, bool plusX) {
        const double ex = x1 - x0, ey = y1 - y0;
        const double len = std::sqrt(ex * ex + ey * ey);
        Edge e{0.5 * (x0 + x1), 0.5 * (y0 + y1), len * 1.0, 0, 0};
        e.nxv = plusX ? ey / len : -ey / len;
        e.nyv = plusX ? -ex / len : ex / len;
        return e;
    };
    auto weight = [](const Edge &e, double ox, double oy, double qx, double qy) {
        const double ax = e.fx - ox, ay = e.fy - oy, bx = e.fx - qx, by = e.fy - qy;
        const double dP = std::sqrt(ax * ax + ay * ay), dN = std::sqrt(bx * bx + by * by);
        const double s = dP + dN;
        return (s > 1e-30) ? dN / s : 0.5;
    };

    for (auto *v : {&m.xa, &m.xnx, &m.xny, &m.xw, &m.xdl, &m.xdx, &m.xdy, &m.xsh, &m.xfx, &m.xfy})
        v->assign(n, 0.0);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) { // east faces; the last column is the wrap face
            const int c = j * nx + i, q = j * nx + (i + 1) % nx;
            const Edge e = edge(xN[i + 1], Y(i + 1, j), xN[i + 1], Y(i + 1, j + 1), true);
            const double sh = (i == nx - 1) ? m.lx : 0.0;
            const double qx = (i == nx - 1) ? m.cx[q] + sh : m.cx[q];
            const double qy = (i == nx - 1) ? m.cy[q] + 0.0 : m.cy[q];
            m.xa[c] = e.a;
            m.xnx[c] = e.nxv;
            m.xny[c] = e.nyv;
            m.xfx[c] = e.fx;
            m.xfy[c] = e.fy;
            m.xsh[c] = sh;
            m.xdx[c] = qx - m.cx[c];
            m.xdy[c] = qy - m.cy[c];
            m.xdl[c] = std::max(std::sqrt(m.xdx[c] * m.xdx[c] + m.xdy[c] * m.xdy[c]), 1e-20);
            m.xw[c] = weight(e, m.cx[c], m.cy[c], qx, qy);
        }
    const int nfy = m.nfy();
    for (auto *v : {&m.ya, &m.ynx, &m.yny, &m.ydl, &m.ydx, &m.ydy, &m.yfx, &m.yfy})
        v->assign(nfy, 0.0);
    m.yw.assign(nfy, 0.5);
    for (int jf = 0; jf <= ny; ++jf)
        for (int i = 0; i < nx; ++i) {
            const int f = jf * nx + i;
            const Edge e = edge(xN[i], Y(i, jf), xN[i + 1], Y(i + 1, jf), jf == 0);
            m.ya[f] = e.a;
            m.ynx[f] = e.nxv;
            m.yny[f] = e.nyv;
            m.yfx[f] = e.fx;
            m.yfy[f] = e.fy;
            if (jf == 0 || jf == ny) { // wall: owner-to-face vector
                const int o = (jf == 0 ? 0 : ny - 1) * nx + i;
                m.ydx[f] = e.fx - m.cx[o];
                m.ydy[f] = e.fy - m.cy[o];
            } else {
                const int o = (jf - 1) * nx + i, q = jf * nx + i;
                m.ydx[f] = m.cx[q] - m.cx[o];
                m.ydy[f] = m.cy[q] - m.cy[o];
                m.yw[f] = weight(e, m.cx[o], m.cy[o], m.cx[q], m.cy[q]);
            }
            m.ydl[f] = std::max(std::sqrt(m.ydx[f] * m.ydx[f] + m.ydy[f] * m.ydy[f]), 1e-20);
        }

    // brute-force wall distance over bottom then top wall-face centres
    m.wd.assign(n, 0.0);
    for (int c = 0; c < n; ++c) {
        double best = std::numeric_limits<double>::max();
        for (int side = 0; side < 2; ++side)
            for (int i = 0; i < nx; ++i) {
                const int f = (side == 0 ? 0 : ny) * nx + i;
                const double dx = m.cx[c] - m.yfx[f], dy = m.cy[c] - m.yfy[f];
                const double d = std::sqrt(dx * dx + dy * dy);
                if (d < best)
                    best = d;
            }
        m.wd[c] = best;
    }
    preparePlanarBalance(m);
    return m;
}

StructMesh makePeriodicChannel(int nx, int ny, double lx, double h, double reTau, double yPlus) {
    if (!(lx > 0) || !(h > 0) || !(reTau > 0) || !(yPlus > 0) || !std::isfinite(lx * h * reTau * yPlus))
        throw std::invalid_argument("channel length, half height, Re_tau and y+ must be positive");
    std::vector<double> xN(nx + 1), yB(nx + 1, 0.0);
    for (int i = 0; i <= nx; ++i)
        xN[i] = lx * i / nx;
    return buildPeriodic(xN, yB, 2.0 * h, ny, yPlus * h / reTau);
}

StructMesh makeCurvedPeriodic(const std::vector<double> &xN, const std::vector<double> &yB,
                              double yTop, int ny, double re, double yPlus) {
    if (!std::isfinite(re) || re < 0 || !(yPlus > 0))
        throw std::invalid_argument("curved mesh Reynolds number and y+ must be valid");
    double y1t = 0.0;
    if (re > 0 && xN.size() == yB.size()) { // skin-friction sizing of the first cell
        double meanH = 0.0;
        for (double v : yB)
            meanH += (yTop - v);
        meanH /= static_cast<double>(yB.size());
        const double cf = 0.058 * std::pow(re, -0.2);
        const double uTau = std::sqrt(cf / 2.0);
        const double nu = meanH / re;
        y1t = yPlus * nu / uTau;
    }
    StructMesh m = buildPeriodic(xN, yB, yTop, ny, y1t);
    m.bottomName = "bottom_wall";
    m.topName = "top_wall";
    return m;
}

std::vector<char> meshBinary(const StructMesh &m) {
    const int nx = m.nx, ny = m.ny, n = m.n, nfy = m.nfy();
    const double dz = 1.0, zc = 0.5 * dz;
    std::vector<char> out;
    auto raw = [&](const void *p, size_t bytes) {
        const char *c = static_cast<const char *>(p);
        out.insert(out.end(), c, c + bytes);
    };
    auto i32 = [&](int v) { raw(&v, sizeof v); };
    auto f64 = [&](double v) { raw(&v, sizeof v); };
    auto vec = [&](double x, double y, double z) {
        f64(x);
        f64(y);
        f64(z);
    };
    const int nInternal = 2 * nx * ny - nx, nFaces = nInternal + 2 * nx;
    const int nNodes = 2 * (nx + 1) * (ny + 1);
    const uint32_t magic = 0x4D534832; // "MSH2"
    raw(&magic, sizeof magic);
    i32(n);
    i32(nFaces);
    i32(nNodes);
    i32(2);
    i32(nInternal);
    for (int k = 0; k < 2; ++k) // front plane z = 0, back plane z = dz
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i)
                vec(m.xNodes[i], m.yNodes[static_cast<size_t>(j) * (nx + 1) + i], k * dz);
    // faces in the generator's order (Mesh.cpp:646-720); fields as Mesh::saveBinary writes
    // them: owner, neighbour, patch, centre, normal, area, delta, d, weight, shift
    std::vector<std::vector<int>> cellFaces(n);
    int fi = 0;
    auto xFace = [&](int c, int q) {
        i32(c);
        i32(q);
        i32(-1);
        vec(m.xfx[c], m.xfy[c], zc);
        vec(m.xnx[c], m.xny[c], 0.0);
        f64(m.xa[c]);
        f64(m.xdl[c]);
        vec(m.xdx[c], m.xdy[c], 0.0);
        f64(m.xw[c]);
        vec(m.xsh[c], 0.0, 0.0);
        cellFaces[c].push_back(fi);
        cellFaces[q].push_back(fi);
        ++fi;
    };
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx - 1; ++i)
            xFace(j * nx + i, j * nx + i + 1);
    for (int j = 0; j < ny; ++j)
        xFace(j * nx + nx - 1, j * nx);
    for (int jf = 1; jf < ny; ++jf)
        for (int i = 0; i < nx; ++i) {
            const int g = jf * nx + i, o = g - nx;
            i32(o);
            i32(g);
            i32(-1);
            vec(m.yfx[g], m.yfy[g], zc);
            vec(m.ynx[g], m.yny[g], 0.0);
            f64(m.ya[g]);
            f64(m.ydl[g]);
            vec(m.ydx[g], m.ydy[g], 0.0);
            f64(m.yw[g]);
            vec(0.0, 0.0, 0.0);
            cellFaces[o].push_back(fi);
            cellFaces[g].push_back(fi);
            ++fi;
        }
    std::vector<int> patchFaces[2];
    for (int side = 0; side < 2; ++side)
        for (int i = 0; i < nx; ++i) {
            const int g = (side == 0 ? 0 : ny) * nx + i;
            const int o = (side == 0 ? 0 : ny - 1) * nx + i;
            i32(o);
            i32(-1);
            i32(side);
            vec(m.yfx[g], m.yfy[g], zc);
            vec(m.ynx[g], m.yny[g], 0.0);
            f64(m.ya[g]);
            f64(m.ydl[g]);
            vec(m.ydx[g], m.ydy[g], 0.0);
            f64(m.yw[g]);
            vec(0.0, 0.0, 0.0);
            cellFaces[o].push_back(fi);
            patchFaces[side].push_back(fi);
            ++fi;
        }
    for (int c = 0; c < n; ++c) {
        vec(m.cx[c], m.cy[c], zc);
        f64(m.vol[c]);
        i32(static_cast<int>(cellFaces[c].size()));
        for (int f : cellFaces[c])
            i32(f);
    }
    for (int side = 0; side < 2; ++side) {
        const std::string &name = side == 0 ? m.bottomName : m.topName;
        const std::string type = "wall";
        i32(static_cast<int>(name.size()));
        raw(name.data(), name.size());
        i32(static_cast<int>(type.size()));
        raw(type.data(), type.size());
        i32(static_cast<int>(patchFaces[side].size()));
        for (int f : patchFaces[side])
            i32(f);
    }
    (void)nfy;
    return out;
}

// Qualifies a mesh bounded by two parallel planar walls with orthogonal faces
// and periodic wrap faces; then s(y) = 1/y^2 + 1/(H-y)^2, its normal face
// gradient and Laplacian are precomputed.
void preparePlanarBalance(StructMesh &m) {
    m.balance = false;
    const int nx = m.nx, ny = m.ny, n = m.n, nfy = m.nfy();
    const int f0 = 0; // first boundary face in reference order: bottom wall, column 0
    const double ix = m.ynx[f0] * -1.0, iy = m.yny[f0] * -1.0;
    const double origin = m.yfx[f0] * ix + m.yfy[f0] * iy;
    double height = 0.0;
    for (int side = 0; side < 2; ++side)
        for (int i = 0; i < nx; ++i) {
            const int f = (side ? ny : 0) * nx + i;
            if (std::abs(std::abs(m.ynx[f] * ix + m.yny[f] * iy) - 1.0) > 1e-12)
                return;
            height = std::max(height, m.yfx[f] * ix + m.yfy[f] * iy - origin);
        }
    if (!(height > 0))
        return;
    const double tol = 1e-12 * height;
    auto orthogonal = [&](double dx, double dy, double nxv, double nyv, double dl) {
        const double ex = dx - nxv * dl, ey = dy - nyv * dl;
        return !(std::sqrt(ex * ex + ey * ey) > 1e-9 * dl);
    };
    bool periodic = false;
    for (int c = 0; c < n; ++c) {
        if (!orthogonal(m.xdx[c], m.xdy[c], m.xnx[c], m.xny[c], m.xdl[c]) ||
            std::abs(m.xsh[c] * ix) > tol)
            return;
        periodic = periodic || m.xsh[c] * m.xsh[c] > 0;
    }
    for (int f = 0; f < nfy; ++f) {
        if (!orthogonal(m.ydx[f], m.ydy[f], m.ynx[f], m.yny[f], m.ydl[f]))
            return;
        const int jf = f / nx;
        if (jf == 0 || jf == ny) {
            const double y = m.yfx[f] * ix + m.yfy[f] * iy - origin;
            if (std::min(std::abs(y), std::abs(y - height)) > tol)
                return;
            if ((y < height / 2 ? -1.0 : 1.0) * (m.ynx[f] * ix + m.yny[f] * iy) < 1 - 1e-12)
                return;
        }
    }
    if (!periodic)
        return;
    std::vector<double> s(n), lap(n), gx(n), gy(nfy, 0.0);
    for (int c = 0; c < n; ++c) {
        const double y = m.cx[c] * ix + m.cy[c] * iy - origin;
        if (!(y > 0 && y < height))
            return;
        s[c] = 1 / (y * y) + 1 / ((height - y) * (height - y));
        lap[c] = 6 * (std::pow(y, -4) + std::pow(height - y, -4));
    }
    auto grad = [&](double fx, double fy, double nxv, double nyv, double &out) {
        const double y = fx * ix + fy * iy - origin;
        if (!(y > 0 && y < height))
            return false;
        out = 2 * (std::pow(height - y, -3) - std::pow(y, -3)) * (nxv * ix + nyv * iy);
        return true;
    };
    for (int c = 0; c < n; ++c)
        if (!grad(m.xfx[c], m.xfy[c], m.xnx[c], m.xny[c], gx[c]))
            return;
    for (int jf = 1; jf < ny; ++jf)
        for (int i = 0; i < nx; ++i) {
            const int f = jf * nx + i;
            if (!grad(m.yfx[f], m.yfy[f], m.ynx[f], m.yny[f], gy[f]))
                return;
        }
    m.sing = std::move(s);
    m.slap = std::move(lap);
    m.sgx = std::move(gx);
    m.sgy = std::move(gy);
    m.balance = true;
}

int cellFaceOrder(const StructMesh &m, int c, int out[4]) {
    const int i = c % m.nx, j = c / m.nx;
    int k = 0;
    if (i >= 1)
        out[k++] = 0;
    if (i <= m.nx - 2)
        out[k++] = 1;
    if (i == 0)
        out[k++] = 0;
    if (i == m.nx - 1)
        out[k++] = 1;
    if (j >= 1)
        out[k++] = 2;
    if (j <= m.ny - 2)
        out[k++] = 3;
    if (j == 0)
        out[k++] = 2;
    if (j == m.ny - 1)
        out[k++] = 3;
    return k;
}

// ------------------------------------------------------------------ AMG
namespace {
struct Csr {
    int n = 0;
    std::vector<int> ptr, col;
    std::vector<double> val, dg;
    int find(int r, int c) const {
        for (int k = ptr[r]; k < ptr[r + 1]; ++k)
            if (col[k] == c)
                return k;
        return -1;
    }
};

void greedyAggregate(const Csr &A, std::vector<int> &map, int &nc) {
    map.assign(A.n, -1);
    nc = 0;
    for (int i = 0; i < A.n; ++i) {
        if (map[i] >= 0)
            continue;
        const int g = nc++;
        map[i] = g;
        const double aii = std::abs(A.dg[i]);
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int c = A.col[k];
            if (c == i || map[c] >= 0)
                continue;
            if (std::abs(A.val[k]) / std::sqrt(aii * std::abs(A.dg[c]) + 1e-30) > 0.25)
                map[c] = g;
        }
    }
    for (int i = 0; i < A.n; ++i) {
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
// Row-relative aggregation, for matrices on which the symmetric strength rule
// stalls (strongly varying cell aspect ratios: the bump-wall meshes keep ~1000
// rows after 20 levels): j is strong for i when |a_ij| >= 0.25 max_k |a_ik|; seeds
// claim their unaggregated strong neighbours, a seed left alone joins its
// strongest neighbour's aggregate, and ids are renumbered in order of first use.
void rowRelativeAggregate(const Csr &A, std::vector<int> &map, int &nc) {
    map.assign(A.n, -1);
    int groups = 0;
    for (int i = 0; i < A.n; ++i) {
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
    for (int i = 0; i < A.n; ++i)
        ++count[map[i]];
    for (int i = 0; i < A.n; ++i) {
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
    for (int i = 0; i < A.n; ++i) {
        if (id[map[i]] < 0)
            id[map[i]] = nc++;
        map[i] = id[map[i]];
    }
}
// Smoothed-aggregation prolongation of one level (weight > 0), or the tentative
// piecewise-constant one (weight 0): P = (I - omega D_F^-1 F) P_tent, where F keeps the
// strong entries of A (|a_ij| / sqrt(a_ii a_jj) > 0.25, the aggregation's rule) and
// lumps the weak ones into its diagonal, and omega = weight / rho(D_F^-1 F) from a
// power iteration. Rows list their coarse columns ascending; exact zeros are dropped.
struct Prolong {
    std::vector<int> ptr, col;
    std::vector<double> val;
};

Prolong smoothedProlongation(const Csr &A, const std::vector<int> &agg, int nc, double weight) {
    const int n = A.n;
    Prolong P;
    P.ptr.assign(n + 1, 0);
    std::vector<double> fd(n, 0.0); // filtered (lumped) diagonal
    auto strongAt = [&](int i, int k) {
        const int c = A.col[k];
        return c != i &&
               std::abs(A.val[k]) / std::sqrt(std::abs(A.dg[i]) * std::abs(A.dg[c]) + 1e-30) > 0.25;
    };
    for (int i = 0; i < n; ++i) {
        double d = A.dg[i];
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (A.col[k] != i && !strongAt(i, k))
                d += A.val[k];
        fd[i] = d;
    }
    // a row whose lumped diagonal vanishes (all its couplings weak) is not smoothed
    auto usable = [&](int i) { return std::abs(fd[i]) > 1e-12 * std::abs(A.dg[i]); };
    double omega = 0.0;
    if (weight > 0.0) {
        std::vector<double> x(n), y(n);
        for (int i = 0; i < n; ++i)
            x[i] = 1.0 + 0.1 * (i % 7);
        double rho = 0.0;
        for (int it = 0; it < 100; ++it) {
            double ny = 0.0, nx = 0.0;
            for (int i = 0; i < n; ++i) {
                double s = 0.0;
                if (usable(i)) {
                    s = fd[i] * x[i];
                    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                        if (strongAt(i, k))
                            s += A.val[k] * x[A.col[k]];
                    s /= fd[i];
                }
                y[i] = s;
                ny += s * s;
                nx += x[i] * x[i];
            }
            rho = std::sqrt(ny / std::max(nx, 1e-300));
            const double inv = 1.0 / std::max(std::sqrt(ny), 1e-300);
            for (int i = 0; i < n; ++i)
                x[i] = y[i] * inv;
        }
        omega = rho > 0.0 ? weight / rho : 0.0;
    }
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
                P.col.push_back(e.first);
                P.val.push_back(e.second);
            }
        P.ptr[i + 1] = static_cast<int>(P.col.size());
    }
    (void)nc;
    return P;
}
} // namespace

AmgHost buildAmg(const StructMesh &m, int minCoarse, int maxLevels) {
    const int nx = m.nx, ny = m.ny, n = m.n;
    // geometric Laplacian with the pressure system's cell-0 pin, as CSR with
    // sorted columns; 'slot' records the structured entry of every nnz
    auto coefX = [&](int c) { return m.xa[c] / std::max(m.xdl[c], 1e-20); };
    auto coefY = [&](int f) { return m.ya[f] / std::max(m.ydl[f], 1e-20); };
    Csr A;
    A.n = n;
    A.ptr.assign(n + 1, 0);
    A.dg.assign(n, 0.0);
    std::vector<int> slot;
    for (int c = 0; c < n; ++c) {
        const int i = c % nx, j = c / nx;
        const int W = j * nx + (i + nx - 1) % nx, E = j * nx + (i + 1) % nx;
        std::vector<std::pair<int, std::pair<int, double>>> row; // col, (slot, value)
        const double cw = coefX(W), ce = coefX(c);
        const double cs = j > 0 ? coefY(c) : 0.0, cn = j < ny - 1 ? coefY(c + nx) : 0.0;
        double d = 0.0;
        int order[4];
        const int nf = cellFaceOrder(m, c, order); // diagonal summed in face-index order
        for (int k = 0; k < nf; ++k) {
            const int code = order[k];
            if (code == 2 && j == 0)
                continue; // walls are Neumann for the pressure correction
            if (code == 3 && j == ny - 1)
                continue;
            d += code == 0 ? cw : code == 1 ? ce : code == 2 ? cs : cn;
        }
        row.push_back({W, {1, -cw}});
        row.push_back({E, {2, -ce}});
        if (j > 0)
            row.push_back({c - nx, {3, -cs}});
        if (j < ny - 1)
            row.push_back({c + nx, {4, -cn}});
        if (c == 0)
            d += d;
        row.push_back({c, {0, d}});
        std::sort(row.begin(), row.end(), [](auto &a, auto &b) { return a.first < b.first; });
        for (auto &e : row) {
            A.col.push_back(e.first);
            A.val.push_back(e.second.second);
            slot.push_back(e.second.first * n + c);
        }
        A.dg[c] = d;
        A.ptr[c + 1] = static_cast<int>(A.col.size());
    }
    // the reference's aggregation first; if it stalls above minCoarse rows, the
    // row-relative rule instead
    AmgHost h;
    for (int attempt = 0; attempt < 2; ++attempt) {
    h = AmgHost{};
    std::vector<Csr> mats{A};
    for (int l = 0; l < maxLevels; ++l) {
        const Csr &F = mats.back();
        if (F.n <= minCoarse)
            break;
        std::vector<int> map;
        int nc = 0;
        if (attempt == 0)
            greedyAggregate(F, map, nc);
        else
            rowRelativeAggregate(F, map, nc);
        if (nc == 0 || nc >= F.n)
            break;
        // prolongation: smoothed aggregation on the reference-rule hierarchy (the
        // tentative piecewise-constant P smoothed by one damped Jacobi step of the
        // filtered geometric matrix), the tentative P itself on the fallback
        const Prolong P = attempt == 0 ? smoothedProlongation(F, map, nc, kProlongWeight)
                                       : smoothedProlongation(F, map, nc, 0.0);
        // coarse pattern and values P^T A P, and per coarse entry the weighted fine
        // entries it sums, both in one fixed order: fine rows ascending, each row's
        // entries in column order, then P's entries of the row and of the column
        std::vector<std::map<int, double>> rows(nc);
        std::vector<std::map<int, std::vector<std::pair<int, double>>>> terms(nc);
        for (int i = 0; i < F.n; ++i)
            for (int k = F.ptr[i]; k < F.ptr[i + 1]; ++k) {
                const int j = F.col[k];
                for (int a = P.ptr[i]; a < P.ptr[i + 1]; ++a)
                    for (int b = P.ptr[j]; b < P.ptr[j + 1]; ++b) {
                        const double w = P.val[a] * P.val[b];
                        rows[P.col[a]][P.col[b]] += w * F.val[k];
                        terms[P.col[a]][P.col[b]].push_back({l == 0 ? slot[k] : k, w});
                    }
            }
        Csr Cm;
        Cm.n = nc;
        Cm.ptr.assign(nc + 1, 0);
        Cm.dg.assign(nc, 0.0);
        for (int I = 0; I < nc; ++I) {
            for (auto &e : rows[I]) {
                Cm.col.push_back(e.first);
                Cm.val.push_back(e.second);
                if (e.first == I)
                    Cm.dg[I] = e.second;
            }
            Cm.ptr[I + 1] = static_cast<int>(Cm.col.size());
        }
        AmgHost::Level L;
        L.n = F.n;
        if (l > 0) {
            L.ptr = F.ptr;
            L.col = F.col;
            L.diagPos.resize(F.n);
            for (int i = 0; i < F.n; ++i)
                L.diagPos[i] = F.find(i, i);
        }
        L.pPtr = P.ptr;
        L.pCol = P.col;
        L.pVal = P.val;
        // restriction R = P^T: coarse row -> (fine row, weight), fine rows ascending
        L.rPtr.assign(nc + 1, 0);
        for (int c : P.col)
            ++L.rPtr[c + 1];
        for (int I = 0; I < nc; ++I)
            L.rPtr[I + 1] += L.rPtr[I];
        L.rCol.resize(P.col.size());
        L.rVal.resize(P.col.size());
        {
            std::vector<int> fill(L.rPtr.begin(), L.rPtr.end() - 1);
            for (int i = 0; i < F.n; ++i)
                for (int a = P.ptr[i]; a < P.ptr[i + 1]; ++a) {
                    const int t = fill[P.col[a]]++;
                    L.rCol[t] = i;
                    L.rVal[t] = P.val[a];
                }
        }
        // gather lists in the coarse CSR order (fine entry id: level 0 -> slot, else nnz)
        const int cnnz = static_cast<int>(Cm.col.size());
        L.gPtr.assign(cnnz + 1, 0);
        for (int I = 0, e = 0; I < nc; ++I)
            for (auto &t : terms[I]) {
                for (auto &sw : t.second) {
                    L.gSrc.push_back(sw.first);
                    L.gW.push_back(sw.second);
                }
                L.gPtr[e + 1] = static_cast<int>(L.gSrc.size());
                ++e;
            }
        h.lev.push_back(std::move(L));
        mats.push_back(std::move(Cm));
    }
    // the coarsest level (dense on the device)
    AmgHost::Level last;
    const Csr &Cl = mats.back();
    last.n = Cl.n;
    if (mats.size() > 1) {
        last.ptr = Cl.ptr;
        last.col = Cl.col;
        last.diagPos.resize(Cl.n);
        for (int i = 0; i < Cl.n; ++i)
            last.diagPos[i] = Cl.find(i, i);
    }
    h.lev.push_back(std::move(last));
    if (attempt == 1) {
        h.w = 0.75;
        h.alpha = 1.7;
        h.sweeps = 2;
    }
    if (h.coarseN() <= minCoarse)
        break;
    }
    return h;
}

// ------------------------------------------------------------------ probes
namespace {
// neighbour across face code k of cell c: returns the neighbour cell (or -1 on
// a wall) and the face's outward normal / centre seen from c and the shift
// that maps a point into the neighbour's frame.
struct FaceView {
    int nb;
    double nxv, nyv, fx, fy, area, toNbShift;
};
FaceView faceView(const StructMesh &m, int c, int code) {
    const int nx = m.nx, ny = m.ny, i = c % nx, j = c / nx;
    FaceView v{};
    if (code == 1) { // east: c is owner
        v.nb = j * nx + (i + 1) % nx;
        v.nxv = m.xnx[c];
        v.nyv = m.xny[c];
        v.fx = m.xfx[c];
        v.fy = m.xfy[c];
        v.area = m.xa[c];
        v.toNbShift = -m.xsh[c];
    } else if (code == 0) { // west: c is the neighbour of cell W's east face
        const int W = j * nx + (i + nx - 1) % nx;
        v.nb = W;
        v.nxv = m.xnx[W] * -1.0;
        v.nyv = m.xny[W] * -1.0;
        v.fx = m.xfx[W] - m.xsh[W];
        v.fy = m.xfy[W];
        v.area = m.xa[W];
        v.toNbShift = m.xsh[W];
    } else if (code == 3) { // north: owner when internal or top wall
        const int f = c + nx;
        v.nb = (j == ny - 1) ? -1 : c + nx;
        v.nxv = m.ynx[f];
        v.nyv = m.yny[f];
        v.fx = m.yfx[f];
        v.fy = m.yfy[f];
        v.area = m.ya[f];
    } else { // south: neighbour of an internal face, owner of the bottom wall
        const int f = c;
        if (j == 0) {
            v.nb = -1;
            v.nxv = m.ynx[f];
            v.nyv = m.yny[f];
        } else {
            v.nb = c - nx;
            v.nxv = m.ynx[f] * -1.0;
            v.nyv = m.yny[f] * -1.0;
        }
        v.fx = m.yfx[f];
        v.fy = m.yfy[f];
        v.area = m.ya[f];
    }
    return v;
}

int nearestCell(const StructMesh &m, double x, double y) {
    int best = 0;
    double bd = 1e30;
    for (int c = 0; c < m.n; ++c) {
        const double dx = m.cx[c] - x, dy = m.cy[c] - y;
        const double d = dx * dx + dy * dy;
        if (d < bd) {
            bd = d;
            best = c;
        }
    }
    return best;
}
} // namespace

ProbeHost prepareProbe(const StructMesh &m, double x, double y) {
    int c = nearestCell(m, x, y);
    double lx = x, ly = y;
    bool inside = false;
    const int maxSteps = 2 * m.n + 10;
    for (int step = 0; step < maxSteps; ++step) { // containing-cell walk
        double worst = 0.0;
        int cross = -1;
        int order[4];
        const int nf = cellFaceOrder(m, c, order);
        for (int k = 0; k < nf; ++k) {
            const FaceView v = faceView(m, c, order[k]);
            const double out = (lx - v.fx) * v.nxv + (ly - v.fy) * v.nyv;
            if (out > worst + 1e-12 * std::sqrt(v.area)) {
                worst = out;
                cross = order[k];
            }
        }
        if (cross < 0) {
            inside = true;
            break;
        }
        const FaceView v = faceView(m, c, cross);
        if (v.nb < 0) {
            inside = true;
            break;
        }
        lx = lx + v.toNbShift;
        c = v.nb;
    }
    if (!inside) {
        c = nearestCell(m, x, y);
        lx = x;
        ly = y;
    }
    ProbeHost p;
    p.cell = c;
    p.ox = lx - m.cx[c];
    p.oy = ly - m.cy[c];
    int order[4];
    const int nf = cellFaceOrder(m, c, order);
    for (int k = 0; k < nf; ++k) {
        const int code = order[k];
        const FaceView v = faceView(m, c, code);
        double dx, dy;
        if (v.nb < 0) {
            dx = v.fx - m.cx[c];
            dy = v.fy - m.cy[c];
        } else {
            dx = m.cx[v.nb] - v.toNbShift - m.cx[c];
            dy = m.cy[v.nb] - m.cy[c];
        }
        const double wt = 1.0 / std::max(dx * dx + dy * dy, 1e-300);
        p.axx += wt * dx * dx;
        p.axy += wt * dx * dy;
        p.ayy += wt * dy * dy;
        p.nb[k] = v.nb;
        p.dx[k] = dx;
        p.dy[k] = dy;
        p.wt[k] = wt;
    }
    p.nnb = nf;
    p.det = p.axx * p.ayy - p.axy * p.axy;
    return p;
}

} // namespace rq
