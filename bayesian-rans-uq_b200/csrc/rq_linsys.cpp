// Host set-up of standalone LDU systems (see rq_linsys.h).
#include "rq_linsys.h"

#include <algorithm>
#include <cmath>
#include <utility>

namespace rq {

void validateLdu(int n, int nf, const double *diag, const double *upper, const double *lower,
                 const double *source, const int32_t *own, const int32_t *nbr) {
    if (n < 0 || nf < 0)
        throw std::invalid_argument("linear system storage must match its declared dimensions");
    if ((n > 0 && (!diag || !source)) || (nf > 0 && (!upper || !lower || !own || !nbr)))
        throw std::invalid_argument("linear system storage must match its declared dimensions");
    for (int f = 0; f < nf; ++f)
        if (own[f] < 0 || own[f] >= n || nbr[f] < 0 || nbr[f] >= n)
            throw std::invalid_argument("linear system connectivity index is out of range");
    auto finite = [](const double *v, int k) {
        for (int i = 0; i < k; ++i)
            if (!std::isfinite(v[i]))
                return false;
        return true;
    };
    if (!finite(diag, n) || !finite(source, n) || !finite(upper, nf) || !finite(lower, nf))
        throw std::invalid_argument("linear system coefficients and source must be finite");
}

namespace {

double recip(double d) { return std::abs(d) > 1e-30 ? 1.0 / d : 1.0; }

// Column-sorted CSR with the diagonal included (the reference's lduToCSR,
// core/include/LinearSolver.hpp:472-532): the order aggregation walks a row in.
void sortedCsr(int n, int nf, const double *diag, const double *upper, const double *lower,
               const int32_t *own, const int32_t *nbr, std::vector<int> &ptr,
               std::vector<int> &col, std::vector<double> &val) {
    ptr.assign(n + 1, 0);
    for (int i = 0; i < n; ++i)
        ptr[i + 1] = 1;
    for (int f = 0; f < nf; ++f) {
        ++ptr[own[f] + 1];
        ++ptr[nbr[f] + 1];
    }
    for (int i = 0; i < n; ++i)
        ptr[i + 1] += ptr[i];
    col.resize(ptr[n]);
    val.resize(ptr[n]);
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < n; ++i) {
        col[fill[i]] = i;
        val[fill[i]++] = diag[i];
    }
    for (int f = 0; f < nf; ++f) {
        col[fill[own[f]]] = nbr[f];
        val[fill[own[f]]++] = upper[f];
        col[fill[nbr[f]]] = own[f];
        val[fill[nbr[f]]++] = lower[f];
    }
    // stable insertion sort of each short row by column
    for (int i = 0; i < n; ++i)
        for (int a = ptr[i] + 1; a < ptr[i + 1]; ++a) {
            const int kc = col[a];
            const double kv = val[a];
            int b = a - 1;
            while (b >= ptr[i] && col[b] > kc) {
                col[b + 1] = col[b];
                val[b + 1] = val[b];
                --b;
            }
            col[b + 1] = kc;
            val[b + 1] = kv;
        }
}

// Aggregation of a general matrix. The reference's greedy pass
// (core/include/LinearSolver.hpp:535-575) with strength measured against the
// row's largest off-diagonal, |a_ij| >= 0.25 max_k |a_ik| (the reference's
// symmetric scaling |a_ij| / sqrt(a_ii a_jj) > 0.25 leaves most rows of a
// high-contrast matrix unclaimed, and coarsening stalls: a 256 x 256 log-normal
// Poisson system keeps 4309 rows after 12 levels). Seeds claim their
// unaggregated strong neighbours; a seed left alone then joins the aggregate
// of its strongest neighbour, so every aggregate of a connected matrix has at
// least two rows; aggregates are renumbered in order of first appearance.
void aggregateRows(int n, const std::vector<int> &ptr, const std::vector<int> &col,
                   const std::vector<double> &val, std::vector<int> &map, int &nc) {
    map.assign(n, -1);
    int groups = 0;
    for (int i = 0; i < n; ++i) {
        if (map[i] >= 0)
            continue;
        const int g = groups++;
        map[i] = g;
        double rowMax = 0.0;
        for (int k = ptr[i]; k < ptr[i + 1]; ++k)
            if (col[k] != i)
                rowMax = std::max(rowMax, std::abs(val[k]));
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
            const int c = col[k];
            if (c != i && map[c] < 0 && std::abs(val[k]) >= 0.25 * rowMax && rowMax > 0.0)
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
        for (int k = ptr[i]; k < ptr[i + 1]; ++k)
            if (col[k] != i && std::abs(val[k]) > best) {
                best = std::abs(val[k]);
                j = col[k];
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

// In-place Gauss-Jordan inverse of a small SPD matrix, no pivoting: row k is
// scaled by the reciprocal of its pivot, then eliminated from every other row.
bool gaussJordanInverse(int m, std::vector<double> a, std::vector<double> &inv) {
    inv.assign(static_cast<size_t>(m) * m, 0.0);
    for (int i = 0; i < m; ++i)
        inv[static_cast<size_t>(i) * m + i] = 1.0;
    for (int k = 0; k < m; ++k) {
        const double piv = a[static_cast<size_t>(k) * m + k];
        if (!(std::abs(piv) > 1e-300))
            return false;
        const double rp = 1.0 / piv;
        for (int j = 0; j < m; ++j) {
            a[static_cast<size_t>(k) * m + j] *= rp;
            inv[static_cast<size_t>(k) * m + j] *= rp;
        }
        for (int i = 0; i < m; ++i) {
            const double f = a[static_cast<size_t>(i) * m + k];
            if (i == k || f == 0.0)
                continue;
            for (int j = 0; j < m; ++j) {
                a[static_cast<size_t>(i) * m + j] -= f * a[static_cast<size_t>(k) * m + j];
                inv[static_cast<size_t>(i) * m + j] -= f * inv[static_cast<size_t>(k) * m + j];
            }
        }
    }
    return true;
}

} // namespace

LinSysHost buildLinSys(int n, int nf, const double *diag, const double *upper,
                       const double *lower, const int32_t *own, const int32_t *nbr, bool withAmg,
                       int minCoarse, int maxLevels, int maxCoarse) {
    LinSysHost S;
    S.n = n;
    S.nf = nf;
    // level 0 in the reference's matvec order (LinearSystem::matvec,
    // LinearSolver.hpp:99-108): the diagonal, then faces in increasing index
    LinLevelHost L0;
    L0.n = n;
    L0.ptr.assign(n + 1, 0);
    for (int i = 0; i < n; ++i)
        L0.ptr[i + 1] = 1;
    for (int f = 0; f < nf; ++f) {
        ++L0.ptr[own[f] + 1];
        ++L0.ptr[nbr[f] + 1];
    }
    for (int i = 0; i < n; ++i)
        L0.ptr[i + 1] += L0.ptr[i];
    L0.col.resize(L0.ptr[n]);
    L0.val.resize(L0.ptr[n]);
    L0.rdg.resize(n);
    {
        std::vector<int> fill(L0.ptr.begin(), L0.ptr.end() - 1);
        for (int i = 0; i < n; ++i) {
            L0.col[fill[i]] = i;
            L0.val[fill[i]++] = diag[i];
            L0.rdg[i] = recip(diag[i]);
        }
        for (int f = 0; f < nf; ++f) {
            L0.col[fill[own[f]]] = nbr[f];
            L0.val[fill[own[f]]++] = upper[f];
            L0.col[fill[nbr[f]]] = own[f];
            L0.val[fill[nbr[f]]++] = lower[f];
        }
    }
    S.lev.push_back(std::move(L0));
    if (!withAmg)
        return S;

    // the hierarchy walks column-sorted rows
    std::vector<int> ptr, col;
    std::vector<double> val;
    sortedCsr(n, nf, diag, upper, lower, own, nbr, ptr, col, val);
    int cur = n;
    for (int l = 0; l + 1 < maxLevels && cur > minCoarse; ++l) {
        std::vector<int> map;
        int nc = 0;
        aggregateRows(cur, ptr, col, val, map, nc);
        if (nc == 0 || nc >= cur)
            break;
        LinLevelHost &F = S.lev.back();
        F.nc = nc;
        F.agg = map;
        F.childPtr.assign(nc + 1, 0);
        for (int i = 0; i < cur; ++i)
            ++F.childPtr[map[i] + 1];
        for (int I = 0; I < nc; ++I)
            F.childPtr[I + 1] += F.childPtr[I];
        F.childIdx.resize(cur);
        {
            std::vector<int> fill(F.childPtr.begin(), F.childPtr.end() - 1);
            for (int i = 0; i < cur; ++i)
                F.childIdx[fill[map[i]]++] = i;
        }
        // coarse pattern: per coarse row the sorted distinct aggregates its children touch
        LinLevelHost C;
        C.n = nc;
        C.ptr.assign(nc + 1, 0);
        std::vector<int> js;
        for (int I = 0; I < nc; ++I) {
            js.clear();
            for (int t = F.childPtr[I]; t < F.childPtr[I + 1]; ++t) {
                const int i = F.childIdx[t];
                for (int k = ptr[i]; k < ptr[i + 1]; ++k)
                    js.push_back(map[col[k]]);
            }
            std::sort(js.begin(), js.end());
            js.erase(std::unique(js.begin(), js.end()), js.end());
            C.col.insert(C.col.end(), js.begin(), js.end());
            C.ptr[I + 1] = static_cast<int>(C.col.size());
        }
        // Galerkin values summed in fine row order, entries in column order
        // (the reference's galerkinIdx summation, LinearSolver.hpp:578-618, 683-690)
        C.val.assign(C.col.size(), 0.0);
        for (int i = 0; i < cur; ++i) {
            const int I = map[i];
            const auto b = C.col.begin() + C.ptr[I], e = C.col.begin() + C.ptr[I + 1];
            for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
                const int pos = static_cast<int>(std::lower_bound(b, e, map[col[k]]) - C.col.begin());
                C.val[pos] += val[k];
            }
        }
        std::vector<double> cdg(nc, 0.0);
        C.rdg.resize(nc);
        for (int I = 0; I < nc; ++I) {
            for (int k = C.ptr[I]; k < C.ptr[I + 1]; ++k)
                if (C.col[k] == I)
                    cdg[I] = C.val[k];
            C.rdg[I] = recip(cdg[I]);
        }
        ptr = C.ptr;
        col = C.col;
        val = C.val;
        cur = nc;
        S.lev.push_back(std::move(C));
    }
    const LinLevelHost &last = S.lev.back();
    S.m = last.n;
    if (S.m > maxCoarse)
        throw LinUnsupported("AMG coarsening stalled above " + std::to_string(maxCoarse) +
                             " rows; use the PCG or BiCGSTAB solver for this system");
    std::vector<double> dense(static_cast<size_t>(S.m) * S.m, 0.0);
    for (int i = 0; i < S.m; ++i)
        for (int k = ptr[i]; k < ptr[i + 1]; ++k)
            dense[static_cast<size_t>(i) * S.m + col[k]] = val[k];
    if (!gaussJordanInverse(S.m, std::move(dense), S.inv))
        throw LinUnsupported("zero pivot in the coarsest AMG level");
    return S;
}

} // namespace rq
