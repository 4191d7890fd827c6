// C ABI: the sequential forward model with its warm-start cache.
//
// WarmStartCache (rans-uq/include/ForwardModel.hpp:21-157) keeps converged
// states keyed by theta; ForwardModel::evaluateWithDiagnostics
// (rans-uq/src/ForwardModel.cpp:35-137) looks the nearest one up after the
// bounds check, solves from it instead of the uniform state, and stores the
// state of a Converged solve. Here every cached state stays in device memory in
// the fields layout (11 x n), and the solve reads it directly: one job, one CTA,
// whose final state lands in a staging buffer that becomes the new entry by a
// pointer move (no copy, no host round trip). The cache's byte count is the
// reference's own payload count, so entries are evicted after the same calls.
#include "rq_capi_common.h"

#include <deque>

using namespace rqc;

struct rq_warm_cache {
    struct Entry {
        std::vector<double> theta;
        std::unique_ptr<DevBuf> state; // 11 x n doubles, fields layout
        double beta1 = 0.0;            // the solve's beta1: its wall-face omega
        size_t bytes = 0;
    };
    rq_problem *p = nullptr;
    int maxSize = 50;
    double threshold = 0.5;
    size_t budget = 64u << 20, retained = 0;
    std::deque<Entry> q; // front = oldest
    std::unique_ptr<DevBuf> staging;
    DevBuf dSnap;
    std::mutex mu;

    // entryBytes (ForwardModel.hpp:39-47): theta, Vec3 over cells + boundary faces,
    // and p, k, omega, nuT, F1, F2, Pk, CDkw over the same
    size_t entryBytes(size_t nTheta) const {
        const size_t cb = static_cast<size_t>(p->mesh.n) + 2u * static_cast<size_t>(p->mesh.nx);
        return nTheta * sizeof(double) + cb * 3 * sizeof(double) + 8 * cb * sizeof(double);
    }
    void evictFront() {
        retained -= q.front().bytes;
        q.pop_front();
    }
    // nearest (:132-144): strictly closer than the threshold, the first of equals wins
    const Entry *nearest(const std::vector<double> &theta) const {
        const Entry *best = nullptr;
        double bestDist = threshold;
        for (const Entry &e : q) {
            double d = std::numeric_limits<double>::infinity();
            if (e.theta.size() == theta.size()) {
                double s = 0.0;
                for (size_t i = 0; i < theta.size(); ++i) {
                    const double t = theta[i] - e.theta[i];
                    s += t * t;
                }
                d = std::sqrt(s);
            }
            if (d < bestDist) {
                bestDist = d;
                best = &e;
            }
        }
        return best;
    }
    // store (:70-92), taking the staging buffer as the entry's state
    void store(const std::vector<double> &theta, double beta1) {
        for (double v : theta)
            if (!std::isfinite(v))
                return;
        for (auto it = q.begin(); it != q.end(); ++it)
            if (it->theta == theta) {
                retained -= it->bytes;
                q.erase(it);
                break;
            }
        const size_t bytes = entryBytes(theta.size());
        if (maxSize == 0 || bytes > budget)
            return;
        while (!q.empty() && (q.size() >= static_cast<size_t>(maxSize) || retained > budget - bytes))
            evictFront();
        q.push_back(Entry{theta, std::move(staging), beta1, bytes});
        retained += bytes;
    }
};

namespace {

// OwnedFlowSnapshot (ForwardModel.hpp:162-186) from the device's final state. Boundary
// values follow the reference's boundary conditions on these all-wall periodic meshes
// (BoundaryCondition.hpp:279-384 via applyAllBCs and the per-iteration updates): U and k
// are zero at the walls, p takes the owner cell's value (zero gradient), omega_b =
// 60 nu / (beta1 y1^2) with the beta1 it was last set with; nuT, Pk and CDkw keep the
// boundary value 0 and F1, F2 the value 1 that initUniform gives them (no later step
// writes them). Face fluxes are reordered from the device layout (x faces c = j nx + i,
// y faces g = jf nx + i) into the generator's face order (Mesh.cpp:646-720): vertical
// internal faces by row, the wrap faces, horizontal internal faces by row, bottom wall,
// top wall.
void writeSnapshot(const rq_problem &P, const double *dFields, const double *dSnap,
                   double *boundary, double *faceFluxes, int32_t *turbEstablished) {
    const rq::StructMesh &m = P.mesh;
    const int nx = m.nx, ny = m.ny, n = m.n, nfy = m.nfy(), nb = 2 * nx;
    std::vector<double> snap(static_cast<size_t>(n) + nfy + 2);
    check(cudaMemcpy(snap.data(), dSnap, sizeof(double) * snap.size(), cudaMemcpyDeviceToHost),
          "snapshot");
    if (turbEstablished)
        *turbEstablished = snap[n + nfy + 1] != 0.0;
    if (boundary) {
        std::vector<double> pc(n);
        check(cudaMemcpy(pc.data(), dFields + 3L * n, sizeof(double) * n, cudaMemcpyDeviceToHost),
              "pressure");
        const double beta = snap[n + nfy];
        const double fill[11] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0};
        for (int b = 0; b < 11; ++b)
            for (int f = 0; f < nb; ++f)
                boundary[static_cast<long>(b) * nb + f] = fill[b];
        for (int f = 0; f < nb; ++f) {
            const int i = f % nx;
            const int owner = f < nx ? i : (ny - 1) * nx + i;
            const int g = f < nx ? i : ny * nx + i; // the wall's y face
            boundary[3L * nb + f] = pc[owner];
            const double y1 = std::max(m.ydl[g], 1e-20);
            boundary[5L * nb + f] = 60.0 * P.cls.nu / (beta * y1 * y1);
        }
    }
    if (faceFluxes) {
        long k = 0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx - 1; ++i)
                faceFluxes[k++] = snap[j * nx + i];
        for (int j = 0; j < ny; ++j)
            faceFluxes[k++] = snap[j * nx + nx - 1];
        for (int j = 0; j < ny - 1; ++j)
            for (int i = 0; i < nx; ++i)
                faceFluxes[k++] = snap[n + (j + 1) * nx + i];
        for (int i = 0; i < nx; ++i)
            faceFluxes[k++] = snap[n + i];
        for (int i = 0; i < nx; ++i)
            faceFluxes[k++] = snap[n + ny * nx + i];
    }
}

} // namespace

extern "C" {

int rq_warm_cache_create(rq_problem *p, int32_t max_size, double threshold, uint64_t byte_budget,
                         rq_warm_cache **out) {
    return guarded([&] {
        if (!p || !out)
            throw std::invalid_argument("null argument");
        requireDevice(*p);
        if (max_size < 0 || !std::isfinite(threshold) || threshold < 0)
            throw std::invalid_argument("Invalid warm-start cache limits");
        auto c = std::make_unique<rq_warm_cache>();
        c->p = p;
        c->maxSize = max_size;
        c->threshold = threshold;
        c->budget = static_cast<size_t>(byte_budget);
        *out = c.release();
    });
}

int rq_warm_cache_destroy(rq_warm_cache *c) {
    return guarded([&] {
        if (!c)
            return;
        DeviceScope on(c->p ? c->p->device : -1);
        delete c;
    });
}

int rq_warm_cache_info(rq_warm_cache *c, int32_t *size, uint64_t *retained_bytes,
                       uint64_t *byte_budget) {
    return guarded([&] {
        if (!c)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(c->mu);
        if (size)
            *size = static_cast<int32_t>(c->q.size());
        if (retained_bytes)
            *retained_bytes = c->retained;
        if (byte_budget)
            *byte_budget = c->budget;
    });
}

int rq_warm_cache_clear(rq_warm_cache *c) {
    return guarded([&] {
        if (!c)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(c->mu);
        c->q.clear();
        c->retained = 0;
    });
}

int rq_warm_cache_set_byte_budget(rq_warm_cache *c, uint64_t byte_budget) {
    return guarded([&] {
        if (!c)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(c->mu);
        c->budget = static_cast<size_t>(byte_budget);
        while (!c->q.empty() && c->retained > c->budget)
            c->evictFront();
    });
}

int rq_evaluate_cached(rq_warm_cache *c, const double *theta, rq_row_out *row,
                       double *predictions, double *fields, double *boundary,
                       double *face_fluxes, int32_t *turb_established,
                       int32_t *used_warm_start) {
    return guarded([&] {
        if (!c || !theta || !row)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(c->mu);
        rq_problem *p = c->p;
        requireDevice(*p);
        std::lock_guard<std::mutex> plock(p->mu);
        const int na = static_cast<int>(p->active.size());
        const int nc = p->mesh.n, no = std::max(p->nObs, 1);
        std::vector<double> th(theta, theta + na);
        // InferenceParameterSet::inBounds, as the kernel admits the draw; only an admitted
        // draw looks the cache up (ForwardModel.cpp:49-53 before :79)
        bool admitted = true;
        double coeff[11];
        std::memcpy(coeff, p->base, sizeof(coeff));
        for (int a = 0; a < na; ++a) {
            const int idx = p->active[a];
            const double v = th[a];
            if (v < p->cls.lo[idx] || v > p->cls.hi[idx] || std::isnan(v) || std::isinf(v))
                admitted = false;
            coeff[idx] = v;
        }
        const rq_warm_cache::Entry *hit = admitted ? c->nearest(th) : nullptr;
        if (!c->staging)
            c->staging = std::make_unique<DevBuf>();
        c->staging->ensure(sizeof(double) * 11L * nc);
        const bool wantSnap = boundary || face_fluxes || turb_established;
        const long nSnap = static_cast<long>(nc) + p->mesh.nfy() + 2;
        if (wantSnap)
            c->dSnap.ensure(sizeof(double) * nSnap);
        p->dTheta.ensure(sizeof(double) * std::max(na, 1));
        p->dRows.ensure(sizeof(rq::RowOut));
        p->dPred.ensure(sizeof(double) * no);
        check(cudaMemcpy(p->dTheta.p, th.data(), sizeof(double) * na, cudaMemcpyHostToDevice), "theta");
        rq::DevJob j{};
        j.cls = p->dCls.as<rq::DevClass>();
        j.theta = p->dTheta.as<double>();
        j.row = p->dRows.as<rq::RowOut>();
        j.pred = p->dPred.as<double>();
        j.fields = c->staging->as<double>();
        j.warm = hit ? hit->state->as<double>() : nullptr;
        j.warmBeta = hit ? hit->beta1 : 0.0;
        j.snap = wantSnap ? c->dSnap.as<double>() : nullptr;
        runOneJob(*p, j);
        rq::RowOut o;
        check(cudaMemcpy(&o, p->dRows.p, sizeof(o), cudaMemcpyDeviceToHost), "row");
        *row = toRow(o);
        if (used_warm_start)
            *used_warm_start = hit != nullptr;
        if (predictions && p->nObs > 0)
            check(cudaMemcpy(predictions, p->dPred.p, sizeof(double) * p->nObs,
                             cudaMemcpyDeviceToHost), "predictions");
        const bool solved = o.status == RQ_CONVERGED || o.status == RQ_UNCONVERGED;
        if (fields && solved)
            check(cudaMemcpy(fields, c->staging->p, sizeof(double) * 11L * nc,
                             cudaMemcpyDeviceToHost), "fields");
        else if (fields) // no state to report (the reference keeps no fields either)
            std::fill(fields, fields + 11L * nc, std::numeric_limits<double>::quiet_NaN());
        if (wantSnap && solved)
            writeSnapshot(*p, c->staging->as<double>(), c->dSnap.as<double>(), boundary,
                          face_fluxes, turb_established);
        // a Converged verdict (finite predictions and likelihood included) seeds the cache
        // (ForwardModel.cpp:114-117)
        if (o.status == RQ_CONVERGED)
            c->store(th, coeff[2]);
    });
}

} // extern "C"
