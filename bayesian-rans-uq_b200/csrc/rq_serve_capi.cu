// C ABI of the serving loop (rq_server_*): a request queue in pinned host
// memory mapped into the device, drained by the persistent serveKernel
// (rq_solver.cu) while the host keeps appending to it.
#include "rq_capi_common.h"

using namespace rqc;

namespace {
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
    int device = -1; // CUDA device of the server's classes, slots and launches
    std::vector<rq_problem *> problems;
    // every slot runs 512 threads whatever the classes' own CTA sizes, so a request's
    // result does not depend on which other classes the server holds (a batch of a
    // class above 1024 cells runs 768 threads; its served requests agree to rounding)
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


extern "C" {
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
        check(cudaGetDevice(&S->device), "cudaGetDevice");
        std::vector<const rq_problem *> cp;
        long ws = 0;
        for (int i = 0; i < n_problems; ++i) {
            if (!problems[i])
                throw std::invalid_argument("null problem");
            requireDevice(*problems[i]);
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
        DeviceScope on(s->device); // a relaunch goes to the server's device
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
        j.warm = nullptr; // served requests start cold, as batch rows do
        j.warmBeta = 0.0;
        j.snap = nullptr;
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
        DeviceScope on(s->device);
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
                DeviceScope on(s->device);
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
    return guarded([&] {
        if (!s)
            return;
        DeviceScope on(s->device);
        delete s;
    });
}

} // extern "C"
