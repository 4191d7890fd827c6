// C ABI of the serving loop (rq_server_*): a request queue in pinned host
// memory mapped into the device, drained by the persistent serveKernel
// (rq_solver.cu) while the host keeps appending to it. Solve workspaces come from
// one device pool: a request is admitted (published to the kernel) once its mesh
// class's workspace fits in the pool, and its region returns to the pool when its
// solve retires.
#include "rq_capi_common.h"

#include <map>

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

// First-fit allocator over one device pool, in 256-byte units; free regions are
// kept by offset and merged with their neighbours when a region returns.
struct PoolAllocator {
    size_t total = 0;
    std::map<size_t, size_t> freeList; // offset -> length
    size_t used = 0;
    void reset(size_t bytes) {
        total = bytes;
        freeList.clear();
        if (bytes)
            freeList[0] = bytes;
        used = 0;
    }
    static size_t round(size_t b) { return (b + 255) / 256 * 256; }
    bool take(size_t bytes, size_t &off) {
        bytes = round(bytes);
        for (auto it = freeList.begin(); it != freeList.end(); ++it)
            if (it->second >= bytes) {
                off = it->first;
                const size_t rest = it->second - bytes;
                freeList.erase(it);
                if (rest)
                    freeList[off + bytes] = rest;
                used += bytes;
                return true;
            }
        return false;
    }
    void give(size_t off, size_t bytes) {
        bytes = round(bytes);
        used -= bytes;
        auto next = freeList.lower_bound(off);
        size_t start = off, len = bytes;
        if (next != freeList.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                start = prev->first;
                len += prev->second;
                freeList.erase(prev);
            }
        }
        if (next != freeList.end() && off + bytes == next->first) {
            len += next->second;
            freeList.erase(next);
        }
        freeList[start] = len;
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
    long long idleNs = 0;
    MappedBuf host; // jobs | theta | rows | predictions | clocks | done | published | closed
    rq::DevJob *jobs = nullptr;
    double *theta = nullptr, *pred = nullptr;
    rq::RowOut *rows = nullptr;
    long long *clock = nullptr;
    int *done = nullptr, *published = nullptr, *closed = nullptr;
    DevBuf dCtl;  // head (next request to claim) and the CTA exit counter
    DevBuf dPool; // solve workspaces of admitted requests
    PoolAllocator pool;
    std::vector<size_t> regionOff, regionLen; // per ticket (len 0: none / returned)
    std::vector<int> problemOf;               // per ticket
    int submitted = 0, nPublished = 0, reaped = 0;
    // launches: CTAs launched in total, kernel launches, and a ring of streams so that
    // a top-up launch runs beside CTAs still in long solves
    static constexpr int kStreams = 4;
    cudaStream_t streams[kStreams] = {};
    cudaStream_t side = nullptr; // for reading the device counters
    int ringNext = 0, launches = 0;
    long long launchedCtas = 0;
    int lastRunning = 0;
    std::chrono::steady_clock::time_point lastCheck{};
    std::mutex mu;
    ~rq_server() {
        if (closed)
            __atomic_store_n(closed, 2, __ATOMIC_RELEASE); // cancel what is not yet claimed
        for (cudaStream_t &st : streams)
            if (st) {
                cudaStreamSynchronize(st); // in-flight solves finish first
                cudaStreamDestroy(st);
            }
        if (side)
            cudaStreamDestroy(side);
    }
    rq::ServeQueue queue() const {
        rq::ServeQueue q{};
        q.jobs = jobs;
        q.published = published;
        q.closed = closed;
        q.done = done;
        q.head = dCtl.as<int>();
        q.exits = dCtl.as<int>() + 1;
        q.capacity = capacity;
        q.idleNs = idleNs;
        return q;
    }
    void launch(int ctas) {
        cudaStream_t st = streams[ringNext];
        ringNext = (ringNext + 1) % kStreams;
        check(rq::launchServe(queue(), nullptr, 0, ctas, block, arena, st), "serve launch");
        ++launches;
        launchedCtas += ctas;
    }
    size_t wsBytes(int problem) const {
        return sizeof(double) * static_cast<size_t>(problems[problem]->cls.wsDoubles);
    }
    // Returns the pool regions of finished requests, then admits waiting requests in
    // submission order while their workspaces fit.
    void reapAndAdmit() {
        for (int t = reaped; t < nPublished; ++t)
            if (regionLen[t] && __atomic_load_n(done + t, __ATOMIC_ACQUIRE)) {
                pool.give(regionOff[t], regionLen[t]);
                regionLen[t] = 0;
            }
        while (reaped < nPublished && !regionLen[reaped])
            ++reaped;
        while (nPublished < submitted) {
            const int t = nPublished;
            size_t off = 0;
            if (!pool.take(wsBytes(problemOf[t]), off))
                break;
            regionOff[t] = off;
            regionLen[t] = wsBytes(problemOf[t]);
            jobs[t].ws = reinterpret_cast<double *>(static_cast<char *>(dPool.p) + off);
            nPublished = t + 1;
            __atomic_store_n(published, nPublished, __ATOMIC_RELEASE);
        }
    }
    // Keeps enough CTAs running: when published requests wait to be claimed and fewer
    // CTAs than slots are alive (some left after the idle timeout, possibly while
    // others still run long solves), launch the difference beside them. The device
    // counters are read at most every 200 us.
    void ensureRunning(bool force = false) {
        reapAndAdmit();
        bool pending = false;
        for (int i = reaped; i < nPublished && !pending; ++i)
            pending = !__atomic_load_n(done + i, __ATOMIC_ACQUIRE);
        if (!pending)
            return;
        const auto now = std::chrono::steady_clock::now();
        if (!force && now - lastCheck < std::chrono::microseconds(200))
            return;
        lastCheck = now;
        int ctl[2] = {0, 0}; // head, exits
        check(cudaMemcpyAsync(ctl, dCtl.p, sizeof(ctl), cudaMemcpyDeviceToHost, side), "counters");
        check(cudaStreamSynchronize(side), "counters");
        const long long running = launchedCtas - ctl[1];
        lastRunning = static_cast<int>(running);
        const int unclaimed = nPublished - ctl[0];
        if (unclaimed > 0 && running < grid)
            launch(static_cast<int>(std::min<long long>(grid - running, unclaimed)));
    }
};

namespace {
rq_server *createServer(rq_problem *const *problems, int32_t n_problems, int32_t capacity,
                        double idle_timeout_s, int32_t max_slots, uint64_t pool_bytes) {
    if (!problems || n_problems < 1)
        throw std::invalid_argument("null argument");
    if (capacity < 1)
        throw std::invalid_argument("server capacity must be positive");
    if (!std::isfinite(idle_timeout_s) || idle_timeout_s <= 0 || idle_timeout_s > 600)
        throw std::invalid_argument("idle timeout must be in (0, 600] seconds");
    if (max_slots < 0)
        throw std::invalid_argument("max_slots must be nonnegative");
    auto S = std::make_unique<rq_server>();
    check(cudaGetDevice(&S->device), "cudaGetDevice");
    std::vector<const rq_problem *> cp;
    size_t wsMax = 0;
    for (int i = 0; i < n_problems; ++i) {
        if (!problems[i])
            throw std::invalid_argument("null problem");
        requireDevice(*problems[i]);
        S->problems.push_back(problems[i]);
        cp.push_back(problems[i]);
        S->thetaStride = std::max<int>(S->thetaStride, static_cast<int>(problems[i]->active.size()));
        S->predStride = std::max(S->predStride, problems[i]->nObs);
        wsMax = std::max(wsMax, S->wsBytes(i));
    }
    S->capacity = capacity;
    S->idleNs = static_cast<long long>(idle_timeout_s * 1e9);
    S->arena = chooseArena(cp);
    int dev = 0, sms = 1;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
    const int perSM = rq::serveBlocksPerSM(S->block, S->arena);
    if (perSM < 1)
        throw RqError(RQ_E_CUDA, "serve kernel does not fit on an SM with this arena");
    long slots = static_cast<long>(sms) * perSM;
    if (max_slots > 0)
        slots = std::min<long>(slots, max_slots);
    S->grid = static_cast<int>(slots);
    // the workspace pool: admission of requests is by free space in it
    size_t freeB = 0, totalB = 0;
    check(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo");
    size_t poolB = pool_bytes ? static_cast<size_t>(pool_bytes)
                              : static_cast<size_t>(0.8 * static_cast<double>(freeB));
    // never more than the slots can use at once
    poolB = std::min(poolB, PoolAllocator::round(wsMax) * static_cast<size_t>(slots));
    if (poolB < PoolAllocator::round(wsMax))
        throw RqError(RQ_E_OOM, "the workspace pool holds no solve of the largest class (" +
                                    std::to_string(wsMax) + " bytes)");
    poolB = poolB / 256 * 256;
    S->dPool.ensure(poolB);
    S->pool.reset(poolB);
    S->dCtl.ensure(2 * sizeof(int));
    check(cudaMemset(S->dCtl.p, 0, 2 * sizeof(int)), "server counters");
    const size_t c = static_cast<size_t>(capacity);
    S->regionOff.assign(c, 0);
    S->regionLen.assign(c, 0);
    S->problemOf.assign(c, 0);
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
    for (cudaStream_t &st : S->streams)
        check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
    check(cudaStreamCreateWithFlags(&S->side, cudaStreamNonBlocking), "stream");
    check(cudaDeviceSynchronize(), "server set-up");
    S->launch(S->grid);
    return S.release();
}
} // namespace

extern "C" {
int rq_server_create(rq_problem *const *problems, int32_t n_problems, int32_t capacity,
                     double idle_timeout_s, int32_t max_slots, rq_server **out) {
    return guarded([&] {
        if (!out)
            throw std::invalid_argument("null argument");
        *out = nullptr;
        *out = createServer(problems, n_problems, capacity, idle_timeout_s, max_slots, 0);
    });
}

int rq_server_create_pooled(rq_problem *const *problems, int32_t n_problems, int32_t capacity,
                            double idle_timeout_s, int32_t max_slots, uint64_t pool_bytes,
                            rq_server **out) {
    return guarded([&] {
        if (!out)
            throw std::invalid_argument("null argument");
        *out = nullptr;
        *out = createServer(problems, n_problems, capacity, idle_timeout_s, max_slots,
                            pool_bytes);
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
        if (PoolAllocator::round(s->wsBytes(problem)) > s->pool.total)
            throw RqError(RQ_E_OOM, "this class's solve workspace exceeds the server's pool");
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
        j.ws = nullptr; // set on admission
        s->problemOf[t] = problem;
        s->submitted = t + 1;
        s->ensureRunning(true);
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
        *done = ticket < s->nPublished && __atomic_load_n(s->done + ticket, __ATOMIC_ACQUIRE) ? 1 : 0;
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
                for (int i = 0; i < s->nPublished; ++i)
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
            for (int i = 0; i < s->nPublished; ++i)
                n += __atomic_load_n(s->done + i, __ATOMIC_ACQUIRE) ? 1 : 0;
            *completed = n;
        }
        if (launches)
            *launches = s->launches;
    });
}

int rq_server_memory(rq_server *s, uint64_t *pool_bytes, uint64_t *in_use_bytes,
                     int64_t *waiting, int32_t *running_ctas) {
    return guarded([&] {
        if (!s)
            throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> lock(s->mu);
        DeviceScope on(s->device);
        s->reapAndAdmit();
        if (pool_bytes)
            *pool_bytes = s->pool.total;
        if (in_use_bytes)
            *in_use_bytes = s->pool.used;
        if (waiting)
            *waiting = s->submitted - s->nPublished;
        if (running_ctas) {
            int ctl[2] = {0, 0};
            check(cudaMemcpyAsync(ctl, s->dCtl.p, sizeof(ctl), cudaMemcpyDeviceToHost, s->side),
                  "counters");
            check(cudaStreamSynchronize(s->side), "counters");
            *running_ctas = static_cast<int32_t>(s->launchedCtas - ctl[1]);
        }
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
