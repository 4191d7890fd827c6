// Internal to the C ABI implementation (rq_capi.cu, rq_serve_capi.cu,
// rq_linear_capi.cu): error plumbing, device buffers, the mesh-class handle and
// the launch helpers the entry points share. Not part of the public interface.
#pragma once
#include "../../include/rq_b200.h"
#include "rq_device.cuh"
#include "rq_kernels.h"
#include "rq_lin.cuh"
#include "rq_linsys.h"
#include "rq_setup.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace rqc {

extern thread_local std::string g_error; // the calling thread's last failure (rq_capi.cu)

struct RqError : std::runtime_error {
    int code;
    RqError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        throw RqError(RQ_E_OOM, std::string(what) + ": " + cudaGetErrorString(e));
    if (e != cudaSuccess)
        throw RqError(RQ_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F> int guarded(F &&f) {
    try {
        f();
        return RQ_OK;
    } catch (const RqError &e) {
        g_error = e.what();
        return e.code;
    } catch (const std::invalid_argument &e) {
        g_error = e.what();
        return RQ_E_INVALID;
    } catch (const std::bad_alloc &e) {
        g_error = "host allocation failed";
        return RQ_E_OOM;
    } catch (const std::exception &e) {
        g_error = e.what();
        return RQ_E_CUDA;
    }
}

// device allocation that frees itself
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void ensure(size_t b) {
        if (b <= bytes)
            return;
        release();
        check(cudaMalloc(&p, b), "cudaMalloc");
        bytes = b;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// The reference's parameter bounds (core/include/InferenceParameters.hpp:147-165).
inline const double kLower[11] = {0.1, 0.1, 0.01, 0.1, 0.1, 0.1, 0.01, 0.1, 0.01, 0.1, 0.35};
inline const double kUpper[11] = {2.0, 2.0, 0.2, 1.5, 2.0, 2.0, 0.2, 1.5, 0.2, 0.8, 0.50};

inline long pad32(long n) { return (n + 31) / 32 * 32; }

} // namespace rqc

struct rq_problem {
    int device = -1;         // CUDA device ordinal the class lives on (current at create)
    double *noallocScratch = nullptr; // device address of the fixed scratch array on `device`
    rq::StructMesh mesh;
    rq::AmgHost amg;
    rq::DevClass cls{};      // host copy with device pointers
    rqc::DevBuf dCls, dDoubles, dInts;
    std::vector<int32_t> active;
    double base[11];
    int32_t nObs = 0;
    int block = 512; // CTA size of this class's launches
    int arenaKb = -1; // shared-memory arena per CTA in KiB: -1 = the default rule, 0 = none
    cudaStream_t stream = nullptr; // for concurrent per-class launches of a multi-class batch
    cudaEvent_t done = nullptr;
    ~rq_problem() {
        if (done)
            cudaEventDestroy(done);
        if (stream)
            cudaStreamDestroy(stream);
    }
    // launch scratch, reused across calls
    rqc::DevBuf dWs, dJobs, dRows, dPred, dFields, dHist, dTheta, dCounter, dClock;
    std::mutex mu;
};

namespace rqc {
// The calling thread's current device must be the one a handle was created on: every
// device pointer behind the handle belongs to that device.
inline void requireDevice(int device, const char *what) {
    int cur = -1;
    check(cudaGetDevice(&cur), "cudaGetDevice");
    if (cur != device)
        throw std::invalid_argument(std::string(what) + " was created on CUDA device " +
                                    std::to_string(device) + " but the current device is " +
                                    std::to_string(cur) + "; call cudaSetDevice first");
}
inline void requireDevice(const rq_problem &p) { requireDevice(p.device, "this problem"); }
// Makes a handle's device current for the scope (destroy paths), then restores.
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess)
            prev = -1;
        if (device >= 0 && device != prev)
            cudaSetDevice(device);
    }
    ~DeviceScope() {
        if (prev >= 0)
            cudaSetDevice(prev);
    }
};
// one job on the problem's own workspace: a grid of one CTA of the class's size, the
// arena the batch path would give the class, queued on the legacy stream and finished
// by the time the caller copies results back (the problem's mutex held by the caller)
void runOneJob(rq_problem &p, const rq::DevJob &job);
int maxSmemOptin();
// shared-memory arena (doubles) of a launch of these classes
int arenaDoublesFor(long wsDoubles, int knobKb, int nmax);
int chooseArena(const std::vector<const rq_problem *> &probs);
inline rq_row_out toRow(const rq::RowOut &o) {
    return rq_row_out{o.status, o.iterations, o.stalled, o.converged, o.loglik, o.finalWorst,
                      o.contractionRate};
}
} // namespace rqc
