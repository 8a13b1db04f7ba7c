// Host runtime shared by the three domain handles: errors, device buffers, the per-handle
// stream and CUDA graphs of N steps, and the device state that carries the ledger and audit.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pantometry_gpu.h"
#include "launch.h"

namespace pm {

void set_error(const std::string& msg);
pm_status fail(pm_status s, const std::string& msg);
pm_status cuda_fail(cudaError_t e, const char* what);

#define PM_CUDA(call)                                       \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// One device allocation.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n) {
        release();
        if (n == 0) n = 16;
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        else p = nullptr;
        return e;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// What every handle carries: its device, its stream, its device state and partials, and the
// cached graphs of G steps (one per ping-pong parity, rebuilt when the step size changes).
// The sample grid of a pm_*_sample call: lo, hi in metres, samples per axis, `n` values in `out`.
pm_status sample_grid_of(const double* lo, const double* hi, const int* samples, const double* out, size_t n,
                         SampleGrid& g);
// Run `launch` into the handle's sample buffer, then copy the n samples to `out` (host).
template <typename H, typename F>
pm_status run_sample(H* h, double* out, size_t n, F launch) {
    if (!h->sampled.p || h->sampled.bytes < n * 8) PM_CUDA(h->sampled.alloc(n * 8));
    PM_CUDA(launch(h->sampled.template as<double>(), h->stream()));
    PM_CUDA(cudaMemcpyAsync(out, h->sampled.p, n * 8, cudaMemcpyDeviceToHost, h->stream()));
    PM_CUDA(cudaStreamSynchronize(h->stream()));
    return PM_OK;
}

struct Handle {
    int device = 0;
    std::string name;
    int precision = PM_PLAIN_F64;
    cudaStream_t own = nullptr;
    cudaStream_t user = nullptr;
    cudaStream_t capture = nullptr;
    DBuf state;      // DevState
    DBuf partials;   // per-block partial sums
    DBuf sampled;    // the samples of the last pm_*_sample call
    DevState* host_state = nullptr;  // pinned mirror
    double tolerance = -1.0;         // no audit: plain `Domain::step`; set one to audit every step
    std::string refusal_site;        // where a step refused on the device (kRefused) is reported
    unsigned resident = 148 * kBlocksPerSM;  // upper bound of any persistent grid (partials sizing)
    unsigned sm_count = 148;
    unsigned wave_of(KernelId id) const { return sm_count * (unsigned)blocks_per_sm(id); }
    int parity = 0;                  // which buffer of a ping-pong pair holds the state
    int call_parity = 0;             // parity when the present call began
    // graph cache
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    double graph_dt = NAN;
    int graph_steps = 0;
    // checkpoint
    bool has_saved = false;
    DevState saved_state;

    static constexpr int kGraphSteps = 64;  // even, so a graph leaves the parity unchanged

    cudaStream_t stream() const { return user ? user : own; }
    pm_status init(int dev, size_t partial_doubles);
    void drop_graphs();
    ~Handle();

    // Host → device copy ordered on the handle's stream and complete on return, so the source
    // may be freed at once and every later launch on the stream sees the bytes.
    cudaError_t put_sync(void* dst, const void* src, size_t bytes) {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream());
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream());
        return e;
    }
    pm_status read_state();                    // device → host_state, synchronising
    pm_status write_state();                   // host_state → device
    pm_status begin_call();                    // clear the previous call's violation
    // Run `n` steps with `one(parity)` launching a single step from buffer `parity`.
    // `pingpong`: each step flips the parity.
    template <typename F>
    pm_status run_steps(long long n, double dt, bool pingpong, F one);
    pm_status finish_call(long long steps_before, pm_violation* out, const std::string& audit_site,
                          const std::string& startup_site, bool pingpong);
};

void fill_violation(pm_violation* v, const char* quantity, const std::string& site, double before, double after,
                    double scale, double tol, long long step);

template <typename F>
pm_status Handle::run_steps(long long n, double dt, bool pingpong, F one) {
    cudaStream_t s = stream();
    const int G = kGraphSteps;
    if (n >= G) {
        if (!(graph_dt == dt) || graph_steps != G) {
            drop_graphs();
            for (int par = 0; par < (pingpong ? 2 : 1); ++par) {
                cudaGraph_t g = nullptr;
                PM_CUDA(cudaStreamBeginCapture(capture, cudaStreamCaptureModeThreadLocal));
                int p = par;
                cudaError_t le = cudaSuccess;
                for (int q = 0; q < G && le == cudaSuccess; ++q) {
                    le = one(p, capture);
                    if (pingpong) p ^= 1;
                }
                cudaError_t ce = cudaStreamEndCapture(capture, &g);
                if (le != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(le, "capture launch"); }
                if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
                cudaError_t ie = cudaGraphInstantiate(&graph[par], g, 0);
                cudaGraphDestroy(g);
                if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate");
            }
            graph_dt = dt;
            graph_steps = G;
        }
    }
    while (n > 0) {
        if (n >= G) {
            PM_CUDA(cudaGraphLaunch(graph[pingpong ? parity : 0], s));
            n -= G;
        } else {
            PM_CUDA(one(parity, s));
            if (pingpong) parity ^= 1;
            n -= 1;
        }
    }
    return PM_OK;
}

}  // namespace pm
