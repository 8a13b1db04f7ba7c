// Host runtime: the Handle base (stream, graphs, device state, audit readout) and the C ABI's
// status and error functions. The three domains live in heat.cu, hall.cu and cavity.cu.
#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <utility>

#include "runtime.h"

namespace pm {

static thread_local std::string g_error;

int occupancy_f64(KernelId id);
int occupancy_f32(KernelId id);

namespace {
std::mutex g_attr_mutex;
std::map<std::pair<const void*, int>, int> g_smem_opt_in;  // (kernel, device) -> bytes allowed
std::map<std::pair<int, int>, int> g_occupancy;             // (kernel id, device) -> blocks per SM
}  // namespace

cudaError_t allow_smem_fn(const void* kernel, int bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    auto it = g_smem_opt_in.find({kernel, dev});
    if (it != g_smem_opt_in.end() && it->second >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) g_smem_opt_in[{kernel, dev}] = bytes;
    return e;
}

int blocks_per_sm(KernelId id) {
    if (id < 0 || id >= kKernelCount) return 1;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    {
        std::lock_guard<std::mutex> lock(g_attr_mutex);
        auto it = g_occupancy.find({(int)id, dev});
        if (it != g_occupancy.end()) return it->second;
    }
    // asked outside the lock: the occupancy queries take it themselves for the opt-in
    int n = occupancy_f64(id);
    if (n < 0) n = occupancy_f32(id);
    if (n < 1) n = 1;
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    g_occupancy[{(int)id, dev}] = n;
    return n;
}

pm_status sample_grid_of(const double* lo, const double* hi, const int* samples, const double* out, size_t n,
                         SampleGrid& g) {
    if (!lo || !hi || !samples || !out) return fail(PM_BAD_ARG, "sample: lo, hi, samples and out are required");
    size_t count = 1;
    for (int a = 0; a < 3; ++a) {
        if (samples[a] < 1) return fail(PM_BAD_ARG, "sample: at least one sample along each axis");
        count *= (size_t)samples[a];
        g.lo[a] = lo[a];
        g.hi[a] = hi[a];
        g.n[a] = samples[a];
    }
    if (count != n) return fail(PM_BAD_ARG, "sample: out holds one value per sample point");
    return PM_OK;
}

void set_error(const std::string& msg) { g_error = msg; }

pm_status fail(pm_status s, const std::string& msg) {
    set_error(msg);
    return s;
}

pm_status cuda_fail(cudaError_t e, const char* what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    set_error(msg);
    if (e == cudaErrorMemoryAllocation) return PM_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return PM_NO_DEVICE;
    return PM_CUDA_ERROR;
}

void fill_violation(pm_violation* v, const char* quantity, const std::string& site, double before, double after,
                    double scale, double tol, long long step) {
    if (!v) return;
    std::memset(v, 0, sizeof(*v));
    std::snprintf(v->quantity, sizeof(v->quantity), "%s", quantity);
    std::snprintf(v->site, sizeof(v->site), "%s", site.c_str());
    v->before = before;
    v->after = after;
    v->scale = scale;
    v->tolerance = tol;
    v->step = step;
}

pm_status Handle::init(int dev, size_t partial_doubles) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(PM_NO_DEVICE, std::string("no CUDA device: ") + (e == cudaSuccess ? "count is 0" : cudaGetErrorString(e)));
    if (dev < 0 || dev >= count) return fail(PM_BAD_ARG, "device index out of range");
    device = dev;
    PM_CUDA(cudaSetDevice(dev));
    cudaDeviceProp prop;
    PM_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10)
        return fail(PM_NO_DEVICE, "the kernels are built for sm_100a (B200); this device is sm_" +
                                      std::to_string(prop.major) + std::to_string(prop.minor));
    int sms = 0;
    PM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    sm_count = (unsigned)sms;
    resident = (unsigned)sms * kBlocksPerSM;
    if (partial_doubles < (size_t)std::max<unsigned>(resident, kMeasureBlocks) * 6)
        partial_doubles = (size_t)std::max<unsigned>(resident, kMeasureBlocks) * 6;
    PM_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
    PM_CUDA(cudaStreamCreateWithFlags(&capture, cudaStreamNonBlocking));
    PM_CUDA(state.alloc(sizeof(DevState)));
    PM_CUDA(partials.alloc(partial_doubles * sizeof(double)));
    PM_CUDA(cudaMallocHost((void**)&host_state, sizeof(DevState)));
    std::memset(host_state, 0, sizeof(DevState));
    host_state->tol = tolerance;
    PM_CUDA(cudaMemcpy(state.p, host_state, sizeof(DevState), cudaMemcpyHostToDevice));
    return PM_OK;
}

void Handle::drop_graphs() {
    for (auto& g : graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    graph_dt = NAN;
    graph_steps = 0;
}

Handle::~Handle() {
    if (own || capture) cudaSetDevice(device);
    drop_graphs();
    if (own) {
        cudaStreamSynchronize(own);
        cudaStreamDestroy(own);
    }
    if (user) cudaStreamSynchronize(user);
    if (capture) cudaStreamDestroy(capture);
    if (host_state) cudaFreeHost(host_state);
}

pm_status Handle::read_state() {
    PM_CUDA(cudaMemcpyAsync(host_state, state.p, sizeof(DevState), cudaMemcpyDeviceToHost, stream()));
    PM_CUDA(cudaStreamSynchronize(stream()));
    return PM_OK;
}

pm_status Handle::write_state() {
    PM_CUDA(cudaMemcpyAsync(state.p, host_state, sizeof(DevState), cudaMemcpyHostToDevice, stream()));
    PM_CUDA(cudaStreamSynchronize(stream()));
    return PM_OK;
}

pm_status Handle::begin_call() {
    // Clear the previous call's violation and set the tolerance; the ledger and books stay.
    PM_CUDA(cudaSetDevice(device));
    pm_status s = read_state();
    if (s != PM_OK) return s;
    host_state->violated = kRunning;
    host_state->violation_step = 0;
    host_state->tol = tolerance;
    host_state->counter = 0u;
    host_state->rate_bits = 0ull;
    call_parity = parity;
    return write_state();
}

pm_status Handle::finish_call(long long steps_before, pm_violation* out, const std::string& audit_site,
                              const std::string& startup_site, bool pingpong) {
    pm_status s = read_state();
    if (s != PM_OK) return s;
    PM_CUDA(cudaGetLastError());
    const long long executed = host_state->steps - steps_before;
    if (pingpong) parity = call_parity ^ (int)(executed & 1);
    if (host_state->violated == kRunning) return PM_OK;
    if (host_state->violated == kDeviceTimeout)
        return fail(PM_DEVICE_TIMEOUT, "a bounded wait inside a " + name + " kernel ran out; the call stopped");
    const long long at = host_state->violation_step - steps_before;
    if (host_state->violated == kRefused) {  // solid.rs:1718-1738, decided on the device
        fill_violation(out, "Fourier number", refusal_site, host_state->v_before, host_state->v_after, host_state->v_scale,
                       host_state->v_tol, at);
        set_error("Fourier number past the explicit limit");
        return PM_VIOLATION;
    }
    if (host_state->violated == kStartupFailed)
        fill_violation(out, "energy", startup_site, host_state->v_before, host_state->v_after, host_state->v_scale,
                       host_state->v_tol, at);
    else
        fill_violation(out, "energy", audit_site, host_state->v_before, host_state->v_after, host_state->v_scale,
                       host_state->v_tol, at);
    set_error("conservation audit failed at " + audit_site);
    return PM_VIOLATION;
}

}  // namespace pm

using namespace pm;

extern "C" {

const char* pm_status_string(pm_status s) {
    switch (s) {
        case PM_OK: return "ok";
        case PM_NO_DEVICE: return "no device";
        case PM_UNSUPPORTED: return "unsupported";
        case PM_VIOLATION: return "violation";
        case PM_DEVICE_TIMEOUT: return "device timeout";
        case PM_BAD_ARG: return "bad argument";
        case PM_CUDA_ERROR: return "cuda error";
        case PM_OUT_OF_MEMORY: return "out of memory";
    }
    return "unknown";
}

const char* pm_last_error(void) { return g_error.c_str(); }

pm_status pm_device_count(int* count) {
    if (!count) return fail(PM_BAD_ARG, "count is null");
    *count = 0;
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        *count = 0;
        return fail(PM_NO_DEVICE, cudaGetErrorString(e));
    }
    return PM_OK;
}

const char* pm_version(void) { return "pantometry_b200 0.1.0 (sm_100a)"; }

}  // extern "C"
