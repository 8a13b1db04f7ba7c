// pm_hall_step_f32_noalloc: one Hall step (FP32 fields, FP64 invariant) on buffers the caller
// owns, for callers that cannot allocate device memory — code running where cudaMalloc is not
// available to it or not allowed: inside a host that owns all device memory through its own pool
// and forbids other allocators, a plugin loaded into such a host, or a caller that must not
// synchronise the device the way cudaMalloc/cudaFree can. It launches the same fused kernel as
// pm_hall_step, with that kernel's scratch (the device state block and the per-block partial
// sums of the invariant) in one fixed file-scope device array instead of handle-owned memory.
//
// The scratch array is modest (kNoallocScratchBytes) and every GPU that loads this library holds
// it until the process exits. Every call shares it and it keeps the last call's contents; the
// parts that must start at zero are cleared by each call before the step. Calls that overlap on
// the GPU (on different streams, or from different threads) race on it and must not be issued.
//
// Host code cannot use the array's name as a device address (it is a host-side stand-in), so the
// first call on each device asks the runtime for the address with cudaGetSymbolAddress, with that
// device current, and caches it; that first call should come before any stream capture.
#include <mutex>

#include "runtime.h"

namespace pm {

constexpr size_t kNoallocScratchBytes = 64 * 1024;
constexpr int kNoallocMaxDevices = 64;

static __device__ __align__(256) unsigned char noalloc_scratch[kNoallocScratchBytes];

// Clear the state block for one independent step: no audit, nothing counted, no violation.
static __global__ void noalloc_reset(DevState* st) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        unsigned char* b = reinterpret_cast<unsigned char*>(st);
        for (size_t q = 0; q < sizeof(DevState); ++q) b[q] = 0;
        st->tol = -1.0;
    }
}

namespace {

struct NoallocDevice {
    unsigned char* scratch = nullptr;  // device address of noalloc_scratch on this device
    int wave = 0;                      // resident blocks of the Hall kernel
};

std::mutex g_noalloc_mutex;
NoallocDevice g_noalloc[kNoallocMaxDevices];

pm_status noalloc_setup(int dev, NoallocDevice& out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoallocDevice& d = g_noalloc[dev];
    if (!d.scratch) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc_scratch)");
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
        d.wave = sms * blocks_per_sm(kHallF32);
        d.scratch = static_cast<unsigned char*>(ptr);
    }
    out = d;
    return PM_OK;
}

}  // namespace

}  // namespace pm

using namespace pm;

extern "C" pm_status pm_hall_step_f32_noalloc(int nx, int ny, int nz, double dx, double speed, double density,
                                              double dt, int first_step, const float* p0, const float* vx0,
                                              const float* vy0, const float* vz0, float* p1, float* vx1, float* vy1,
                                              float* vz1, void* stream, double* invariant) {
    if (!p0 || !vx0 || !vy0 || !vz0 || !p1 || !vx1 || !vy1 || !vz1)
        return fail(PM_BAD_ARG, "noalloc: null field pointer");
    {
        // the kernel reads old values of neighbouring nodes while it writes the new ones, so
        // every output must be a buffer of its own, apart from every input and other output
        const void* all[8] = {p0, vx0, vy0, vz0, p1, vx1, vy1, vz1};
        for (int o = 4; o < 8; ++o)
            for (int q = 0; q < o; ++q)
                if (all[o] == all[q]) return fail(PM_BAD_ARG, "noalloc: an output buffer is also an input or another output");
    }
    if (nx < 2 || ny < 1 || nz < 1) return fail(PM_BAD_ARG, "noalloc: a hall has at least 2 x 1 x 1 nodes");
    if ((unsigned long long)nx * ny * nz >= (1ull << 32)) return fail(PM_BAD_ARG, "noalloc: grid above 2^32 nodes");
    if (!(dx > 0.0) || !(density > 0.0) || !(speed > 0.0) || !(dt > 0.0))
        return fail(PM_BAD_ARG, "noalloc: dx, speed, density and dt must be positive");
    const double courant = speed * dt * std::sqrt(3.0) / dx;  // hall.rs:319, refused as at hall.rs:410
    if (courant > 1.0 + 1e-12) return fail(PM_VIOLATION, "noalloc: Courant number past the three-dimensional limit");
    int dev = 0;
    PM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoallocMaxDevices) return fail(PM_BAD_ARG, "noalloc: device index beyond the set-up table");
    NoallocDevice d;
    pm_status s = noalloc_setup(dev, d);
    if (s != PM_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    HallArgs<float> a{};
    a.p0 = p0; a.vx0 = vx0; a.vy0 = vy0; a.vz0 = vz0;
    a.p1 = p1; a.vx1 = vx1; a.vy1 = vy1; a.vz1 = vz1;
    a.nx = nx; a.ny = ny; a.nz = nz;
    const double vh = first_step ? 0.5 * dt : dt;  // hall.rs:428
    a.gain = (float)(vh / (density * dx));         // hall.rs:433
    a.scale = (float)(dt * (density * speed * speed) / dx);  // hall.rs:464
    const double volume = dx * dx * dx;
    a.knode = volume / (2.0 * (density * speed * speed));
    a.kface = 0.5 * density * volume;
    a.src = -1;
    a.src_i = a.src_j = a.src_k = -1;
    a.starting = 0;
    a.tiles = make_tiles(nx, ny, nz, choose_zc(nx, ny, nz, (unsigned)d.wave));
    a.nblocks = grid_for(a.tiles, (unsigned)d.wave);
    // scratch layout: the state block, then 3 partial sums per block
    const size_t state_bytes = (sizeof(DevState) + 255) & ~size_t(255);
    const size_t need = state_bytes + (size_t)a.nblocks * 3 * sizeof(double);
    if (need > kNoallocScratchBytes)
        return fail(PM_BAD_ARG, "noalloc: this grid needs " + std::to_string(need) + " bytes of scratch; the fixed maximum is " +
                                    std::to_string(kNoallocScratchBytes));
    a.st = reinterpret_cast<DevState*>(d.scratch);
    a.partials = reinterpret_cast<double*>(d.scratch + state_bytes);

    noalloc_reset<<<1, 1, 0, st>>>(a.st);
    PM_CUDA(cudaGetLastError());
    PM_CUDA(launch_hall<float>(a, st));
    if (invariant) {
        PM_CUDA(cudaMemcpyAsync(invariant, &a.st->invariant, sizeof(double), cudaMemcpyDeviceToHost, st));
        PM_CUDA(cudaStreamSynchronize(st));
    }
    return PM_OK;
}
