// Device-side pieces shared by every stepping kernel: the per-handle state word block, the
// fixed-order FP64 reduction tree and the on-device audit.
//
// Determinism. Every step kernel leaves one partial per block (a warp-shuffle tree, then a tree
// over the block's warps, both in a fixed order). The last block to finish — found with one
// atomic ticket — sums the partials in a fixed strided order followed by the same fixed tree.
// Which block happens to finish last changes nothing about the order of the additions, so the
// ledger is bit-reproducible from run to run on one launch geometry. This is the GPU form of
// `Ensemble::blocks`' rule that the association of a sum must not depend on scheduling
// (crates/pantometry-core/src/ensemble.rs:180-230).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pm {

// The tiling every step kernel walks: 32 × 8 columns of cells (one warp row per y), each
// marched through `zc` planes by its thread. A persistent grid of blocks takes tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... in that fixed order, so every thread's share of a
// reduction is summed in the same order on every run.
struct Tiles {
    int nx, ny, nz, zc;
    int ntx, nty, ntz;
    long long ntiles;
    int rows;  // rows of a tile: the block's y extent (8 but in the many-step heat kernels)
};

__host__ __device__ inline Tiles make_tiles(int nx, int ny, int nz, int zc, int rows = 8) {
    Tiles t;
    t.nx = nx; t.ny = ny; t.nz = nz; t.zc = zc;
    t.rows = rows;
    t.ntx = (nx + 31) / 32;
    t.nty = (ny + rows - 1) / rows;
    t.ntz = (nz + zc - 1) / zc;
    t.ntiles = (long long)t.ntx * t.nty * t.ntz;
    return t;
}

// Asynchronous global → shared copies (cp.async, sm_80 and later): each thread queues element
// copies for planes ahead of the one it computes, so the bytes in flight are set by the ring of
// shared-memory stages rather than by registers or thread count.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
// The same copy to a shared address given as a 32-bit offset, issued only where `pred` holds
// (a predicated instruction: no branch, no divergence).
template <int BYTES>
__device__ __forceinline__ void cp_async_if(unsigned saddr, const void* gmem, bool pred) {
    asm volatile(
        "{\n .reg .pred q;\n setp.ne.b32 q, %2, 0;\n @q cp.async.ca.shared.global [%0], [%1], %3;\n}\n" ::"r"(saddr),
        "l"(gmem), "r"((int)pred), "n"(BYTES)
        : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Why the run stopped, in DevState::violated.
// kDeviceTimeout: a bounded wait inside a kernel ran out (the kernel gave up and returned).
// kRefused: a step was refused before anything moved (a state-dependent stability limit, checked
// on the device at the start of each step; the v_* fields hold the refusal's numbers).
enum : int { kRunning = 0, kAuditFailed = 1, kStartupFailed = 2, kDeviceTimeout = 3, kRefused = 4 };

// One per handle, in device memory. Written only by the last block of a step kernel (and by
// the host between calls), read by every block of the next kernel: stream order is the only
// synchronisation, nothing ever spins.
struct DevState {
    int violated;       // kRunning / kAuditFailed / kStartupFailed / kDeviceTimeout
    int has_invariant;  // cavity: an invariant exists (after release_mode or a first step)
    long long steps;    // steps completed since the state was uploaded or released
    long long violation_step;
    double tol;         // relative audit tolerance; negative disables the audit
    double prev_total, prev_scale;  // the ledger after the last completed step
    double v_before, v_after, v_scale, v_tol;
    double total, scale;  // the ledger's energy entry after the last step
    double part[4];       // its contributions, in `Ledger::with` order
    // Solid3D books (solid.rs:256-270)
    double lost, supplied;
    // Hall books (hall.rs:84-88) and the source extension
    double datum, offset, injected, last_delta;
    // Cavity books (cavity.rs:161-162) and the source extension
    double invariant, dissipated, work;
    double work_booked;  // cavity source work already in the ledger: through the previous step
    // Solid3D with radiating films: `worst_rate_now` of the present state (solid.rs:1148-1185),
    // and the max over boundary cells the step kernel gathers for the next state (the bits of a
    // non-negative double, so an integer atomicMax orders them)
    double rate_now;
    unsigned long long rate_bits;
    unsigned int counter;  // arrival ticket for the last-block reduction; always 0 between kernels
    unsigned int pad;
};

// Rust's f64::max (NaN-ignoring) is CUDA's fmax.
__device__ __forceinline__ double rmax(double a, double b) { return fmax(a, b); }

__device__ __forceinline__ int linear_tid() {
    return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
__device__ __forceinline__ unsigned linear_bid() {
    return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
}

template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV]) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
    }
}

// Sum over the block, result valid in linear thread 0. `smem` holds 32*NV doubles.
// blockDim (all three axes multiplied) must be a multiple of 32.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem) {
    const int tid = linear_tid();
    const int lane = tid & 31, warp = tid >> 5;
    const int nwarps = (blockDim.x * blockDim.y * blockDim.z) >> 5;
    warp_sum<NV>(v);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) smem[warp * NV + q] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] = lane < nwarps ? smem[lane * NV + q] : 0.0;
        warp_sum<NV>(v);
    }
    __syncthreads();
}

// Reduce this block's values, publish them as partials[bid], and if this block is the last of
// `nblocks` to arrive, reduce all partials in fixed order. Returns true in the last block, with
// the totals in v (valid in linear thread 0). The counter is reset for the next kernel.
template <int NV>
__device__ __forceinline__ bool finish_blocks(double (&v)[NV], double* partials, unsigned nblocks,
                                              unsigned* counter) {
    __shared__ double smem[32 * NV];
    __shared__ int is_last;
    const int tid = linear_tid();
    const unsigned bid = linear_bid();
    block_sum<NV>(v, smem);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) partials[(size_t)bid * NV + q] = v[q];
        __threadfence();
        unsigned ticket = atomicAdd(counter, 1u);
        is_last = (ticket == nblocks - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = 0.0;
    for (unsigned b = tid; b < nblocks; b += nthreads) {
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] += __ldcg(&partials[(size_t)b * NV + q]);
    }
    block_sum<NV>(v, smem);
    if (tid == 0) *counter = 0u;
    return true;
}

// `audit_with` (crates/pantometry-core/src/conserved.rs:323-363) for the one quantity on this
// path, against the ledger the previous step left; then commit this step's ledger. The same
// arithmetic is `attribute` with no bus traffic (sim.rs:1169-1223): only the site differs,
// and the host names it.
__device__ __forceinline__ void audit_and_commit(DevState* st, double total, double scale) {
    st->steps += 1;
    if (st->tol >= 0.0 && st->violated == kRunning) {
        double b = st->prev_total;
        double sc = rmax(rmax(rmax(fabs(b), fabs(total)), st->prev_scale), scale);
        if (!(sc < 1e-300) && fabs(total - b) / sc > st->tol) {
            st->violated = kAuditFailed;
            st->violation_step = st->steps;
            st->v_before = b;
            st->v_after = total;
            st->v_scale = sc;
            st->v_tol = st->tol;
        }
    }
    st->prev_total = total;
    st->prev_scale = scale;
    st->total = total;
    st->scale = scale;
}

// The many-step kernels' grid-wide wait: arrival counters 128 bytes apart (so the blocks' arrivals do
// not queue on one address), then a word of their own for the books' verdict.
constexpr int kWaitCounters = 8;
constexpr int kWaitWords = 32 * kWaitCounters + 32;

// Arrive at the grid's n-th wait and wait until every block has arrived n times, polling at most
// `budget` times after the first look. The arrival is a release, so what the block wrote before it
// is seen by every block after its own wait, which ends with an acquire. A block may add
// kWaitStop to its arrival to say the grid is to stop after this wait: every block sees it in the
// sum it polls, with no further read. Returns 0 when the wait ran out, 1 when every block has
// arrived, 2 when every block has arrived and one said stop.
constexpr unsigned kWaitStop = 1u << 30;
__device__ __forceinline__ int grid_wait(unsigned* base, unsigned n, unsigned budget, bool stop_after = false) {
    __shared__ int passed;
    __syncthreads();
    if (linear_tid() == 0) {
        const unsigned arrive = stop_after ? 1u + kWaitStop : 1u;
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(base + 32 * (blockIdx.x % kWaitCounters)), "r"(arrive)
                     : "memory");
        const unsigned target = n * gridDim.x;
        int ok = 0;
        for (unsigned it = 0;; ++it) {
            unsigned v[kWaitCounters];
#pragma unroll
            for (int r = 0; r < kWaitCounters; ++r)
                asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v[r]) : "l"(base + 32 * r) : "memory");
            unsigned sum = 0;
#pragma unroll
            for (int r = 0; r < kWaitCounters; ++r) sum += v[r];
            if (sum % kWaitStop >= target) {
                ok = sum >= kWaitStop ? 2 : 1;
                break;
            }
            if (it >= budget) break;
            __nanosleep(32);
        }
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        passed = ok;
    }
    __syncthreads();
    return passed;
}

// `Ledger::add` (conserved.rs:86-90) into an entry that starts at zero.
__device__ __forceinline__ void ledger_add(double& total, double& scale, double x) {
    total += x;
    scale = rmax(scale, fabs(x));
}

}  // namespace pm
