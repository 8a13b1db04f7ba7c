// The FP32 form of a uniform Solid3D block staged by the Tensor Memory Accelerator: the ensemble's
// TMA stage (ens_tma.cuh) over the columns of one block. A work item is one stage: the 32 × 8
// column at (x0, y0) and the planes kb .. kb+P−1, for which one thread issues one tiled TMA load of
//   x0−4 .. x0+35, y0−1 .. y0+8, kb−1 .. kb+P
// of the old deviations into a ring of S shared-memory stages (rows of a multiple of 4 cells, so
// x0 − 4 starts on 16 bytes; the hardware fills outside the block with zeros). Each of the eight
// consumer warps steps its row of the stage with tma_stage_row, the arithmetic heat_f32_step and
// the ensemble's TMA kernel share, so the three agree bit for bit. Work items go to the persistent
// CTAs in turn (w = blockIdx.x, blockIdx.x + gridDim.x, ...), x fastest, so the stages in flight at
// one time are neighbours and share their halo rows and planes in L2. Every wait on a stage's
// mbarrier is bounded; a wait that runs out stops the call with kDeviceTimeout.
//
// The books: each thread sums its cells' new deviations and the heat its films shed in FP64; the
// grid's sums are reduced in fixed order by the last CTA (finish_blocks), which runs the ledger and
// the audit as heat_f32_step does.
#pragma once

#include "ens_tma.cuh"

namespace pm {

struct HeatTmaArgs {
    float* __restrict__ dnew;
    int nx, ny, nz;
    unsigned ntx, nty, ntz;   // stages: 32-cell columns along x, 8-row columns along y, P-plane slabs
    EnsBrickInfo cell;        // the block's coefficients (a, b, off, exposed) and extents
    double capacity;          // per cell
    DevState* st;
    double* partials;
    unsigned nblocks;
};

template <int P, int S>
static __global__ void __launch_bounds__(kEnsConsumers + 32, PM_ENS_TMA_MIN_BLOCKS)
    heat_tma_step(const HeatTmaArgs a, const __grid_constant__ CUtensorMap map) {
    using St = EnsTmaStage<P>;
    DevState* st = a.st;
    if (st->violated) return;
    extern __shared__ __align__(128) unsigned char heat_tma_smem[];
    __shared__ int stage_w[S];  // the slot's work item; −1: the walk is over
    const St* ring = reinterpret_cast<const St*>(heat_tma_smem);
    const unsigned ring_base = static_cast<unsigned>(__cvta_generic_to_shared(heat_tma_smem));
    const unsigned full_base = ring_base + S * (unsigned)sizeof(St), empty_base = full_base + 8 * S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned nitems = a.ntx * a.nty * a.ntz;
    if (tid == 0) {
        for (int q = 0; q < S; ++q) {
            mbar_init(full_base + 8 * q, 1);
            mbar_init(empty_base + 8 * q, kEnsConsumers / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    double acc[2] = {0.0, 0.0};  // Σ deviation of the new state, Σ heat shed (per cell capacity to come)
    bool timed_out = false;
    if (warp == kEnsConsumers / 32) {  // the producer
        if (lane == 0) {
            int q = 0;
            for (unsigned w = blockIdx.x;; w += gridDim.x, ++q) {
                const int slot = q % S;
                if (q >= S && !mbar_wait(empty_base + 8 * slot, (unsigned)(((q / S) - 1) & 1))) {
                    timed_out = true;
                    break;
                }
                if (w >= nitems) {  // the end of the walk, released with a plain arrive
                    stage_w[slot] = -1;
                    mbar_arrive(full_base + 8 * slot);
                    break;
                }
                stage_w[slot] = (int)w;
                const unsigned r = w / a.ntx, cx = w - r * a.ntx, cy = r % a.nty, cz = r / a.nty;
                const unsigned full = full_base + 8 * slot;
                mbar_expect_tx(full, (unsigned)sizeof(St));
                tma_load_3d(ring_base + slot * (unsigned)sizeof(St), &map, (int)(32 * cx) - 4, (int)(8 * cy) - 1,
                            (int)(P * cz) - 1, full);
            }
            if (timed_out) st->violated = kDeviceTimeout;
            // The last load of each slot lands before this block gives up its shared memory: at once
            // where the consumers took it, bounded where they stopped waiting. After the end of the
            // walk, slot q % S holds the end marker, a later phase than its last load's (whose parity
            // the marker's successor shares), so its last load, consumed before the marker was
            // written, is not waited on; after a wait that ran out, stage q was never issued and the
            // slot's last load is load q − S.
            for (int u = q >= S ? q - S + (timed_out ? 0 : 1) : 0; u < q; ++u)
                mbar_wait(full_base + 8 * (u % S), (unsigned)((u / S) & 1));
        }
        timed_out = __shfl_sync(0xffffffffu, timed_out ? 1 : 0, 0) != 0;
    } else {
        const int tx = lane, ty = warp;
        const size_t plane = (size_t)a.nx * a.ny;
        int slot = 0;
        unsigned phase = 0;  // of the slot's full barrier: flips each time the ring wraps
        for (;; slot = slot + 1 == S ? 0 : slot + 1, phase ^= slot == 0 ? 1u : 0u) {
            const bool got = mbar_wait(full_base + 8 * slot, phase);
            if (__any_sync(0xffffffffu, !got)) {
                if (lane == 0) st->violated = kDeviceTimeout;
                timed_out = true;
                break;
            }
            const int w = stage_w[slot];
            if (w < 0) break;  // the walk is over (every consumer reads the same word)
            const unsigned r = (unsigned)w / a.ntx, cx = (unsigned)w - r * a.ntx, cy = r % a.nty, cz = r / a.nty;
            const int x0 = 32 * (int)cx, i = x0 + tx, j = 8 * (int)cy + ty, kb = P * (int)cz;
            if (i < a.nx && j < a.ny) {
                float* __restrict__ out = a.dnew + ((size_t)i + (size_t)a.nx * ((size_t)j + (size_t)a.ny * kb));
                tma_stage_row<P>(ring[slot], a.cell, x0, tx, ty, i, j, kb, min(P, a.nz - kb), out, plane, acc);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty_base + 8 * slot);
        }
    }
    if (__syncthreads_or(timed_out ? 1 : 0)) return;
    if (finish_blocks<2>(acc, a.partials, a.nblocks, &st->counter) && tid == 0) {
        const double stored = a.capacity * acc[0];
        st->lost += a.capacity * acc[1];
        double total = 0.0, scale = 0.0;
        ledger_add(total, scale, stored);
        ledger_add(total, scale, st->lost);
        ledger_add(total, scale, -st->supplied);
        st->part[0] = stored;
        st->part[1] = st->lost;
        st->part[2] = -st->supplied;
        audit_and_commit(st, total, scale);
    }
}

}  // namespace pm
