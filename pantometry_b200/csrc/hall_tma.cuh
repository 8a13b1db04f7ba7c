// Hall step, FP32 form for halls whose x extent is a multiple of 4 nodes, staged by the Tensor
// Memory Accelerator.
//
// Layout. The handle keeps all four fields in the nodes' own index order n = i + nx·(j + ny·k):
// the pressure as the reference does (hall.rs:67-77), and each face array padded to nx·ny·nz,
// the face on the high side of node n at index n (the padding — x faces at i = nx−1, y faces at
// j = ny−1, z faces at k = nz−1 — is zero and never written). One index then addresses every
// array, and every array is a 3D tensor whose row pitch nx·4 bytes is a multiple of 16, so TMA
// can tile it.
//
// Walk. Tiles are 32 × 8 columns of nodes over a z-chunk (the same tiling as hall_step), taken
// by a persistent grid in order; each tile is streamed P planes at a time. For a stage of planes
// k .. k+P−1 one thread issues four tiled TMA loads into a ring of S shared-memory stages:
//   p   x0−4 .. x0+35, y0−1 .. y0+8, k−1 .. k+P      (the node, its six neighbours)
//   vx  x0−4 .. x0+31, y0   .. y0+7, k   .. k+P−1    (faces i−1 and i)
//   vy  x0   .. x0+31, y0−1 .. y0+7, k   .. k+P−1    (faces j−1 and j)
//   vz  x0   .. x0+31, y0   .. y0+7, k−1 .. k+P−1    (faces k−1 and k)
// The x start is a multiple of 4 elements (16 bytes); parts of a box outside the hall are
// filled with zeros by the hardware. Completion is tracked by one mbarrier per stage; every wait
// on it is bounded and a wait that runs out stops the kernel with kDeviceTimeout.
//
// Arithmetic. Per node, exactly hall_step's: the six face velocities from the old state (the low
// ones recomputed rather than exchanged), the pressure with the wall weights (hall.rs:433-505),
// the source extension, and the FP64 invariant of the node and its own faces (hall.rs:334-384).
#pragma once

#include <cuda.h>

#include "hall_kernels.cuh"

namespace pm {

// The four old fields of one parity as TMA tensor maps.
struct HallMaps {
    CUtensorMap p, vx, vy, vz;
};

template <int P>
struct HallTmaStage {
    float p[P + 2][10][40];
    float vx[P][8][36];
    float vy[P][9][32];
    float vz[P + 1][8][32];
};

// The tile shapes a hall can step with: planes per stage, stages in the ring, resident blocks per
// SM the kernel is held to. Shape 0 (8 planes in each of 2 stages, 87 KB of shared memory, two
// blocks per SM) measured fastest on B200 at 256³ among 2-8 planes and 2-5 stages in hand sweeps
// (176 Gcell/s, against 166 for 6 × 2 at three blocks and 141 for 4 × 3); the others are the
// runners-up, which pm_hall_autotune times on a hall's own grid. Every shape computes each node
// with the same expressions, so they agree bit for bit.
struct HallTmaShape {
    int planes, stages, min_blocks;
};
constexpr HallTmaShape kHallTmaShapes[] = {{8, 2, 2}, {6, 2, 3}, {4, 3, 3}, {4, 2, 4}};
constexpr int kHallTmaShapeCount = sizeof(kHallTmaShapes) / sizeof(kHallTmaShapes[0]);
constexpr int kHallTmaPlanes = kHallTmaShapes[0].planes;
constexpr int kHallTmaStages = kHallTmaShapes[0].stages;
constexpr unsigned kMbarSpinLimit = 1u << 22;  // try_wait rounds before a wait gives up

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred q;\n mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n selp.b32 %0, 1, 0, q;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for phase `parity` of the barrier to complete, at most kMbarSpinLimit rounds. After the
// first few rounds each failed round sleeps, so waiting warps leave the issue slots to the warps
// of other blocks that have work (about a second in all before the wait gives up).
#ifndef PM_MBAR_SLEEP_NS
#define PM_MBAR_SLEEP_NS 64
#endif
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
    for (unsigned n = 0; n < kMbarSpinLimit; ++n) {
        if (mbar_try_wait(bar, parity)) return true;
        if (PM_MBAR_SLEEP_NS > 0 && n >= 4) __nanosleep(PM_MBAR_SLEEP_NS);
    }
    return false;
}
__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap* map, int x, int y, int z, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// Tile cursor stepping P planes at a time.
__device__ __forceinline__ bool hall_cursor_advance(HallCursor& c, const Tiles& T, int planes) {
    c.k += planes;
    if (c.k < c.k1) return false;
    hall_cursor_at(c, T, c.t + gridDim.x);
    return true;
}

template <int P>
__device__ __forceinline__ void hall_tma_issue(const HallMaps& m, unsigned stage, unsigned bar, const HallCursor& c) {
    using St = HallTmaStage<P>;
    const St* z = nullptr;
    auto off = [&](const void* q) { return (unsigned)((const char*)q - (const char*)z); };
    mbar_expect_tx(bar, (unsigned)sizeof(St));
    tma_load_3d(stage + off(&z->p[0][0][0]), &m.p, c.x0 - 4, c.y0 - 1, c.k - 1, bar);
    tma_load_3d(stage + off(&z->vx[0][0][0]), &m.vx, c.x0 - 4, c.y0, c.k, bar);
    tma_load_3d(stage + off(&z->vy[0][0][0]), &m.vy, c.x0, c.y0 - 1, c.k, bar);
    tma_load_3d(stage + off(&z->vz[0][0][0]), &m.vz, c.x0, c.y0, c.k - 1, bar);
}

template <int P, int S, bool HET, int MINB>
static __global__ void __launch_bounds__(256, MINB) hall_tma_step(HallArgs<float> a, const __grid_constant__ HallMaps m) {
    DevState* st = a.st;
    if (st->violated) return;
    using St = HallTmaStage<P>;
    extern __shared__ __align__(128) unsigned char hall_tma_smem[];
    const St* ring = reinterpret_cast<const St*>(hall_tma_smem);
    const unsigned ring_base = static_cast<unsigned>(__cvta_generic_to_shared(hall_tma_smem));
    const unsigned bar_base = ring_base + S * (unsigned)sizeof(St);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = tx + 32 * ty;
    const long long step = st->steps;
    const double delta = (a.src_i >= 0 && step < a.nwave) ? a.wave[step] : 0.0;
    const double last_delta = st->last_delta;
    double acc[3] = {0.0, 0.0, 0.0};  // invariant, immediate source term, injected increment

    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(bar_base + 8 * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const Tiles T = a.tiles;
    const float gain = a.gain;
    HallCursor pf, cc;  // producer (thread 0 only) and consumer cursors
    hall_cursor_at(cc, T, blockIdx.x);
    int issued = 0;
    if (tid == 0) {
        hall_cursor_at(pf, T, blockIdx.x);
        for (; issued < S - 1 && pf.valid; ++issued) {
            hall_tma_issue<P>(m, ring_base + issued * (unsigned)sizeof(St), bar_base + 8 * issued, pf);
            hall_cursor_advance(pf, T, P);
        }
    }
    float sc = a.scale;
    double kn = a.knode;
    bool timed_out = false;
    int it = 0;
    while (cc.valid) {
        const int slot = it % S;
        const bool got = mbar_wait(bar_base + 8 * slot, (unsigned)((it / S) & 1));
        // everyone's copies of this stage have landed, and everyone is done with the previous one
        if (!__syncthreads_and(got)) {
            timed_out = true;
            break;
        }
        if (tid == 0 && pf.valid) {
            const int fill = (it + S - 1) % S;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            hall_tma_issue<P>(m, ring_base + fill * (unsigned)sizeof(St), bar_base + 8 * fill, pf);
            hall_cursor_advance(pf, T, P);
            ++issued;
        }
        const St& s = ring[slot];
        const int i = cc.x0 + tx, j = cc.y0 + ty;
        if (i < nx && j < ny) {
            const bool xl = i > 0, xh = i + 1 < nx, yl = j > 0, yh = j + 1 < ny;
            // hall.rs:675-681: weight 2 on a wall, 1 inside; the share 1/w is an exact power of two
            const float wi = (xl && xh) ? 1.0f : 2.0f, wj = (yl && yh) ? 1.0f : 2.0f;
            const double si = (xl && xh) ? 1.0 : 0.5, sj = (yl && yh) ? 1.0 : 0.5;
            const bool src_col = i == a.src_i && j == a.src_j;
            double cn = si * sj * kn;
            const double cxf = a.kface * sj, cyf = a.kface * si, czf = a.kface * si * sj;
            unsigned n = (unsigned)i + (unsigned)nx * ((unsigned)j + (unsigned)ny * (unsigned)cc.k);
            const unsigned sp = (unsigned)nx * (unsigned)ny;
#pragma unroll
            for (int h = 0; h < P; ++h) {
                const int k = cc.k + h;
                if (k >= cc.k1) break;
                if (HET) {
                    const int b = i / a.block + a.nbx * (j / a.block + a.nby * (k / a.block));
                    sc = a.block_scale[b];
                    kn = a.block_knode[b];
                    cn = si * sj * kn;
                }
                const float pc = s.p[h + 1][ty + 1][tx + 4];
                const bool zh = k + 1 < nz, zl = k > 0;
                const float hx0 = s.vx[h][ty][tx + 4] - gain * (s.p[h + 1][ty + 1][tx + 5] - pc);
                const float lx0 = s.vx[h][ty][tx + 3] - gain * (pc - s.p[h + 1][ty + 1][tx + 3]);
                const float hy0 = s.vy[h][ty + 1][tx] - gain * (s.p[h + 1][ty + 2][tx + 4] - pc);
                const float ly0 = s.vy[h][ty][tx] - gain * (pc - s.p[h + 1][ty][tx + 4]);
                const float hz0 = s.vz[h + 1][ty][tx] - gain * (s.p[h + 2][ty + 1][tx + 4] - pc);
                const float lz0 = s.vz[h][ty][tx] - gain * (pc - s.p[h][ty + 1][tx + 4]);
                const float hx = xh ? hx0 : 0.0f, lx = xl ? lx0 : 0.0f;
                const float hy = yh ? hy0 : 0.0f, ly = yl ? ly0 : 0.0f;
                const float hz = zh ? hz0 : 0.0f, lz = zl ? lz0 : 0.0f;
                if (xh) a.vx1[n] = hx;
                if (yh) a.vy1[n] = hy;
                if (zh) a.vz1[n] = hz;
                const bool zin = zl && zh;
                const float wk = zin ? 1.0f : 2.0f;
                // hall.rs:499-502
                float np = pc - sc * (wi * (hx - lx) + wj * (hy - ly) + wk * (hz - lz));
                if (src_col && k == a.src_k) {
                    // deferred term of the previous injection, then this one's
                    acc[2] += a.wsrc * (last_delta + delta) * (double)pc;
                    acc[1] += a.wsrc * delta * (double)pc;
                    np = (float)((double)np + delta);
                }
                a.p1[n] = np;
                const double dhx = (double)hx, dhy = (double)hy, dhz = (double)hz;
                const double sk = zin ? 1.0 : 0.5;
                acc[0] += sk * (cn * (double)np * (double)pc + cxf * dhx * dhx + cyf * dhy * dhy) + czf * dhz * dhz;
                n += sp;
            }
        }
        hall_cursor_advance(cc, T, P);
        ++it;
    }
    if (timed_out) {
        // stop every later kernel of the call, and let the copies still in flight land before
        // the block's shared memory is given up
        if (tid == 0) {
            st->violated = kDeviceTimeout;
            for (int q = it; q < issued; ++q) mbar_wait(bar_base + 8 * (q % S), (unsigned)((q / S) & 1));
        }
        return;
    }
    hall_finish<float>(a, acc, delta);
}

}  // namespace pm
