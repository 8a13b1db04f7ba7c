// Batched Solid3D stepping, FP32 form, staged by the Tensor Memory Accelerator: the brick list of
// ensemble_kernels.cuh walked by a persistent grid, each 32 × 8-column brick streamed P planes at
// a time through a ring of S shared-memory stages. For a stage of planes kb .. kb+P−1 of block g
// one thread issues one tiled TMA load of the block's deviations
//   x0−4 .. x0+35, y0−1 .. y0+8, kb−1 .. kb+P
// (rows padded to a multiple of 4 elements, so every row starts on 16 bytes; the hardware fills
// outside the block with zeros) through block g's own tensor map. The per-cell arithmetic is
// heat_f32_step's, the per-brick FP64 partials and the per-block ticket reduction are ens_step's.
// Every wait on a stage's mbarrier is bounded; a wait that runs out stops the kernel with
// kDeviceTimeout in every block's books.
//
// Order of the walk. Bricks differ in cost (blocks of 16 to 128 cells per axis), so a fixed share
// per CTA (brick c, c + gridDim, ...) lets the CTAs drift apart, and the bricks running at one time
// stop being neighbours: the halo rows and planes one brick reads from its neighbours are then
// gone from L2 by the time the neighbour runs. The producers therefore take bricks in list order
// from one atomic counter, so the bricks in flight are always a contiguous run of the list and a
// brick's x, y and z neighbours run beside it. Which CTA takes which brick changes nothing in the
// results: every partial is stored by brick and warp, and each block's are summed in fixed order.
//
// No barrier spans the consumer warps. Each warp waits for its stage, computes its row of the
// brick, hands the slot back, and at the end of a brick stores its own two partials; after the step
// ens_tma_books sums each block's partials in a fixed order and runs its ledger and audit.
#pragma once

#include "ensemble_kernels.cuh"
#include "hall_tma.cuh"

namespace pm {

// Planes per stage, stages in the ring, blocks per SM. Measured on B200 over the 512-grid ensemble:
// 16 × 2 at three blocks per SM 405 Gcell/s, 16 × 3 at two 398, 8 × 3 at four 371-378, 12 × 4 at
// two 378, 24 × 2 at two 379, 32 × 2 at two 328, 4 × 6 at three 307. A deeper stage reads its
// two halo planes over more planes of its own.
#ifndef PM_ENS_TMA_PLANES
#define PM_ENS_TMA_PLANES 16
#endif
#ifndef PM_ENS_TMA_STAGES
#define PM_ENS_TMA_STAGES 2
#endif
#ifndef PM_ENS_TMA_MIN_BLOCKS
#define PM_ENS_TMA_MIN_BLOCKS 3
#endif
constexpr int kEnsTmaPlanes = PM_ENS_TMA_PLANES;
constexpr int kEnsTmaStages = PM_ENS_TMA_STAGES;

template <int P>
struct EnsTmaStage {
    float t[P + 2][10][40];
};

inline size_t ens_tma_smem_bytes() { return sizeof(EnsTmaStage<kEnsTmaPlanes>) * kEnsTmaStages + 16 * kEnsTmaStages; }

// Everything a stage's consumers need about its brick, one 128-byte record per brick built on the
// host; the producer bulk-copies it into the stage's slot with the stage's tile, on the same
// mbarrier, so neither side ever waits on a dependent chain of global loads.
struct alignas(16) EnsBrickInfo {
    unsigned long long offset;
    unsigned grid;
    int x0, y0, nx, ny, nz, pitch, exposed;
    float a, b[6], off[6];
    unsigned pad[9];
};
static_assert(sizeof(EnsBrickInfo) == 128, "one record is one 128-byte bulk copy");

template <bool B>
struct Flag {
    static constexpr bool value = B;
};

constexpr unsigned kEnsHoldBlocks = 16384;  // blocks whose stop flags fit the shared bitmask

struct EnsTmaArgs {
    EnsArgs<float> e;
    const CUtensorMap* maps;    // per block: the old field's map (this launch's parity)
    const EnsBrickInfo* infos;  // per brick
    // work[0]: the next brick of the walk; work[1]: CTAs done. Zero at every launch's start: the
    // last CTA to finish puts both back to zero.
    unsigned* work;
};
// Partials per brick: two for each consumer warp (Σ deviation of the new state, Σ heat shed).
constexpr int kEnsTmaPartialsPerBrick = 2 * 8;

__device__ __forceinline__ void bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
constexpr int kEnsConsumers = 256;

// One warp's row of one stage: the cells (i, j, kb .. kb + hn − 1) of a block of m.nx × m.ny × m.nz
// cells, read from the stage tile `s` (x0−4 .. x0+35, y0−1 .. y0+8, kb−1 .. kb+P, the block's own
// tile at x0, y0) and written through `out`, one plane apart. The per-cell arithmetic of
// heat_f32_step in the same order and roundings, shared by the ensemble's TMA kernel and the single
// block's (heat_tma_step), so all three agree bit for bit.
template <int P>
__device__ __forceinline__ void tma_stage_row(const EnsTmaStage<P>& s, const EnsBrickInfo& m, int x0, int tx, int ty,
                                              int i, int j, int kb, int hn, float* __restrict__ out, size_t plane,
                                              double (&acc)[2]) {
    const int nx = m.nx, ny = m.ny, nz = m.nz;
    const bool xl = i > 0, xh = i + 1 < nx, yl = j > 0, yh = j + 1 < ny;
    const bool xedge = x0 == 0 || x0 + 32 >= nx;  // the brick holds an x face
    const float ga = m.a;
    if (!xedge && yl && yh && hn == P && kb > 0 && kb + P < nz) {
        // a whole stage of interior cells: no film, no bound, the planes below and
        // above carried in registers; the general form's arithmetic without its zeros
        float below = s.t[0][ty + 1][tx + 4], here = s.t[1][ty + 1][tx + 4];
#pragma unroll
        for (int h = 0; h < P; ++h) {
            const float above = s.t[h + 2][ty + 1][tx + 4];
            const float xm = s.t[h + 1][ty + 1][tx + 3], xp = s.t[h + 1][ty + 1][tx + 5];
            const float ym = s.t[h + 1][ty][tx + 4], yp = s.t[h + 1][ty + 2][tx + 4];
            const float sum = (((((xm - here) + (xp - here)) + (ym - here)) + (yp - here)) + (below - here)) + (above - here);
            const float nd = __fadd_rn(here, __fmaf_rn(ga, sum, -0.0f));
            *out = nd;
            out += plane;
            acc[0] += (double)nd;
            below = here;
            here = above;
        }
    } else if (yl && yh && nx > 1) {
        // a stage of a row inside the block in y (a brick on an x face, a stage holding a
        // z face, or a partial stage): the general form's sums and films term for term, so
        // the stage stays one straight run of planes. Adding +0 for an absent neighbour is
        // adding nothing, since a sum that starts at +0 is never −0 here. An absent x
        // neighbour is read at the cell itself, so its term is here − here = +0 with no
        // select; a lane lies on one x face at most (the block is two cells wide or more),
        // and its film b·(here + off) + 0 takes that face's coefficients, or 0 · (here + 0)
        // + 0 = +0 off the faces.
        const int exposed = m.exposed;
        const bool fx0 = ((exposed >> 0) & 1) && !xl, fx1 = ((exposed >> 1) & 1) && !xh;
        const bool fz0 = ((exposed >> 4) & 1) && kb == 0, fz1 = (exposed >> 5) & 1;
        const float bx = fx0 ? m.b[0] : fx1 ? m.b[1] : 0.0f, ox = fx0 ? m.off[0] : fx1 ? m.off[1] : 0.0f;
        const int xmi = xl ? tx + 3 : tx + 4, xpi = xh ? tx + 5 : tx + 4;
        const int zlast = nz - 1 - kb;  // the stage's plane on the z+ face, if below hn
        double col_shed = 0.0;
        float below = s.t[0][ty + 1][tx + 4], here = s.t[1][ty + 1][tx + 4];
#pragma unroll
        for (int h = 0; h < P; ++h) {
            if (h >= hn) break;
            const bool zl = h > 0 || kb > 0, zh = h < zlast;
            const float above = s.t[h + 2][ty + 1][tx + 4];
            const float xm = s.t[h + 1][ty + 1][xmi], xp = s.t[h + 1][ty + 1][xpi];
            const float ym = s.t[h + 1][ty][tx + 4], yp = s.t[h + 1][ty + 2][tx + 4];
            float sum = 0.0f;
            sum += xm - here;
            sum += xp - here;
            sum += ym - here;
            sum += yp - here;
            sum += zl ? below - here : 0.0f;
            sum += zh ? above - here : 0.0f;
            float shed = __fmaf_rn(bx, here + ox, 0.0f);
            if (h == 0 && fz0) shed = __fmaf_rn(m.b[4], here + m.off[4], shed);
            if (fz1 && !zh) shed = __fmaf_rn(m.b[5], here + m.off[5], shed);
            if (exposed) col_shed += (double)shed;
            const float nd = __fadd_rn(here, __fmaf_rn(ga, sum, -shed));
            *out = nd;
            out += plane;
            acc[0] += (double)nd;
            below = here;
            here = above;
        }
        acc[1] += col_shed;
    } else {
        // The general form, taken by the whole warp: its row (y) and each plane (z) are
        // the same for every lane, so those tests are uniform, and a lane on an x face
        // selects its terms rather than diverging. The sums start at +0 and so are never
        // −0, which makes adding +0 for an absent neighbour or film exact; the film terms
        // are the fused b·(here + off) + shed that the plain `shed += ...` contracts to.
        const int exposed = m.exposed;
        const bool ex0 = xedge && ((exposed >> 0) & 1), ex1 = xedge && ((exposed >> 1) & 1);
        const bool ey0 = ((exposed >> 2) & 1) && !yl, ey1 = ((exposed >> 3) & 1) && !yh;
        const bool ez0 = ((exposed >> 4) & 1) && kb == 0;  // plane 0 of the stage is the z− face
        const bool ez1 = (exposed >> 5) & 1;
        const int zlast = nz - 1 - kb;  // the stage's plane on the z+ face, if below P
        // the y and z films are taken only by stages on a face row or a face plane
        const bool faces = ey0 || ey1 || ez0 || (ez1 && zlast < hn);
        // the x faces' film coefficients, used by every cell of the stage, in registers
        const float b0 = m.b[0], o0 = m.off[0], b1 = m.b[1], o1 = m.off[1];
        double col_shed = 0.0;
        auto run = [&](auto faces_tag, auto full_tag) {
            constexpr bool FACES = decltype(faces_tag)::value, FULL = decltype(full_tag)::value;
            float below = s.t[0][ty + 1][tx + 4], here = s.t[1][ty + 1][tx + 4];
#pragma unroll
            for (int h = 0; h < P; ++h) {
                if (!FULL && h >= hn) break;
                const bool zl = h > 0 || kb > 0, zh = h < zlast;
                const float above = s.t[h + 2][ty + 1][tx + 4];
                const float xm = s.t[h + 1][ty + 1][tx + 3], xp = s.t[h + 1][ty + 1][tx + 5];
                float sum = 0.0f;  // the neighbours present, in the reference's order
                sum += xl ? xm - here : 0.0f;
                sum += xh ? xp - here : 0.0f;
                if (yl) sum += s.t[h + 1][ty][tx + 4] - here;
                if (yh) sum += s.t[h + 1][ty + 2][tx + 4] - here;
                if (zl) sum += below - here;
                if (zh) sum += above - here;
                float shed = 0.0f;
                if (exposed) {
                    if (ex0) {
                        const float v = __fmaf_rn(b0, here + o0, shed);
                        shed = xl ? shed : v;
                    }
                    if (ex1) {
                        const float v = __fmaf_rn(b1, here + o1, shed);
                        shed = xh ? shed : v;
                    }
                    if constexpr (FACES) {
                        if (ey0) shed = __fmaf_rn(m.b[2], here + m.off[2], shed);
                        if (ey1) shed = __fmaf_rn(m.b[3], here + m.off[3], shed);
                        if (ez0 && h == 0) shed = __fmaf_rn(m.b[4], here + m.off[4], shed);
                        if (ez1 && !zh) shed = __fmaf_rn(m.b[5], here + m.off[5], shed);
                    }
                    col_shed += (double)shed;
                }
                const float nd = __fadd_rn(here, __fmaf_rn(ga, sum, -shed));
                *out = nd;
                out += plane;
                acc[0] += (double)nd;
                below = here;
                here = above;
            }
        };
        if (faces) {
            if (hn == P) run(Flag<true>{}, Flag<true>{});
            else run(Flag<true>{}, Flag<false>{});
        } else {
            if (hn == P) run(Flag<false>{}, Flag<true>{});
            else run(Flag<false>{}, Flag<false>{});
        }
        acc[1] += col_shed;
    }
}

// Warps 0-7 consume (the cells of a 32 × 8 brick column each); warp 8 produces: it takes the
// bricks of the walk from the shared counter, one brick ahead, and for every stage issues the
// brick's record and the tile, S − 1 stages ahead. Slots are handed back and forth with a full and
// an empty mbarrier each; every wait is bounded.
template <int P, int S>
static __global__ void __launch_bounds__(kEnsConsumers + 32, PM_ENS_TMA_MIN_BLOCKS) ens_tma_step(const EnsTmaArgs t) {
    using St = EnsTmaStage<P>;
    const EnsArgs<float>& a = t.e;
    extern __shared__ __align__(128) unsigned char ens_tma_smem[];
    __shared__ EnsBrickInfo info[S];
    __shared__ unsigned stage_brick[S];
    __shared__ int stage_kb[S], stage_z1[S];  // stage_z1 < 0: the walk is over
    __shared__ unsigned holdmask[kEnsHoldBlocks / 32];
    const St* ring = reinterpret_cast<const St*>(ens_tma_smem);
    const unsigned ring_base = static_cast<unsigned>(__cvta_generic_to_shared(ens_tma_smem));
    const unsigned full_base = ring_base + S * (unsigned)sizeof(St), empty_base = full_base + 8 * S;
    const unsigned info_base = static_cast<unsigned>(__cvta_generic_to_shared(info));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // A block's flag changes only after all its bricks of a launch are done, so the flags read
    // at the start hold for the whole launch (the host keeps this path to ≤ kEnsHoldBlocks blocks).
    for (unsigned w = tid; w < (a.ngrids + 31) / 32; w += blockDim.x) {
        unsigned bits = 0;
        for (unsigned q = 0; q < 32 && 32 * w + q < a.ngrids; ++q)
            if (a.states[32 * w + q].violated) bits |= 1u << q;
        holdmask[w] = bits;
    }
    if (tid == 0) {
        for (int q = 0; q < S; ++q) {
            mbar_init(full_base + 8 * q, 1);
            mbar_init(empty_base + 8 * q, kEnsConsumers / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp == kEnsConsumers / 32) {  // the producer
        if (lane != 0) return;
        unsigned b = atomicAdd(&t.work[0], 1u);
        EnsBrick br{}, nbr{};
        if (b < a.nbricks) br = a.bricks[b];
        unsigned nb = b < a.nbricks ? atomicAdd(&t.work[0], 1u) : a.nbricks;
        if (nb < a.nbricks) nbr = a.bricks[nb];
        int kb = br.z0;
        int q = 0;
        bool ok = true;
        for (;; ++q) {
            const int slot = q % S;
            if (q >= S && !mbar_wait(empty_base + 8 * slot, (unsigned)(((q / S) - 1) & 1))) {
                ok = false;
                break;
            }
            if (b >= a.nbricks) {  // the end of the walk, released with a plain arrive
                stage_z1[slot] = -1;
                mbar_arrive(full_base + 8 * slot);
                break;
            }
            stage_brick[slot] = b;
            stage_kb[slot] = kb;
            stage_z1[slot] = br.z1;
            const unsigned full = full_base + 8 * slot;
            mbar_expect_tx(full, (unsigned)sizeof(St) + (unsigned)sizeof(EnsBrickInfo));
            bulk_load(info_base + slot * (unsigned)sizeof(EnsBrickInfo), t.infos + b, sizeof(EnsBrickInfo), full);
            tma_load_3d(ring_base + slot * (unsigned)sizeof(St), t.maps + br.grid, (int)br.x0 - 4, (int)br.y0 - 1, kb - 1,
                        full);
            kb += P;
            if (kb >= br.z1) {  // to the next brick, and take the one after it
                b = nb;
                br = nbr;
                kb = br.z0;
                nb = b < a.nbricks ? atomicAdd(&t.work[0], 1u) : a.nbricks;
                if (nb < a.nbricks) nbr = a.bricks[nb];
            }
        }
        if (!ok) {
            for (unsigned g = 0; g < a.ngrids; ++g) a.states[g].violated = kDeviceTimeout;
        }
        // the last use of each slot: its copies land before this thread (and the block) is done
        for (int u = (q >= S ? q - S + 1 : 0); u < q; ++u) mbar_wait(full_base + 8 * (u % S), (unsigned)((u / S) & 1));
        // this CTA takes no more bricks; the last CTA to get here zeroes the counters for the next
        // launch (every other CTA's last take precedes its arrival here)
        __threadfence();
        if (atomicAdd(&t.work[1], 1u) == gridDim.x - 1) {
            t.work[0] = 0u;
            t.work[1] = 0u;
            __threadfence();
        }
        return;
    }
    const int tx = lane, ty = warp;
    double acc[2] = {0.0, 0.0};  // this warp's row of the brick: Σ deviation of the new state, Σ heat shed
    int slot = 0;
    unsigned phase = 0;  // of the slot's full barrier: flips each time the ring wraps
    for (;; slot = slot + 1 == S ? 0 : slot + 1, phase ^= slot == 0 ? 1u : 0u) {
        const bool got = mbar_wait(full_base + 8 * slot, phase);
        if (__any_sync(0xffffffffu, !got)) {  // this warp stops; the others and the producer run out too
            if (lane == 0)
                for (unsigned g = 0; g < a.ngrids; ++g) a.states[g].violated = kDeviceTimeout;
            return;
        }
        const int z1 = stage_z1[slot];
        if (z1 < 0) return;  // the walk is over (every consumer reads the same word)
        const EnsBrickInfo& m = info[slot];
        const St& s = ring[slot];
        const int kb = stage_kb[slot];
        const unsigned brick = stage_brick[slot], gi = m.grid;
        const int nx = m.nx, ny = m.ny, pitch = m.pitch;
        const bool hold = (holdmask[gi >> 5] >> (gi & 31)) & 1u;
        const int i = m.x0 + tx, j = m.y0 + ty;
        if (i < nx && j < ny) {
            const size_t plane = (size_t)pitch * ny;
            // this lane's cell of the stage's first plane; each plane's store steps it by a plane
            float* __restrict__ out = a.nu + m.offset + ((size_t)i + (size_t)pitch * ((size_t)j + (size_t)ny * kb));
            const int hn = min(P, z1 - kb);  // planes of this stage in the brick
            if (hold) {
                for (int h = 0; h < hn; ++h, out += plane) *out = s.t[h + 1][ty + 1][tx + 4];
            } else {
                tma_stage_row<P>(s, m, m.x0, tx, ty, i, j, kb, hn, out, plane, acc);
            }
        }
        const bool brick_done = kb + P >= z1;
        // this warp is done with the slot (the tile and the record)
        __syncwarp();
        if (lane == 0) mbar_arrive(empty_base + 8 * slot);
        if (brick_done && !hold) {
            // this warp's two partials of the brick, stored by brick and warp; ens_tma_books sums
            // them per block once the step is done (no ordering inside this kernel, so no warp waits
            // for its field stores to land)
            warp_sum<2>(acc);
            if (lane == 0) {
                const size_t at = ((size_t)brick * 8 + (size_t)warp) * 2;
                a.partials[at] = acc[0];
                a.partials[at + 1] = acc[1];
            }
        }
        if (brick_done) acc[0] = acc[1] = 0.0;
    }
}

// The books of every block after ens_tma_step: one warp per block sums its bricks' partials in a
// fixed order (lane-strided, then the warp's tree), then runs its ledger and audit. A block held at
// the step's start (violated) was copied, not stepped, and is left alone.
static __global__ void __launch_bounds__(256) ens_tma_books(const EnsArgs<float> a) {
    const int lane = threadIdx.x & 31;
    const unsigned gi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (gi >= a.ngrids) return;
    DevState* st = a.states + gi;
    if (st->violated) return;
    const EnsGrid& g = a.grids[gi];
    double v[2] = {0.0, 0.0};
    const size_t first = (size_t)g.first_brick * 8, count = (size_t)g.nbricks * 8;
    for (size_t q = lane; q < count; q += 32) {
        v[0] += a.partials[(first + q) * 2];
        v[1] += a.partials[(first + q) * 2 + 1];
    }
    warp_sum<2>(v);
    if (lane == 0) {
        const double stored = g.capacity * v[0];
        st->lost += g.capacity * v[1];
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

// One block's cells between the caller's kelvin (x fastest, rows of nx) and the device's f32
// deviations T − T0 on rows of `pitch` (to_dev = 1; the padding zeroed by the caller), and back.
static __global__ void ens_relayout(const double* __restrict__ kelvin, float* __restrict__ dev, double* __restrict__ out,
                                    int nx, int ny, int nz, int pitch, double t0, int to_dev) {
    const size_t n = (size_t)nx * ny * nz;
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
        const size_t i = r % (size_t)nx, rest = r / (size_t)nx;
        const size_t p = i + (size_t)pitch * rest;  // rest = j + ny·k
        if (to_dev) dev[p] = (float)(kelvin[r] - t0);
        else out[r] = (double)dev[p] + t0;
    }
}

}  // namespace pm
