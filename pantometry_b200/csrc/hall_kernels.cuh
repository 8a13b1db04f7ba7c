// Hall stepping kernel (crates/pantometry-acoustic/src/hall.rs:408-530), fused.
//
// The reference makes four passes per step — three face-velocity passes, a copy of the
// pressure into `pressure_prev`, then the node pass — and a sixth pass for the ledger
// (`invariant_si`, hall.rs:334-384). Here one kernel does all of it per node:
//   * the new velocity on the node's three high faces (which it owns and writes) and on its
//     three low faces (which it recomputes from the old state rather than waits for),
//   * the new pressure from those six velocities with the wall weights (hall.rs:675-681),
//   * the invariant terms of the node and of its owned faces, in FP64.
// Old and new states are separate buffers (a ping-pong pair), so no thread ever reads a value
// another thread has already advanced, and `pressure_prev` is simply the old pressure buffer.
//
// Real = double with --fmad=false is the plain form, bit-exact with `Hall::step`: every field
// value is formed by the reference's own expression in its own order. Real = float is the
// chosen form; its invariant is still accumulated in FP64.
#pragma once

#include "common.cuh"

namespace pm {

template <typename Real>
struct HallArgs {
    const Real* __restrict__ p0;
    const Real* __restrict__ vx0;
    const Real* __restrict__ vy0;
    const Real* __restrict__ vz0;
    Real* __restrict__ p1;
    Real* __restrict__ vx1;
    Real* __restrict__ vy1;
    Real* __restrict__ vz1;
    int nx, ny, nz;
    Real gain;   // vh / (ρ·dx)          (hall.rs:433)
    Real scale;  // h·ρc² / dx           (hall.rs:464)
    // Heterogeneous speed (extension): per-block scale and invariant weight; null = uniform.
    const Real* __restrict__ block_scale;
    const double* __restrict__ block_knode;
    int block, nbx, nby;
    double knode;    // V / (2ρc²): weight of p·p_prev in the invariant
    double kface;    // ½ρ·V: weight of v² in the invariant
    // Point source (extension): wave[steps] added at `src` after the pressure update.
    long long src;
    int src_i, src_j, src_k;  // the source node (src_i = -1: none)
    const double* __restrict__ wave;
    long long nwave;
    double wsrc;     // the source node's share · V/(2ρc²)
    int starting;    // first step: half-step velocities, and the startup offset (hall.rs:513-528)
    Tiles tiles;
    DevState* st;
    double* partials;
    unsigned nblocks;
};

__device__ __forceinline__ double wall_weight(int k, int n) { return (k == 0 || k + 1 == n) ? 2.0 : 1.0; }

// The walk. Block b takes tiles b, b + G, b + 2G, ... (a tile is a 32 × 8 column of nodes over a
// z-chunk) and steps through each tile's planes two at a time; neighbouring blocks hold
// neighbouring tiles at the same time, so a tile's x and y halos come out of L2.
//
// Staging. Each pair of planes of a tile — the pressures of both planes with a one-node halo in
// x and y, the pressures of the plane above the pair, and the face velocities — is copied into a
// ring of HallDepth::stages shared-memory stages with cp.async, running ahead of the pair being
// computed and on across tile boundaries. Every thread copies its own nodes' values plus at most
// one fixed halo value per plane, so a pair costs a handful of copy instructions and one barrier.
template <typename Real> struct HallDepth;
template <> struct HallDepth<float> { static constexpr int stages = 4, min_blocks = 3; };
template <> struct HallDepth<double> { static constexpr int stages = 3, min_blocks = 2; };

template <typename Real>
struct HallStage {
    Real p[2][10][34];  // p(x0-1 .. x0+32, y0-1 .. y0+8, k + h), h = 0, 1
    Real pa[8][32];     // p(x0 .. x0+31, y0 .. y0+7, k+2)
    Real vx[2][8][33];  // x faces x0-1 .. x0+31
    Real vy[2][9][32];  // y faces y0-1 .. y0+7
    Real vz[2][8][32];  // z faces at k + h
    Real pb[8][32];     // p(.., k-1) and vz(.., k-1): the plane below, at a tile's first pair only
    Real vzb[8][32];
};

struct HallCursor {
    unsigned t;
    int x0, y0, k, k0, k1;
    bool valid;
};

// Tile t of the tiling (fewer than 2^32 tiles): 32-bit divisions only, once per tile.
__device__ __forceinline__ void hall_cursor_at(HallCursor& c, const Tiles& T, unsigned t) {
    c.t = t;
    c.valid = t < (unsigned)T.ntiles;
    if (!c.valid) return;
    const unsigned r = t / (unsigned)T.ntx;
    const unsigned tz = r / (unsigned)T.nty;
    c.x0 = (int)(t - r * (unsigned)T.ntx) * 32;
    c.y0 = (int)(r - tz * (unsigned)T.nty) * 8;
    c.k0 = c.k = (int)tz * T.zc;
    c.k1 = min(T.nz, c.k + T.zc);
}
// to the next pair of planes; returns whether a new tile began
__device__ __forceinline__ bool hall_cursor_next(HallCursor& c, const Tiles& T) {
    c.k += 2;
    if (c.k < c.k1) return false;
    hall_cursor_at(c, T, c.t + gridDim.x);
    return true;
}

// The one halo value thread `tid` copies per plane, as (row, column) in the p tile (kind 0), the
// x-face column (kind 1) or the y-face row (kind 2); kind -1 for none.
struct HallHalo {
    int kind, r, c;
};
__device__ __forceinline__ HallHalo hall_halo(int tid) {
    HallHalo h{-1, 0, 0};
    if (tid < 34) h = HallHalo{0, 0, tid};
    else if (tid < 68) h = HallHalo{0, 9, tid - 34};
    else if (tid < 76) h = HallHalo{0, tid - 68 + 1, 0};
    else if (tid < 84) h = HallHalo{0, tid - 76 + 1, 33};
    else if (tid < 92) h = HallHalo{1, tid - 84, 0};
    else if (tid < 124) h = HallHalo{2, 0, tid - 92};
    return h;
}

// What a thread copies for one tile: the global offsets of its node at plane k (every array here
// has fewer than 2^32 elements), whether each value exists, and its halo value's array, offset and
// plane stride, chosen once per tile so that the copies themselves never branch.
struct HallCopy {
    unsigned p, fx, fy;      // p and vz share the node index
    unsigned halo, hstride;  // the halo value's offset and per-plane stride
    unsigned hplane;         // bytes from the halo value's slot in the pair's first plane to its second
    bool live, xh, yh, halo_live;
};

template <typename Real>
__device__ __forceinline__ HallCopy hall_copy_at(const HallCursor& c, const HallArgs<Real>& a, const HallHalo& h,
                                                 unsigned sp, unsigned sx, unsigned sy) {
    HallCopy o;
    const int nx = a.nx, ny = a.ny;
    const int i = c.x0 + threadIdx.x, j = c.y0 + threadIdx.y, k = c.k;
    o.live = i < nx && j < ny;
    o.xh = o.live && i + 1 < nx;
    o.yh = o.live && j + 1 < ny;
    o.p = (unsigned)i + (unsigned)nx * ((unsigned)j + (unsigned)ny * (unsigned)k);
    o.fx = (unsigned)i + (unsigned)(nx - 1) * ((unsigned)j + (unsigned)ny * (unsigned)k);
    o.fy = (unsigned)i + (unsigned)nx * ((unsigned)j + (unsigned)(ny - 1) * (unsigned)k);
    o.halo = 0;
    o.hstride = 0;
    o.hplane = 0;
    o.halo_live = false;
    if (h.kind == 0) {
        const int gi = c.x0 - 1 + h.c, gj = c.y0 - 1 + h.r;
        o.halo_live = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
        o.halo = (unsigned)gi + (unsigned)nx * ((unsigned)gj + (unsigned)ny * (unsigned)k);
        o.hstride = sp;
        o.hplane = sizeof(Real) * 10 * 34;
    } else if (h.kind == 1) {
        const int fi = c.x0 - 1, gj = c.y0 + h.r;
        o.halo_live = fi >= 0 && gj < ny;
        o.halo = (unsigned)fi + (unsigned)(nx - 1) * ((unsigned)gj + (unsigned)ny * (unsigned)k);
        o.hstride = sx;
        o.hplane = sizeof(Real) * 8 * 33;
    } else if (h.kind == 2) {
        const int gi = c.x0 + h.c, fj = c.y0 - 1;
        o.halo_live = gi < nx && fj >= 0;
        o.halo = (unsigned)gi + (unsigned)nx * ((unsigned)fj + (unsigned)(ny - 1) * (unsigned)k);
        o.hstride = sy;
        o.hplane = sizeof(Real) * 9 * 32;
    }
    return o;
}

__device__ __forceinline__ void hall_copy_next(HallCopy& o, unsigned sp, unsigned sx, unsigned sy) {
    o.p += 2 * sp;
    o.fx += 2 * sx;
    o.fy += 2 * sy;
    o.halo += 2 * o.hstride;
}

// Byte offset within a stage of one of this thread's values.
template <typename Real>
__device__ __forceinline__ unsigned hall_at(const Real* q) {
    return (unsigned)((const char*)q - (const char*)static_cast<const HallStage<Real>*>(nullptr));
}

// Byte offset within a stage of this thread's halo value (plane h).
template <typename Real>
__device__ __forceinline__ unsigned hall_halo_at(const HallHalo& h, int plane) {
    const HallStage<Real>* z = nullptr;
    if (h.kind == 0) return hall_at<Real>(&z->p[plane][h.r][h.c]);
    if (h.kind == 1) return hall_at<Real>(&z->vx[plane][h.r][0]);
    return hall_at<Real>(&z->vy[plane][0][h.c < 32 ? h.c : 0]);
}

// Queue the copies of the pair (k, k+1) of cursor c into the stage at shared address `base`.
template <typename Real>
__device__ __forceinline__ void hall_stage(unsigned base, unsigned halo_at, const HallArgs<Real>& a,
                                           const HallCursor& c, const HallCopy& o, const Real* hsrc, unsigned sp,
                                           unsigned sx, unsigned sy) {
    constexpr int B = sizeof(Real);
    constexpr unsigned PLANE_P = sizeof(Real) * 10 * 34, PLANE_VX = sizeof(Real) * 8 * 33, PLANE_VY = sizeof(Real) * 9 * 32,
                       PLANE_VZ = sizeof(Real) * 8 * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const HallStage<Real>* z = nullptr;
    const unsigned sp0 = base + hall_at<Real>(&z->p[0][ty + 1][tx + 1]);
    const unsigned svx = base + hall_at<Real>(&z->vx[0][ty][tx + 1]);
    const unsigned svy = base + hall_at<Real>(&z->vy[0][ty + 1][tx]);
    const unsigned svz = base + hall_at<Real>(&z->vz[0][ty][tx]);
    const unsigned spa = base + hall_at<Real>(&z->pa[ty][tx]);
    const int nz = a.nz, k = c.k;
    const bool two = k + 1 < c.k1;  // the pair's second plane is computed here
    const bool z1 = o.live && k + 1 < nz, z2 = o.live && two && k + 2 < nz;
    cp_async_if<B>(sp0, a.p0 + o.p, o.live);
    cp_async_if<B>(sp0 + PLANE_P, a.p0 + o.p + sp, z1);
    cp_async_if<B>(svz, a.vz0 + o.p, z1);
    cp_async_if<B>(svx, a.vx0 + o.fx, o.xh);
    cp_async_if<B>(svy, a.vy0 + o.fy, o.yh);
    cp_async_if<B>(spa, a.p0 + o.p + 2 * sp, z2);
    cp_async_if<B>(svz + PLANE_VZ, a.vz0 + o.p + sp, z2);
    cp_async_if<B>(svx + PLANE_VX, a.vx0 + o.fx + sx, o.xh && two);
    cp_async_if<B>(svy + PLANE_VY, a.vy0 + o.fy + sy, o.yh && two);
    // the plane below a tile's first pair, for the low z face of its first node
    const bool below = o.live && k == c.k0 && k > 0;
    cp_async_if<B>(base + hall_at<Real>(&z->pb[ty][tx]), a.p0 + (below ? o.p - sp : o.p), below);
    cp_async_if<B>(base + hall_at<Real>(&z->vzb[ty][tx]), a.vz0 + (below ? o.p - sp : o.p), below);
    cp_async_if<B>(base + halo_at, hsrc + o.halo, o.halo_live);
    cp_async_if<B>(base + halo_at + o.hplane, hsrc + o.halo + o.hstride, o.halo_live && two);
}

// The step's ledger, in the last block: the invariant of the new state, the source's injected
// work, the startup offset on the first step (hall.rs:513-528) and the audit.
template <typename Real>
__device__ __forceinline__ void hall_finish(const HallArgs<Real>& a, double (&acc)[3], double delta) {
    DevState* st = a.st;
    if (finish_blocks<3>(acc, a.partials, a.nblocks, &st->counter) && linear_tid() == 0) {
        const double plus = acc[0];
        st->injected += acc[2];
        st->last_delta = delta;
        if (a.starting) {
            // hall.rs:513-528, with the invariant taken before this step's injection
            const double invariant = plus - acc[1];
            const double off = st->datum - invariant;
            const double sc = rmax(fabs(st->datum), fabs(invariant));
            if (sc > 0.0 && fabs(off) / sc > 0.25) {
                st->violated = kStartupFailed;
                st->violation_step = st->steps + 1;
                st->v_before = st->datum;
                st->v_after = invariant;
                st->v_scale = sc;
                st->v_tol = 0.25;
            } else {
                st->offset = off;
            }
        }
        // the energy, then the source's injected work as an entry of its own (zero without a
        // source): the total is the same sum, and the scale covers what the source moved
        double total = 0.0, scale = 0.0;
        ledger_add(total, scale, plus + st->offset);
        ledger_add(total, scale, -st->injected);
        st->part[0] = total;
        st->invariant = plus;
        audit_and_commit(st, total, scale);
    }
}

template <typename Real, bool HET>
static __global__ void __launch_bounds__(256, HallDepth<Real>::min_blocks) hall_step(HallArgs<Real> a) {
    DevState* st = a.st;
    if (st->violated) return;
    constexpr int S = HallDepth<Real>::stages;
    constexpr unsigned STAGE = sizeof(HallStage<Real>);
    extern __shared__ __align__(16) unsigned char hall_smem[];
    HallStage<Real>* ring = reinterpret_cast<HallStage<Real>*>(hall_smem);
    const unsigned ring_base = static_cast<unsigned>(__cvta_generic_to_shared(hall_smem));
    const long long step = st->steps;
    const double delta = (a.src_i >= 0 && step < a.nwave) ? a.wave[step] : 0.0;
    const double last_delta = st->last_delta;
    double acc[3] = {0.0, 0.0, 0.0};  // invariant, immediate source term, injected increment

    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const unsigned sp = (unsigned)nx * (unsigned)ny, sx = (unsigned)(nx - 1) * (unsigned)ny,
                   sy = (unsigned)nx * (unsigned)(ny - 1);
    const Real gain = a.gain;
    const Tiles T = a.tiles;
    const HallHalo halo = hall_halo(tx + 32 * ty);
    const unsigned halo_at = hall_halo_at<Real>(halo, 0);
    const Real* hsrc = halo.kind == 1 ? a.vx0 : (halo.kind == 2 ? a.vy0 : a.p0);

    HallCursor pf, cc;
    hall_cursor_at(pf, T, blockIdx.x);
    hall_cursor_at(cc, T, blockIdx.x);
    HallCopy po = hall_copy_at<Real>(pf, a, halo, sp, sx, sy);
    for (int d = 0; d < S - 1; ++d) {
        if (pf.valid) hall_stage<Real>(ring_base + d * STAGE, halo_at, a, pf, po, hsrc, sp, sx, sy);
        cp_async_commit();
        if (hall_cursor_next(pf, T)) po = hall_copy_at<Real>(pf, a, halo, sp, sx, sy);
        else hall_copy_next(po, sp, sx, sy);
    }
    // per tile: this thread's node offsets and its invariant weights
    HallCopy co = hall_copy_at<Real>(cc, a, halo, sp, sx, sy);
    bool fresh = true;
    double cn = 0.0, cxf = 0.0, cyf = 0.0, czf = 0.0;  // node, x-face, y-face, z-face weights
    Real wi = Real(1), wj = Real(1);
    bool xl = false, yl = false, src_col = false;
    Real sc = a.scale;
    double kn = a.knode;
    Real lz = Real(0);
    int slot = 0;
    while (cc.valid) {
        cp_async_wait<S - 2>();  // this thread's copies of the pair have landed
        __syncthreads();         // ... and everyone's; and everyone is done with the previous pair
        {
            const int fill = slot == 0 ? S - 1 : slot - 1;
            if (pf.valid) hall_stage<Real>(ring_base + fill * STAGE, halo_at, a, pf, po, hsrc, sp, sx, sy);
            cp_async_commit();
            if (hall_cursor_next(pf, T)) po = hall_copy_at<Real>(pf, a, halo, sp, sx, sy);
            else hall_copy_next(po, sp, sx, sy);
        }
        const int i = cc.x0 + tx, j = cc.y0 + ty;
        if (fresh) {  // a new tile: the weights that are constant over a column
            fresh = false;
            xl = i > 0;
            yl = j > 0;
            // hall.rs:675-681: weight 2 on a wall, 1 inside; the share 1/w is an exact power of two
            wi = (xl && co.xh) ? Real(1) : Real(2);
            wj = (yl && co.yh) ? Real(1) : Real(2);
            const double si = (xl && co.xh) ? 1.0 : 0.5, sj = (yl && co.yh) ? 1.0 : 0.5;
            src_col = i == a.src_i && j == a.src_j;
            cn = si * sj * kn;
            cxf = a.kface * sj;
            cyf = a.kface * si;
            czf = a.kface * si * sj;
        }
        const HallStage<Real>& c = ring[slot];
        if (cc.k == cc.k0) {
            // the low z face of the tile's first node, from the old state staged with the pair:
            // vz(k-1) − gain·(p(k) − p(k-1))
            lz = cc.k > 0 ? c.vzb[ty][tx] - gain * (c.p[0][ty + 1][tx + 1] - c.pb[ty][tx]) : Real(0);
        }
        if (co.live) {
            unsigned op = co.p, ofx = co.fx, ofy = co.fy;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = cc.k + h;
                if (h == 1 && k >= cc.k1) break;
                if (HET && (h == 0 || (k % a.block) == 0)) {
                    const int b = i / a.block + a.nbx * (j / a.block + a.nby * (k / a.block));
                    sc = a.block_scale[b];
                    kn = a.block_knode[b];
                    cn = (((xl && co.xh) ? 1.0 : 0.5) * ((yl && co.yh) ? 1.0 : 0.5)) * kn;
                }
                // Every staged read is in bounds; a value with no face behind it is computed
                // and then replaced by the reference's 0.0.
                const Real pc = c.p[h][ty + 1][tx + 1];
                const bool zh = k + 1 < nz;
                const Real above = h == 0 ? c.p[1][ty + 1][tx + 1] : c.pa[ty][tx];
                const Real hx0 = c.vx[h][ty][tx + 1] - gain * (c.p[h][ty + 1][tx + 2] - pc);
                const Real lx0 = c.vx[h][ty][tx] - gain * (pc - c.p[h][ty + 1][tx]);
                const Real hy0 = c.vy[h][ty + 1][tx] - gain * (c.p[h][ty + 2][tx + 1] - pc);
                const Real ly0 = c.vy[h][ty][tx] - gain * (pc - c.p[h][ty][tx + 1]);
                const Real hz0 = c.vz[h][ty][tx] - gain * (above - pc);
                const Real hx = co.xh ? hx0 : Real(0), lx = xl ? lx0 : Real(0);
                const Real hy = co.yh ? hy0 : Real(0), ly = yl ? ly0 : Real(0);
                const Real hz = zh ? hz0 : Real(0);
                if (co.xh) a.vx1[ofx] = hx;
                if (co.yh) a.vy1[ofy] = hy;
                if (zh) a.vz1[op] = hz;
                const bool zin = k > 0 && zh;
                const Real wk = zin ? Real(1) : Real(2);
                // hall.rs:499-502
                Real np = pc - sc * (wi * (hx - lx) + wj * (hy - ly) + wk * (hz - lz));
                if (src_col && k == a.src_k) {
                    // deferred term of the previous injection, then this one's
                    acc[2] += a.wsrc * (last_delta + delta) * (double)pc;
                    acc[1] += a.wsrc * delta * (double)pc;
                    np = (Real)((double)np + delta);
                }
                a.p1[op] = np;
                // hall.rs:345-349 (share · p · p_prev / 2ρc² · V) and 356-382 (share · ½ρv² · V
                // on the node's own high faces)
                const double dhx = (double)hx, dhy = (double)hy, dhz = (double)hz;
                const double sk = zin ? 1.0 : 0.5;
                acc[0] += sk * (cn * (double)np * (double)pc + cxf * dhx * dhx + cyf * dhy * dhy) + czf * dhz * dhz;
                lz = hz;
                op += sp;
                ofx += sx;
                ofy += sy;
            }
        }
        if (hall_cursor_next(cc, T)) {
            co = hall_copy_at<Real>(cc, a, halo, sp, sx, sy);
            fresh = true;
        } else {
            hall_copy_next(co, sp, sx, sy);
        }
        slot = slot + 1 == S ? 0 : slot + 1;
    }
    cp_async_wait<0>();
    hall_finish<Real>(a, acc, delta);
}

// `invariant_si` of an uploaded state (hall.rs:334-384), for `released_from`'s datum.
template <typename Real>
struct HallMeasureArgs {
    const Real* p;
    const Real* pp;
    const Real* vx;
    const Real* vy;
    const Real* vz;
    int nx, ny, nz;
    double knode, kface;
    const double* __restrict__ block_knode;
    int block, nbx, nby;
    int padded;  // face arrays laid out like the nodes (nx·ny·nz each), as the TMA form keeps them
    Tiles tiles;
    DevState* st;
    double* partials;
    unsigned nblocks;
};

template <typename Real>
static __global__ void __launch_bounds__(256) hall_measure(HallMeasureArgs<Real> a) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    double acc[1] = {0.0};
    for (long long t = blockIdx.x; t < a.tiles.ntiles; t += gridDim.x) {
        const int tx = (int)(t % a.tiles.ntx);
        const long long r = t / a.tiles.ntx;
        const int i = tx * 32 + threadIdx.x;
        const int j = (int)(r % a.tiles.nty) * 8 + threadIdx.y;
        const int k0 = (int)(r / a.tiles.nty) * a.tiles.zc;
        const int k1 = min(nz, k0 + a.tiles.zc);
        if (i >= nx || j >= ny) continue;
        for (int k = k0; k < k1; ++k) {
            const size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
            const double wi = wall_weight(i, nx), wj = wall_weight(j, ny), wk = wall_weight(k, nz);
            double kn = a.knode;
            if (a.block_knode) kn = a.block_knode[i / a.block + a.nbx * (j / a.block + a.nby * (k / a.block))];
            double inv = (1.0 / (wi * wj * wk)) * (double)a.p[idx] * (double)a.pp[idx] * kn;
            if (i + 1 < nx) {
                const double v = a.vx[a.padded ? idx : (size_t)i + (size_t)(nx - 1) * ((size_t)j + (size_t)ny * k)];
                inv += (1.0 / (wj * wk)) * a.kface * v * v;
            }
            if (j + 1 < ny) {
                const double v = a.vy[a.padded ? idx : (size_t)i + (size_t)nx * ((size_t)j + (size_t)(ny - 1) * k)];
                inv += (1.0 / (wi * wk)) * a.kface * v * v;
            }
            if (k + 1 < nz) {
                const double v = a.vz[idx];
                inv += (1.0 / (wi * wj)) * a.kface * v * v;
            }
            acc[0] += inv;
        }
    }
    if (finish_blocks<1>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) {
        a.st->invariant = acc[0];
    }
}

}  // namespace pm
