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
// z-chunk) and steps through each tile's planes; neighbouring blocks hold neighbouring tiles at
// the same time, so a tile's x and y halos come out of L2.
//
// Staging. Each plane of a tile — the pressures with a one-node halo in x and y, the pressures
// of the plane above, the face velocities on both sides of the nodes — is copied into a ring of
// kStages shared-memory stages with cp.async, up to kStages − 1 planes ahead of the plane being
// computed, and the copies run on across tile boundaries. Every thread copies its own node's
// five values plus at most one fixed halo value, so a plane costs a handful of instructions and
// one barrier.
template <typename Real> struct HallDepth;
template <> struct HallDepth<float> { static constexpr int stages = 6, min_blocks = 4; };
template <> struct HallDepth<double> { static constexpr int stages = 4, min_blocks = 3; };

template <typename Real>
struct HallStage {
    Real p[10][34];  // p(x0-1 .. x0+32, y0-1 .. y0+8, k)
    Real pa[8][32];  // p(x0 .. x0+31, y0 .. y0+7, k+1)
    Real vx[8][33];  // x faces x0-1 .. x0+31
    Real vy[9][32];  // y faces y0-1 .. y0+7
    Real vz[8][32];  // z faces at k
};

struct HallCursor {
    long long t;
    int x0, y0, k, k0, k1;
    bool valid;
};

__device__ __forceinline__ void hall_cursor_at(HallCursor& c, const Tiles& T, long long t) {
    c.t = t;
    c.valid = t < T.ntiles;
    if (!c.valid) return;
    const int tx = (int)(t % T.ntx);
    const long long r = t / T.ntx;
    c.x0 = tx * 32;
    c.y0 = (int)(r % T.nty) * 8;
    c.k0 = c.k = (int)(r / T.nty) * T.zc;
    c.k1 = min(T.nz, c.k + T.zc);
}
__device__ __forceinline__ void hall_cursor_next(HallCursor& c, const Tiles& T) {
    if (++c.k >= c.k1) hall_cursor_at(c, T, c.t + gridDim.x);
}

// The one halo value thread `tid` copies, as (row, column) in the stage's p tile (kind 0), the
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

// A thread's offsets into the four arrays for its node of one tile, at the tile's first plane,
// and the per-plane strides. Every array here has fewer than 2^32 elements.
struct HallOffsets {
    unsigned p, fx, fy;  // p and vz share the node index
    unsigned halo;       // the thread's halo value, if any
    bool live, xh, yh, halo_live;
};

__device__ __forceinline__ HallOffsets hall_offsets(const HallCursor& c, int nx, int ny, const HallHalo& h) {
    HallOffsets o;
    const int i = c.x0 + threadIdx.x, j = c.y0 + threadIdx.y, k = c.k;
    o.live = i < nx && j < ny;
    o.xh = i + 1 < nx;
    o.yh = j + 1 < ny;
    o.p = (unsigned)i + (unsigned)nx * ((unsigned)j + (unsigned)ny * (unsigned)k);
    o.fx = (unsigned)i + (unsigned)(nx - 1) * ((unsigned)j + (unsigned)ny * (unsigned)k);
    o.fy = (unsigned)i + (unsigned)nx * ((unsigned)j + (unsigned)(ny - 1) * (unsigned)k);
    o.halo = 0;
    o.halo_live = false;
    if (h.kind == 0) {
        const int gi = c.x0 - 1 + h.c, gj = c.y0 - 1 + h.r;
        o.halo_live = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
        o.halo = (unsigned)gi + (unsigned)nx * ((unsigned)gj + (unsigned)ny * (unsigned)k);
    } else if (h.kind == 1) {
        const int fi = c.x0 - 1, gj = c.y0 + h.r;
        o.halo_live = fi >= 0 && gj < ny;
        o.halo = (unsigned)fi + (unsigned)(nx - 1) * ((unsigned)gj + (unsigned)ny * (unsigned)k);
    } else if (h.kind == 2) {
        const int gi = c.x0 + h.c, fj = c.y0 - 1;
        o.halo_live = gi < nx && fj >= 0;
        o.halo = (unsigned)gi + (unsigned)nx * ((unsigned)fj + (unsigned)(ny - 1) * (unsigned)k);
    }
    return o;
}

template <typename Real>
__device__ __forceinline__ void hall_stage(HallStage<Real>& st, const HallArgs<Real>& a, const HallOffsets& o,
                                           bool zh, const HallHalo& h) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    if (o.live) {
        cp_async<sizeof(Real)>(&st.p[ty + 1][tx + 1], a.p0 + o.p);
        if (zh) {
            cp_async<sizeof(Real)>(&st.pa[ty][tx], a.p0 + o.p + (unsigned)a.nx * (unsigned)a.ny);
            cp_async<sizeof(Real)>(&st.vz[ty][tx], a.vz0 + o.p);
        }
        if (o.xh) cp_async<sizeof(Real)>(&st.vx[ty][tx + 1], a.vx0 + o.fx);
        if (o.yh) cp_async<sizeof(Real)>(&st.vy[ty + 1][tx], a.vy0 + o.fy);
    }
    if (o.halo_live) {
        if (h.kind == 0) cp_async<sizeof(Real)>(&st.p[h.r][h.c], a.p0 + o.halo);
        else if (h.kind == 1) cp_async<sizeof(Real)>(&st.vx[h.r][0], a.vx0 + o.halo);
        else cp_async<sizeof(Real)>(&st.vy[0][h.c], a.vy0 + o.halo);
    }
}

__device__ __forceinline__ void hall_offsets_next(HallOffsets& o, const HallHalo& h, unsigned sp, unsigned sx,
                                                  unsigned sy) {
    o.p += sp;
    o.fx += sx;
    o.fy += sy;
    o.halo += h.kind == 0 ? sp : (h.kind == 1 ? sx : sy);
}

template <typename Real, bool HET>
static __global__ void __launch_bounds__(256, HallDepth<Real>::min_blocks) hall_step(HallArgs<Real> a) {
    DevState* st = a.st;
    if (st->violated) return;
    constexpr int S = HallDepth<Real>::stages;
    extern __shared__ __align__(16) unsigned char hall_smem[];
    HallStage<Real>* ring = reinterpret_cast<HallStage<Real>*>(hall_smem);
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

    HallCursor pf, cc;
    hall_cursor_at(pf, T, blockIdx.x);
    hall_cursor_at(cc, T, blockIdx.x);
    HallOffsets po = hall_offsets(pf, nx, ny, halo);
    for (int d = 0; d < S - 1; ++d) {
        if (pf.valid) hall_stage<Real>(ring[d], a, po, pf.k + 1 < nz, halo);
        cp_async_commit();
        const long long t = pf.t;
        hall_cursor_next(pf, T);
        if (pf.t != t) po = hall_offsets(pf, nx, ny, halo);
        else hall_offsets_next(po, halo, sp, sx, sy);
    }
    // per tile: this thread's node offsets and its invariant weights
    HallOffsets co = hall_offsets(cc, nx, ny, halo);
    double cn = 0.0, cxf = 0.0, cyf = 0.0, czf = 0.0;  // node, x-face, y-face, z-face weights
    Real wi = Real(1), wj = Real(1);
    bool xl = false, yl = false, src_col = false;
    Real sc = a.scale;
    double kn = a.knode;
    Real lz = Real(0);
    long long tile = -1;
    int slot = 0;
    while (cc.valid) {
        cp_async_wait<S - 2>();  // this thread's copies of the plane have landed
        __syncthreads();         // ... and everyone's; and everyone is done with the previous plane
        if (pf.valid) hall_stage<Real>(ring[(slot + S - 1) % S], a, po, pf.k + 1 < nz, halo);
        cp_async_commit();
        {
            const long long t = pf.t;
            hall_cursor_next(pf, T);
            if (pf.t != t) po = hall_offsets(pf, nx, ny, halo);
            else hall_offsets_next(po, halo, sp, sx, sy);
        }
        const int i = cc.x0 + tx, j = cc.y0 + ty, k = cc.k;
        if (cc.t != tile) {  // a new tile: the weights that are constant over a column
            tile = cc.t;
            xl = i > 0;
            yl = j > 0;
            // hall.rs:675-681: weight 2 on a wall, 1 inside; the share 1/w is an exact power of two
            wi = (xl && co.xh) ? Real(1) : Real(2);
            wj = (yl && co.yh) ? Real(1) : Real(2);
            const double si = (xl && co.xh) ? 1.0 : 0.5, sj = (yl && co.yh) ? 1.0 : 0.5;
            src_col = i == a.src_i && j == a.src_j;
            if (HET) {
                const int b = i / a.block + a.nbx * (j / a.block + a.nby * (k / a.block));
                sc = a.block_scale[b];
                kn = a.block_knode[b];
            }
            cn = si * sj * kn;
            cxf = a.kface * sj;
            cyf = a.kface * si;
            czf = a.kface * si * sj;
            if (co.live) {
                // the low z face of the tile's first node, from the old state:
                // vz(k-1) − gain·(p(k) − p(k-1))
                lz = Real(0);
                if (k > 0) lz = a.vz0[co.p - sp] - gain * (a.p0[co.p] - a.p0[co.p - sp]);
            }
        }
        const HallStage<Real>& c = ring[slot];
        if (co.live) {
            if (HET && (k % a.block) == 0) {
                const int b = i / a.block + a.nbx * (j / a.block + a.nby * (k / a.block));
                sc = a.block_scale[b];
                kn = a.block_knode[b];
                cn = (((xl && co.xh) ? 1.0 : 0.5) * ((yl && co.yh) ? 1.0 : 0.5)) * kn;
            }
            const Real pc = c.p[ty + 1][tx + 1];
            const bool zh = k + 1 < nz;
            Real hx = Real(0), lx = Real(0), hy = Real(0), ly = Real(0), hz = Real(0);
            if (co.xh) {
                hx = c.vx[ty][tx + 1] - gain * (c.p[ty + 1][tx + 2] - pc);
                a.vx1[co.fx] = hx;
            }
            if (xl) lx = c.vx[ty][tx] - gain * (pc - c.p[ty + 1][tx]);
            if (co.yh) {
                hy = c.vy[ty + 1][tx] - gain * (c.p[ty + 2][tx + 1] - pc);
                a.vy1[co.fy] = hy;
            }
            if (yl) ly = c.vy[ty][tx] - gain * (pc - c.p[ty][tx + 1]);
            if (zh) {
                hz = c.vz[ty][tx] - gain * (c.pa[ty][tx] - pc);
                a.vz1[co.p] = hz;
            }
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
            a.p1[co.p] = np;
            // hall.rs:345-349 (share · p · p_prev / 2ρc² · V) and 356-382 (share · ½ρv² · V on
            // the node's own high faces)
            const double dhx = (double)hx, dhy = (double)hy, dhz = (double)hz;
            const double sk = zin ? 1.0 : 0.5;
            acc[0] += sk * (cn * (double)np * (double)pc + cxf * dhx * dhx + cyf * dhy * dhy) + czf * dhz * dhz;
            lz = hz;
        }
        {
            const long long t = cc.t;
            hall_cursor_next(cc, T);
            if (cc.t != t) co = hall_offsets(cc, nx, ny, halo);
            else hall_offsets_next(co, halo, sp, sx, sy);
        }
        slot = (slot + 1) % S;
    }
    cp_async_wait<0>();
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
        double total = 0.0, scale = 0.0;
        const double energy = plus + st->offset - st->injected;
        ledger_add(total, scale, energy);
        st->part[0] = energy;
        st->invariant = plus;
        audit_and_commit(st, total, scale);
    }
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
                const double v = a.vx[(size_t)i + (size_t)(nx - 1) * ((size_t)j + (size_t)ny * k)];
                inv += (1.0 / (wj * wk)) * a.kface * v * v;
            }
            if (j + 1 < ny) {
                const double v = a.vy[(size_t)i + (size_t)nx * ((size_t)j + (size_t)(ny - 1) * k)];
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
