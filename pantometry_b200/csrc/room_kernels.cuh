// Room stepping kernels (crates/pantometry-acoustic/src/room.rs:368-478): the two-dimensional
// staggered scheme, pressure at the nodes (i + nx·j), vx on the (nx−1)·ny faces between
// horizontal neighbours (i + (nx−1)·j), vy on the nx·(ny−1) faces between vertical ones
// (i + nx·j), rigid walls.
//
// room_step — one thread per node over a persistent grid. The reference updates every face from
//   the old pressure, then every pressure from the new faces; here each node forms its four faces
//   from the old state with the reference's own expression (so a face shared by two nodes is
//   computed twice, identically), writes the faces it owns (right and upper) into the other buffer
//   of each ping-pong pair, then its new pressure. The plain f64 form (built with --fmad=false)
//   is bit-exact with `Room::step`. Fused: the FP64 invariant of the new state (room.rs:243-281:
//   share·pⁿ⁺¹·pⁿ·V/(2ρc²) per node, ρu²/2·V over the wall weight per face), the startup offset
//   on the first step (room.rs:448-476) and the audit, in the last block.
//
// room_measure — the invariant of a state, for the datum of a release and for a restore.
#pragma once

#include "common.cuh"

namespace pm {

template <typename Real>
struct RoomArgs {
    const Real* __restrict__ p0;
    const Real* __restrict__ vx0;
    const Real* __restrict__ vy0;
    Real* __restrict__ p1;
    Real* __restrict__ vx1;
    Real* __restrict__ vy1;
    int nx, ny;
    Real gain;      // vh/(ρ·dx), vh = h/2 on the first step (room.rs:387-409)
    Real scale;     // h·ρc²/dx (room.rs:443)
    double knode;   // V/(2ρc²), V = dx²·depth; 0 with ρc² ≤ 0 (room.rs:246-248)
    double kface;   // ρ/2·V; 0 with ρc² ≤ 0
    int starting;
    DevState* st;
    double* partials;
    unsigned nblocks;
};

__device__ __forceinline__ double room_share(int k, int n) { return (k == 0 || k + 1 == n) ? 0.5 : 1.0; }

template <typename Real>
static __global__ void __launch_bounds__(256) room_step(RoomArgs<Real> a) {
    DevState* st = a.st;
    if (st->violated) return;
    const int nx = a.nx, ny = a.ny;
    const size_t n = (size_t)nx * ny, fx = (size_t)(nx - 1);
    const Real gain = a.gain, scale = a.scale;
    double acc[1] = {0.0};
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % (size_t)nx), j = (int)(c / (size_t)nx);
        const Real pc = a.p0[c];
        // room.rs:405-418: ρ du/dt = −∇p on every face, from the old pressure
        const Real left = i > 0 ? a.vx0[fx * j + i - 1] - gain * (pc - a.p0[c - 1]) : Real(0);
        const Real right = i < nx - 1 ? a.vx0[fx * j + i] - gain * (a.p0[c + 1] - pc) : Real(0);
        const Real below = j > 0 ? a.vy0[c - nx] - gain * (pc - a.p0[c - nx]) : Real(0);
        const Real above = j < ny - 1 ? a.vy0[c] - gain * (a.p0[c + nx] - pc) : Real(0);
        if (i < nx - 1) a.vx1[fx * j + i] = right;
        if (j < ny - 1) a.vy1[c] = above;
        // room.rs:420-446: dp/dt = −ρc² ∇·u, a wall node's divergence over half the spacing
        const Real wi = (i == 0 || i == nx - 1) ? Real(2) : Real(1);
        const Real wj = (j == 0 || j == ny - 1) ? Real(2) : Real(1);
        const Real np = pc - scale * (wi * (right - left) + wj * (above - below));
        a.p1[c] = np;
        const double si = room_share(i, nx), sj = room_share(j, ny);
        const double dr = (double)right, da = (double)above;
        acc[0] += (si * sj) * a.knode * (double)np * (double)pc + sj * a.kface * (dr * dr) + si * a.kface * (da * da);
    }
    if (finish_blocks<1>(acc, a.partials, a.nblocks, &st->counter) && linear_tid() == 0) {
        const double invariant = acc[0];
        if (a.starting) {
            // room.rs:448-476: the released state's datum against the staggered invariant
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
        double total = 0.0, scale_l = 0.0;
        ledger_add(total, scale_l, invariant + st->offset);  // room.rs:480-482
        st->part[0] = total;
        st->invariant = invariant;
        audit_and_commit(st, total, scale_l);
    }
}

template <typename Real>
struct RoomMeasureArgs {
    const Real* p;
    const Real* pp;
    const Real* vx;
    const Real* vy;
    int nx, ny;
    double knode, kface;
    DevState* st;
    double* partials;
    unsigned nblocks;
};

template <typename Real>
static __global__ void __launch_bounds__(256) room_measure(RoomMeasureArgs<Real> a) {
    const int nx = a.nx, ny = a.ny;
    const size_t n = (size_t)nx * ny, fx = (size_t)(nx - 1);
    double acc[1] = {0.0};
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % (size_t)nx), j = (int)(c / (size_t)nx);
        const double si = room_share(i, nx), sj = room_share(j, ny);
        const double dr = i < nx - 1 ? (double)a.vx[fx * j + i] : 0.0;
        const double da = j < ny - 1 ? (double)a.vy[c] : 0.0;
        acc[0] += (si * sj) * a.knode * (double)a.p[c] * (double)a.pp[c] + sj * a.kface * (dr * dr) + si * a.kface * (da * da);
    }
    if (finish_blocks<1>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) a.st->invariant = acc[0];
}

}  // namespace pm
