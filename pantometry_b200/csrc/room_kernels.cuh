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

// ---------------------------------------------------------------------------------------------
// Tube (crates/pantometry-acoustic/src/lib.rs:107-560): the same scheme in one dimension, n
// pressure samples, n−1 faces, and ends that are closed, open or matched to an impedance.
//
// tube_step — one thread per sample. Its faces come from the old pressure with the reference's
//   expression (lib.rs:402-405); an end sample's outer face is the wall's velocity from its own
//   old pressure (lib.rs:368-382, 411-412). The new pressure follows lib.rs:424-433. Fused: the
//   FP64 invariant (lib.rs:301-327), the work the moving ends publish, |p u| A dt with the new
//   pressure (lib.rs:441-450), the startup offset (lib.rs:457-462: taken only within 25%, never
//   refused), and the audit of the tube's books: its energy plus what it has published.
// ---------------------------------------------------------------------------------------------
template <typename Real>
struct TubeArgs {
    const Real* __restrict__ p0;
    const Real* __restrict__ v0;
    Real* __restrict__ p1;
    Real* __restrict__ v1;
    int n;
    Real gain;       // vh/(ρ·dx)
    Real coef;       // dt·ρc²/dx
    double outward[2];  // end k's outward sign (−1 left, +1 right), 0 when closed
    double z[2];        // the impedance end k's wall velocity divides by (lib.rs:368-382)
    double knode;       // V/(2ρc²), V = area·dx; 0 with ρc² ≤ 0
    double kface;       // ρ/2·V; 0 with ρc² ≤ 0
    double area, dt;    // for the published work
    int starting;
    DevState* st;
    double* partials;
    unsigned nblocks;
};

template <typename Real>
static __global__ void __launch_bounds__(256) tube_step(TubeArgs<Real> a) {
    DevState* st = a.st;
    if (st->violated) return;
    const int n = a.n;
    const Real gain = a.gain;
    double acc[2] = {0.0, 0.0};  // the invariant of the new state, the work published this step
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Real pc = a.p0[i];
        Real inflow, outflow;
        // u = outward·p/Z at an open or matched end, 0 at a closed one
        if (i == 0) inflow = a.outward[0] == 0.0 ? Real(0) : (Real)(a.outward[0] * (double)pc / a.z[0]);
        else inflow = a.v0[i - 1] - gain * (pc - a.p0[i - 1]);
        if (i == n - 1) outflow = a.outward[1] == 0.0 ? Real(0) : (Real)(a.outward[1] * (double)pc / a.z[1]);
        else outflow = a.v0[i] - gain * (a.p0[i + 1] - pc);
        if (i < n - 1) a.v1[i] = outflow;
        const bool end = i == 0 || i == n - 1;
        const Real share = end ? Real(2) : Real(1);
        const Real np = pc - a.coef * share * (outflow - inflow);
        a.p1[i] = np;
        const double dn = (double)np, dof = (double)outflow;
        acc[0] += (end ? 0.5 : 1.0) * a.knode * dn * (double)pc + (i < n - 1 ? a.kface * (dof * dof) : 0.0);
        if (i == 0) acc[1] += fabs(dn * (double)inflow) * a.area * a.dt;
        if (i == n - 1) acc[1] += fabs(dn * (double)outflow) * a.area * a.dt;
    }
    if (finish_blocks<2>(acc, a.partials, a.nblocks, &st->counter) && linear_tid() == 0) {
        const double invariant = acc[0];
        if (a.starting) {
            const double off = st->datum - invariant;
            const double sc = rmax(fabs(st->datum), fabs(invariant));
            if (sc > 0.0 && fabs(off) / sc <= 0.25) st->offset = off;
        }
        st->injected += acc[1];  // the published total
        const double energy = invariant + st->offset;
        double total = 0.0, scale_l = 0.0;
        ledger_add(total, scale_l, energy);
        ledger_add(total, scale_l, st->injected);
        st->part[0] = energy;
        st->part[1] = st->injected;
        st->invariant = invariant;
        audit_and_commit(st, total, scale_l);
    }
}

template <typename Real>
struct TubeMeasureArgs {
    const Real* p;
    const Real* pp;
    const Real* v;
    int n;
    double knode, kface;
    DevState* st;
    double* partials;
    unsigned nblocks;
};

template <typename Real>
static __global__ void __launch_bounds__(256) tube_measure(TubeMeasureArgs<Real> a) {
    const int n = a.n;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double u = i < n - 1 ? (double)a.v[i] : 0.0;
        acc[0] += ((i == 0 || i == n - 1) ? 0.5 : 1.0) * a.knode * (double)a.p[i] * (double)a.pp[i] + a.kface * (u * u);
    }
    if (finish_blocks<1>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) a.st->invariant = acc[0];
}

}  // namespace pm
