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
    const double* __restrict__ wave;
    long long nwave;
    double wsrc;     // the source node's share · V/(2ρc²)
    int starting;    // first step: half-step velocities, and the startup offset (hall.rs:513-528)
    DevState* st;
    double* partials;
    unsigned nblocks;
};

__device__ __forceinline__ double wall_weight(int k, int n) { return (k == 0 || k + 1 == n) ? 2.0 : 1.0; }

template <typename Real>
static __global__ void __launch_bounds__(256) hall_step(HallArgs<Real> a) {
    DevState* st = a.st;
    if (st->violated) return;
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int k = blockIdx.z;
    const long long step = st->steps;
    const double delta = (a.src >= 0 && step < a.nwave) ? a.wave[step] : 0.0;
    double acc[3] = {0.0, 0.0, 0.0};  // invariant, immediate source term, injected increment
    if (i < a.nx && j < a.ny) {
        const int nx = a.nx, ny = a.ny, nz = a.nz;
        const size_t plane = (size_t)nx * ny;
        const size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
        const Real gain = a.gain;
        const Real pc = a.p0[idx];
        Real hx = Real(0), lx = Real(0), hy = Real(0), ly = Real(0), hz = Real(0), lz = Real(0);
        const size_t fx = (size_t)i + (size_t)(nx - 1) * ((size_t)j + (size_t)ny * k);
        const size_t fy = (size_t)i + (size_t)nx * ((size_t)j + (size_t)(ny - 1) * k);
        if (i + 1 < nx) {
            const Real d = a.p0[idx + 1] - pc;
            hx = a.vx0[fx] - gain * d;
            a.vx1[fx] = hx;
        }
        if (i > 0) {
            const Real d = pc - a.p0[idx - 1];
            lx = a.vx0[fx - 1] - gain * d;
        }
        if (j + 1 < ny) {
            const Real d = a.p0[idx + nx] - pc;
            hy = a.vy0[fy] - gain * d;
            a.vy1[fy] = hy;
        }
        if (j > 0) {
            const Real d = pc - a.p0[idx - nx];
            ly = a.vy0[fy - nx] - gain * d;
        }
        if (k + 1 < nz) {
            const Real d = a.p0[idx + plane] - pc;
            hz = a.vz0[idx] - gain * d;
            a.vz1[idx] = hz;
        }
        if (k > 0) {
            const Real d = pc - a.p0[idx - plane];
            lz = a.vz0[idx - plane] - gain * d;
        }
        const Real wi = (Real)wall_weight(i, nx), wj = (Real)wall_weight(j, ny), wk = (Real)wall_weight(k, nz);
        Real sc = a.scale;
        double kn = a.knode;
        if (a.block_scale) {
            const int b = i / a.block + a.nbx * (j / a.block + a.nby * (k / a.block));
            sc = a.block_scale[b];
            kn = a.block_knode[b];
        }
        Real np = pc - sc * (wi * (hx - lx) + wj * (hy - ly) + wk * (hz - lz));
        if ((long long)idx == a.src) {
            // deferred term of the previous injection, then this one's (see oracle derivation)
            acc[2] = a.wsrc * (st->last_delta + delta) * (double)pc;
            acc[1] = a.wsrc * delta * (double)pc;
            np = (Real)((double)np + delta);
        }
        a.p1[idx] = np;
        // hall.rs:345-349: share · p · p_prev / (2ρc²) · V
        const double share = 1.0 / ((double)wi * (double)wj * (double)wk);
        double inv = share * (double)np * (double)pc * kn;
        // hall.rs:356-382: share · ½ρ · v² · V on the owned (high) faces
        if (i + 1 < nx) inv += (1.0 / ((double)wj * (double)wk)) * a.kface * (double)hx * (double)hx;
        if (j + 1 < ny) inv += (1.0 / ((double)wi * (double)wk)) * a.kface * (double)hy * (double)hy;
        if (k + 1 < nz) inv += (1.0 / ((double)wi * (double)wj)) * a.kface * (double)hz * (double)hz;
        acc[0] = inv;
    }
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
    DevState* st;
    double* partials;
    unsigned nblocks;
};

template <typename Real>
static __global__ void __launch_bounds__(256) hall_measure(HallMeasureArgs<Real> a) {
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int k = blockIdx.z;
    double acc[1] = {0.0};
    if (i < a.nx && j < a.ny) {
        const int nx = a.nx, ny = a.ny, nz = a.nz;
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
        acc[0] = inv;
    }
    if (finish_blocks<1>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) {
        DevState* st = a.st;
        st->invariant = acc[0];
    }
}

}  // namespace pm
