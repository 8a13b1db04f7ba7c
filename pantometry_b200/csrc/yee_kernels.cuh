// Cavity (Yee FDTD) stepping kernels (crates/pantometry-em/src/cavity.rs:1346-1501).
//
// Per step the reference runs: three H passes; a clone of H; the invariant — two full passes
// that pair Eⁿ with H⁻ and H⁺ (cavity.rs:1490-1496); three E passes; the wall pass; the
// obstacle pass. Here a step is two kernels over the (nx+1)(ny+1)(nz+1) node lattice:
//
//   yee_h  — H⁺ = H⁻ − (dt/dx)/μ · curl Eⁿ for every face (cavity.rs:1346-1379), in place
//            (each face is read and written by its own thread only), with the invariant's two
//            halves accumulated in the same pass: ½εEⁿ² over the edges that share the thread's
//            lattice index (cavity.rs:776-847) and ½μ H⁺·H⁻ over its faces (cavity.rs:854-905).
//            H⁻ is the value in the register before the store, so the clone disappears.
//   yee_e  — Eⁿ⁺¹ on interior edges with the semi-implicit loss (cavity.rs:1383-1452), zero on
//            conducting walls (cavity.rs:1239-1293), zero on edges touching a solid cell
//            (cavity.rs:304-331); the Joule loss and the source work in FP64; then the ledger
//            `invariant + dissipated` (cavity.rs:1520-1524) and the audit in the last block.
//
// Real = double with --fmad=false is the plain form, bit-exact with `Cavity::step`.
#pragma once

#include "common.cuh"

namespace pm {

template <typename Real>
struct YeeHArgs {
    const Real* __restrict__ ex;
    const Real* __restrict__ ey;
    const Real* __restrict__ ez;
    Real* __restrict__ hx;
    Real* __restrict__ hy;
    Real* __restrict__ hz;
    int nx, ny, nz;
    double g;                        // dt / dx
    int uniform;
    Real ch;                         // uniform: g / μ
    const double* __restrict__ mu0;  // general: μ per face component
    const double* __restrict__ mu1;
    const double* __restrict__ mu2;
    int energy;                      // 1: accumulate the invariant and store it
    double eps_u, mu_u;              // uniform ε (edge mean) and μ
    const double* __restrict__ eps0;
    const double* __restrict__ eps1;
    const double* __restrict__ eps2;
    double volume;                   // dx³
    DevState* st;
    double* partials;
    unsigned nblocks;
};

__device__ __forceinline__ double half_if(bool end) { return end ? 0.5 : 1.0; }

template <typename Real>
static __global__ void __launch_bounds__(256) yee_h(YeeHArgs<Real> a) {
    if (a.st->violated) return;
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    // index helpers, cavity.rs:1044-1067
    auto iex = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)nx * ((size_t)jj + (size_t)(ny + 1) * kk); };
    auto iey = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)(nx + 1) * ((size_t)jj + (size_t)ny * kk); };
    auto iez = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)(nx + 1) * ((size_t)jj + (size_t)(ny + 1) * kk); };
    auto ihx = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)(nx + 1) * ((size_t)jj + (size_t)ny * kk); };
    auto ihy = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)nx * ((size_t)jj + (size_t)(ny + 1) * kk); };
    auto ihz = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)nx * ((size_t)jj + (size_t)ny * kk); };
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // Σ wεEx², Σ wεEy², Σ wεEz², Σ wμHx⁺Hx⁻, ...
    if (i <= nx && j <= ny && k <= nz) {
        if (j < ny && k < nz) {  // hx over (nx+1) × ny × nz
            const Real curl = (a.ez[iez(i, j + 1, k)] - a.ez[iez(i, j, k)]) - (a.ey[iey(i, j, k + 1)] - a.ey[iey(i, j, k)]);
            const size_t idx = ihx(i, j, k);
            const Real was = a.hx[idx];
            double mu = a.mu_u;
            Real c = a.ch;
            if (!a.uniform) { mu = a.mu0[idx]; c = (Real)(a.g / mu); }
            const Real now = was - c * curl;
            a.hx[idx] = now;
            if (a.energy) acc[3] = half_if(i == 0 || i == nx) * mu * (double)now * (double)was;
        }
        if (i < nx && k < nz) {  // hy over nx × (ny+1) × nz
            const Real curl = (a.ex[iex(i, j, k + 1)] - a.ex[iex(i, j, k)]) - (a.ez[iez(i + 1, j, k)] - a.ez[iez(i, j, k)]);
            const size_t idx = ihy(i, j, k);
            const Real was = a.hy[idx];
            double mu = a.mu_u;
            Real c = a.ch;
            if (!a.uniform) { mu = a.mu1[idx]; c = (Real)(a.g / mu); }
            const Real now = was - c * curl;
            a.hy[idx] = now;
            if (a.energy) acc[4] = half_if(j == 0 || j == ny) * mu * (double)now * (double)was;
        }
        if (i < nx && j < ny) {  // hz over nx × ny × (nz+1)
            const Real curl = (a.ey[iey(i + 1, j, k)] - a.ey[iey(i, j, k)]) - (a.ex[iex(i, j + 1, k)] - a.ex[iex(i, j, k)]);
            const size_t idx = ihz(i, j, k);
            const Real was = a.hz[idx];
            double mu = a.mu_u;
            Real c = a.ch;
            if (!a.uniform) { mu = a.mu2[idx]; c = (Real)(a.g / mu); }
            const Real now = was - c * curl;
            a.hz[idx] = now;
            if (a.energy) acc[5] = half_if(k == 0 || k == nz) * mu * (double)now * (double)was;
        }
        if (a.energy) {
            if (i < nx) {  // ex: cell-centred in x, node-centred in y and z
                const size_t idx = iex(i, j, k);
                const double e = a.uniform ? a.eps_u : a.eps0[idx];
                const double f = (double)a.ex[idx];
                acc[0] = 1.0 * half_if(j == 0 || j == ny) * half_if(k == 0 || k == nz) * e * f * f;
            }
            if (j < ny) {
                const size_t idx = iey(i, j, k);
                const double e = a.uniform ? a.eps_u : a.eps1[idx];
                const double f = (double)a.ey[idx];
                acc[1] = half_if(i == 0 || i == nx) * 1.0 * half_if(k == 0 || k == nz) * e * f * f;
            }
            if (k < nz) {
                const size_t idx = iez(i, j, k);
                const double e = a.uniform ? a.eps_u : a.eps2[idx];
                const double f = (double)a.ez[idx];
                acc[2] = half_if(i == 0 || i == nx) * half_if(j == 0 || j == ny) * 1.0 * e * f * f;
            }
        }
    }
    if (!a.energy) return;
    if (finish_blocks<6>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) {
        const double v = a.volume;
        const double electric = 0.5 * ((acc[0] + acc[1]) + acc[2]) * v;
        const double paired = 0.5 * v * ((acc[3] + acc[4]) + acc[5]);
        a.st->invariant = electric + paired;
        a.st->has_invariant = 1;
    }
}

template <typename Real>
struct YeeEArgs {
    Real* __restrict__ ex;
    Real* __restrict__ ey;
    Real* __restrict__ ez;
    const Real* __restrict__ hx;
    const Real* __restrict__ hy;
    const Real* __restrict__ hz;
    int nx, ny, nz;
    double dt, dx, volume;
    int uniform;
    Real decay[3], gain[3];             // uniform: per component, from the edge-mean ε and σ
    double sigma_u[3];
    const double* __restrict__ eps0;    // general: ε, σ per edge component
    const double* __restrict__ eps1;
    const double* __restrict__ eps2;
    const double* __restrict__ sig0;
    const double* __restrict__ sig1;
    const double* __restrict__ sig2;
    const uint8_t* __restrict__ solid;  // per cell, or null
    long long src;                      // Ez edge with a soft current (extension), or -1
    const double* __restrict__ current;
    long long ncurrent;
    double eps_src, sig_src;            // ε, σ at the source edge
    int with_source;
    DevState* st;
    double* partials;
    unsigned nblocks;
};

template <typename Real>
__device__ __forceinline__ void coefficients(double eps, double sigma, double dt, double dx, Real& decay, Real& gain) {
    // cavity.rs:1391-1397
    const double half = sigma * dt / (2.0 * eps);
    decay = (Real)((1.0 - half) / (1.0 + half));
    gain = (Real)((dt / (eps * dx)) / (1.0 + half));
}

__device__ __forceinline__ bool touches_solid(const uint8_t* solid, int nx, int ny, int nz, int ci0, int ci1,
                                              int cj0, int cj1, int ck0, int ck1) {
    for (int kk = ck0; kk <= ck1; ++kk)
        for (int jj = cj0; jj <= cj1; ++jj)
            for (int ii = ci0; ii <= ci1; ++ii)
                if (ii >= 0 && ii < nx && jj >= 0 && jj < ny && kk >= 0 && kk < nz &&
                    solid[(size_t)ii + (size_t)nx * ((size_t)jj + (size_t)ny * kk)])
                    return true;
    return false;
}

template <typename Real>
static __global__ void __launch_bounds__(256) yee_e(YeeEArgs<Real> a) {
    DevState* st = a.st;
    if (st->violated) return;
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    auto iex = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)nx * ((size_t)jj + (size_t)(ny + 1) * kk); };
    auto iey = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)(nx + 1) * ((size_t)jj + (size_t)ny * kk); };
    auto iez = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)(nx + 1) * ((size_t)jj + (size_t)(ny + 1) * kk); };
    auto ihx = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)(nx + 1) * ((size_t)jj + (size_t)ny * kk); };
    auto ihy = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)nx * ((size_t)jj + (size_t)(ny + 1) * kk); };
    auto ihz = [&](int ii, int jj, int kk) { return (size_t)ii + (size_t)nx * ((size_t)jj + (size_t)ny * kk); };
    const long long step = st->steps;
    const double jsrc = (a.with_source && step < a.ncurrent) ? a.current[step] : 0.0;
    const double dt = a.dt;
    double acc[2] = {0.0, 0.0};  // Joule loss, source work
    if (i <= nx && j <= ny && k <= nz) {
        if (i < nx) {  // ex over nx × (ny+1) × (nz+1); interior j in 1..ny-1, k in 1..nz-1
            const size_t idx = iex(i, j, k);
            Real v = Real(0);
            if (j >= 1 && j < ny && k >= 1 && k < nz) {
                const Real curl = (a.hz[ihz(i, j, k)] - a.hz[ihz(i, j - 1, k)]) - (a.hy[ihy(i, j, k)] - a.hy[ihy(i, j, k - 1)]);
                Real decay = a.decay[0], gain = a.gain[0];
                double s = a.sigma_u[0];
                if (!a.uniform) { s = a.sig0[idx]; coefficients<Real>(a.eps0[idx], s, dt, a.dx, decay, gain); }
                const Real before = a.ex[idx];
                v = decay * before + gain * curl;
                const double mid = 0.5 * ((double)before + (double)v);
                acc[0] += s * mid * mid * dt * a.volume;
            }
            if (a.solid && touches_solid(a.solid, nx, ny, nz, i, i, j - 1, j, k - 1, k)) v = Real(0);
            a.ex[idx] = v;
        }
        if (j < ny) {  // ey over (nx+1) × ny × (nz+1); interior i in 1..nx-1, k in 1..nz-1
            const size_t idx = iey(i, j, k);
            Real v = Real(0);
            if (i >= 1 && i < nx && k >= 1 && k < nz) {
                const Real curl = (a.hx[ihx(i, j, k)] - a.hx[ihx(i, j, k - 1)]) - (a.hz[ihz(i, j, k)] - a.hz[ihz(i - 1, j, k)]);
                Real decay = a.decay[1], gain = a.gain[1];
                double s = a.sigma_u[1];
                if (!a.uniform) { s = a.sig1[idx]; coefficients<Real>(a.eps1[idx], s, dt, a.dx, decay, gain); }
                const Real before = a.ey[idx];
                v = decay * before + gain * curl;
                const double mid = 0.5 * ((double)before + (double)v);
                acc[0] += s * mid * mid * dt * a.volume;
            }
            if (a.solid && touches_solid(a.solid, nx, ny, nz, i - 1, i, j, j, k - 1, k)) v = Real(0);
            a.ey[idx] = v;
        }
        if (k < nz) {  // ez over (nx+1) × (ny+1) × nz; interior i in 1..nx-1, j in 1..ny-1
            const size_t idx = iez(i, j, k);
            Real v = Real(0);
            if (i >= 1 && i < nx && j >= 1 && j < ny) {
                const Real curl = (a.hy[ihy(i, j, k)] - a.hy[ihy(i - 1, j, k)]) - (a.hx[ihx(i, j, k)] - a.hx[ihx(i, j - 1, k)]);
                Real decay = a.decay[2], gain = a.gain[2];
                double s = a.sigma_u[2];
                if (!a.uniform) { s = a.sig2[idx]; coefficients<Real>(a.eps2[idx], s, dt, a.dx, decay, gain); }
                const Real before = a.ez[idx];
                v = decay * before + gain * curl;
                if ((long long)idx == a.src) {
                    // soft current: ε dE/dt = ∇×H − J, with the σ term's semi-implicit divisor
                    const double e = a.eps_src, ss = a.sig_src;
                    v = (Real)((double)v - (dt / e) / (1.0 + (ss * dt / (2.0 * e))) * jsrc);
                    acc[1] += -(dt * a.volume) * jsrc * (0.5 * ((double)before + (double)v));
                }
                const double mid = 0.5 * ((double)before + (double)v);
                acc[0] += s * mid * mid * dt * a.volume;
            }
            if (a.solid && touches_solid(a.solid, nx, ny, nz, i - 1, i, j - 1, j, k, k)) v = Real(0);
            a.ez[idx] = v;
        }
    }
    if (finish_blocks<2>(acc, a.partials, a.nblocks, &st->counter) && linear_tid() == 0) {
        st->dissipated += fmax(acc[0], 0.0);
        st->work += acc[1];
        double total = 0.0, scale = 0.0;
        ledger_add(total, scale, st->invariant);
        ledger_add(total, scale, st->dissipated);
        if (a.with_source) ledger_add(total, scale, -st->work);
        st->part[0] = st->invariant;
        st->part[1] = st->dissipated;
        st->part[2] = -st->work;
        audit_and_commit(st, total, scale);
    }
}

// ½εE² and ½μH² of the present state (cavity.rs:824-847, 919-940): the naive energy the
// ledger reports before any invariant exists, and what pm_cavity_energies returns.
template <typename Real>
static __global__ void __launch_bounds__(256) yee_measure(YeeHArgs<Real> a, double* out2) {
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i <= nx && j <= ny && k <= nz) {
        if (i < nx) {
            const size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)(ny + 1) * k);
            const double f = (double)a.ex[idx];
            acc[0] = half_if(j == 0 || j == ny) * half_if(k == 0 || k == nz) * (a.uniform ? a.eps_u : a.eps0[idx]) * f * f;
        }
        if (j < ny) {
            const size_t idx = (size_t)i + (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k);
            const double f = (double)a.ey[idx];
            acc[1] = half_if(i == 0 || i == nx) * half_if(k == 0 || k == nz) * (a.uniform ? a.eps_u : a.eps1[idx]) * f * f;
        }
        if (k < nz) {
            const size_t idx = (size_t)i + (size_t)(nx + 1) * ((size_t)j + (size_t)(ny + 1) * k);
            const double f = (double)a.ez[idx];
            acc[2] = half_if(i == 0 || i == nx) * half_if(j == 0 || j == ny) * (a.uniform ? a.eps_u : a.eps2[idx]) * f * f;
        }
        if (j < ny && k < nz) {
            const size_t idx = (size_t)i + (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k);
            const double f = (double)a.hx[idx];
            acc[3] = half_if(i == 0 || i == nx) * (a.uniform ? a.mu_u : a.mu0[idx]) * f * f;
        }
        if (i < nx && k < nz) {
            const size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)(ny + 1) * k);
            const double f = (double)a.hy[idx];
            acc[4] = half_if(j == 0 || j == ny) * (a.uniform ? a.mu_u : a.mu1[idx]) * f * f;
        }
        if (i < nx && j < ny) {
            const size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
            const double f = (double)a.hz[idx];
            acc[5] = half_if(k == 0 || k == nz) * (a.uniform ? a.mu_u : a.mu2[idx]) * f * f;
        }
    }
    if (finish_blocks<6>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) {
        const double v = a.volume;
        out2[0] = 0.5 * ((acc[0] + acc[1]) + acc[2]) * v;
        out2[1] = 0.5 * ((acc[3] + acc[4]) + acc[5]) * v;
    }
}

}  // namespace pm
