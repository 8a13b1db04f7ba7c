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
    Tiles tiles;                     // over the (nx+1) × (ny+1) × (nz+1) node lattice
    DevState* st;
    double* partials;
    unsigned nblocks;
};

__device__ __forceinline__ double half_if(bool end) { return end ? 0.5 : 1.0; }

template <typename Real>
static __global__ void __launch_bounds__(256) yee_h(YeeHArgs<Real> a) {
    if (a.st->violated) return;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    // strides of the six arrays (cavity.rs:1044-1067): x fastest, then y, then z
    const size_t sEx = (size_t)nx * (ny + 1), sEy = (size_t)(nx + 1) * ny, sEz = (size_t)(nx + 1) * (ny + 1);
    const size_t sHx = (size_t)(nx + 1) * ny, sHy = (size_t)nx * (ny + 1), sHz = (size_t)nx * ny;
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // Σ wεEx², Σ wεEy², Σ wεEz², Σ wμHx⁺Hx⁻, ...
    for (long long t = blockIdx.x; t < a.tiles.ntiles; t += gridDim.x) {
        const int tx = (int)(t % a.tiles.ntx);
        const long long r = t / a.tiles.ntx;
        const int i = tx * 32 + threadIdx.x;
        const int j = (int)(r % a.tiles.nty) * 8 + threadIdx.y;
        const int k0 = (int)(r / a.tiles.nty) * a.tiles.zc;
        const int k1 = min(nz + 1, k0 + a.tiles.zc);
        if (i > nx || j > ny) continue;
        const bool hx_col = j < ny, hy_col = i < nx, hz_col = i < nx && j < ny;
        const size_t ex0 = (size_t)i + (size_t)nx * j, ey0 = (size_t)i + (size_t)(nx + 1) * j;
        const size_t ez0 = (size_t)i + (size_t)(nx + 1) * j;
        const size_t hx0 = (size_t)i + (size_t)(nx + 1) * j, hy0 = (size_t)i + (size_t)nx * j, hz0 = (size_t)i + (size_t)nx * j;
        // Ey(i, j, k) and Ex(i, j, k) of the present plane, carried from the previous plane's k+1
        Real ey_k = (j < ny) ? a.ey[ey0 + sEy * k0] : Real(0);
        Real ex_k = (i < nx) ? a.ex[ex0 + sEx * k0] : Real(0);
        for (int k = k0; k < k1; ++k) {
            const bool zin = k < nz;
            const Real ey_k1 = (j < ny && zin) ? a.ey[ey0 + sEy * (k + 1)] : Real(0);
            const Real ex_k1 = (i < nx && zin) ? a.ex[ex0 + sEx * (k + 1)] : Real(0);
            if (hx_col && zin) {  // hx over (nx+1) × ny × nz (cavity.rs:1349-1358)
                const Real curl = (a.ez[ez0 + (nx + 1) + sEz * k] - a.ez[ez0 + sEz * k]) - (ey_k1 - ey_k);
                const size_t idx = hx0 + sHx * k;
                const Real was = a.hx[idx];
                double mu = a.mu_u;
                Real c = a.ch;
                if (!a.uniform) { mu = a.mu0[idx]; c = (Real)(a.g / mu); }
                const Real now = was - c * curl;
                a.hx[idx] = now;
                if (a.energy) acc[3] += half_if(i == 0 || i == nx) * mu * (double)now * (double)was;
            }
            if (hy_col && zin) {  // hy over nx × (ny+1) × nz (cavity.rs:1359-1368)
                const Real curl = (ex_k1 - ex_k) - (a.ez[ez0 + 1 + sEz * k] - a.ez[ez0 + sEz * k]);
                const size_t idx = hy0 + sHy * k;
                const Real was = a.hy[idx];
                double mu = a.mu_u;
                Real c = a.ch;
                if (!a.uniform) { mu = a.mu1[idx]; c = (Real)(a.g / mu); }
                const Real now = was - c * curl;
                a.hy[idx] = now;
                if (a.energy) acc[4] += half_if(j == 0 || j == ny) * mu * (double)now * (double)was;
            }
            if (hz_col) {  // hz over nx × ny × (nz+1) (cavity.rs:1369-1378)
                const Real curl = (a.ey[ey0 + 1 + sEy * k] - ey_k) - (a.ex[ex0 + nx + sEx * k] - ex_k);
                const size_t idx = hz0 + sHz * k;
                const Real was = a.hz[idx];
                double mu = a.mu_u;
                Real c = a.ch;
                if (!a.uniform) { mu = a.mu2[idx]; c = (Real)(a.g / mu); }
                const Real now = was - c * curl;
                a.hz[idx] = now;
                if (a.energy) acc[5] += half_if(k == 0 || k == nz) * mu * (double)now * (double)was;
            }
            if (a.energy) {
                if (i < nx) {  // ex: cell-centred in x, node-centred in y and z
                    const double e = a.uniform ? a.eps_u : a.eps0[ex0 + sEx * k];
                    const double f = (double)ex_k;
                    acc[0] += 1.0 * half_if(j == 0 || j == ny) * half_if(k == 0 || k == nz) * e * f * f;
                }
                if (j < ny) {
                    const double e = a.uniform ? a.eps_u : a.eps1[ey0 + sEy * k];
                    const double f = (double)ey_k;
                    acc[1] += half_if(i == 0 || i == nx) * 1.0 * half_if(k == 0 || k == nz) * e * f * f;
                }
                if (zin) {
                    const double e = a.uniform ? a.eps_u : a.eps2[ez0 + sEz * k];
                    const double f = (double)a.ez[ez0 + sEz * k];
                    acc[2] += half_if(i == 0 || i == nx) * half_if(j == 0 || j == ny) * 1.0 * e * f * f;
                }
            }
            ey_k = ey_k1;
            ex_k = ex_k1;
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
    Tiles tiles;
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
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t sEx = (size_t)nx * (ny + 1), sEy = (size_t)(nx + 1) * ny, sEz = (size_t)(nx + 1) * (ny + 1);
    const size_t sHx = (size_t)(nx + 1) * ny, sHy = (size_t)nx * (ny + 1), sHz = (size_t)nx * ny;
    const long long step = st->steps;
    const double jsrc = (a.with_source && step < a.ncurrent) ? a.current[step] : 0.0;
    const double dt = a.dt;
    double acc[2] = {0.0, 0.0};  // Joule loss, source work
    for (long long t = blockIdx.x; t < a.tiles.ntiles; t += gridDim.x) {
        const int tx = (int)(t % a.tiles.ntx);
        const long long r = t / a.tiles.ntx;
        const int i = tx * 32 + threadIdx.x;
        const int j = (int)(r % a.tiles.nty) * 8 + threadIdx.y;
        const int k0 = (int)(r / a.tiles.nty) * a.tiles.zc;
        const int k1 = min(nz + 1, k0 + a.tiles.zc);
        if (i > nx || j > ny) continue;
        const size_t ex0 = (size_t)i + (size_t)nx * j, ey0 = (size_t)i + (size_t)(nx + 1) * j;
        const size_t ez0 = (size_t)i + (size_t)(nx + 1) * j;
        const size_t hx0 = (size_t)i + (size_t)(nx + 1) * j, hy0 = (size_t)i + (size_t)nx * j, hz0 = (size_t)i + (size_t)nx * j;
        // hy(i, j, k-1) and hx(i, j, k-1), carried from the previous plane
        const bool xin = i >= 1 && i < nx, yin = j >= 1 && j < ny;
        Real hy_km = (k0 >= 1 && i < nx && k0 - 1 < nz) ? a.hy[hy0 + sHy * (k0 - 1)] : Real(0);
        Real hx_km = (k0 >= 1 && j < ny && k0 - 1 < nz) ? a.hx[hx0 + sHx * (k0 - 1)] : Real(0);
        for (int k = k0; k < k1; ++k) {
            const bool zin = k < nz, kint = k >= 1 && k < nz;
            const Real hy_k = (i < nx && zin) ? a.hy[hy0 + sHy * k] : Real(0);
            const Real hx_k = (j < ny && zin) ? a.hx[hx0 + sHx * k] : Real(0);
            if (i < nx) {  // ex over nx × (ny+1) × (nz+1); interior j in 1..ny-1, k in 1..nz-1
                const size_t idx = ex0 + sEx * k;
                Real v = Real(0);
                if (yin && kint) {
                    const Real curl = (a.hz[hz0 + sHz * k] - a.hz[hz0 - nx + sHz * k]) - (hy_k - hy_km);
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
                const size_t idx = ey0 + sEy * k;
                Real v = Real(0);
                if (xin && kint) {
                    const Real curl = (hx_k - hx_km) - (a.hz[hz0 + sHz * k] - a.hz[hz0 - 1 + sHz * k]);
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
            if (zin) {  // ez over (nx+1) × (ny+1) × nz; interior i in 1..nx-1, j in 1..ny-1
                const size_t idx = ez0 + sEz * k;
                Real v = Real(0);
                if (xin && yin) {
                    const Real curl = (hy_k - a.hy[hy0 - 1 + sHy * k]) - (hx_k - a.hx[hx0 - (nx + 1) + sHx * k]);
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
            hy_km = hy_k;
            hx_km = hx_k;
        }
    }
    if (finish_blocks<2>(acc, a.partials, a.nblocks, &st->counter) && linear_tid() == 0) {
        st->dissipated += fmax(acc[0], 0.0);
        // The invariant of this step was taken before this step's electric update, so the work
        // that update did is booked against the next step's invariant.
        st->work_booked = st->work;
        st->work += acc[1];
        double total = 0.0, scale = 0.0;
        ledger_add(total, scale, st->invariant);
        ledger_add(total, scale, st->dissipated);
        if (a.with_source) ledger_add(total, scale, -st->work_booked);
        st->part[0] = st->invariant;
        st->part[1] = st->dissipated;
        st->part[2] = -st->work_booked;
        audit_and_commit(st, total, scale);
    }
}

// ½εE² and ½μH² of the present state (cavity.rs:824-847, 919-940): the naive energy the
// ledger reports before any invariant exists, and what pm_cavity_energies returns.
template <typename Real>
static __global__ void __launch_bounds__(256) yee_measure(YeeHArgs<Real> a, double* out2) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (long long t = blockIdx.x; t < a.tiles.ntiles; t += gridDim.x) {
        const int tx = (int)(t % a.tiles.ntx);
        const long long r = t / a.tiles.ntx;
        const int i = tx * 32 + threadIdx.x;
        const int j = (int)(r % a.tiles.nty) * 8 + threadIdx.y;
        const int k0 = (int)(r / a.tiles.nty) * a.tiles.zc;
        const int k1 = min(nz + 1, k0 + a.tiles.zc);
        if (i > nx || j > ny) continue;
        for (int k = k0; k < k1; ++k) {
            if (i < nx) {
                const size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)(ny + 1) * k);
                const double f = (double)a.ex[idx];
                acc[0] += half_if(j == 0 || j == ny) * half_if(k == 0 || k == nz) * (a.uniform ? a.eps_u : a.eps0[idx]) * f * f;
            }
            if (j < ny) {
                const size_t idx = (size_t)i + (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k);
                const double f = (double)a.ey[idx];
                acc[1] += half_if(i == 0 || i == nx) * half_if(k == 0 || k == nz) * (a.uniform ? a.eps_u : a.eps1[idx]) * f * f;
            }
            if (k < nz) {
                const size_t idx = (size_t)i + (size_t)(nx + 1) * ((size_t)j + (size_t)(ny + 1) * k);
                const double f = (double)a.ez[idx];
                acc[2] += half_if(i == 0 || i == nx) * half_if(j == 0 || j == ny) * (a.uniform ? a.eps_u : a.eps2[idx]) * f * f;
            }
            if (j < ny && k < nz) {
                const size_t idx = (size_t)i + (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k);
                const double f = (double)a.hx[idx];
                acc[3] += half_if(i == 0 || i == nx) * (a.uniform ? a.mu_u : a.mu0[idx]) * f * f;
            }
            if (i < nx && k < nz) {
                const size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)(ny + 1) * k);
                const double f = (double)a.hy[idx];
                acc[4] += half_if(j == 0 || j == ny) * (a.uniform ? a.mu_u : a.mu1[idx]) * f * f;
            }
            if (i < nx && j < ny) {
                const size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
                const double f = (double)a.hz[idx];
                acc[5] += half_if(k == 0 || k == nz) * (a.uniform ? a.mu_u : a.mu2[idx]) * f * f;
            }
        }
    }
    if (finish_blocks<6>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) {
        const double v = a.volume;
        out2[0] = 0.5 * ((acc[0] + acc[1]) + acc[2]) * v;
        out2[1] = 0.5 * ((acc[3] + acc[4]) + acc[5]) * v;
    }
}

}  // namespace pm
