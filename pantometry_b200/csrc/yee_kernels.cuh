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

// ---------------------------------------------------------------------------------------------
// The fused step. One pass per step over ping-pong copies of E and H: H⁺ from Eⁿ, the invariant
// ½ε|Eⁿ|² + ½μ H⁻·H⁺, then Eⁿ⁺¹ from H⁺ — the reference's order inside `Cavity::step`
// (cavity.rs:1490-1500), with nothing written in place.
//
// Block b walks tiles b, b + G, ... of the (nx+1) × (ny+1) lattice (32 × 8 columns over a
// z-chunk), streaming planes k0 − 1 .. k1 through a ring of kYeeStages shared-memory stages with
// cp.async. A stage holds one plane of all six old components over the tile and a one-cell halo
// (289 halo values, at most two per thread). Per plane:
//   1. H⁺ on the tile's own faces and on the halo faces its edges need (the x0 − 1 column and
//      the y0 − 1 row — a neighbouring block computes those too, from the same old values, and
//      gets the same bits), into shared memory; the tile's own H⁺ to the new buffer; the
//      invariant's terms for the tile's own edges and faces.
//   2. one barrier, then Eⁿ⁺¹ on the tile's own edges: interior edges by the semi-implicit
//      update (cavity.rs:1383-1452), conducting walls 0, edges touching a solid cell 0. H⁺ of the
//      plane below comes from registers carried up the column (at a tile's first plane, from
//      the extra plane k0 − 1 the tile streams first).
// ---------------------------------------------------------------------------------------------
constexpr int kYeeHalo = 289;

template <typename Real> struct YeeDepth;
// At least 3: the plane computed, the plane above it, and one in flight.
template <> struct YeeDepth<float> { static constexpr int stages = 6, min_blocks = 2; };
template <> struct YeeDepth<double> { static constexpr int stages = 4, min_blocks = 2; };
static_assert(YeeDepth<float>::stages >= 3 && YeeDepth<double>::stages >= 3, "the ring holds two planes being read");

template <typename Real>
struct YeeStage {
    Real ex[10][33];  // lattice (x0-1 .. x0+31, y0-1 .. y0+8)
    Real ey[9][34];   // (x0-1 .. x0+32, y0-1 .. y0+7)
    Real ez[10][34];  // (x0-1 .. x0+32, y0-1 .. y0+8)
    Real hx[9][32];   // (x0 .. x0+31, y0-1 .. y0+7)
    Real hy[8][33];   // (x0-1 .. x0+31, y0 .. y0+7)
    Real hz[9][33];   // (x0-1 .. x0+31, y0-1 .. y0+7)
};

template <typename Real>
struct YeeHp {        // H⁺ of the present plane over the tile and its halo
    Real hx[9][32];
    Real hy[8][33];
    Real hz[9][33];
};

template <typename Real>
struct YeeStepArgs {
    const Real* old[6];  // ex ey ez hx hy hz at step n (H at n − ½)
    Real* neu[6];        // at n + 1 (H at n + ½)
    unsigned pstride[6]; // elements per plane of each component
    int nx, ny, nz;
    double g;            // dt / dx
    int uniform;
    Real ch;             // uniform: g / μ
    const double* __restrict__ mu0;
    const double* __restrict__ mu1;
    const double* __restrict__ mu2;
    double mu_u, eps_u;
    double dt, dx, volume;
    Real decay[3], gain[3];
    double sigma_u[3];
    const double* __restrict__ eps0;
    const double* __restrict__ eps1;
    const double* __restrict__ eps2;
    const double* __restrict__ sig0;
    const double* __restrict__ sig1;
    const double* __restrict__ sig2;
    const uint8_t* __restrict__ solid;
    int src_i, src_j, src_k;  // the Ez edge with a soft current (extension); src_i < 0: none
    const double* __restrict__ current;
    long long ncurrent;
    double eps_src, sig_src;
    Tiles tiles;              // over the (nx+1) × (ny+1) × (nz+1) lattice
    DevState* st;
    double* partials;
    unsigned nblocks;
    // Mixed media, the coefficients of this dt computed once by yee_coefs: gain and decay per
    // edge component, g/μ per face component. lossless: σ is 0 on every edge (decay 1, no Joule
    // term; cdecay and σ never read). mu_var: μ differs between faces (otherwise every face holds
    // mu_u and its coefficient ch; cch and μ never read).
    const Real* __restrict__ cgain[3];
    const Real* __restrict__ cdecay[3];
    const Real* __restrict__ cch[3];
    int lossless, mu_var;
    // FP32 TMA form only: a box of nb_w³ lattice nodes from (nb_x0, nb_y0, nb_z0) whose six
    // components the kernel's last block steps again in f64 (yee_near_body) once the grid's cells
    // are in; the box's energy terms are left to it, and it closes the books. nb_w = 0: none.
    int nb_x0, nb_y0, nb_z0, nb_w;
    // FP32 TMA form only: the tiles cover [0, nx) × [0, ny) of the lattice and the last column and
    // row are stepped by the wall pass (yee_tma_wall_pass). 0: the tiles cover the whole lattice.
    int wall_split;
};

// The per-edge and per-face coefficients of one dt for a cavity of mixed media, exactly the values
// the update would otherwise form at every edge and face of every step (cavity.rs:1355 and
// 1391-1397): gain and decay from ε and σ, g/μ from μ.
template <typename Real>
struct YeeCoefArgs {
    const double* eps[3];
    const double* sig[3];
    const double* mu[3];
    Real* gain[3];
    Real* decay[3];  // null: lossless
    Real* ch[3];     // null: one μ
    size_t ne[3], nf[3];
    double dt, dx, g;
    // L > 0: gain and decay go to the padded lattice (row pitch L, ny1 rows per plane) of a
    // TMA-staged cavity; ext[q] = the x and y extents of edge component q
    unsigned L, ny1;
    int ext[3][2];
};

template <typename Real>
static __global__ void yee_coefs(YeeCoefArgs<Real> a) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int q = 0; q < 3; ++q) {
        for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < a.ne[q]; c += stride) {
            Real d, g;
            coefficients<Real>(a.eps[q][c], a.sig[q][c], a.dt, a.dx, d, g);
            size_t p = c;
            if (a.L) {
                const size_t i = c % (size_t)a.ext[q][0], r = c / (size_t)a.ext[q][0];
                p = i + (size_t)a.L * (r % (size_t)a.ext[q][1] + (size_t)a.ny1 * (r / (size_t)a.ext[q][1]));
            }
            a.gain[q][p] = g;
            if (a.decay[q]) a.decay[q][p] = d;
        }
        if (a.ch[q])
            for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < a.nf[q]; c += stride)
                a.ch[q][c] = (Real)(a.g / a.mu[q][c]);
    }
}

// Halo value e (0 .. 288) of a stage: component, row, column.
__device__ __forceinline__ void yee_halo_elem(int e, int& q, int& r, int& c) {
    // ex [10][33]: column 0 (10), rows 0 and 9 of columns 1..32 (64)
    if (e < 74) { q = 0; if (e < 10) { r = e; c = 0; } else { e -= 10; r = e < 32 ? 0 : 9; c = 1 + (e & 31); } return; }
    e -= 74;
    // ey [9][34]: columns 0 and 33 (18), row 0 of columns 1..32 (32)
    if (e < 50) { q = 1; if (e < 18) { r = e % 9; c = e < 9 ? 0 : 33; } else { r = 0; c = 1 + (e - 18); } return; }
    e -= 50;
    // ez [10][34]: columns 0 and 33 (20), rows 0 and 9 of columns 1..32 (64)
    if (e < 84) { q = 2; if (e < 20) { r = e % 10; c = e < 10 ? 0 : 33; } else { e -= 20; r = e < 32 ? 0 : 9; c = 1 + (e & 31); } return; }
    e -= 84;
    // hx [9][32]: row 0 (32)
    if (e < 32) { q = 3; r = 0; c = e; return; }
    e -= 32;
    // hy [8][33]: column 0 (8)
    if (e < 8) { q = 4; r = e; c = 0; return; }
    e -= 8;
    // hz [9][33]: column 0 (9), row 0 of columns 1..32 (32)
    q = 5;
    if (e < 9) { r = e; c = 0; } else { r = 0; c = 1 + (e - 9); }
}

// Lattice origin (column 0, row 0) of each component's stage array relative to (x0, y0), and
// its row width; the component's own extents.
__device__ __forceinline__ void yee_geom(int q, int nx, int ny, int nz, int& ox, int& oy, int& W, int& ext_x, int& ext_y,
                                         int& ext_z) {
    switch (q) {
        case 0: ox = -1; oy = -1; W = 33; ext_x = nx; ext_y = ny + 1; ext_z = nz + 1; break;
        case 1: ox = -1; oy = -1; W = 34; ext_x = nx + 1; ext_y = ny; ext_z = nz + 1; break;
        case 2: ox = -1; oy = -1; W = 34; ext_x = nx + 1; ext_y = ny + 1; ext_z = nz; break;
        case 3: ox = 0; oy = -1; W = 32; ext_x = nx + 1; ext_y = ny; ext_z = nz; break;
        case 4: ox = -1; oy = 0; W = 33; ext_x = nx; ext_y = ny + 1; ext_z = nz; break;
        default: ox = -1; oy = -1; W = 33; ext_x = nx; ext_y = ny; ext_z = nz + 1; break;
    }
}

__device__ __forceinline__ unsigned yee_stage_offset(int q, int r, int c, unsigned esize) {
    // element offsets of the six arrays inside YeeStage, in order
    const unsigned start[6] = {0u, 330u, 330u + 306u, 330u + 306u + 340u, 330u + 306u + 340u + 288u,
                               330u + 306u + 340u + 288u + 264u};
    const unsigned W[6] = {33u, 34u, 34u, 32u, 33u, 33u};
    return (start[q] + (unsigned)r * W[q] + (unsigned)c) * esize;
}

struct YeeWalk {
    unsigned t;
    int x0, y0, k0, k1, k, first, last;
    bool valid;
};

__device__ __forceinline__ void yee_walk_at(YeeWalk& w, const Tiles& T, unsigned t, int nz) {
    w.t = t;
    w.valid = t < (unsigned)T.ntiles;
    if (!w.valid) return;
    const unsigned r = t / (unsigned)T.ntx;
    const unsigned tz = r / (unsigned)T.nty;
    w.x0 = (int)(t - r * (unsigned)T.ntx) * 32;
    w.y0 = (int)(r - tz * (unsigned)T.nty) * 8;
    w.k0 = (int)tz * T.zc;
    w.k1 = min(T.nz, w.k0 + T.zc);  // T.nz = nz + 1 lattice planes
    w.first = w.k0 > 0 ? w.k0 - 1 : 0;
    w.last = min(w.k1, nz);
    w.k = w.first;
}
__device__ __forceinline__ void yee_walk_next(YeeWalk& w, const Tiles& T, int nz) {
    if (++w.k > w.last) yee_walk_at(w, T, w.t + gridDim.x, nz);
}

// Per-tile copy state of one thread: its own lattice position's six offsets at the tile's first
// streamed plane and their validity, and its (up to two) halo values'.
struct YeeCopy {
    unsigned own[6];
    unsigned hoff[2];
    unsigned ownmask, hmask;  // bit q: own value q exists (in x, y); bit h: halo value h exists
};

template <typename Real>
__device__ __forceinline__ YeeCopy yee_copy_at(const YeeStepArgs<Real>& a, const YeeWalk& w, const int (&hq)[2],
                                               const int (&hr)[2], const int (&hc)[2]) {
    YeeCopy o;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int tx = threadIdx.x, ty = threadIdx.y;
    o.ownmask = 0;
    for (int q = 0; q < 6; ++q) {
        int ox, oy, W, ex, ey, ez;
        yee_geom(q, nx, ny, nz, ox, oy, W, ex, ey, ez);
        const int i = w.x0 + tx, j = w.y0 + ty;
        if (i < ex && j < ey) o.ownmask |= 1u << q;
        o.own[q] = (unsigned)(i < ex ? i : 0) + (unsigned)ex * ((unsigned)(j < ey ? j : 0) + (unsigned)ey * (unsigned)w.k);
    }
    o.hmask = 0;
    for (int h = 0; h < 2; ++h) {
        o.hoff[h] = 0;
        if (hq[h] < 0) continue;
        int ox, oy, W, ex, ey, ez;
        yee_geom(hq[h], nx, ny, nz, ox, oy, W, ex, ey, ez);
        const int gi = w.x0 + ox + hc[h], gj = w.y0 + oy + hr[h];
        if (gi >= 0 && gi < ex && gj >= 0 && gj < ey) {
            o.hmask |= 1u << h;
            o.hoff[h] = (unsigned)gi + (unsigned)ex * ((unsigned)gj + (unsigned)ey * (unsigned)w.k);
        }
    }
    return o;
}

template <typename Real>
__device__ __forceinline__ void yee_copy_next(YeeCopy& o, const YeeStepArgs<Real>& a, const int (&hq)[2]) {
#pragma unroll
    for (int q = 0; q < 6; ++q) o.own[q] += a.pstride[q];
    if (hq[0] >= 0) o.hoff[0] += a.pstride[hq[0]];
    if (hq[1] >= 0) o.hoff[1] += a.pstride[hq[1]];
}

// Queue the copies of plane w.k into the stage at shared address `base`.
template <typename Real>
__device__ __forceinline__ void yee_stage(unsigned base, const YeeStepArgs<Real>& a, const YeeWalk& w, const YeeCopy& o,
                                          const int (&hq)[2], const unsigned (&hs)[2]) {
    constexpr int B = sizeof(Real);
    const int tx = threadIdx.x, ty = threadIdx.y, nz = a.nz, k = w.k;
    const YeeStage<Real>* z = nullptr;
    auto at = [&](const Real* q) { return base + (unsigned)((const char*)q - (const char*)z); };
    const bool zin = k < nz;  // components with nz planes (ez, hx, hy) exist at this plane
    cp_async_if<B>(at(&z->ex[ty + 1][tx + 1]), a.old[0] + o.own[0], (o.ownmask >> 0) & 1);
    cp_async_if<B>(at(&z->ey[ty + 1][tx + 1]), a.old[1] + o.own[1], (o.ownmask >> 1) & 1);
    cp_async_if<B>(at(&z->ez[ty + 1][tx + 1]), a.old[2] + o.own[2], ((o.ownmask >> 2) & 1) && zin);
    cp_async_if<B>(at(&z->hx[ty + 1][tx]), a.old[3] + o.own[3], ((o.ownmask >> 3) & 1) && zin);
    cp_async_if<B>(at(&z->hy[ty][tx + 1]), a.old[4] + o.own[4], ((o.ownmask >> 4) & 1) && zin);
    cp_async_if<B>(at(&z->hz[ty + 1][tx + 1]), a.old[5] + o.own[5], (o.ownmask >> 5) & 1);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        if (hq[h] < 0) continue;
        const bool planar = hq[h] == 0 || hq[h] == 1 || hq[h] == 5;  // nz + 1 planes
        cp_async_if<B>(base + hs[h], a.old[hq[h]] + o.hoff[h], ((o.hmask >> h) & 1) && (planar || zin));
    }
}

// UNIFORM: one medium everywhere (no media arrays read); SOLID: some cells are obstacles.
template <typename Real, bool UNIFORM, bool SOLID>
static __global__ void __launch_bounds__(256, YeeDepth<Real>::min_blocks) yee_step(YeeStepArgs<Real> a) {
    DevState* st = a.st;
    if (st->violated) return;
    constexpr int S = YeeDepth<Real>::stages;
    constexpr unsigned STAGE = sizeof(YeeStage<Real>);
    extern __shared__ __align__(16) unsigned char yee_smem[];
    const YeeStage<Real>* ring = reinterpret_cast<const YeeStage<Real>*>(yee_smem);
    YeeHp<Real>* hp = reinterpret_cast<YeeHp<Real>*>(yee_smem + S * STAGE);
    const unsigned ring_base = static_cast<unsigned>(__cvta_generic_to_shared(yee_smem));
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
    const Tiles T = a.tiles;
    const long long step = st->steps;
    const double jsrc = (a.src_i >= 0 && step < a.ncurrent) ? a.current[step] : 0.0;
    const double dt = a.dt;
    const bool lossy = UNIFORM ? a.sigma_u[0] != 0.0 : !a.lossless;
    // Σ wεE², Σ wμH⁺H⁻ (each already weighted), Joule loss, source work
    double acc[4] = {0.0, 0.0, 0.0, 0.0};

    int hq[2], hr[2], hc[2];
    unsigned hs[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int e = tid + 256 * h;
        hq[h] = -1; hr[h] = 0; hc[h] = 0; hs[h] = 0;
        if (e < kYeeHalo) {
            yee_halo_elem(e, hq[h], hr[h], hc[h]);
            hs[h] = yee_stage_offset(hq[h], hr[h], hc[h], sizeof(Real));
        }
    }

    YeeWalk pf, cw;
    yee_walk_at(pf, T, blockIdx.x, nz);
    yee_walk_at(cw, T, blockIdx.x, nz);
    YeeCopy po = yee_copy_at<Real>(a, pf, hq, hr, hc);
    for (int d = 0; d < S - 1; ++d) {
        if (pf.valid) yee_stage<Real>(ring_base + d * STAGE, a, pf, po, hq, hs);
        cp_async_commit();
        const unsigned t = pf.t;
        yee_walk_next(pf, T, nz);
        if (pf.t != t) po = yee_copy_at<Real>(a, pf, hq, hr, hc);
        else yee_copy_next<Real>(po, a, hq);
    }
    Real hx_below = Real(0), hy_below = Real(0);  // H⁺ of this column at the plane below
    unsigned own_h[6];                            // this thread's offsets at the computed plane
    {
        YeeCopy co = yee_copy_at<Real>(a, cw, hq, hr, hc);
#pragma unroll
        for (int q = 0; q < 6; ++q) own_h[q] = co.own[q];
    }
    const Real ch = a.ch;
    const Real dec0 = a.decay[0], gain0 = a.gain[0];
    int slot = 0;
    while (cw.valid) {
        // This plane (slot) and the next (slot + 1, whose ex and ey the H⁺ update reads) must have
        // landed: of the S − 1 + n groups committed before plane n, all but the newest S − 3.
        cp_async_wait<S - 3>();
        __syncthreads();  // ... everyone's; and everyone is done with the oldest stage and H⁺
        {
            const int fill = slot == 0 ? S - 1 : slot - 1;
            if (pf.valid) yee_stage<Real>(ring_base + fill * STAGE, a, pf, po, hq, hs);
            cp_async_commit();
            const unsigned t = pf.t;
            yee_walk_next(pf, T, nz);
            if (pf.t != t) po = yee_copy_at<Real>(a, pf, hq, hr, hc);
            else yee_copy_next<Real>(po, a, hq);
        }
        const YeeStage<Real>& S0 = ring[slot];
        const YeeStage<Real>& S1 = ring[slot + 1 == S ? 0 : slot + 1];
        const int k = cw.k;
        const int i = cw.x0 + tx, j = cw.y0 + ty;
        const bool compute = k >= cw.k0 && k < cw.k1;  // else the extra plane below or above the chunk
        const bool zin = k < nz;
        const bool in_x = i <= nx, in_y = j <= ny;
        // node-centred half weights of the boundary samples (cavity.rs:766-772)
        const double hi = (i == 0 || i == nx) ? 0.5 : 1.0, hj = (j == 0 || j == ny) ? 0.5 : 1.0,
                     hk = (k == 0 || k == nz) ? 0.5 : 1.0;
        // ---- 1. H⁺ (cavity.rs:1346-1379) on own faces, into shared memory and the new buffer
        const bool fx = in_x && j < ny && zin, fy = i < nx && in_y && zin, fz = i < nx && j < ny;
        const Real wx = S0.hx[ty + 1][tx], wy = S0.hy[ty][tx + 1], wz = S0.hz[ty + 1][tx + 1];
        const Real ex0 = S0.ex[ty + 1][tx + 1], ey0 = S0.ey[ty + 1][tx + 1], ez0 = S0.ez[ty + 1][tx + 1];
        Real cx = ch, cy = ch, cz = ch;
        double mux = a.mu_u, muy = a.mu_u, muz = a.mu_u;
        if constexpr (!UNIFORM) {
            if (a.mu_var) {
                if (fx) { mux = a.mu0[own_h[3]]; cx = a.cch[0][own_h[3]]; }
                if (fy) { muy = a.mu1[own_h[4]]; cy = a.cch[1][own_h[4]]; }
                if (fz) { muz = a.mu2[own_h[5]]; cz = a.cch[2][own_h[5]]; }
            }
        }
        const Real hxn = wx - cx * ((S0.ez[ty + 2][tx + 1] - ez0) - (S1.ey[ty + 1][tx + 1] - ey0));
        const Real hyn = wy - cy * ((S1.ex[ty + 1][tx + 1] - ex0) - (S0.ez[ty + 1][tx + 2] - ez0));
        const Real hzn = wz - cz * ((S0.ey[ty + 1][tx + 2] - ey0) - (S0.ex[ty + 2][tx + 1] - ex0));
        hp->hx[ty + 1][tx] = hxn;
        hp->hy[ty][tx + 1] = hyn;
        hp->hz[ty + 1][tx + 1] = hzn;
        if (compute) {
            if (fx) a.neu[3][own_h[3]] = hxn;
            if (fy) a.neu[4][own_h[4]] = hyn;
            if (fz) a.neu[5][own_h[5]] = hzn;
            // ½μ H⁻·H⁺ (cavity.rs:854-905) and ½εEⁿ² (cavity.rs:776-847) on own faces and edges
            double m = 0.0, e = 0.0;
            m += fx ? hi * mux * (double)hxn * (double)wx : 0.0;
            m += fy ? hj * muy * (double)hyn * (double)wy : 0.0;
            m += fz ? hk * muz * (double)hzn * (double)wz : 0.0;
            double epx = a.eps_u, epy = a.eps_u, epz = a.eps_u;
            if constexpr (!UNIFORM) {
                if (i < nx && in_y) epx = a.eps0[own_h[0]];
                if (in_x && j < ny) epy = a.eps1[own_h[1]];
                if (in_x && in_y && zin) epz = a.eps2[own_h[2]];
            }
            const double dex = (double)ex0, dey = (double)ey0, dez = (double)ez0;
            e += (i < nx && in_y) ? hj * hk * epx * dex * dex : 0.0;
            e += (in_x && j < ny) ? hi * hk * epy * dey * dey : 0.0;
            e += (in_x && in_y && zin) ? hi * hj * epz * dez * dez : 0.0;
            acc[0] += e;
            acc[1] += m;
        }
        // halo faces: the y0 − 1 row (hx, hz) by warp 7, the x0 − 1 column (hy, hz) by warp 6
        if (compute && ty == 7) {
            Real c1 = ch, c2 = ch;
            if constexpr (!UNIFORM) {
                const int ii = cw.x0 + tx, jj = cw.y0 - 1;
                if (a.mu_var && jj >= 0 && ii <= nx && zin) c1 = a.cch[0][(unsigned)ii + (unsigned)(nx + 1) * ((unsigned)jj + (unsigned)ny * (unsigned)k)];
                if (a.mu_var && jj >= 0 && ii < nx) c2 = a.cch[2][(unsigned)ii + (unsigned)nx * ((unsigned)jj + (unsigned)ny * (unsigned)k)];
            }
            hp->hx[0][tx] = S0.hx[0][tx] - c1 * ((S0.ez[1][tx + 1] - S0.ez[0][tx + 1]) - (S1.ey[0][tx + 1] - S0.ey[0][tx + 1]));
            hp->hz[0][tx + 1] = S0.hz[0][tx + 1] - c2 * ((S0.ey[0][tx + 2] - S0.ey[0][tx + 1]) - (S0.ex[1][tx + 1] - S0.ex[0][tx + 1]));
        }
        if (compute && ty == 6 && tx < 9) {
            // column x0 − 1, rows y0 − 1 .. y0 + 7 (row index r = tx)
            const int r = tx;
            Real c1 = ch, c2 = ch;
            if constexpr (!UNIFORM) {
                const int ii = cw.x0 - 1, jj = cw.y0 - 1 + r;
                if (a.mu_var && ii >= 0 && jj >= 0 && jj <= ny && zin) c1 = a.cch[1][(unsigned)ii + (unsigned)nx * ((unsigned)jj + (unsigned)(ny + 1) * (unsigned)k)];
                if (a.mu_var && ii >= 0 && jj >= 0 && jj < ny) c2 = a.cch[2][(unsigned)ii + (unsigned)nx * ((unsigned)jj + (unsigned)ny * (unsigned)k)];
            }
            if (r >= 1) hp->hy[r - 1][0] = S0.hy[r - 1][0] - c1 * ((S1.ex[r][0] - S0.ex[r][0]) - (S0.ez[r][1] - S0.ez[r][0]));
            hp->hz[r][0] = S0.hz[r][0] - c2 * ((S0.ey[r][1] - S0.ey[r][0]) - (S0.ex[r + 1][0] - S0.ex[r][0]));
        }
        __syncthreads();
        // ---- 2. Eⁿ⁺¹ on own edges (cavity.rs:1383-1452): interior by the semi-implicit update,
        // conducting walls 0 (cavity.rs:1239-1293), edges touching a solid cell 0 (cavity.rs:304-331)
        if (compute) {
            const bool ix = i >= 1 && i < nx, iy = j >= 1 && j < ny, iz = k >= 1 && k < nz;
            const Real cex = (hp->hz[ty + 1][tx + 1] - hp->hz[ty][tx + 1]) - (hyn - hy_below);
            const Real cey = (hxn - hx_below) - (hp->hz[ty + 1][tx + 1] - hp->hz[ty + 1][tx]);
            const Real cez = (hyn - hp->hy[ty][tx]) - (hxn - hp->hx[ty][tx]);
            Real d0 = dec0, g0 = gain0, d1 = dec0, g1 = gain0, d2 = dec0, g2 = gain0;
            double s0 = a.sigma_u[0], s1 = s0, s2 = s0;
            if constexpr (!UNIFORM) {
                const bool e0 = i < nx && in_y && iy && iz, e1 = in_x && j < ny && ix && iz,
                           e2 = in_x && in_y && zin && ix && iy;
                if (e0) g0 = a.cgain[0][own_h[0]];
                if (e1) g1 = a.cgain[1][own_h[1]];
                if (e2) g2 = a.cgain[2][own_h[2]];
                if (!a.lossless) {
                    if (e0) { s0 = a.sig0[own_h[0]]; d0 = a.cdecay[0][own_h[0]]; }
                    if (e1) { s1 = a.sig1[own_h[1]]; d1 = a.cdecay[1][own_h[1]]; }
                    if (e2) { s2 = a.sig2[own_h[2]]; d2 = a.cdecay[2][own_h[2]]; }
                }
            }
            Real vx = d0 * ex0 + g0 * cex;
            Real vy = d1 * ey0 + g1 * cey;
            Real vz = d2 * ez0 + g2 * cez;
            if (i == a.src_i && j == a.src_j && k == a.src_k) {
                // soft current: ε dE/dt = ∇×H − J, with the σ term's semi-implicit divisor
                const double e = a.eps_src, ss = a.sig_src;
                vz = (Real)((double)vz - (dt / e) / (1.0 + (ss * dt / (2.0 * e))) * jsrc);
                acc[3] += -(dt * a.volume) * jsrc * (0.5 * ((double)ez0 + (double)vz));
            }
            const bool lx = iy && iz, ly = ix && iz, lz = ix && iy;  // interior edges
            vx = lx ? vx : Real(0);
            vy = ly ? vy : Real(0);
            vz = lz ? vz : Real(0);
            if (lossy) {
                const double mx = 0.5 * ((double)ex0 + (double)vx), my = 0.5 * ((double)ey0 + (double)vy),
                             mz = 0.5 * ((double)ez0 + (double)vz);
                acc[2] += (lx && i < nx && in_y) ? s0 * mx * mx * dt * a.volume : 0.0;
                acc[2] += (ly && in_x && j < ny) ? s1 * my * my * dt * a.volume : 0.0;
                acc[2] += (lz && in_x && in_y && zin) ? s2 * mz * mz * dt * a.volume : 0.0;
            }
            if constexpr (SOLID) {
                if (touches_solid(a.solid, nx, ny, nz, i, i, j - 1, j, k - 1, k)) vx = Real(0);
                if (touches_solid(a.solid, nx, ny, nz, i - 1, i, j, j, k - 1, k)) vy = Real(0);
                if (touches_solid(a.solid, nx, ny, nz, i - 1, i, j - 1, j, k, k)) vz = Real(0);
            }
            if (i < nx && in_y) a.neu[0][own_h[0]] = vx;
            if (in_x && j < ny) a.neu[1][own_h[1]] = vy;
            if (in_x && in_y && zin) a.neu[2][own_h[2]] = vz;
        }
        hx_below = hxn;
        hy_below = hyn;
        {
            const unsigned t = cw.t;
            yee_walk_next(cw, T, nz);
            if (cw.t != t) {
                YeeCopy co = yee_copy_at<Real>(a, cw, hq, hr, hc);
#pragma unroll
                for (int q = 0; q < 6; ++q) own_h[q] = co.own[q];
            } else {
#pragma unroll
                for (int q = 0; q < 6; ++q) own_h[q] += a.pstride[q];
            }
        }
        slot = slot + 1 == S ? 0 : slot + 1;
    }
    cp_async_wait<0>();
    if (finish_blocks<4>(acc, a.partials, a.nblocks, &st->counter) && linear_tid() == 0) {
        const double v = a.volume;
        const double electric = 0.5 * acc[0] * v;   // cavity.rs:846
        const double paired = 0.5 * v * acc[1];     // cavity.rs:885-904
        st->invariant = electric + paired;
        st->has_invariant = 1;
        st->dissipated += fmax(acc[2], 0.0);
        st->work_booked = st->work;
        st->work += acc[3];
        double total = 0.0, scale = 0.0;
        ledger_add(total, scale, st->invariant);
        ledger_add(total, scale, st->dissipated);
        if (a.src_i >= 0) ledger_add(total, scale, -st->work_booked);
        st->part[0] = st->invariant;
        st->part[1] = st->dissipated;
        st->part[2] = -st->work_booked;
        audit_and_commit(st, total, scale);
    }
}

// Magnetic and open walls (cavity.rs:1074-1236), applied to the new E after a step, one wall at a
// time in the reference's order, so edges shared by two walls end as they do there. Any layout:
// component q's edge (i, j, k) is at i + rx[q]·(j + ry[q]·k).
template <typename Real>
struct YeeWallArgs {
    Real* e[3];         // the new ex, ey, ez
    const Real* pe[3];  // the previous step's E after its walls (Mur's history)
    int nx, ny, nz;
    unsigned rx[3], ry[3];
    int wall;           // 0..5: XLow, XHigh, YLow, YHigh, ZLow, ZHigh
    int kind;           // 1 mirror (magnetic), 2 Mur (open), 3 zero (open, no history yet)
    Real k;             // Mur's coefficient (cΔt − Δ)/(cΔt + Δ)
};

// cavity.rs:304-331 `enforce_solid` as a pass of its own: the twelve edges of every solid cell to
// zero. Run after the walls when a cavity has both obstacles and magnetic or open walls, since the
// reference applies its walls (and takes Mur's history) before it zeroes the obstacles' edges
// (cavity.rs:1497-1499); the step kernels then leave those edges to this pass. Neighbouring solid
// cells share edges and write the same zero.
template <typename Real>
static __global__ void yee_enforce_solid(YeeWallArgs<Real> a, const uint8_t* __restrict__ solid) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t cells = (size_t)nx * ny * nz;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
        if (!solid[c]) continue;
        const size_t i = c % (size_t)nx, r = c / (size_t)nx;
        const size_t j = r % (size_t)ny, k = r / (size_t)ny;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const size_t u = q & 1, v = q >> 1;
            a.e[0][i + a.rx[0] * ((j + u) + a.ry[0] * (k + v))] = Real(0);
            a.e[1][(i + u) + a.rx[1] * (j + a.ry[1] * (k + v))] = Real(0);
            a.e[2][(i + u) + a.rx[2] * ((j + v) + a.ry[2] * k)] = Real(0);
        }
    }
}

template <typename Real>
static __global__ void yee_walls(YeeWallArgs<Real> a) {
    const int nx = a.nx, ny = a.ny, nz = a.nz, w = a.wall;
    // the wall's two tangential components (cavity.rs:1096-1157): x walls ey, ez; y walls ex, ez;
    // z walls ex, ey; each over (u, v) = its two in-plane lattice coordinates
    const int q0 = w < 2 ? 1 : 0, q1 = w < 4 ? 2 : 1;
    int n0u, n0v, n1u, n1v;  // extents of (u, v) for each component
    if (w < 2) { n0u = ny; n0v = nz + 1; n1u = ny + 1; n1v = nz; }
    else if (w < 4) { n0u = nx; n0v = nz + 1; n1u = nx + 1; n1v = nz; }
    else { n0u = nx; n0v = ny + 1; n1u = nx + 1; n1v = ny; }
    const int edge = (w & 1) ? (w < 2 ? nx : w < 4 ? ny : nz) : 0;
    const int inner = (w & 1) ? edge - 1 : 1;
    const size_t c0 = (size_t)n0u * n0v, total = c0 + (size_t)n1u * n1v;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const bool first = t < c0;
        const int q = first ? q0 : q1;
        const size_t r = first ? t : t - c0;
        const int nu = first ? n0u : n1u;
        const int u = (int)(r % (size_t)nu), v = (int)(r / (size_t)nu);
        int ia, ja, ka, ib, jb, kb;
        if (w < 2) { ia = edge; ib = inner; ja = jb = u; ka = kb = v; }
        else if (w < 4) { ja = edge; jb = inner; ia = ib = u; ka = kb = v; }
        else { ka = edge; kb = inner; ia = ib = u; ja = jb = v; }
        const size_t ai = (size_t)ia + (size_t)a.rx[q] * ((size_t)ja + (size_t)a.ry[q] * ka);
        const size_t bi = (size_t)ib + (size_t)a.rx[q] * ((size_t)jb + (size_t)a.ry[q] * kb);
        Real* e = a.e[q];
        if (a.kind == 1) e[ai] = e[bi];                                        // cavity.rs:1170-1236
        else if (a.kind == 2) e[ai] = a.pe[q][bi] + a.k * (e[bi] - a.pe[q][ai]);  // cavity.rs:1096-1157
        else e[ai] = Real(0);                                                  // cavity.rs:1087-1089
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
