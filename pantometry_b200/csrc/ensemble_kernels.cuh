// Batched Solid3D stepping: many independent uneven blocks advanced by one persistent kernel per
// step that walks a list of bricks (the GPU form of `Ensemble::run` over `Solid3D` samples,
// crates/pantometry-core/src/ensemble.rs:102-140, with each sample's own `Solid3D::step`,
// crates/pantometry-thermal/src/solid.rs:1717-1901).
//
// Layout. The blocks' cells are concatenated in block order, each block in the reference's
// index order i + pitch·(j + ny·k) (pitch = nx rounded up to 2 for f64 and to 4 for f32, the
// padding columns zero, so that every pair or quad of a row starts on 16 bytes and TMA can tile
// each f32 block). A brick is a bx × by × zc box of one block (bx·by = 256
// threads, each marching one column of zc planes); the brick list holds every brick of every
// block, block by block, and a persistent grid of thread blocks takes bricks blockIdx.x,
// blockIdx.x + gridDim.x, ... in that fixed order. Brick shapes are chosen at run time (the
// autotuner times each candidate on the real state).
//
// Per-cell arithmetic. The f64 form is heat_plain_step's uniform path (the reference's operand
// order, compiled with --fmad=false: bit-exact with `Solid3D::step` for each block on its own).
// The f32 form is heat_f32_step's (deviations T − T0, temperature-independent films).
//
// Ledgers. Every brick leaves one FP64 partial per quantity (fixed thread order, fixed tree).
// The last brick of a block to finish — found with the block's own atomic ticket — sums that
// block's partials in fixed order and runs the block's ledger and audit. The sums therefore do
// not depend on which thread block ran which brick, only on the brick shape.
#pragma once

#include "heat_kernels.cuh"

namespace pm {

// One block of the ensemble, as the kernel reads it.
struct EnsGrid {
    int nx, ny, nz;
    unsigned nbricks;
    unsigned long long offset;  // first cell in the concatenated field
    int pitch;                  // elements per row: nx rounded up to 2 (f64) or 4 (f32)
    int pad0;
    unsigned first_brick;
    int exposed;                // film faces (bit f: XMin, XMax, YMin, YMax, ZMin, ZMax)
    // plain f64 coefficients (`resolve` of a one-material block, solid.rs:588-784)
    double kface, mobility, capacity, k_cell, eps_cell;
    double dts, dx, reference;
    double share[6], ambient[6], convection[6];
    // f32 coefficients
    float a;      // dt · mobility · k_face
    float b[6];   // dt · mobility · g_f / dx per film face
    float off[6]; // T0 − ambient per film face
    float pad;
    // h = +inf: per face the film's series with the half cell, the same for every cell of the face
    // (bare / gap is +inf for every finite nonzero gap; see film_flux)
    double g_inf[6];
};

struct EnsBrick {
    unsigned grid;
    unsigned short x0, y0, z0, z1;
    unsigned pad;
};

template <typename Real>
struct EnsArgs {
    const Real* __restrict__ old;
    Real* __restrict__ nu;
    const EnsGrid* __restrict__ grids;
    const EnsBrick* __restrict__ bricks;
    unsigned nbricks;
    unsigned ngrids;
    int bxs;             // log2 of the threads along the brick's x extent (2 to 6)
    int wide;            // each thread takes adjacent cells of its row: four (f32) or two (f64)
    DevState* states;    // one per block: its books, ledger and audit
    double* partials;    // two per brick
};

// `film_flux` (solid.rs:1192-1219) of a block's cell, read off the old state.
__device__ __forceinline__ double ens_film_flux(const EnsGrid& g, int i, int j, int k, double here) {
    double out = 0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (!((g.exposed >> f) & 1)) continue;
        if (!face_holds(f, i, j, k, g.nx, g.ny, g.nz)) continue;
        const double share = g.share[f];
        const double ambient = g.ambient[f];
        const double gap = here - ambient;
        if (gap == 0.0) continue;
        double cond;
        if (isinf(g.convection[f]) && g.convection[f] > 0.0) {
            cond = g.g_inf[f];
        } else {
            // crates/pantometry-thermal/src/lib.rs:104-110 `Environment::loss_from`, area = share
            const double convective = g.convection[f] * share * (here - ambient);
            const double radiative = g.eps_cell * kStefanBoltzmann * share * (powi4(here) - powi4(ambient));
            const double bare = convective + radiative;
            cond = series_with_half_cell(bare / gap, g.k_cell, share, g.dx);
        }
        out += cond * gap / g.dx;
    }
    return out;
}

// One step of every live block (MEASURE = false), or the opening ledger of the present state
// (MEASURE = true: nothing is written, stored heat is summed and committed without an audit).
template <typename Real, bool MEASURE>
__device__ __forceinline__ void ens_brick(const EnsArgs<Real>& a, const EnsGrid& g, const EnsBrick& br,
                                          double (&acc)[2]) {
    const int tid = threadIdx.x;
    const int bx = 1 << a.bxs;
    const int i = br.x0 + (tid & (bx - 1));
    const int j = br.y0 + (tid >> a.bxs);
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny) return;
    const int pitch = g.pitch;
    const size_t plane = (size_t)pitch * ny;
    const Real* __restrict__ told = a.old + g.offset;
    Real* __restrict__ tnew = a.nu + g.offset;
    const int k0 = br.z0, k1 = br.z1;
    size_t c = (size_t)i + (size_t)pitch * ((size_t)j + (size_t)ny * k0);
    if (MEASURE) {
        for (int k = k0; k < k1; ++k, c += plane) {
            if constexpr (sizeof(Real) == 8) acc[0] += g.capacity * ((double)told[c] - g.reference);  // solid.rs:1583-1590
            else acc[0] += (double)told[c];
        }
        return;
    }
    if constexpr (sizeof(Real) == 8) {
        // heat_plain_step, uniform block: the reference's order of the six face terms
        double below = k0 > 0 ? told[c - plane] : 0.0;
        double here = told[c];
        const double kf = g.kface;
        for (int k = k0; k < k1; ++k, c += plane) {
            const double above = k + 1 < nz ? told[c + plane] : 0.0;
            const double t0 = here;
            double flux = 0.0;
            if (i > 0) flux += kf * (told[c - 1] - t0);
            if (i + 1 < nx) flux += kf * (told[c + 1] - t0);
            if (j > 0) flux += kf * (told[c - pitch] - t0);
            if (j + 1 < ny) flux += kf * (told[c + pitch] - t0);
            if (k > 0) flux += kf * (below - t0);
            if (k + 1 < nz) flux += kf * (above - t0);
            const double shed = g.exposed ? ens_film_flux(g, i, j, k, t0) : 0.0;
            const double nt = t0 + g.dts * g.mobility * (flux - shed);  // add_kelvin (solid.rs:1620-1635)
            tnew[c] = nt;
            acc[0] += g.capacity * (nt - g.reference);
            if (shed != 0.0) acc[1] += g.dts * g.mobility * shed * g.capacity;  // solid.rs:1821-1823
            below = here;
            here = above;
        }
    } else {
        // heat_f32_step on deviations
        float below = k0 > 0 ? __ldg(told + c - plane) : 0.0f;
        float here = __ldg(told + c);
        const bool xl = i > 0, xh = i + 1 < nx, yl = j > 0, yh = j + 1 < ny;
        const bool edge_xy = !(xl && xh && yl && yh);
        const float ga = g.a;
        double col_shed = 0.0;
        for (int k = k0; k < k1; ++k, c += plane) {
            const float above = (k + 1 < nz) ? __ldg(told + c + plane) : 0.0f;
            float s = 0.0f;
            if (xl) s += __ldg(told + c - 1) - here;
            if (xh) s += __ldg(told + c + 1) - here;
            if (yl) s += __ldg(told + c - pitch) - here;
            if (yh) s += __ldg(told + c + pitch) - here;
            if (k > 0) s += below - here;
            if (k + 1 < nz) s += above - here;
            float shed = 0.0f;
            if (g.exposed && (edge_xy || k == 0 || k + 1 == nz)) {
                if (((g.exposed >> 0) & 1) && !xl) shed += g.b[0] * (here + g.off[0]);
                if (((g.exposed >> 1) & 1) && !xh) shed += g.b[1] * (here + g.off[1]);
                if (((g.exposed >> 2) & 1) && !yl) shed += g.b[2] * (here + g.off[2]);
                if (((g.exposed >> 3) & 1) && !yh) shed += g.b[3] * (here + g.off[3]);
                if (((g.exposed >> 4) & 1) && k == 0) shed += g.b[4] * (here + g.off[4]);
                if (((g.exposed >> 5) & 1) && k + 1 == nz) shed += g.b[5] * (here + g.off[5]);
                col_shed += (double)shed;
            }
            const float nd = here + (ga * s - shed);
            tnew[c] = nd;
            acc[0] += (double)nd;
            below = here;
            here = above;
        }
        acc[1] += col_shed;
    }
}

// Four adjacent cells of a row per thread (the f32 quad shapes): heat_f32_quad_step's arithmetic
// on a brick of one block, which is ens_brick's f32 arithmetic cell for cell (the same order and
// roundings), so the fields agree with every other brick shape bit for bit. Rows are padded to a
// multiple of 4 cells, so every quad starts on 16 bytes; cells of a quad past the block's last
// column (the padding) are neither used as neighbours nor written nor summed.
template <bool MEASURE>
__device__ __forceinline__ void ens_brick_quad(const EnsArgs<float>& a, const EnsGrid& g, const EnsBrick& br,
                                               double (&acc)[2]) {
    const int tid = threadIdx.x;
    const int i = br.x0 + 4 * (tid & ((1 << a.bxs) - 1));
    const int j = br.y0 + (tid >> a.bxs);
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny) return;
    const int pitch = g.pitch;
    const size_t plane = (size_t)pitch * ny;
    const int k0 = br.z0, k1 = br.z1;
    const size_t c = g.offset + (size_t)i + (size_t)pitch * ((size_t)j + (size_t)ny * k0);
    const float* p = a.old + c;
    float* o = a.nu + c;
    const int valid = min(4, nx - i);  // cells of the quad inside the block
    if (MEASURE) {
        for (int k = k0; k < k1; ++k, p += plane) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(p));
            acc[0] += (double)v.x;
            if (valid > 1) acc[0] += (double)v.y;
            if (valid > 2) acc[0] += (double)v.z;
            if (valid > 3) acc[0] += (double)v.w;
        }
        return;
    }
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const bool xl = i > 0, xh = i + 4 < nx, yl = j > 0, yh = j + 1 < ny;
    const float ga = g.a;
    float4 below = k0 > 0 ? __ldg(reinterpret_cast<const float4*>(p - plane)) : zero;
    float4 here = __ldg(reinterpret_cast<const float4*>(p));
    double col_shed = 0.0;
    for (int k = k0; k < k1; ++k, p += plane, o += plane) {
        const bool zl = k > 0, zh = k + 1 < nz;
        const float4 above = zh ? __ldg(reinterpret_cast<const float4*>(p + plane)) : zero;
        const float4 ym = yl ? __ldg(reinterpret_cast<const float4*>(p - pitch)) : zero;
        const float4 yp = yh ? __ldg(reinterpret_cast<const float4*>(p + pitch)) : zero;
        const float xm = xl ? __ldg(p - 1) : 0.0f, xp = xh ? __ldg(p + 4) : 0.0f;
        const float hv[4] = {here.x, here.y, here.z, here.w}, bv[4] = {below.x, below.y, below.z, below.w};
        const float av[4] = {above.x, above.y, above.z, above.w};
        const float mv[4] = {ym.x, ym.y, ym.z, ym.w}, pv[4] = {yp.x, yp.y, yp.z, yp.w};
        float nd[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float h = hv[e];
            const bool l = e > 0 || xl, r = e < 3 ? i + e + 1 < nx : xh;  // x neighbours in the block
            float sum = 0.0f;
            if (l) sum += (e == 0 ? xm : hv[e - 1]) - h;
            if (r) sum += (e == 3 ? xp : hv[e + 1]) - h;
            if (yl) sum += mv[e] - h;
            if (yh) sum += pv[e] - h;
            if (zl) sum += bv[e] - h;
            if (zh) sum += av[e] - h;
            float shed = 0.0f;
            if (g.exposed && (!(l && r && yl && yh) || !zl || !zh)) {
                if (((g.exposed >> 0) & 1) && !l) shed = __fmaf_rn(g.b[0], h + g.off[0], shed);
                if (((g.exposed >> 1) & 1) && !r) shed = __fmaf_rn(g.b[1], h + g.off[1], shed);
                if (((g.exposed >> 2) & 1) && !yl) shed = __fmaf_rn(g.b[2], h + g.off[2], shed);
                if (((g.exposed >> 3) & 1) && !yh) shed = __fmaf_rn(g.b[3], h + g.off[3], shed);
                if (((g.exposed >> 4) & 1) && !zl) shed = __fmaf_rn(g.b[4], h + g.off[4], shed);
                if (((g.exposed >> 5) & 1) && !zh) shed = __fmaf_rn(g.b[5], h + g.off[5], shed);
                if (e < valid) col_shed += (double)shed;
            }
            nd[e] = __fadd_rn(h, __fmaf_rn(ga, sum, -shed));
            if (e < valid) acc[0] += (double)nd[e];
        }
        if (valid == 4) {
            *reinterpret_cast<float4*>(o) = make_float4(nd[0], nd[1], nd[2], nd[3]);
        } else {
            for (int e = 0; e < valid; ++e) o[e] = nd[e];
        }
        below = here;
        here = above;
    }
    acc[1] += col_shed;
}

// Two adjacent cells of a row per thread (the f64 pair shapes): ens_brick's f64 arithmetic for each
// cell, expression for expression (the reference's operand order, compiled without contraction),
// with 16-byte loads of the pair, the plane above and the rows either side and one 16-byte store,
// so the fields agree with the one-cell shapes, and with the reference, bit for bit. Rows are
// padded to an even length; a pair's second cell past the block's last column (the padding) is
// neither used as a neighbour nor written nor summed.
template <bool MEASURE>
__device__ __forceinline__ void ens_brick_pair(const EnsArgs<double>& a, const EnsGrid& g, const EnsBrick& br,
                                               double (&acc)[2]) {
    const int tid = threadIdx.x;
    const int i = br.x0 + 2 * (tid & ((1 << a.bxs) - 1));
    const int j = br.y0 + (tid >> a.bxs);
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny) return;
    const int pitch = g.pitch;
    const size_t plane = (size_t)pitch * ny;
    const int k0 = br.z0, k1 = br.z1;
    const double* p = a.old + g.offset + ((size_t)i + (size_t)pitch * ((size_t)j + (size_t)ny * k0));
    double* o = a.nu + (p - a.old);
    const bool two = i + 1 < nx;  // the pair's second cell is in the block
    if (MEASURE) {
        for (int k = k0; k < k1; ++k, p += plane) {
            const double2 v = *reinterpret_cast<const double2*>(p);
            acc[0] += g.capacity * (v.x - g.reference);  // solid.rs:1583-1590
            if (two) acc[0] += g.capacity * (v.y - g.reference);
        }
        return;
    }
    const double2 zero = make_double2(0.0, 0.0);
    const double kf = g.kface;
    const bool xl = i > 0, xh = i + 2 < nx, yl = j > 0, yh = j + 1 < ny;
    double2 below = k0 > 0 ? *reinterpret_cast<const double2*>(p - plane) : zero;
    double2 here = *reinterpret_cast<const double2*>(p);
    for (int k = k0; k < k1; ++k, p += plane, o += plane) {
        const double2 above = k + 1 < nz ? *reinterpret_cast<const double2*>(p + plane) : zero;
        const double2 ym = yl ? *reinterpret_cast<const double2*>(p - pitch) : zero;
        const double2 yp = yh ? *reinterpret_cast<const double2*>(p + pitch) : zero;
        const double xm = xl ? p[-1] : 0.0, xp = xh ? p[2] : 0.0;
        const double hv[2] = {here.x, here.y}, bv[2] = {below.x, below.y}, av[2] = {above.x, above.y};
        const double mv[2] = {ym.x, ym.y}, pv[2] = {yp.x, yp.y};
        double nt[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const double t0 = hv[e];
            double flux = 0.0;  // heat_plain_step's uniform path: the reference's order of the six face terms
            if (e > 0 || xl) flux += kf * ((e == 0 ? xm : hv[0]) - t0);
            if (e == 0 ? two : xh) flux += kf * ((e == 1 ? xp : hv[1]) - t0);
            if (yl) flux += kf * (mv[e] - t0);
            if (yh) flux += kf * (pv[e] - t0);
            if (k > 0) flux += kf * (bv[e] - t0);
            if (k + 1 < nz) flux += kf * (av[e] - t0);
            const double shed = g.exposed ? ens_film_flux(g, i + e, j, k, t0) : 0.0;
            nt[e] = t0 + g.dts * g.mobility * (flux - shed);  // add_kelvin (solid.rs:1620-1635)
            if (e == 0 || two) {
                acc[0] += g.capacity * (nt[e] - g.reference);
                if (shed != 0.0) acc[1] += g.dts * g.mobility * shed * g.capacity;  // solid.rs:1821-1823
            }
        }
        if (two) *reinterpret_cast<double2*>(o) = make_double2(nt[0], nt[1]);
        else o[0] = nt[0];
        below = here;
        here = above;
    }
}

// A block whose audit failed keeps its state: its bricks copy old to new, so the ping-pong
// parity stays the same for every block of the ensemble.
template <typename Real, bool WIDE>
__device__ __forceinline__ void ens_hold(const EnsArgs<Real>& a, const EnsGrid& g, const EnsBrick& br) {
    constexpr int kWidth = WIDE ? (sizeof(Real) == 8 ? 2 : 4) : 1;
    const int tid = threadIdx.x;
    const int i = br.x0 + kWidth * (tid & ((1 << a.bxs) - 1));
    const int j = br.y0 + (tid >> a.bxs);
    if (i >= g.nx || j >= g.ny) return;
    const int cells = min(kWidth, g.nx - i);
    const size_t plane = (size_t)g.pitch * g.ny;
    size_t c = g.offset + (size_t)i + (size_t)g.pitch * ((size_t)j + (size_t)g.ny * br.z0);
    for (int k = br.z0; k < br.z1; ++k, c += plane)
        for (int e = 0; e < cells; ++e) a.nu[c + e] = a.old[c + e];
}

// WIDE: four cells of a row per thread (f32) or two (f64, held to PM_ENS_PAIR_MIN_BLOCKS blocks per
// SM: occupancy sets the speed of the f64 wide forms, as for heat_plain_pair_step).
#ifndef PM_ENS_PAIR_MIN_BLOCKS
#define PM_ENS_PAIR_MIN_BLOCKS 4
#endif
template <typename Real, bool MEASURE, bool WIDE = false>
static __global__ void __launch_bounds__(256, (WIDE && sizeof(Real) == 8) ? PM_ENS_PAIR_MIN_BLOCKS : 1)
    ens_step(EnsArgs<Real> a) {
    __shared__ double red[32 * 2];
    __shared__ int last;
    const int tid = threadIdx.x;
    for (unsigned b = blockIdx.x; b < a.nbricks; b += gridDim.x) {
        const EnsBrick br = a.bricks[b];
        const EnsGrid& g = a.grids[br.grid];
        DevState* st = a.states + br.grid;
        if (!MEASURE && st->violated) {  // block-uniform: every thread reads the same word
            ens_hold<Real, WIDE>(a, g, br);
            continue;
        }
        double acc[2] = {0.0, 0.0};
        if constexpr (WIDE && sizeof(Real) == 4) ens_brick_quad<MEASURE>(a, g, br, acc);
        else if constexpr (WIDE) ens_brick_pair<MEASURE>(a, g, br, acc);
        else ens_brick<Real, MEASURE>(a, g, br, acc);
        block_sum<2>(acc, red);
        if (tid == 0) {
            a.partials[2 * (size_t)b] = acc[0];
            a.partials[2 * (size_t)b + 1] = acc[1];
            __threadfence();
            const unsigned ticket = atomicAdd(&st->counter, 1u);
            last = ticket == g.nbricks - 1 ? 1 : 0;
        }
        __syncthreads();
        if (!last) continue;
        // The block's last brick: its partials in fixed order, then the ledger and the audit.
        __threadfence();
        double v[2] = {0.0, 0.0};
        for (unsigned q = tid; q < g.nbricks; q += blockDim.x) {
            v[0] += __ldcg(&a.partials[2 * (size_t)(g.first_brick + q)]);
            v[1] += __ldcg(&a.partials[2 * (size_t)(g.first_brick + q) + 1]);
        }
        block_sum<2>(v, red);
        if (tid == 0) {
            st->counter = 0u;
            const double stored = sizeof(Real) == 8 ? v[0] : g.capacity * v[0];
            if (!MEASURE) st->lost += sizeof(Real) == 8 ? v[1] : g.capacity * v[1];
            double total = 0.0, scale = 0.0;
            ledger_add(total, scale, stored);
            ledger_add(total, scale, st->lost);
            ledger_add(total, scale, -st->supplied);
            st->part[0] = stored;
            st->part[1] = st->lost;
            st->part[2] = -st->supplied;
            if (MEASURE) {
                st->total = total;
                st->scale = scale;
                st->prev_total = total;
                st->prev_scale = scale;
            } else {
                audit_and_commit(st, total, scale);
            }
        }
    }
}

// One f64 block between the caller's dense layout (x fastest, rows of nx) and the device's rows
// of `pitch` (to_dev = 1; the padding zeroed by the caller), and back.
static __global__ void ens_relayout64(const double* __restrict__ dense, double* __restrict__ padded,
                                      double* __restrict__ out, int nx, int ny, int nz, int pitch, int to_dev) {
    const size_t n = (size_t)nx * ny * nz;
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
        const size_t i = r % (size_t)nx, rest = r / (size_t)nx;
        const size_t q = i + (size_t)pitch * rest;  // rest = j + ny·k
        if (to_dev) padded[q] = dense[r];
        else out[r] = padded[q];
    }
}

}  // namespace pm
