// Solid3D stepping kernels (crates/pantometry-thermal/src/solid.rs:1717-1901).
//
// heat_plain_step — IEEE f64, the reference's operand order, compiled with --fmad=false so no
//   multiply-add is contracted: bit-exact with `Solid3D::step` cell by cell. One thread per
//   cell, reading the old field and writing the new one (the reference's `old = cells.clone()`
//   becomes a ping-pong pair). Films (`losing_from`) are evaluated in the same update, from the
//   old state, exactly as `film_flux` does. Fused: this step's stored heat and shed heat, summed
//   in FP64 by the fixed-order tree, then the ledger and the audit in the last block.
//
// heat_f32_step — the chosen form. The field is stored as the deviation T − T0 in f32, which
//   keeps the subtraction `T_nb − T` on numbers of order the deviation rather than of 300 K
//   (the reference's own finding, runtime/gpu/src/lib.rs:37-51). Films with a temperature-
//   independent conductance. A uniform block folds dt·mobility·k into one coefficient; a filled
//   block (FILLED) reads its per-face conductivities in f32, each cell's dt·mobility (formed once
//   per step size) and each boundary cell's film conductance, with `Solid3D::step`'s arithmetic
//   in f32. Stored heat, shed heat and the ledger stay FP64 (per-cell capacities in f64).
#pragma once

#include "common.cuh"

namespace pm {

constexpr double kStefanBoltzmann = 5.670374419e-8;  // pantometry-units/src/lib.rs:899

// Rust `powi` with a constant exponent: binary-decomposition multiplies.
__device__ __forceinline__ double powi4(double x) {
    double s = x * x;
    return s * s;
}
__device__ __forceinline__ double powi3(double x) { return x * (x * x); }

// solid.rs:110-122
__device__ __forceinline__ double series_with_half_cell(double film, double conductivity, double area,
                                                        double dx) {
    if (film <= 0.0) return 0.0;
    double half = 2.0 * conductivity * area / dx;
    if (!isfinite(half)) return film;
    if (half <= 0.0) return 0.0;
    return 1.0 / (1.0 / film + 1.0 / half);
}

__device__ __forceinline__ bool face_holds(int f, int i, int j, int k, int nx, int ny, int nz) {
    switch (f) {
        case 0: return i == 0;
        case 1: return i + 1 == nx;
        case 2: return j == 0;
        case 3: return j + 1 == ny;
        case 4: return k == 0;
        default: return k + 1 == nz;
    }
}

struct HeatFilms {
    int exposed;  // bit f set: face f (XMin, XMax, YMin, YMax, ZMin, ZMax) loses heat
    double ambient[6];
    double convection[6];
    double share[6];  // area / cells_on(face), computed on the host as the reference does
    // Faces with h = +inf on a block of one material: bit f set, and g_inf[f] the film's series
    // with the half cell there, which is the same for every cell of the face (see film_flux).
    int dirichlet;
    double g_inf[6];
};

// One cell's side of a radiative gap: a pair of solid cells facing each other along a grid line
// across a run of void (solid.rs:786-838), in the order the pairs were found, which is the order
// the step applies them (solid.rs:1866-1878).
struct HeatGapEntry {
    long long partner;   // the cell across the void
    double coefficient;  // σA/(1/ε₁ + 1/ε₂ − 1)
    int lower;           // 1: this cell is the pair's first cell, the one the exchange is taken from
    int last;            // 1: the cell's last entry
};

struct HeatPlainArgs {
    const double* __restrict__ told;
    double* __restrict__ tnew;
    // General (filled) blocks: per-face conductivities and per-cell coefficients, as
    // `resolve` builds them (solid.rs:588-784). Null in uniform mode.
    const double* __restrict__ kx;
    const double* __restrict__ ky;
    const double* __restrict__ kz;
    const double* __restrict__ mob;
    const double* __restrict__ cap;
    const uint32_t* __restrict__ which;  // per-cell material, for the film (general mode)
    const double* __restrict__ mat_k;    // per-material conductivity (+inf: `thermal: None`)
    const double* __restrict__ mat_eps;  // per-material emissivity
    // Heat that has a place (null where nothing generates): watts per cell, zero on void
    // (solid.rs:1045-1085); the gaps (null without any): per cell the first of its entries or −1
    const double* __restrict__ src;
    const int* __restrict__ gap_of;
    const HeatGapEntry* __restrict__ gaps;
    // Uniform blocks: the single values every interior face and cell holds.
    double kface, mobility, capacity, k_cell, eps_cell;
    int uniform;
    int nx, ny, nz;
    double dts, dx, reference;
    HeatFilms films;
    int pairs;  // uniform blocks with rows of an even number of cells: heat_plain_pair_step
    int quads;  // rows of a multiple of 4 cells, four a thread: heat_plain_quad_step (pairs is 0)
    // Radiating films (some exposed cell with emissivity > 0) or radiative gaps: the step limit
    // depends on the state, so each step checks dt against the rate its own state gives
    // (solid.rs:1718-1738) and gathers the rate of the state it leaves. static_rate: `worst_rate`
    // of `resolve`.
    int radiating;
    double static_rate;
    Tiles tiles;
    DevState* st;
    double* partials;
    unsigned nblocks;  // the launch's grid: min(tiles, resident blocks)
};

// solid.rs:1192-1219 `film_flux`, read off the old state.
__device__ __forceinline__ double film_flux(const HeatPlainArgs& a, int i, int j, int k, size_t c,
                                            double here) {
    double emissivity, conductivity;
    if (a.uniform) {
        emissivity = a.eps_cell;
        conductivity = a.k_cell;
    } else {
        uint32_t m = a.which[c];
        emissivity = a.mat_eps[m];
        conductivity = a.mat_k[m];
    }
    double out = 0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (!((a.films.exposed >> f) & 1)) continue;
        if (!face_holds(f, i, j, k, a.nx, a.ny, a.nz)) continue;
        double share = a.films.share[f];
        double ambient = a.films.ambient[f];
        double gap = here - ambient;
        if (gap == 0.0) continue;
        double g;
        if ((a.films.dirichlet >> f) & 1) {
            // h = +inf: the convective term is ±inf with the gap's sign and the radiative one finite,
            // so bare / gap is +inf for every finite nonzero gap, and series_with_half_cell(+inf, k,
            // share, dx) is the face's constant, formed once on the host by the same expression
            g = a.films.g_inf[f];
        } else {
            // crates/pantometry-thermal/src/lib.rs:104-110 `Environment::loss_from`, area = share
            double convective = a.films.convection[f] * share * (here - ambient);
            double radiative = emissivity * kStefanBoltzmann * share * (powi4(here) - powi4(ambient));
            double bare = convective + radiative;
            g = series_with_half_cell(bare / gap, conductivity, share, a.dx);
        }
        out += g * gap / a.dx;
    }
    return out;
}

// solid.rs:1269-1288 `loss_conductance_at`: the films' tangent conductance at temperature `at`,
// h + 4εσ·max(T, T∞)³ per exposed face with the half cell in series, summed from −0.0 as Rust's
// `Sum for f64` does.
__device__ __forceinline__ double loss_conductance(const HeatPlainArgs& a, int i, int j, int k, size_t c, double at) {
    double emissivity, conductivity;
    if (a.uniform) {
        emissivity = a.eps_cell;
        conductivity = a.k_cell;
    } else {
        uint32_t m = a.which[c];
        emissivity = a.mat_eps[m];
        conductivity = a.mat_k[m];
    }
    double total = -0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (!((a.films.exposed >> f) & 1)) continue;
        if (!face_holds(f, i, j, k, a.nx, a.ny, a.nz)) continue;
        const double share = a.films.share[f];
        const double hot = fmax(at, a.films.ambient[f]);
        const double h = a.films.convection[f] + 4.0 * emissivity * kStefanBoltzmann * powi3(hot);
        total += series_with_half_cell(h * share, conductivity, share, a.dx);
    }
    return total;
}

// One boundary cell's term of `worst_rate_now` (solid.rs:1172-1183) at its new temperature, or
// −1 where it has no film: mobility·(face_sum + loss/dx), face_sum summed as `resolve` sums it
// (solid.rs:757-762).
__device__ __forceinline__ double heat_cell_rate(const HeatPlainArgs& a, int i, int j, int k, size_t c, double t) {
    const double loss = loss_conductance(a, i, j, k, c, t);
    if (loss == 0.0) return -1.0;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    double face_sum, mob;
    if (a.uniform) {
        const double kf = a.kface;
        face_sum = ((((((i > 0 && i < nx) ? kf : 0.0) + ((i + 1 < nx) ? kf : 0.0)) + ((j > 0 && j < ny) ? kf : 0.0)) +
                     ((j + 1 < ny) ? kf : 0.0)) + ((k > 0 && k < nz) ? kf : 0.0)) + ((k + 1 < nz) ? kf : 0.0);
        mob = a.mobility;
    } else {
        const size_t plane = (size_t)nx * ny;
        const size_t xr = (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k);
        const size_t yr = (size_t)nx * ((size_t)j + (size_t)(ny + 1) * k);
        face_sum = ((((a.kx[i + xr] + a.kx[i + 1 + xr]) + a.ky[i + yr]) + a.ky[i + nx + yr]) + a.kz[c]) + a.kz[c + plane];
        mob = a.mob[c];
    }
    return mob * (face_sum + loss / a.dx);
}

// The refusal a radiating block's step makes before anything moves (solid.rs:1718-1738), against
// the rate of the state the step starts from. Every block reads the same rate and takes the same
// decision; block 0 records it.
__device__ __forceinline__ bool heat_refused(const HeatPlainArgs& a) {
    if (!a.radiating) return false;
    DevState* st = a.st;
    const double ratio = a.dts * st->rate_now;
    if (!(ratio > 1.0 + 6e-12)) return false;
    if (blockIdx.x == 0 && linear_tid() == 0) {
        constexpr double fourier = 1.0 / 6.0;  // solid.rs:84
        st->violated = kRefused;
        st->violation_step = st->steps + 1;
        st->v_before = fourier;
        st->v_after = ratio * fourier;
        st->v_scale = fourier;
        st->v_tol = 1e-12;
    }
    return true;
}

// The block's largest boundary-cell rate into the launch's max, before the block's ticket: a
// warp tree, then the warps' values, then one integer atomicMax on the bits (every candidate is
// a non-negative double or −1, which is left out).
__device__ __forceinline__ void heat_rate_publish(const HeatPlainArgs& a, double r) {
    __shared__ double wmax[32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, off));
    const int tid = linear_tid(), lane = tid & 31, warp = tid >> 5;
    const int nwarps = (blockDim.x * blockDim.y * blockDim.z) >> 5;
    if (lane == 0) wmax[warp] = r;
    __syncthreads();
    if (tid == 0) {
        double m = -1.0;
        for (int w = 0; w < nwarps; ++w) m = fmax(m, wmax[w]);
        if (m >= 0.0) atomicMax(&a.st->rate_bits, (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
}

// A gap cell's exchanges after the sweep and the source (solid.rs:1866-1878): each pair's watts
// read off the old state, the cell's share added in the pairs' order. Where the limit follows the
// state, the pairs' terms of `worst_rate_now` (solid.rs:1159-1171) at the cell's new temperature:
// each side offers 4σA·T³/(...)/C of both cells at its own T, and since every operation there is
// monotone in T the larger side's offers are the reference's value at the hotter of the two.
__device__ __forceinline__ double heat_gap_cell(const HeatPlainArgs& a, int g, double here, double capc, double nt,
                                                double& rate) {
    for (int e = g;; ++e) {
        const HeatGapEntry x = a.gaps[e];
        const double other = a.told[x.partner];
        const double ta = x.lower ? here : other, tb = x.lower ? other : here;
        const double watts = x.coefficient * (powi4(ta) - powi4(tb));
        if (watts != 0.0) {
            const double joules = watts * a.dts;
            nt += x.lower ? -joules / capc : joules / capc;
        }
        if (x.last) break;
    }
    if (a.radiating) {
        for (int e = g;; ++e) {
            const HeatGapEntry x = a.gaps[e];
            const double cond = 4.0 * x.coefficient * powi3(nt);
            rate = fmax(rate, fmax(cond / capc, cond / a.cap[x.partner]));
            if (x.last) break;
        }
    }
    return nt;
}

// Decode tile t of a tiling into the thread's column (i, j) and plane range [k0, k1).
// In 32-bit arithmetic where the tiling allows (a 64-bit division is a long software sequence, and the
// many-step kernels decode a tile every step).
__device__ __forceinline__ void tile_column(const Tiles& T, long long t, int& i, int& j, int& k0, int& k1) {
    int tx, ty, tz;
    if (T.ntiles <= 0x7fffffffLL) {
        const unsigned u = (unsigned)t, ntx = (unsigned)T.ntx, nty = (unsigned)T.nty;
        const unsigned r = u / ntx;
        tx = (int)(u - r * ntx);
        ty = (int)(r % nty);
        tz = (int)(r / nty);
    } else {
        tx = (int)(t % T.ntx);
        const long long r = t / T.ntx;
        ty = (int)(r % T.nty);
        tz = (int)(r / T.nty);
    }
    i = tx * 32 + threadIdx.x;
    j = ty * T.rows + threadIdx.y;
    k0 = tz * T.zc;
    k1 = min(T.nz, k0 + T.zc);
}

// The books of a plain step, after its cells: the blocks' partials reduced in fixed order by the
// last block to finish, then the ledger and the audit.
// acc: stored heat, heat shed, and (filled blocks) heat generated.
template <int NV>
__device__ __forceinline__ void heat_plain_books(const HeatPlainArgs& a, double (&acc)[NV]) {
    if (finish_blocks<NV>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) {
        DevState* st = a.st;
        st->lost += acc[1];
        if constexpr (NV > 2) st->supplied += acc[2];
        double total = 0.0, scale = 0.0;
        ledger_add(total, scale, acc[0]);
        ledger_add(total, scale, st->lost);
        ledger_add(total, scale, -st->supplied);
        st->part[0] = acc[0];
        st->part[1] = st->lost;
        st->part[2] = -st->supplied;
        audit_and_commit(st, total, scale);
        if (a.radiating) {  // worst_rate_now of the state this step leaves (solid.rs:1148-1185)
            const unsigned long long bits = atomicExch(&st->rate_bits, 0ull);
            st->rate_now = bits ? fmax(a.static_rate, __longlong_as_double((long long)bits)) : a.static_rate;
        }
    }
}

// Plain form. Each thread marches its column through the tile's planes, holding the cell
// below, the cell and the cell above in registers.
// Held to four blocks of 256 per SM (64 registers, no spill; 90 and two blocks unbounded).
#ifndef PM_HEAT_PLAIN_MIN_BLOCKS
#define PM_HEAT_PLAIN_MIN_BLOCKS 4
#endif
static __global__ void __launch_bounds__(256, PM_HEAT_PLAIN_MIN_BLOCKS) heat_plain_step(HeatPlainArgs a) {
    if (a.st->violated || heat_refused(a)) return;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t plane = (size_t)nx * ny;
    double acc[3] = {0.0, 0.0, 0.0};  // stored heat of the new state, heat shed and generated this step
    double rate = -1.0;  // a state-dependent limit: the largest rate of the new state
    for (long long t = blockIdx.x; t < a.tiles.ntiles; t += gridDim.x) {
        int i, j, k0, k1;
        tile_column(a.tiles, t, i, j, k0, k1);
        if (i >= nx || j >= ny) continue;
        size_t c = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k0);
        double below = k0 > 0 ? a.told[c - plane] : 0.0;
        double here = a.told[c];
        for (int k = k0; k < k1; ++k, c += plane) {
            const double above = k + 1 < nz ? a.told[c + plane] : 0.0;
            const double t0 = here;
            double flux = 0.0;
            if (a.uniform) {
                const double kf = a.kface;
                if (i > 0) flux += kf * (a.told[c - 1] - t0);
                if (i + 1 < nx) flux += kf * (a.told[c + 1] - t0);
                if (j > 0) flux += kf * (a.told[c - nx] - t0);
                if (j + 1 < ny) flux += kf * (a.told[c + nx] - t0);
                if (k > 0) flux += kf * (below - t0);
                if (k + 1 < nz) flux += kf * (above - t0);
            } else {
                const size_t xr = (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k);
                const size_t yr = (size_t)nx * ((size_t)j + (size_t)(ny + 1) * k);
                if (i > 0) flux += a.kx[i + xr] * (a.told[c - 1] - t0);
                if (i + 1 < nx) flux += a.kx[i + 1 + xr] * (a.told[c + 1] - t0);
                if (j > 0) flux += a.ky[i + yr] * (a.told[c - nx] - t0);
                if (j + 1 < ny) flux += a.ky[i + nx + yr] * (a.told[c + nx] - t0);
                if (k > 0) flux += a.kz[c] * (below - t0);
                if (k + 1 < nz) flux += a.kz[c + plane] * (above - t0);
            }
            const bool face = i == 0 || i + 1 == nx || j == 0 || j + 1 == ny || k == 0 || k + 1 == nz;
            const double shed = (a.films.exposed && face) ? film_flux(a, i, j, k, c, t0) : 0.0;
            const double mob = a.uniform ? a.mobility : a.mob[c];
            const double capc = a.uniform ? a.capacity : a.cap[c];
            double nt = t0 + a.dts * mob * (flux - shed);  // add_kelvin, latent <= 0 (solid.rs:1620-1635)
            if (a.src) {  // solid.rs:1854-1864, after the sweep
                const double w = a.src[c];
                if (w != 0.0) {
                    const double joules = w * a.dts;
                    nt += joules / capc;
                    acc[2] += joules;
                }
            }
            if (a.gap_of) {
                const int g = a.gap_of[c];
                if (g >= 0) nt = heat_gap_cell(a, g, t0, capc, nt, rate);
            }
            a.tnew[c] = nt;
            acc[0] += capc * (nt - a.reference);                  // solid.rs:1583-1590
            if (shed != 0.0) acc[1] += a.dts * mob * shed * capc;  // solid.rs:1821-1823
            if (a.radiating && face) rate = fmax(rate, heat_cell_rate(a, i, j, k, c, nt));
            below = here;
            here = above;
        }
    }
    if (a.radiating) heat_rate_publish(a, rate);
    heat_plain_books(a, acc);
}

// The plain form of a uniform block with two adjacent cells of a row per thread (rows of an even
// number of cells, so every pair starts on 16 bytes): per plane one 16-byte load each for the
// plane above and the rows either side, two scalar loads for the cells left and right of the
// pair, one 16-byte store. Each cell's arithmetic is heat_plain_step's uniform path, expression
// for expression (the reference's operand order, no contraction in the plain unit), so the fields
// agree with it, and with the reference, bit for bit; only the order of the FP64 sums within a
// block differs.
// Four blocks of 256 per SM (64 registers, a few bytes spilled) ran 164.8 Gcell/s on a 256³ block,
// against 143.0 at three (80 registers) and 114.4 at two (98 registers, the compiler's own choice).
#ifndef PM_HEAT_PAIR_MIN_BLOCKS
#define PM_HEAT_PAIR_MIN_BLOCKS 4
#endif
// A load of the old field: through L1 within one launch (its inputs never change while it runs), or
// from L2 alone (`ld.global.cg`) in the many-step kernel, where a buffer read two steps ago has since
// been rewritten by other blocks and a line kept in this SM's L1 would be stale.
template <bool CG>
__device__ __forceinline__ double2 heat_ld2(const double* p) {
    if constexpr (CG) return __ldcg(reinterpret_cast<const double2*>(p));
    else return *reinterpret_cast<const double2*>(p);
}
template <bool CG>
__device__ __forceinline__ double heat_ld(const double* p) {
    if constexpr (CG) return __ldcg(p);
    else return *p;
}

// One tile of the wide form for one step, from `told` into `tnew`: W adjacent cells of a row per
// thread (W = 2, the pair form, or 4), the arithmetic the one-step kernels and the persistent
// many-step kernel run, so they agree bit for bit. Each row of W cells comes in 16-byte loads.
template <bool CG, int W = 2>
__device__ __forceinline__ void heat_pair_tile(const HeatPlainArgs& a, long long t, const double* told, double* tnew,
                                               double (&acc)[2], double& rate) {
    static_assert(W == 2 || W == 4, "two or four cells of a row per thread");
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t plane = (size_t)nx * ny;
    const double kf = a.kface;
    int q, j, k0, k1;
    tile_column(a.tiles, t, q, j, k0, k1);  // q: the group's place along the row
    const int i = W * q;
    if (i >= nx || j >= ny) return;
    const size_t c0 = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k0);
    const double* p = told + c0;
    double* o = tnew + c0;
    const bool xl = i > 0, xh = i + W < nx, yl = j > 0, yh = j + 1 < ny;
    auto row = [&](double (&v)[W], const double* at, bool present) {
#pragma unroll
        for (int w = 0; w < W / 2; ++w) {
            const double2 d = present ? heat_ld2<CG>(at + 2 * w) : make_double2(0.0, 0.0);
            v[2 * w] = d.x;
            v[2 * w + 1] = d.y;
        }
    };
    double bv[W], hv[W];
    row(bv, p - plane, k0 > 0);
    row(hv, p, true);
    size_t c = c0;
    for (int k = k0; k < k1; ++k, p += plane, o += plane, c += plane) {
        double av[W], mv[W], pv[W];
        row(av, p + plane, k + 1 < nz);
        row(mv, p - nx, yl);
        row(pv, p + nx, yh);
        const double xm = xl ? heat_ld<CG>(p - 1) : 0.0, xp = xh ? heat_ld<CG>(p + W) : 0.0;
        double nt[W];
#pragma unroll
        for (int e = 0; e < W; ++e) {
            const double t0 = hv[e];
            double flux = 0.0;
            if (e > 0 || xl) flux += kf * ((e == 0 ? xm : hv[e > 0 ? e - 1 : 0]) - t0);
            if (e < W - 1 || xh) flux += kf * ((e == W - 1 ? xp : hv[e + 1 < W ? e + 1 : W - 1]) - t0);
            if (yl) flux += kf * (mv[e] - t0);
            if (yh) flux += kf * (pv[e] - t0);
            if (k > 0) flux += kf * (bv[e] - t0);
            if (k + 1 < nz) flux += kf * (av[e] - t0);
            // only a cell on a face can have a film: film_flux is +0 everywhere else
            const bool face = i + e == 0 || i + e + 1 == nx || !yl || !yh || k == 0 || k + 1 == nz;
            const double shed = (a.films.exposed && face) ? film_flux(a, i + e, j, k, c + e, t0) : 0.0;
            nt[e] = t0 + a.dts * a.mobility * (flux - shed);  // add_kelvin, latent <= 0 (solid.rs:1620-1635)
            acc[0] += a.capacity * (nt[e] - a.reference);     // solid.rs:1583-1590
            if (shed != 0.0) acc[1] += a.dts * a.mobility * shed * a.capacity;  // solid.rs:1821-1823
            if (a.radiating && face)
                rate = fmax(rate, heat_cell_rate(a, i + e, j, k, c + e, nt[e]));
        }
#pragma unroll
        for (int w = 0; w < W / 2; ++w) reinterpret_cast<double2*>(o)[w] = make_double2(nt[2 * w], nt[2 * w + 1]);
#pragma unroll
        for (int e = 0; e < W; ++e) {
            bv[e] = hv[e];
            hv[e] = av[e];
        }
    }
}

static __global__ void __launch_bounds__(256, PM_HEAT_PAIR_MIN_BLOCKS) heat_plain_pair_step(HeatPlainArgs a) {
    if (a.st->violated || heat_refused(a)) return;
    double acc[2] = {0.0, 0.0};  // stored heat of the new state, heat shed this step
    double rate = -1.0;  // a state-dependent limit: the largest rate of the new state
    for (long long t = blockIdx.x; t < a.tiles.ntiles; t += gridDim.x) heat_pair_tile<false>(a, t, a.told, a.tnew, acc, rate);
    if (a.radiating) heat_rate_publish(a, rate);
    heat_plain_books(a, acc);
}

// Four cells of a row per thread (rows of a multiple of 4 cells): four independent FP64 chains a
// thread, where the reference's sequential flux sum makes each cell one chain. Measured on a 256³
// block: 170 Gcell/s at two blocks of 256 per SM (no bound on registers), 159 at three (80
// registers, a few bytes spilled), against the pair form's 161.
#ifndef PM_HEAT_QUAD64_MIN_BLOCKS
#define PM_HEAT_QUAD64_MIN_BLOCKS 2
#endif
static __global__ void __launch_bounds__(256, PM_HEAT_QUAD64_MIN_BLOCKS) heat_plain_quad_step(HeatPlainArgs a) {
    if (a.st->violated || heat_refused(a)) return;
    double acc[2] = {0.0, 0.0};  // stored heat of the new state, heat shed this step
    double rate = -1.0;  // a state-dependent limit: the largest rate of the new state
    for (long long t = blockIdx.x; t < a.tiles.ntiles; t += gridDim.x)
        heat_pair_tile<false, 4>(a, t, a.told, a.tnew, acc, rate);
    if (a.radiating) heat_rate_publish(a, rate);
    heat_plain_books(a, acc);
}

struct HeatPersist {
    unsigned* barrier;  // kWaitWords words, zero at launch: the grid wait's counters
    int nsteps;
    unsigned budget;    // polls per grid wait before giving up
};

// The many-step kernels of small uniform blocks: every step of a call in one cooperative launch.
// Block 0 keeps the books and takes no cells; blocks 1.. take the tiles. In step s the workers step
// their tiles and store their partials (two sets, by the step's parity) while block 0 sums step
// s−1's in a fixed order and audits them; then every block arrives at the grid's s-th wait, block 0
// adding the stop mark to its arrival if the audit failed, and every block learns of it from the
// sum it polls. A failed audit of step s−1 ends the call with step s−1's state, which is intact:
// step s wrote the other buffer. After the last wait block 0 audits the last step and writes the
// books back. So the books' arithmetic never sits between the steps, and only block 0 reads the
// partials.
template <typename Args, typename StepTiles>
__device__ __forceinline__ void heat_persist(const Args& a, const HeatPersist& p, double cap_scale,
                                             StepTiles step_tiles) {
    __shared__ DevState books;
    __shared__ double red[32 * 2];
    __shared__ int stop;
    const int tid = linear_tid();
    const int nthreads = blockDim.x * blockDim.y;
    const bool keeper = blockIdx.x == 0;
    const unsigned workers = gridDim.x - 1;
    if (tid == 0) {
        stop = a.st->violated;
        if (keeper) books = *a.st;
    }
    __syncthreads();
    if (stop) return;
    auto audit = [&](int s) {  // block 0: step s's partials into the books
        const double* part = a.partials + (size_t)(s & 1) * 2 * workers;
        double v[2] = {0.0, 0.0};
        for (unsigned b = tid; b < workers; b += nthreads) {
            v[0] += __ldcg(&part[2 * (size_t)b]);
            v[1] += __ldcg(&part[2 * (size_t)b + 1]);
        }
        block_sum<2>(v, red);
        if (tid == 0) {
            const double stored = cap_scale * v[0];
            books.lost += cap_scale * v[1];
            double total = 0.0, scale = 0.0;
            ledger_add(total, scale, stored);
            ledger_add(total, scale, books.lost);
            ledger_add(total, scale, -books.supplied);
            books.part[0] = stored;
            books.part[1] = books.lost;
            books.part[2] = -books.supplied;
            audit_and_commit(&books, total, scale);
            stop = books.violated ? 1 : 0;
        }
    };
    bool timed_out = false;
    int s = 0;
    for (; s < p.nsteps; ++s) {
        if (!keeper) {
            double acc[2] = {0.0, 0.0};
            step_tiles(s, (long long)blockIdx.x - 1, (long long)workers, acc);
            block_sum<2>(acc, red);
            if (tid == 0) {
                double* part = a.partials + (size_t)(s & 1) * 2 * workers;
                part[2 * (size_t)(blockIdx.x - 1)] = acc[0];
                part[2 * (size_t)(blockIdx.x - 1) + 1] = acc[1];
            }
        } else if (s > 0) {
            audit(s - 1);  // sets `stop` in block 0 when the audit failed (read after the wait's barrier)
        }
        const int w = grid_wait(p.barrier, (unsigned)(s + 1), p.budget, keeper && stop);
        if (w == 0) {
            timed_out = true;
            break;
        }
        if (w == 2) {
            stop = 1;
            break;
        }
    }
    if (timed_out) {
        if (tid == 0) atomicExch(&a.st->violated, kDeviceTimeout);
        return;
    }
    if (!keeper) return;
    if (!stop) audit(p.nsteps - 1);
    if (tid == 0) {
        DevState* st = a.st;
        const int seen = atomicAdd(&st->violated, 0);  // a block that gave up has already said so
        books.counter = 0u;
        *st = books;
        if (seen == kDeviceTimeout) st->violated = kDeviceTimeout;
    }
}

// The pair form's many-step kernel: blocks of 32 × ROWS threads (8 rows: four blocks per SM; 32 rows:
// one block of 1024 per SM, so a 64³ block is 128 workers and the keeper).
template <int ROWS>
static __global__ void __launch_bounds__(32 * ROWS, ROWS == 8 ? PM_HEAT_PAIR_MIN_BLOCKS : 1)
    heat_plain_pair_steps(HeatPlainArgs a, HeatPersist p) {
    heat_persist(a, p, 1.0, [&](int s, long long first, long long stride, double (&acc)[2]) {
        const double* told = (s & 1) ? a.tnew : a.told;
        double* tnew = const_cast<double*>((s & 1) ? a.told : a.tnew);
        double rate = -1.0;
        for (long long t = first; t < a.tiles.ntiles; t += stride) heat_pair_tile<true>(a, t, told, tnew, acc, rate);
    });
}

struct HeatF32Args {
    const float* __restrict__ dold;
    float* __restrict__ dnew;
    int nx, ny, nz;
    float a;         // dt · mobility · k_face
    int exposed;     // film faces
    float b[6];      // dt · mobility · g_f / dx per film face
    float off[6];    // T0 − ambient per film face
    double capacity; // per cell
    // Filled blocks (null otherwise): per-face conductivities (solid.rs:686-713), dt · mobility
    // per cell, capacity per cell, and per exposed face f the film conductance g/dx of each cell
    // on it (film[f] indexed j + ny·k on the x faces, i + nx·k on the y faces, i + nx·j on z)
    const float* __restrict__ kx;
    const float* __restrict__ ky;
    const float* __restrict__ kz;
    const float* __restrict__ m;
    const double* __restrict__ cap;
    const float* film[6];
    double dts;                       // the step, for the sources
    const double* __restrict__ src;   // filled blocks that generate: watts per cell, zero on void
    int quads;  // uniform blocks with rows of a multiple of 4: heat_f32_quad_step, tiles of quads
    Tiles tiles;
    DevState* st;
    double* partials;
    unsigned nblocks;
    // Uniform blocks whose films radiate (heat_f32_step only): each face cell's film is the plain
    // form's film_flux at its kelvin T0 + deviation, and its new rate joins the state's limit, both
    // through `rad` (the plain form's film, conductance and limit parameters; no field is read)
    int radiating;
    double t0;
    HeatPlainArgs rad;
};

// The books of an FP32 step, after its cells: the block's partials reduced in fixed order by the
// last block to finish, then the ledger and the audit.
// acc: stored heat, heat shed, and (filled blocks) heat generated.
template <int NV>
__device__ __forceinline__ void heat_f32_books(const HeatF32Args& a, double (&acc)[NV], bool filled) {
    if (finish_blocks<NV>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) {
        DevState* st = a.st;
        const double stored = filled ? acc[0] : a.capacity * acc[0];
        st->lost += filled ? acc[1] : a.capacity * acc[1];
        if constexpr (NV > 2) st->supplied += acc[2];
        double total = 0.0, scale = 0.0;
        ledger_add(total, scale, stored);
        ledger_add(total, scale, st->lost);
        ledger_add(total, scale, -st->supplied);
        st->part[0] = stored;
        st->part[1] = st->lost;
        st->part[2] = -st->supplied;
        audit_and_commit(st, total, scale);
        if (a.radiating) {  // worst_rate_now of the state this step leaves (solid.rs:1148-1185)
            const unsigned long long bits = atomicExch(&st->rate_bits, 0ull);
            st->rate_now = bits ? fmax(a.rad.static_rate, __longlong_as_double((long long)bits)) : a.rad.static_rate;
        }
    }
}

// Chosen form, z-marching like the plain form; neighbours in the plane come from L1/L2.
template <bool FILLED>
static __global__ void __launch_bounds__(256) heat_f32_step(HeatF32Args a) {
    if (a.st->violated || (a.radiating && heat_refused(a.rad))) return;
    double rate = -1.0;  // radiating films: the largest rate of the new state
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t plane = (size_t)nx * ny;
    double acc[FILLED ? 3 : 2] = {};
    for (long long t = blockIdx.x; t < a.tiles.ntiles; t += gridDim.x) {
        int i, j, k0, k1;
        tile_column(a.tiles, t, i, j, k0, k1);
        if (i >= nx || j >= ny) continue;
        size_t c = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k0);
        float below = k0 > 0 ? __ldg(a.dold + c - plane) : 0.0f;
        float here = __ldg(a.dold + c);
        const bool xl = i > 0, xh = i + 1 < nx, yl = j > 0, yh = j + 1 < ny;
        const bool edge_xy = !(xl && xh && yl && yh);
        double col_shed = 0.0;
        for (int k = k0; k < k1; ++k, c += plane) {
            const float above = (k + 1 < nz) ? __ldg(a.dold + c + plane) : 0.0f;
            float s = 0.0f;
            if constexpr (FILLED) {
                // solid.rs:1773-1826 in the reference's arm order, each face's own conductivity
                const size_t xr = (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k);
                const size_t yr = (size_t)nx * ((size_t)j + (size_t)(ny + 1) * k);
                if (xl) s += __ldg(a.kx + i + xr) * (__ldg(a.dold + c - 1) - here);
                if (xh) s += __ldg(a.kx + i + 1 + xr) * (__ldg(a.dold + c + 1) - here);
                if (yl) s += __ldg(a.ky + i + yr) * (__ldg(a.dold + c - nx) - here);
                if (yh) s += __ldg(a.ky + i + nx + yr) * (__ldg(a.dold + c + nx) - here);
                if (k > 0) s += __ldg(a.kz + c) * (below - here);
                if (k + 1 < nz) s += __ldg(a.kz + c + plane) * (above - here);
            } else {
                if (xl) s += __ldg(a.dold + c - 1) - here;
                if (xh) s += __ldg(a.dold + c + 1) - here;
                if (yl) s += __ldg(a.dold + c - nx) - here;
                if (yh) s += __ldg(a.dold + c + nx) - here;
                if (k > 0) s += below - here;
                if (k + 1 < nz) s += above - here;
            }
            float shed = 0.0f;
            if (a.exposed && (edge_xy || k == 0 || k + 1 == nz)) {
                if constexpr (FILLED) {
                    const unsigned px = (unsigned)j + (unsigned)ny * (unsigned)k, py = (unsigned)i + (unsigned)nx * (unsigned)k,
                                   pz = (unsigned)i + (unsigned)nx * (unsigned)j;
                    if (((a.exposed >> 0) & 1) && !xl) shed += __ldg(a.film[0] + px) * (here + a.off[0]);
                    if (((a.exposed >> 1) & 1) && !xh) shed += __ldg(a.film[1] + px) * (here + a.off[1]);
                    if (((a.exposed >> 2) & 1) && !yl) shed += __ldg(a.film[2] + py) * (here + a.off[2]);
                    if (((a.exposed >> 3) & 1) && !yh) shed += __ldg(a.film[3] + py) * (here + a.off[3]);
                    if (((a.exposed >> 4) & 1) && k == 0) shed += __ldg(a.film[4] + pz) * (here + a.off[4]);
                    if (((a.exposed >> 5) & 1) && k + 1 == nz) shed += __ldg(a.film[5] + pz) * (here + a.off[5]);
                } else if (a.radiating) {
                    // solid.rs:1192-1219 at the cell's kelvin, as dt · mobility · flux
                    shed = (float)(a.rad.dts * a.rad.mobility * film_flux(a.rad, i, j, k, c, a.t0 + (double)here));
                    col_shed += (double)shed;
                } else {
                    if (((a.exposed >> 0) & 1) && !xl) shed += a.b[0] * (here + a.off[0]);
                    if (((a.exposed >> 1) & 1) && !xh) shed += a.b[1] * (here + a.off[1]);
                    if (((a.exposed >> 2) & 1) && !yl) shed += a.b[2] * (here + a.off[2]);
                    if (((a.exposed >> 3) & 1) && !yh) shed += a.b[3] * (here + a.off[3]);
                    if (((a.exposed >> 4) & 1) && k == 0) shed += a.b[4] * (here + a.off[4]);
                    if (((a.exposed >> 5) & 1) && k + 1 == nz) shed += a.b[5] * (here + a.off[5]);
                    col_shed += (double)shed;
                }
            }
            float nd;
            if constexpr (FILLED) {
                // add_kelvin (solid.rs:1620-1635); stored heat C·dev and shed heat C·dt·mob·shed
                const float mc = __ldg(a.m + c);
                nd = here + mc * (s - shed);
                const double capc = __ldg(a.cap + c);
                if (a.src) {  // solid.rs:1854-1864, after the sweep: the joules in FP64, the rise in f32
                    const double w = __ldg(a.src + c);
                    if (w != 0.0) {
                        const double joules = w * a.dts;
                        nd += (float)(joules / capc);
                        acc[FILLED ? 2 : 0] += joules;
                    }
                }
                acc[0] += capc * (double)nd;
                if (shed != 0.0f) acc[1] += capc * (double)(mc * shed);
            } else {
                nd = here + (a.a * s - shed);
                acc[0] += (double)nd;
                if (a.radiating && (edge_xy || k == 0 || k + 1 == nz))
                    rate = fmax(rate, heat_cell_rate(a.rad, i, j, k, c, a.t0 + (double)nd));
            }
            a.dnew[c] = nd;
            below = here;
            here = above;
        }
        acc[1] += col_shed;
    }
    if (a.radiating) heat_rate_publish(a.rad, rate);
    heat_f32_books(a, acc, FILLED);
}

// The uniform FP32 form with four adjacent cells of a row per thread (rows of a multiple of 4
// cells, so every quad starts on 16 bytes): per plane one 16-byte load each for the plane above
// and the rows either side, two scalar loads for the cells left and right of the quad, one 16-byte
// store. Each cell's arithmetic is heat_f32_step's uniform case in the same order and roundings
// (the sums from +0 with the neighbours present, the films as the fused b·(here + off) + shed,
// then here + (a·sum − shed) as a fused multiply-add and an add), so the fields agree with it bit
// for bit; only the order of the FP64 sums within a block differs.
template <bool CG>
__device__ __forceinline__ float4 heat_ld4(const float* p) {
    if constexpr (CG) return __ldcg(reinterpret_cast<const float4*>(p));
    else return __ldg(reinterpret_cast<const float4*>(p));
}
template <bool CG>
__device__ __forceinline__ float heat_ldf(const float* p) {
    if constexpr (CG) return __ldcg(p);
    else return __ldg(p);
}

// One tile of the quad form for one step, from `dold` into `dnew` (loads as heat_ld2 describes):
// the arithmetic of the one-step and the many-step kernels.
template <bool CG>
__device__ __forceinline__ void heat_quad_tile(const HeatF32Args& a, long long t, const float* dold, float* dnew,
                                               double (&acc)[2]) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t plane = (size_t)nx * ny;
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    int q, j, k0, k1;
    tile_column(a.tiles, t, q, j, k0, k1);  // q: the quad's place along the row
    const int i = 4 * q;
    if (i >= nx || j >= ny) return;
    const size_t c = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k0);
    const float* p = dold + c;
    float* o = dnew + c;
    const bool xl = i > 0, xh = i + 4 < nx, yl = j > 0, yh = j + 1 < ny;
    float4 below = k0 > 0 ? heat_ld4<CG>(p - plane) : zero;
    float4 here = heat_ld4<CG>(p);
    double col_shed = 0.0;
    for (int k = k0; k < k1; ++k, p += plane, o += plane) {
        const bool zl = k > 0, zh = k + 1 < nz;
        const float4 above = zh ? heat_ld4<CG>(p + plane) : zero;
        const float4 ym = yl ? heat_ld4<CG>(p - nx) : zero;
        const float4 yp = yh ? heat_ld4<CG>(p + nx) : zero;
        const float xm = xl ? heat_ldf<CG>(p - 1) : 0.0f, xp = xh ? heat_ldf<CG>(p + 4) : 0.0f;
        const float hv[4] = {here.x, here.y, here.z, here.w}, bv[4] = {below.x, below.y, below.z, below.w};
        const float av[4] = {above.x, above.y, above.z, above.w};
        const float mv[4] = {ym.x, ym.y, ym.z, ym.w}, pv[4] = {yp.x, yp.y, yp.z, yp.w};
        float nd[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float h = hv[e];
            const bool l = e > 0 || xl, r = e < 3 || xh;  // the cell's x neighbours are in the block
            float s = 0.0f;
            if (l) s += (e == 0 ? xm : hv[e - 1]) - h;
            if (r) s += (e == 3 ? xp : hv[e + 1]) - h;
            if (yl) s += mv[e] - h;
            if (yh) s += pv[e] - h;
            if (zl) s += bv[e] - h;
            if (zh) s += av[e] - h;
            float shed = 0.0f;
            if (a.exposed && (!(l && r && yl && yh) || !zl || !zh)) {
                if (((a.exposed >> 0) & 1) && !l) shed = __fmaf_rn(a.b[0], h + a.off[0], shed);
                if (((a.exposed >> 1) & 1) && !r) shed = __fmaf_rn(a.b[1], h + a.off[1], shed);
                if (((a.exposed >> 2) & 1) && !yl) shed = __fmaf_rn(a.b[2], h + a.off[2], shed);
                if (((a.exposed >> 3) & 1) && !yh) shed = __fmaf_rn(a.b[3], h + a.off[3], shed);
                if (((a.exposed >> 4) & 1) && !zl) shed = __fmaf_rn(a.b[4], h + a.off[4], shed);
                if (((a.exposed >> 5) & 1) && !zh) shed = __fmaf_rn(a.b[5], h + a.off[5], shed);
                col_shed += (double)shed;
            }
            nd[e] = __fadd_rn(h, __fmaf_rn(a.a, s, -shed));
            acc[0] += (double)nd[e];
        }
        *reinterpret_cast<float4*>(o) = make_float4(nd[0], nd[1], nd[2], nd[3]);
        below = here;
        here = above;
    }
    acc[1] += col_shed;
}

static __global__ void __launch_bounds__(256) heat_f32_quad_step(HeatF32Args a) {
    if (a.st->violated) return;
    double acc[2] = {0.0, 0.0};
    for (long long t = blockIdx.x; t < a.tiles.ntiles; t += gridDim.x) heat_quad_tile<false>(a, t, a.dold, a.dnew, acc);
    heat_f32_books(a, acc, false);
}

// The quad form's many-step kernel, as heat_plain_pair_steps.
template <int ROWS>
static __global__ void __launch_bounds__(32 * ROWS, ROWS == 8 ? 3 : 1) heat_f32_quad_steps(HeatF32Args a, HeatPersist p) {
    heat_persist(a, p, a.capacity, [&](int s, long long first, long long stride, double (&acc)[2]) {
        const float* dold = (s & 1) ? a.dnew : a.dold;
        float* dnew = const_cast<float*>((s & 1) ? a.dold : a.dnew);
        for (long long t = first; t < a.tiles.ntiles; t += stride) heat_quad_tile<true>(a, t, dold, dnew, acc);
    });
}

// The opening ledger of a freshly uploaded block: stored heat only (lost and supplied are zero
// until something steps). Plain: Σ C·(T − T_ref); f32: C·Σ dev.
struct HeatMeasureArgs {
    const double* t64;
    const float* d32;
    const double* cap;  // null: uniform `capacity`
    double capacity, reference;
    size_t n;
    DevState* st;
    double* partials;
    unsigned nblocks;
};

static __global__ void __launch_bounds__(256) heat_measure(HeatMeasureArgs a) {
    double acc[1] = {0.0};
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < a.n; c += (size_t)gridDim.x * blockDim.x) {
        if (a.t64) {
            const double capc = a.cap ? a.cap[c] : a.capacity;
            acc[0] += capc * (a.t64[c] - a.reference);
        } else {
            acc[0] += a.cap ? a.cap[c] * (double)a.d32[c] : (double)a.d32[c];
        }
    }
    if (finish_blocks<1>(acc, a.partials, a.nblocks, &a.st->counter) && linear_tid() == 0) {
        DevState* st = a.st;
        const double stored = (a.t64 || a.cap) ? acc[0] : a.capacity * acc[0];
        double total = 0.0, scale = 0.0;
        ledger_add(total, scale, stored);
        ledger_add(total, scale, st->lost);
        ledger_add(total, scale, -st->supplied);
        st->part[0] = stored;
        st->part[1] = st->lost;
        st->part[2] = -st->supplied;
        st->total = total;
        st->scale = scale;
        st->prev_total = total;
        st->prev_scale = scale;
    }
}

// Conversions between the caller's kelvin (f64) and the f32 deviation store.
static __global__ void heat_to_deviation(const double* __restrict__ t, float* __restrict__ d, double t0, size_t n) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        d[c] = (float)(t[c] - t0);
}
static __global__ void heat_from_deviation(const float* __restrict__ d, double* __restrict__ t, double t0, size_t n) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        t[c] = t0 + (double)d[c];
}
// solid.rs:1752-1765 + 1620-1635: a uniform rise over every cell but the void ones (`vd`, null
// where there is none).
static __global__ void heat_add_rise64(double* __restrict__ t, double rise, size_t n, const uint8_t* __restrict__ vd) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        if (!vd || !vd[c]) t[c] += rise;
}
static __global__ void heat_add_rise32(float* __restrict__ d, float rise, size_t n, const uint8_t* __restrict__ vd) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        if (!vd || !vd[c]) d[c] += rise;
}

// ---------------------------------------------------------------------------------------------
// Bar1D (crates/pantometry-thermal/src/lib.rs:425-660): explicit conduction along a bar with
// insulated ends, `prev + f·(left − 2·prev + right)` with the end cells' missing neighbour their
// own value (lib.rs:614-620). One thread per cell; the plain f64 form (built with --fmad=false)
// is bit-exact with `Bar1D::step`, the FP32 form keeps T − T_ref. Fused: the stored heat
// C·Σ(T − T_ref) (lib.rs:536-538) and the audit of the bar's books against the heat it took from
// the bus (its `attribute` check, books_balance at lib.rs:555-557).
//
// bar_deposit — the heat a step takes from the bus before it conducts (lib.rs:590-606): lumped
// joules into the first cell, then joules per cell, each divided by the cell's capacity.
// ---------------------------------------------------------------------------------------------
template <typename Real>
struct BarArgs {
    const Real* __restrict__ told;
    Real* __restrict__ tnew;
    int n;
    Real f;            // α·dt/dx² (lib.rs:546-551)
    double capacity;   // (ρ·area·dx)·c (lib.rs:514-520)
    double reference;  // T_ref in the plain form; 0 for the FP32 deviations
    DevState* st;
    double* partials;
    unsigned nblocks;
};

template <typename Real>
static __global__ void __launch_bounds__(256) bar_step(BarArgs<Real> a) {
    DevState* st = a.st;
    if (st->violated) return;
    const int n = a.n, last = n - 1;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Real prev = a.told[i];
        const Real left = a.told[i > 0 ? i - 1 : 0];
        const Real right = a.told[i + 1 < last ? i + 1 : last];
        const Real nt = prev + a.f * (left - Real(2) * prev + right);
        a.tnew[i] = nt;
        acc[0] += (double)nt - a.reference;
    }
    if (finish_blocks<1>(acc, a.partials, a.nblocks, &st->counter) && linear_tid() == 0) {
        const double stored = a.capacity * acc[0];
        double total = 0.0, scale = 0.0;
        ledger_add(total, scale, stored);
        ledger_add(total, scale, -st->injected);  // what it has taken from the bus
        st->part[0] = stored;
        st->part[1] = st->injected;
        audit_and_commit(st, total, scale);
    }
}

template <typename Real>
static __global__ void bar_deposit(Real* __restrict__ t, const double* __restrict__ per_cell, double lumped,
                                   double capacity, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Real v = t[i];
        if (i == 0 && lumped != 0.0) v = (Real)((double)v + lumped / capacity);
        if (per_cell) v = (Real)((double)v + per_cell[i] / capacity);
        t[i] = v;
    }
}

}  // namespace pm
