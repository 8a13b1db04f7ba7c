// pm_ensemble: many independent one-material `Solid3D` blocks of uneven sizes, each with its own
// substance, step and films, advanced together by one persistent brick-list kernel per step
// (ensemble_kernels.cuh) and CUDA graphs of 64 steps. Each block keeps its own FP64 books,
// ledger and audit, exactly as a `Solid3D` driven alone would (solid.rs:1904-1927).
#include <algorithm>
#include <limits>
#include <new>

#include "runtime.h"

namespace pm {

namespace {

constexpr double kStableFourier3D = 1.0 / 6.0;  // solid.rs:84

double ens_series_with_half_cell(double film, double conductivity, double area, double dx) {  // solid.rs:110-122
    if (film <= 0.0) return 0.0;
    double half = 2.0 * conductivity * area / dx;
    if (!std::isfinite(half)) return film;
    if (half <= 0.0) return 0.0;
    return 1.0 / (1.0 / film + 1.0 / half);
}

double ens_rust_max(double a, double b) {  // f64::max
    if (std::isnan(a)) return b;
    if (std::isnan(b)) return a;
    return a > b ? a : b;
}

// The brick shapes the autotuner chooses among: log2 of the threads along x (256 threads, so
// y = 256 >> bxs rows), the planes each thread marches, and the cells of its row each thread takes
// (1; 4 for the f32 quad shapes; 2 for the f64 pair shapes). Every shape has its own x and y
// extents in cells.
struct EnsShape {
    int bxs, zc, cells;
    int x() const { return cells << bxs; }
    int y() const { return 256 >> bxs; }
};
constexpr EnsShape kEnsShapes[] = {{5, 16, 1}, {5, 8, 1},  {5, 32, 1}, {5, 64, 1}, {4, 8, 1},  {4, 16, 1},
                                   {4, 32, 1}, {4, 64, 1}, {6, 8, 1},  {6, 16, 1}, {6, 32, 1}, {6, 64, 1},
                                   {2, 32, 4}, {2, 64, 4}, {3, 32, 4}, {3, 64, 4}, {4, 32, 4}, {4, 64, 4},
                                   {5, 32, 4}, {5, 64, 4}, {3, 32, 2}, {3, 64, 2}, {4, 32, 2}, {4, 64, 2},
                                   {5, 32, 2}, {5, 64, 2}};
// whether a shape runs at this precision: the quads are f32 only, the pairs f64 only
inline bool ens_shape_fits(const EnsShape& s, int p) {
    return s.cells == 1 || (s.cells == 4) == (p != PM_PLAIN_F64);
}
constexpr int kEnsShapeCount = sizeof(kEnsShapes) / sizeof(kEnsShapes[0]);

// What `Solid3D::resolve` and `worst_rate_now` give for one uniform block with films on all six
// faces (solid.rs:588-784, 1148-1185), with the same arithmetic the single-block handle uses.
struct UniformBlock {
    double kface, mobility, capacity, k_cell;
    double share[6];
    double rate;  // worst rate now; NaN: no diffusivity
};

UniformBlock uniform_block(const pm_ensemble_grid& d) {
    UniformBlock u{};
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const double dx = d.dx;
    const double volume = dx * dx * dx;
    const pm_substance& s = d.substance;
    const double k = s.thermal ? s.conductivity : NAN;
    const double C = s.thermal ? (s.density * volume) * s.specific_heat : NAN;
    const double sum = k + k;
    u.kface = sum > 0.0 ? 2.0 * k * k / sum : 0.0;
    u.capacity = C;
    u.mobility = dx / C;
    u.k_cell = s.thermal ? s.conductivity : std::numeric_limits<double>::infinity();
    const double areas[6] = {((double)ny * dx) * ((double)nz * dx), ((double)ny * dx) * ((double)nz * dx),
                             ((double)nx * dx) * ((double)nz * dx), ((double)nx * dx) * ((double)nz * dx),
                             ((double)nx * dx) * ((double)ny * dx), ((double)nx * dx) * ((double)ny * dx)};
    const double cells_on[6] = {(double)ny * nz, (double)ny * nz, (double)nx * nz,
                                (double)nx * nz, (double)nx * ny, (double)nx * ny};
    for (int f = 0; f < 6; ++f) u.share[f] = areas[f] / cells_on[f];  // solid.rs:1203
    const bool films = d.convection_w_per_m2_k != 0.0;
    auto fx = [&](int i) { return (i > 0 && i < nx) ? u.kface : 0.0; };
    auto fy = [&](int j) { return (j > 0 && j < ny) ? u.kface : 0.0; };
    auto fz = [&](int q) { return (q > 0 && q < nz) ? u.kface : 0.0; };
    double worst = 0.0;
    bool nowhere = false;
    for (int k3 : {0, 1, nz - 2, nz - 1}) {
        if (k3 < 0 || k3 >= nz) continue;
        for (int j3 : {0, 1, ny - 2, ny - 1}) {
            if (j3 < 0 || j3 >= ny) continue;
            for (int i3 : {0, 1, nx - 2, nx - 1}) {
                if (i3 < 0 || i3 >= nx) continue;
                const double face_sum = fx(i3) + fx(i3 + 1) + fy(j3) + fy(j3 + 1) + fz(k3) + fz(k3 + 1);
                const double rate = u.mobility * face_sum;
                if (std::isnan(rate)) nowhere = true;
                else worst = ens_rust_max(worst, rate);
            }
        }
    }
    if (nowhere) {
        u.rate = NAN;
        return u;
    }
    if (films) {
        const double base = worst;
        double now = base;
        for (int k3 : {0, 1, nz - 2, nz - 1}) {
            if (k3 < 0 || k3 >= nz) continue;
            for (int j3 : {0, 1, ny - 2, ny - 1}) {
                if (j3 < 0 || j3 >= ny) continue;
                for (int i3 : {0, 1, nx - 2, nx - 1}) {
                    if (i3 < 0 || i3 >= nx) continue;
                    double loss = -0.0;  // solid.rs:1269-1288 at zero emissivity
                    for (int f = 0; f < 6; ++f) {
                        const bool holds = f == 0 ? i3 == 0 : f == 1 ? i3 + 1 == nx : f == 2 ? j3 == 0
                                         : f == 3 ? j3 + 1 == ny : f == 4 ? k3 == 0 : k3 + 1 == nz;
                        if (!holds) continue;
                        loss += ens_series_with_half_cell(d.convection_w_per_m2_k * u.share[f], u.k_cell, u.share[f], dx);
                    }
                    if (loss == 0.0) continue;
                    const double face_sum = fx(i3) + fx(i3 + 1) + fy(j3) + fy(j3 + 1) + fz(k3) + fz(k3 + 1);
                    now = ens_rust_max(now, u.mobility * (face_sum + loss / dx));
                }
            }
        }
        worst = now;
    }
    u.rate = worst;
    return u;
}

pm_status check_grid(const pm_ensemble_grid& d, int g) {
    const std::string where = "block " + std::to_string(g) + ": ";
    if (d.nx < 1 || d.ny < 1 || d.nz < 1 || d.nx > 65535 || d.ny > 65535 || d.nz > 65535)
        return fail(PM_BAD_ARG, where + "each axis holds 1..65535 cells");
    if (!(d.dx > 0.0)) return fail(PM_BAD_ARG, where + "dx must be positive");
    if (!d.substance.thermal) return fail(PM_UNSUPPORTED, where + "a substance without thermal properties");
    if (d.convection_w_per_m2_k != 0.0 && d.substance.emissivity != 0.0)
        return fail(PM_UNSUPPORTED, where + "radiating films (emissivity > 0) make the step limit state-dependent");
    if (!(d.convection_w_per_m2_k >= 0.0)) return fail(PM_BAD_ARG, where + "film convection must be >= 0");
    if (!(d.dt > 0.0)) return fail(PM_BAD_ARG, where + "dt must be positive");
    return PM_OK;
}

}  // namespace

struct Ensemble : Handle {
    std::vector<pm_ensemble_grid> desc;
    std::vector<UniformBlock> blocks;
    std::vector<EnsGrid> grids;
    std::vector<EnsBrick> bricks;
    std::vector<DevState> states;  // host mirror of the per-block books
    size_t cells = 0;                     // cells of every block, in the caller's layout
    size_t dcells = 0;                    // elements on the device (f32 rows padded to a multiple of 4)
    std::vector<size_t> ref_offset;       // each block's first cell in the caller's layout
    // FP32: bricks 32 wide step with the TMA-staged kernel; maps[par * blocks + g] is block g's map
    bool tma = false;
    std::vector<CUtensorMap> maps;
    DBuf dmaps, dinfos;
    DBuf dwork;  // the TMA walk's two counters (next brick, CTAs done), zero between launches
    int shape = 0;
    long long generation = 0;  // bumped when the brick list changes (the graph cache key)
    DBuf field[2], stage, dgrids, dbricks, dstates, bpartials, saved, saved_states;

    size_t esize() const { return precision == PM_PLAIN_F64 ? sizeof(double) : sizeof(float); }
    unsigned wave() const {
        const bool wide = kEnsShapes[shape].cells != 1;
        return wave_of(precision == PM_PLAIN_F64 ? (wide ? kEnsF64Pair : kEnsF64) : (wide ? kEnsF32Quad : kEnsF32));
    }

    // Brick list and block table for a shape; uploads both.
    pm_status set_shape(int sh) {
        const EnsShape s = kEnsShapes[sh];
        if (!ens_shape_fits(s, precision))
            return fail(PM_BAD_ARG, s.cells == 4 ? "quad brick shapes are f32 only" : "pair brick shapes are f64 only");
        const int bx = s.x(), by = s.y();
        bricks.clear();
        for (size_t g = 0; g < grids.size(); ++g) {
            EnsGrid& e = grids[g];
            e.first_brick = (unsigned)bricks.size();
            for (int z = 0; z < e.nz; z += s.zc)
                for (int y = 0; y < e.ny; y += by)
                    for (int x = 0; x < e.nx; x += bx) {
                        EnsBrick b{};
                        b.grid = (unsigned)g;
                        b.x0 = (unsigned short)x;
                        b.y0 = (unsigned short)y;
                        b.z0 = (unsigned short)z;
                        b.z1 = (unsigned short)std::min(e.nz, z + s.zc);
                        bricks.push_back(b);
                    }
            e.nbricks = (unsigned)bricks.size() - e.first_brick;
        }
        if (bricks.size() >= (size_t)UINT32_MAX) return fail(PM_BAD_ARG, "too many bricks");
        if (tma) {  // the per-brick records the TMA kernel copies with each stage
            std::vector<EnsBrickInfo> infos(bricks.size());
            for (size_t q = 0; q < bricks.size(); ++q) {
                const EnsGrid& g = grids[bricks[q].grid];
                EnsBrickInfo& f = infos[q];
                std::memset(&f, 0, sizeof(f));
                f.offset = g.offset;
                f.grid = bricks[q].grid;
                f.x0 = bricks[q].x0; f.y0 = bricks[q].y0;
                f.nx = g.nx; f.ny = g.ny; f.nz = g.nz; f.pitch = g.pitch; f.exposed = g.exposed;
                f.a = g.a;
                for (int k = 0; k < 6; ++k) { f.b[k] = g.b[k]; f.off[k] = g.off[k]; }
            }
            PM_CUDA(cudaStreamSynchronize(stream()));
            if (dinfos.bytes < infos.size() * sizeof(EnsBrickInfo)) PM_CUDA(dinfos.alloc(infos.size() * sizeof(EnsBrickInfo)));
            PM_CUDA(put_sync(dinfos.p, infos.data(), infos.size() * sizeof(EnsBrickInfo)));
        }
        drop_graphs();
        PM_CUDA(cudaStreamSynchronize(stream()));
        if (dbricks.bytes < bricks.size() * sizeof(EnsBrick)) PM_CUDA(dbricks.alloc(bricks.size() * sizeof(EnsBrick)));
        // two partials per brick, or two per consumer warp of a brick on the TMA path
        const size_t per_brick = tma ? (size_t)kEnsTmaPartialsPerBrick : 2;
        if (bpartials.bytes < bricks.size() * per_brick * sizeof(double))
            PM_CUDA(bpartials.alloc(bricks.size() * per_brick * sizeof(double)));
        if (tma && !dwork.p) {
            PM_CUDA(dwork.alloc(2 * sizeof(unsigned)));
            PM_CUDA(cudaMemsetAsync(dwork.p, 0, 2 * sizeof(unsigned), stream()));
        }
        PM_CUDA(put_sync(dbricks.p, bricks.data(), bricks.size() * sizeof(EnsBrick)));
        PM_CUDA(put_sync(dgrids.p, grids.data(), grids.size() * sizeof(EnsGrid)));
        shape = sh;
        ++generation;
        return PM_OK;
    }

    template <typename Real>
    EnsArgs<Real> args(int par) const {
        EnsArgs<Real> a{};
        a.old = field[par].as<Real>();
        a.nu = field[par ^ 1].as<Real>();
        a.grids = dgrids.as<EnsGrid>();
        a.bricks = dbricks.as<EnsBrick>();
        a.nbricks = (unsigned)bricks.size();
        a.ngrids = (unsigned)grids.size();
        a.bxs = kEnsShapes[shape].bxs;
        a.wide = kEnsShapes[shape].cells != 1 ? 1 : 0;
        a.states = dstates.as<DevState>();
        a.partials = bpartials.as<double>();
        return a;
    }
    unsigned nblocks() const { return std::min<unsigned>(wave(), (unsigned)std::max<size_t>(bricks.size(), 1)); }

    cudaError_t launch(int par, bool measure, cudaStream_t s) const {
        if (precision == PM_PLAIN_F64) return launch_ens<double>(args<double>(par), measure, nblocks(), s);
        if (!measure && tma && kEnsShapes[shape].bxs == 5 && kEnsShapes[shape].cells == 1) {
            EnsTmaArgs t{};
            t.e = args<float>(par);
            t.maps = dmaps.as<CUtensorMap>() + (size_t)par * grids.size();
            t.infos = dinfos.as<EnsBrickInfo>();
            t.work = dwork.as<unsigned>();
            const unsigned w = wave_of(kEnsTma);
            return launch_ens_tma(t, std::min<unsigned>(w, (unsigned)std::max<size_t>(bricks.size(), 1)), s);
        }
        return launch_ens<float>(args<float>(par), measure, nblocks(), s);
    }

    // Tensor maps of every block's field in both parities (box 40 × 10 × (P + 2), x from x0 − 4).
    pm_status build_maps() {
        const size_t G = grids.size();
        maps.assign(2 * G, CUtensorMap{});
        for (int par = 0; par < 2; ++par)
            for (size_t g = 0; g < G; ++g) {
                const EnsGrid& q = grids[g];
                if (!hall_tma_map(&maps[par * G + g], field[par].as<float>() + q.offset, q.pitch, q.ny, q.nz, 40, 10,
                                  kEnsTmaPlanes + 2))
                    return fail(PM_CUDA_ERROR, "cuTensorMapEncodeTiled refused an ensemble block");
            }
        PM_CUDA(dmaps.alloc(maps.size() * sizeof(CUtensorMap)));
        PM_CUDA(put_sync(dmaps.p, maps.data(), maps.size() * sizeof(CUtensorMap)));
        return PM_OK;
    }

    pm_status read_states() {
        PM_CUDA(cudaMemcpyAsync(states.data(), dstates.p, states.size() * sizeof(DevState), cudaMemcpyDeviceToHost, stream()));
        PM_CUDA(cudaStreamSynchronize(stream()));
        return PM_OK;
    }
    pm_status write_states() {
        PM_CUDA(cudaMemcpyAsync(dstates.p, states.data(), states.size() * sizeof(DevState), cudaMemcpyHostToDevice, stream()));
        PM_CUDA(cudaStreamSynchronize(stream()));
        return PM_OK;
    }

    // The opening ledger of every block's present state (books kept).
    pm_status measure() {
        PM_CUDA(launch(parity, true, stream()));
        return read_states();
    }

    pm_status run(long long n) {
        return run_steps(n, (double)generation, true, [this](int par, cudaStream_t st) { return launch(par, false, st); });
    }
};

}  // namespace pm

using namespace pm;

#define ENS_GUARD(e)                                              \
    do {                                                          \
        if (!(e)) return fail(PM_BAD_ARG, "null pm_ensemble");    \
        cudaSetDevice((e)->device);                               \
    } while (0)

extern "C" {

pm_status pm_ensemble_max_stable_dt(const pm_ensemble_grid* grids, int count, double* seconds) {
    if (!grids || !seconds || count < 0) return fail(PM_BAD_ARG, "null argument");
    for (int g = 0; g < count; ++g) {
        pm_ensemble_grid d = grids[g];
        d.dt = 1.0;  // not asked for here
        pm_status s = check_grid(d, g);
        if (s != PM_OK) return s;
        const double rate = uniform_block(d).rate;
        seconds[g] = std::isnan(rate) ? std::numeric_limits<double>::infinity() : 1.0 / rate;  // solid.rs:1709-1715
    }
    return PM_OK;
}

pm_status pm_ensemble_create(const pm_ensemble_grid* grids, int count, int precision, int device, pm_ensemble** out) {
    if (!grids || !out || count < 1) return fail(PM_BAD_ARG, "grids, a count of at least one, and out");
    *out = nullptr;
    if (precision != PM_PLAIN_F64 && precision != PM_FIELDS_F32) return fail(PM_BAD_ARG, "unknown precision");
    for (int g = 0; g < count; ++g) {
        pm_status s = check_grid(grids[g], g);
        if (s != PM_OK) return s;
    }
    Ensemble* e = new (std::nothrow) Ensemble();
    if (!e) return fail(PM_OUT_OF_MEMORY, "host allocation");
    e->name = "ensemble";
    e->precision = precision;
    e->desc.assign(grids, grids + count);
    e->grids.resize(count);
    e->blocks.resize(count);
    size_t offset = 0;
    for (int g = 0; g < count; ++g) {
        const pm_ensemble_grid& d = grids[g];
        const UniformBlock u = uniform_block(d);
        e->blocks[g] = u;
        EnsGrid& q = e->grids[g];
        std::memset(&q, 0, sizeof(q));
        q.nx = d.nx; q.ny = d.ny; q.nz = d.nz;
        q.pitch = precision == PM_PLAIN_F64 ? (d.nx + 1) & ~1 : (d.nx + 3) & ~3;
        q.offset = offset;
        offset += (size_t)q.pitch * d.ny * d.nz;
        q.exposed = d.convection_w_per_m2_k != 0.0 ? 0x3f : 0;
        q.kface = u.kface; q.mobility = u.mobility; q.capacity = u.capacity;
        q.k_cell = u.k_cell; q.eps_cell = d.substance.emissivity;
        q.dts = d.dt; q.dx = d.dx; q.reference = d.initial_kelvin;
        const double dm = d.dt * u.mobility;
        q.a = (float)(dm * u.kface);
        for (int f = 0; f < 6; ++f) {
            q.share[f] = u.share[f];
            q.ambient[f] = d.initial_kelvin;
            q.convection[f] = d.convection_w_per_m2_k;
            const double gf = q.exposed ? ens_series_with_half_cell(d.convection_w_per_m2_k * u.share[f], u.k_cell, u.share[f], d.dx) : 0.0;
            q.b[f] = (float)(dm * gf / d.dx);
            q.off[f] = 0.0f;  // the films' ambient is the block's own T0
            if (d.convection_w_per_m2_k == std::numeric_limits<double>::infinity())
                q.g_inf[f] = ens_series_with_half_cell(d.convection_w_per_m2_k, u.k_cell, u.share[f], d.dx);
        }
    }
    e->dcells = offset;
    e->ref_offset.resize(count);
    e->cells = 0;
    for (int g = 0; g < count; ++g) {
        e->ref_offset[g] = e->cells;
        e->cells += (size_t)grids[g].nx * grids[g].ny * grids[g].nz;
    }
    pm_status s = e->init(device, 0);
    if (s != PM_OK) { delete e; return s; }
    auto bail = [&](pm_status st) { delete e; return st; };
    for (auto& f : e->field) {
        cudaError_t ce = f.alloc(e->dcells * e->esize());
        if (ce == cudaSuccess) ce = cudaMemset(f.p, 0, e->dcells * e->esize());
        if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaMalloc ensemble field"));
    }
    cudaError_t ce = e->dgrids.alloc(count * sizeof(EnsGrid));
    if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaMalloc block table"));
    ce = e->dstates.alloc(count * sizeof(DevState));
    if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaMalloc block books"));
    e->states.assign(count, DevState{});
    for (auto& st : e->states) st.tol = e->tolerance;
    if ((s = e->write_states()) != PM_OK) return bail(s);
    // FP32 bricks 32 wide step with the TMA kernel when the driver tiles every block
    if (precision == PM_FIELDS_F32 && count <= (int)kEnsHoldBlocks) e->tma = e->build_maps() == PM_OK;
    if ((s = e->set_shape(0)) != PM_OK) return bail(s);
    // every block starts at its own T0 (Solid3D::new)
    std::vector<double> t(e->cells);
    for (int g = 0; g < count; ++g)
        std::fill(t.begin() + e->ref_offset[g], t.begin() + e->ref_offset[g] + (size_t)grids[g].nx * grids[g].ny * grids[g].nz,
                  grids[g].initial_kelvin);
    *out = reinterpret_cast<pm_ensemble*>(e);
    s = pm_ensemble_upload(*out, t.data(), t.size());
    if (s != PM_OK) { *out = nullptr; return bail(s); }
    return PM_OK;
}

pm_status pm_ensemble_upload(pm_ensemble* ep, const double* kelvin, size_t n) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    if (!kelvin || n != e->cells) return fail(PM_BAD_ARG, "upload: one value per cell of every block, in block order");
    e->parity = 0;
    if (e->precision == PM_PLAIN_F64) {
        // rows padded to an even length: the caller's dense blocks moved onto them, the padding zero
        if (e->stage.bytes < n * 8) PM_CUDA(e->stage.alloc(n * 8));
        PM_CUDA(cudaMemcpyAsync(e->stage.p, kelvin, n * 8, cudaMemcpyHostToDevice, e->stream()));
        for (int par = 0; par < 2; ++par) PM_CUDA(cudaMemsetAsync(e->field[par].p, 0, e->dcells * 8, e->stream()));
        for (size_t g = 0; g < e->grids.size(); ++g) {
            const EnsGrid& q = e->grids[g];
            PM_CUDA(launch_ens_relayout64(e->stage.as<double>() + e->ref_offset[g], e->field[0].as<double>() + q.offset,
                                          nullptr, q.nx, q.ny, q.nz, q.pitch, 1, e->stream()));
        }
    } else {
        if (e->stage.bytes < n * 8) PM_CUDA(e->stage.alloc(n * 8));
        PM_CUDA(cudaMemcpyAsync(e->stage.p, kelvin, n * 8, cudaMemcpyHostToDevice, e->stream()));
        for (size_t g = 0; g < e->grids.size(); ++g) {
            const EnsGrid& q = e->grids[g];
            PM_CUDA(launch_ens_relayout(e->stage.as<double>() + e->ref_offset[g], e->field[0].as<float>() + q.offset, nullptr,
                                        q.nx, q.ny, q.nz, q.pitch, q.reference, 1, e->stream()));
        }
    }
    // fresh books: nothing lost or supplied, no audit history
    for (auto& st : e->states) {
        std::memset(&st, 0, sizeof(st));
        st.tol = e->tolerance;
    }
    pm_status s = e->write_states();
    if (s != PM_OK) return s;
    return e->measure();
}

pm_status pm_ensemble_download(pm_ensemble* ep, double* kelvin, size_t n) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    if (!kelvin || n != e->cells) return fail(PM_BAD_ARG, "download: one value per cell of every block, in block order");
    if (e->precision == PM_PLAIN_F64) {
        if (e->stage.bytes < n * 8) PM_CUDA(e->stage.alloc(n * 8));
        for (size_t g = 0; g < e->grids.size(); ++g) {
            const EnsGrid& q = e->grids[g];
            PM_CUDA(launch_ens_relayout64(nullptr, e->field[e->parity].as<double>() + q.offset,
                                          e->stage.as<double>() + e->ref_offset[g], q.nx, q.ny, q.nz, q.pitch, 0,
                                          e->stream()));
        }
        PM_CUDA(cudaMemcpyAsync(kelvin, e->stage.p, n * 8, cudaMemcpyDeviceToHost, e->stream()));
    } else {
        if (e->stage.bytes < n * 8) PM_CUDA(e->stage.alloc(n * 8));
        for (size_t g = 0; g < e->grids.size(); ++g) {
            const EnsGrid& q = e->grids[g];
            PM_CUDA(launch_ens_relayout(nullptr, e->field[e->parity].as<float>() + q.offset,
                                        e->stage.as<double>() + e->ref_offset[g], q.nx, q.ny, q.nz, q.pitch, q.reference, 0,
                                        e->stream()));
        }
        PM_CUDA(cudaMemcpyAsync(kelvin, e->stage.p, n * 8, cudaMemcpyDeviceToHost, e->stream()));
    }
    PM_CUDA(cudaStreamSynchronize(e->stream()));
    return PM_OK;
}

pm_status pm_ensemble_set_tolerance(pm_ensemble* ep, double tol) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    e->tolerance = tol;
    return PM_OK;
}

pm_status pm_ensemble_step(pm_ensemble* ep, long long nsteps, pm_violation* out) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    if (nsteps < 0) return fail(PM_BAD_ARG, "nsteps must be >= 0");
    if (nsteps == 0) return PM_OK;
    // solid.rs:1718-1738 for each block: the stability refusal, before anything moves
    for (size_t g = 0; g < e->desc.size(); ++g) {
        const std::string site = "block " + std::to_string(g) + " (explicit 3D conduction)";
        const double ratio = e->desc[g].dt * e->blocks[g].rate;
        if (std::isnan(ratio)) {
            const double inf = std::numeric_limits<double>::infinity();
            fill_violation(out, "substance has no diffusivity", site, inf, inf, inf, 0.0, 1);
            set_error("substance has no diffusivity");
            return PM_VIOLATION;
        }
        if (ratio > 1.0 + 6e-12) {
            fill_violation(out, "Fourier number", site, kStableFourier3D, ratio * kStableFourier3D, kStableFourier3D, 1e-12, 1);
            set_error("Fourier number past the explicit limit in " + site);
            return PM_VIOLATION;
        }
    }
    // clear the previous call's violations, set the tolerance; books stay
    pm_status s = e->read_states();
    if (s != PM_OK) return s;
    std::vector<long long> before(e->states.size());
    for (size_t g = 0; g < e->states.size(); ++g) {
        DevState& st = e->states[g];
        st.violated = kRunning;
        st.violation_step = 0;
        st.tol = e->tolerance;
        st.counter = 0u;
        before[g] = st.steps;
    }
    if ((s = e->write_states()) != PM_OK) return s;
    if ((s = e->run(nsteps)) != PM_OK) return s;
    if ((s = e->read_states()) != PM_OK) return s;
    PM_CUDA(cudaGetLastError());
    for (size_t g = 0; g < e->states.size(); ++g) {
        const DevState& st = e->states[g];
        if (st.violated == kRunning) continue;
        const std::string site = "block " + std::to_string(g) + " (its own books, against what it moved on the bus)";
        fill_violation(out, "energy", site, st.v_before, st.v_after, st.v_scale, st.v_tol, st.violation_step - before[g]);
        set_error("conservation audit failed at " + site);
        return PM_VIOLATION;
    }
    return PM_OK;
}

pm_status pm_ensemble_ledgers(pm_ensemble* ep, pm_ledger* out, int count) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    if (!out || count != (int)e->states.size()) return fail(PM_BAD_ARG, "one pm_ledger per block");
    pm_status s = e->read_states();
    if (s != PM_OK) return s;
    for (int g = 0; g < count; ++g) {
        const DevState& st = e->states[g];
        std::memset(&out[g], 0, sizeof(pm_ledger));
        out[g].total = st.total;
        out[g].scale = st.scale;
        out[g].n_parts = 3;
        for (int q = 0; q < 3; ++q) out[g].parts[q] = st.part[q];
        out[g].steps = st.steps;
    }
    return PM_OK;
}

pm_status pm_ensemble_set_shape(pm_ensemble* ep, int brick_x, int planes) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    for (int q = 0; q < kEnsShapeCount; ++q)
        if (kEnsShapes[q].cells == 1 && kEnsShapes[q].x() == brick_x && kEnsShapes[q].zc == planes) return e->set_shape(q);
    return fail(PM_BAD_ARG, "brick shape: x extent 16, 32 or 64 and 8, 16, 32 or 64 planes");
}

pm_status pm_ensemble_set_brick(pm_ensemble* ep, int brick_x, int brick_y, int planes) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    for (int q = 0; q < kEnsShapeCount; ++q)
        if (kEnsShapes[q].x() == brick_x && kEnsShapes[q].y() == brick_y && kEnsShapes[q].zc == planes) return e->set_shape(q);
    return fail(PM_BAD_ARG, "brick: one of the listed shapes (x × y × planes)");
}

pm_status pm_ensemble_shape(pm_ensemble* ep, int* brick_x, int* brick_y, int* planes) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    const EnsShape s = kEnsShapes[e->shape];
    if (brick_x) *brick_x = s.x();
    if (brick_y) *brick_y = s.y();
    if (planes) *planes = s.zc;
    return PM_OK;
}

pm_status pm_ensemble_autotune(pm_ensemble* ep, int trial_steps, int* brick_x, int* planes) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    if (trial_steps < 1) return fail(PM_BAD_ARG, "trial_steps must be >= 1");
    // keep the present state and books; every trial runs on a copy of them and is undone
    const size_t bytes = e->dcells * e->esize();
    if (e->saved.bytes < bytes) PM_CUDA(e->saved.alloc(bytes));
    PM_CUDA(cudaMemcpyAsync(e->saved.p, e->field[e->parity].p, bytes, cudaMemcpyDeviceToDevice, e->stream()));
    pm_status s = e->read_states();
    if (s != PM_OK) return s;
    const std::vector<DevState> kept = e->states;
    const int kept_parity = e->parity;
    for (auto& st : e->states) { st.tol = -1.0; st.violated = kRunning; }
    if ((s = e->write_states()) != PM_OK) return s;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    PM_CUDA(cudaEventCreate(&t0));
    PM_CUDA(cudaEventCreate(&t1));
    int best = e->shape;
    float best_ms = std::numeric_limits<float>::infinity();
    pm_status result = PM_OK;
    for (int q = 0; q < kEnsShapeCount && result == PM_OK; ++q) {
        if (!ens_shape_fits(kEnsShapes[q], e->precision)) continue;  // quads are f32 only, pairs f64 only
        if ((result = e->set_shape(q)) != PM_OK) break;
        cudaError_t ce = cudaSuccess;
        for (int w = 0; w < 2 && ce == cudaSuccess; ++w) { ce = e->launch(e->parity, false, e->stream()); e->parity ^= 1; }
        if (ce == cudaSuccess) ce = cudaEventRecord(t0, e->stream());
        for (int w = 0; w < trial_steps && ce == cudaSuccess; ++w) { ce = e->launch(e->parity, false, e->stream()); e->parity ^= 1; }
        if (ce == cudaSuccess) ce = cudaEventRecord(t1, e->stream());
        if (ce == cudaSuccess) ce = cudaEventSynchronize(t1);
        float ms = 0.0f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, t0, t1);
        if (ce != cudaSuccess) { result = cuda_fail(ce, "autotune trial"); break; }
        if (ms < best_ms) { best_ms = ms; best = q; }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (result != PM_OK) return result;
    e->parity = kept_parity;
    PM_CUDA(cudaMemcpyAsync(e->field[e->parity].p, e->saved.p, bytes, cudaMemcpyDeviceToDevice, e->stream()));
    e->states = kept;
    if ((s = e->write_states()) != PM_OK) return s;
    if ((s = e->set_shape(best)) != PM_OK) return s;
    // the ledger's association follows the brick shape: re-take the present books in it
    std::vector<DevState> books = e->states;
    if ((s = e->measure()) != PM_OK) return s;
    for (size_t g = 0; g < books.size(); ++g) {
        e->states[g].steps = books[g].steps;
        e->states[g].tol = books[g].tol;
    }
    if ((s = e->write_states()) != PM_OK) return s;
    if (brick_x) *brick_x = kEnsShapes[best].x();
    if (planes) *planes = kEnsShapes[best].zc;
    return PM_OK;
}

pm_status pm_ensemble_set_stream(pm_ensemble* ep, void* stream) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    ENS_GUARD(e);
    PM_CUDA(cudaStreamSynchronize(e->stream()));
    e->user = static_cast<cudaStream_t>(stream);
    return PM_OK;
}

void pm_ensemble_destroy(pm_ensemble* ep) {
    Ensemble* e = reinterpret_cast<Ensemble*>(ep);
    if (!e) return;
    cudaSetDevice(e->device);
    delete e;
}

}  // extern "C"
