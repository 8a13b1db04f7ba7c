// pm_heat: the device form of `Solid3D` (crates/pantometry-thermal/src/solid.rs).
#include <algorithm>
#include <limits>
#include <new>

#include "runtime.h"

namespace pm {

namespace {

constexpr double kStableFourier3D = 1.0 / 6.0;  // solid.rs:84

double host_series_with_half_cell(double film, double conductivity, double area, double dx) {  // solid.rs:110-122
    if (film <= 0.0) return 0.0;
    double half = 2.0 * conductivity * area / dx;
    if (!std::isfinite(half)) return film;
    if (half <= 0.0) return 0.0;
    return 1.0 / (1.0 / film + 1.0 / half);
}

double rust_max(double a, double b) {  // f64::max
    if (std::isnan(a)) return b;
    if (std::isnan(b)) return a;
    return a > b ? a : b;
}

}  // namespace

struct Heat : Handle {
    int nx = 1, ny = 1, nz = 1;
    double dx = 0.0, reference = 0.0;
    std::vector<pm_substance> mats;
    std::vector<uint32_t> which;  // empty while the block is one material
    // solid.rs:238-266: void cells (empty while there are none), the watts each cell generates
    // (empty while nothing does) and the gap pairs across the void, in the order they were found
    std::vector<uint8_t> vd;
    std::vector<double> source;
    struct Gap { size_t a, b; double coefficient; };
    std::vector<Gap> gaps;
    HeatFilms films{};
    double film_conv[6] = {0, 0, 0, 0, 0, 0};
    // `resolve` products (solid.rs:588-784)
    bool uniform = true;
    double kface = 0.0, mobility = 0.0, capacity = 0.0;
    std::vector<double> kx, ky, kz, mob, cap;
    double worst_rate = 0.0;
    double cap_sum = 0.0;
    // device buffers
    DBuf field[2];  // f64 kelvin (plain) or f32 deviations
    DBuf dkx, dky, dkz, dmob, dcap, dwhich, dmatk, dmateps;
    DBuf dsrc, dvoid, dgap_of, dgaps;  // watts per cell (zero on void), void flags, the gap table
    // the FP32 form of a filled block: face conductivities and film conductances in f32, and
    // dt·mobility per cell for the step size m_dt
    DBuf dkx32, dky32, dkz32, dm32, dfilm32;
    size_t film_off[6] = {0, 0, 0, 0, 0, 0};
    double m_dt = NAN;
    // the wide forms, where the block is uniform and its rows allow: two cells of a row per thread
    // in the plain form (heat_plain_pair_step, even rows), four in the FP32 form
    // (heat_f32_quad_step, rows of a multiple of 4); false: one cell per thread throughout
    bool wide = true;
    bool quads64 = true;  // plain f64, rows of a multiple of 4: four cells a thread (else two)
    double pending = 0.0; // placeless heat handed in for the next step (pm_heat_absorb)
    DBuf saved;
    DBuf stage;     // f64 staging for uploads/downloads of the f32 form
    // the TMA-staged FP32 form of a uniform block whose rows hold a multiple of 4 cells: the tensor
    // maps of the two parities' deviations (heat_tma_step)
    CUtensorMap tmaps[2];
    bool tma_maps = false;
    // the persistent many-step path of small plain f64 blocks (heat_plain_pair_steps)
    DBuf dbarrier;
    unsigned wait_budget = 1u << 24;  // polls per grid-barrier wait, about 100 ns apart
    static constexpr size_t kPersistMaxCells = size_t(1) << 22;
    static constexpr int kPersistChunk = 1024;  // steps per cooperative launch
    double saved_lost = 0.0, saved_supplied = 0.0;

    size_t n() const { return (size_t)nx * ny * nz; }
    size_t esize() const { return precision == PM_PLAIN_F64 ? sizeof(double) : sizeof(float); }

    double mat_k(uint32_t m) const { return mats[m].thermal ? mats[m].conductivity : std::numeric_limits<double>::infinity(); }
    double mat_eps(uint32_t m) const { return mats[m].thermal ? mats[m].emissivity : 0.0; }
    uint32_t mat_of(size_t c) const { return which.empty() ? 0u : which[c]; }
    bool is_void(size_t c) const { return !vd.empty() && vd[c]; }

    // Per-cell (k, C) of a one-phase block (solid.rs:600-702 with φ = 0); nothing for void.
    void cell_props(size_t c, double& k, double& C) const {
        if (is_void(c)) { k = 0.0; C = 0.0; return; }
        const pm_substance& s = mats[mat_of(c)];
        const double volume = dx * dx * dx;
        const double ks = s.thermal ? s.conductivity : NAN;
        const double cs = s.thermal ? (s.density * volume) * s.specific_heat : NAN;
        const double phi = 0.0;
        k = ks + phi * (ks - ks);
        C = cs + phi * (cs - cs);
    }
    static double series(double a, double b) {
        double sum = a + b;
        return sum > 0.0 ? 2.0 * a * b / sum : 0.0;
    }

    // Face conductivities of a uniform block: zero on the outer faces, `kface` inside.
    double face_x(int i) const { return (i > 0 && i < nx) ? kface : 0.0; }
    double face_y(int j) const { return (j > 0 && j < ny) ? kface : 0.0; }
    double face_z(int k) const { return (k > 0 && k < nz) ? kface : 0.0; }

    double face_sum_at(int i, int j, int k) const {  // solid.rs:757-762
        if (uniform)
            return face_x(i) + face_x(i + 1) + face_y(j) + face_y(j + 1) + face_z(k) + face_z(k + 1);
        return kx[i + (size_t)(nx + 1) * (j + (size_t)ny * k)] + kx[i + 1 + (size_t)(nx + 1) * (j + (size_t)ny * k)] +
               ky[i + (size_t)nx * (j + (size_t)(ny + 1) * k)] + ky[i + (size_t)nx * (j + 1 + (size_t)(ny + 1) * k)] +
               kz[i + (size_t)nx * (j + (size_t)ny * k)] + kz[i + (size_t)nx * (j + (size_t)ny * (k + 1))];
    }
    double mob_at(size_t c) const { return uniform ? mobility : mob[c]; }

    // solid.rs:588-784 for a one-phase block; a block with void or a source is a filled one.
    void resolve() {
        uniform = mats.size() == 1 && vd.empty() && source.empty();
        gaps.clear();
        const size_t N = n();
        if (uniform) {
            double k, C;
            cell_props(0, k, C);
            kface = series(k, k);
            capacity = C;
            mobility = dx / C;
            kx.clear(); ky.clear(); kz.clear(); mob.clear(); cap.clear();
            cap_sum = -0.0;
            for (size_t c = 0; c < N; ++c) cap_sum += C;
            // The rate is the same within each class of cell (interior, face, edge, corner), so
            // sampling i, j, k at 0, 1, n-2, n-1 visits every distinct value.
            worst_rate = 0.0;
            bool nowhere = false;
            for (int k3 : {0, 1, nz - 2, nz - 1}) {
                if (k3 < 0 || k3 >= nz) continue;
                for (int j3 : {0, 1, ny - 2, ny - 1}) {
                    if (j3 < 0 || j3 >= ny) continue;
                    for (int i3 : {0, 1, nx - 2, nx - 1}) {
                        if (i3 < 0 || i3 >= nx) continue;
                        double rate = mobility * face_sum_at(i3, j3, k3);
                        if (std::isnan(rate)) nowhere = true;
                        else worst_rate = rust_max(worst_rate, rate);
                    }
                }
            }
            if (nowhere) worst_rate = NAN;
            return;
        }
        std::vector<double> km(N), cm(N);
        for (size_t c = 0; c < N; ++c) cell_props(c, km[c], cm[c]);
        kx.assign((size_t)(nx + 1) * ny * nz, 0.0);
        ky.assign((size_t)nx * (ny + 1) * nz, 0.0);
        kz.assign((size_t)nx * ny * (nz + 1), 0.0);
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    size_t c = i + (size_t)nx * (j + (size_t)ny * k);
                    if (i > 0) kx[i + (size_t)(nx + 1) * (j + (size_t)ny * k)] = series(km[c - 1], km[c]);
                    if (j > 0) ky[i + (size_t)nx * (j + (size_t)(ny + 1) * k)] = series(km[c - nx], km[c]);
                    if (k > 0) kz[i + (size_t)nx * (j + (size_t)ny * k)] = series(km[c - (size_t)nx * ny], km[c]);
                }
        cap.assign(N, 0.0);
        mob.assign(N, 0.0);
        worst_rate = 0.0;
        cap_sum = -0.0;
        bool nowhere = false;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    size_t c = i + (size_t)nx * (j + (size_t)ny * k);
                    cap[c] = cm[c];
                    mob[c] = is_void(c) ? 0.0 : dx / cm[c];  // solid.rs:753-756
                    cap_sum += cm[c];
                    double rate = mob[c] * face_sum_at(i, j, k);
                    if (std::isnan(rate)) nowhere = true;
                    else worst_rate = rust_max(worst_rate, rate);
                }
        if (nowhere) worst_rate = NAN;
        find_gaps();
    }

    // solid.rs:786-838 `find_gaps`: along every row, then every column, then every pillar, a run
    // of void with solid at both ends pairs its two end cells, with the parallel-plate series.
    void find_gaps() {
        gaps.clear();
        if (vd.empty()) return;
        const double area = dx * dx;
        auto walk = [&](size_t first, size_t stride, int len) {
            bool have_last = false, void_between = false;
            size_t last = 0;
            for (int q = 0; q < len; ++q) {
                const size_t c = first + stride * (size_t)q;
                if (vd[c]) { void_between = have_last; continue; }
                if (have_last && void_between) {
                    const double ea = mat_eps(mat_of(last)), eb = mat_eps(mat_of(c));
                    if (ea > 0.0 && eb > 0.0) {
                        const double resistance = 1.0 / ea + 1.0 / eb - 1.0;
                        if (resistance > 0.0) gaps.push_back(Gap{last, c, kStefanBoltzmann * area / resistance});
                    }
                }
                last = c;
                have_last = true;
                void_between = false;
            }
        };
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j) walk((size_t)nx * (j + (size_t)ny * k), 1, nx);
        for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nx; ++i) walk(i + (size_t)nx * ny * k, (size_t)nx, ny);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) walk(i + (size_t)nx * j, (size_t)nx * ny, nz);
    }

    // Radiating films: the step limit follows the state (solid.rs:1148-1185).
    bool radiating() const { return films.exposed && any_radiative_film(); }
    // Radiating films or radiative gaps: the limit follows the state.
    bool state_dependent() const { return radiating() || !gaps.empty(); }

    // solid.rs:1269-1288 `loss_conductance_at` at temperature `at`, summed from −0.0 (Rust's
    // `Sum for f64`), radiating term included.
    double loss_conductance_at(double at, int i, int j, int k, size_t c) const {
        double total = -0.0;
        const double eps = mat_eps(mat_of(c));
        for (int f = 0; f < 6; ++f) {
            if (!((films.exposed >> f) & 1)) continue;
            bool holds = f == 0 ? i == 0 : f == 1 ? i + 1 == nx : f == 2 ? j == 0 : f == 3 ? j + 1 == ny : f == 4 ? k == 0 : k + 1 == nz;
            if (!holds) continue;
            const double share = films.share[f];
            const double hot = rust_max(at, films.ambient[f]);
            const double h = film_conv[f] + 4.0 * eps * kStefanBoltzmann * (hot * (hot * hot));  // powi(3)
            total += host_series_with_half_cell(h * share, mat_k(mat_of(c)), share, dx);
        }
        return total;
    }
    // solid.rs:1148-1185 over a state `t` (kelvin, reference order); a void cell's temperature is
    // not a number (solid.rs:1324-1335).
    double worst_rate_of(const std::vector<double>& t) const {
        if ((films.exposed == 0 && gaps.empty()) || std::isnan(worst_rate)) return worst_rate;
        double worst = worst_rate;
        for (const Gap& g : gaps) {
            const double hotter = rust_max(t[g.a], t[g.b]);
            const double cond = 4.0 * g.coefficient * (hotter * (hotter * hotter));  // powi(3)
            for (size_t c : {g.a, g.b})
                if (cap[c] > 0.0) worst = rust_max(worst, cond / cap[c]);
        }
        if (films.exposed == 0) return worst;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    if (!(i == 0 || i + 1 == nx || j == 0 || j + 1 == ny || k == 0 || k + 1 == nz)) continue;
                    const size_t c = i + (size_t)nx * (j + (size_t)ny * k);
                    const double loss = loss_conductance_at(is_void(c) ? NAN : t[c], i, j, k, c);
                    if (loss == 0.0) continue;
                    worst = rust_max(worst, mob_at(c) * (face_sum_at(i, j, k) + loss / dx));
                }
        return worst;
    }
    // The rate of the present state into the device books, where the films radiate: the step
    // kernels keep it from then on, step by step.
    pm_status refresh_rate() {
        if (!state_dependent() || (precision != PM_PLAIN_F64 && !radiating_f32())) return PM_OK;
        std::vector<double> t(n());
        if (precision == PM_PLAIN_F64) {
            PM_CUDA(cudaMemcpyAsync(t.data(), field[parity].p, n() * 8, cudaMemcpyDeviceToHost, stream()));
        } else {  // the kelvin the FP32 deviations hold
            if (!stage.p || stage.bytes < n() * 8) PM_CUDA(stage.alloc(n() * 8));
            PM_CUDA(launch_heat_convert(nullptr, field[parity].as<float>(), reference, n(), 0, stage.as<double>(), stream()));
            PM_CUDA(cudaMemcpyAsync(t.data(), stage.p, n() * 8, cudaMemcpyDeviceToHost, stream()));
        }
        PM_CUDA(cudaStreamSynchronize(stream()));
        pm_status s = read_state();
        if (s != PM_OK) return s;
        host_state->rate_now = worst_rate_of(t);
        host_state->rate_bits = 0ull;
        return write_state();
    }

    bool any_radiative_film() const {
        for (int f = 0; f < 6; ++f)
            if (((films.exposed >> f) & 1)) {
                for (uint32_t m = 0; m < mats.size(); ++m)
                    if (mat_eps(m) != 0.0) return true;
            }
        return false;
    }

    size_t cells_on(int f) const {  // solid.rs:1222-1229
        return f < 2 ? (size_t)ny * nz : (f < 4 ? (size_t)nx * nz : (size_t)nx * ny);
    }

    // solid.rs:1269-1288 at a temperature-independent film (emissivity zero).
    double loss_at(int i, int j, int k, size_t c) const {
        double total = -0.0;
        for (int f = 0; f < 6; ++f) {
            if (!((films.exposed >> f) & 1)) continue;
            bool holds = f == 0 ? i == 0 : f == 1 ? i + 1 == nx : f == 2 ? j == 0 : f == 3 ? j + 1 == ny : f == 4 ? k == 0 : k + 1 == nz;
            if (!holds) continue;
            double share = films.share[f];
            // h + 4εσ·max(T, T∞)³ with ε = 0 (radiating films are refused before this runs)
            double h = film_conv[f];
            total += host_series_with_half_cell(h * share, mat_k(mat_of(c)), share, dx);
        }
        return total;
    }

    // solid.rs:1148-1185
    double worst_rate_now() const {
        if (films.exposed == 0 || std::isnan(worst_rate)) return worst_rate;
        double worst = worst_rate;
        auto visit = [&](int i, int j, int k) {
            size_t c = i + (size_t)nx * (j + (size_t)ny * k);
            double loss = loss_at(i, j, k, c);
            if (loss == 0.0) return;
            worst = rust_max(worst, mob_at(c) * (face_sum_at(i, j, k) + loss / dx));
        };
        if (uniform) {
            for (int k3 : {0, 1, nz - 2, nz - 1}) {
                if (k3 < 0 || k3 >= nz) continue;
                for (int j3 : {0, 1, ny - 2, ny - 1}) {
                    if (j3 < 0 || j3 >= ny) continue;
                    for (int i3 : {0, 1, nx - 2, nx - 1})
                        if (i3 >= 0 && i3 < nx) visit(i3, j3, k3);
                }
            }
        } else {
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i)
                        if (i == 0 || i + 1 == nx || j == 0 || j + 1 == ny || k == 0 || k + 1 == nz) visit(i, j, k);
        }
        return worst;
    }

    pm_status put_buf(DBuf& b, const void* src, size_t bytes) {
        PM_CUDA(b.alloc(bytes));
        PM_CUDA(put_sync(b.p, src, bytes));
        return PM_OK;
    }

    // A filled block in the FP32 form: the face conductivities rounded to f32, the capacities in
    // f64 for the stored heat, the film conductances; dt·mobility follows with the step size.
    pm_status upload_coefficients_f32() {
        auto put32 = [&](DBuf& b, const std::vector<double>& v) -> pm_status {
            std::vector<float> f(v.size());
            for (size_t q = 0; q < v.size(); ++q) f[q] = (float)v[q];
            return put_buf(b, f.data(), f.size() * 4);
        };
        pm_status s;
        if ((s = put32(dkx32, kx)) != PM_OK) return s;
        if ((s = put32(dky32, ky)) != PM_OK) return s;
        if ((s = put32(dkz32, kz)) != PM_OK) return s;
        if ((s = put_buf(dcap, cap.data(), cap.size() * 8)) != PM_OK) return s;
        if ((s = upload_places()) != PM_OK) return s;
        m_dt = NAN;
        return upload_films_f32();
    }

    // Per exposed face, each cell's film conductance g/dx with the half cell of its own material
    // in series (solid.rs:1192-1219 at zero emissivity, where g does not depend on the gap).
    pm_status upload_films_f32() {
        if (uniform || precision == PM_PLAIN_F64) return PM_OK;
        drop_graphs();
        std::vector<float> v;
        for (int f = 0; f < 6; ++f) {
            film_off[f] = v.size();
            if (!((films.exposed >> f) & 1)) continue;
            const double share = films.share[f];
            const int a1 = f < 2 ? ny : nx, a2 = f < 4 ? nz : ny;  // the plane's two extents
            for (int q2 = 0; q2 < a2; ++q2)
                for (int q1 = 0; q1 < a1; ++q1) {
                    int i, j, k;
                    if (f < 2) { i = f == 0 ? 0 : nx - 1; j = q1; k = q2; }
                    else if (f < 4) { i = q1; j = f == 2 ? 0 : ny - 1; k = q2; }
                    else { i = q1; j = q2; k = f == 4 ? 0 : nz - 1; }
                    const size_t c = i + (size_t)nx * (j + (size_t)ny * k);
                    const double g = host_series_with_half_cell(film_conv[f] * share, mat_k(mat_of(c)), share, dx);
                    v.push_back((float)(g / dx));
                }
        }
        if (v.empty()) v.push_back(0.0f);
        return put_buf(dfilm32, v.data(), v.size() * 4);
    }

    // dt·mobility per cell for step size dt, once per change of dt or of the block.
    pm_status prepare_f32(double dt) {
        if (uniform || precision == PM_PLAIN_F64 || m_dt == dt) return PM_OK;
        std::vector<float> m(n());
        for (size_t c = 0; c < n(); ++c) m[c] = (float)(dt * mob[c]);
        if (!dm32.p || dm32.bytes < n() * 4) PM_CUDA(dm32.alloc(n() * 4));
        PM_CUDA(put_sync(dm32.p, m.data(), n() * 4));
        m_dt = dt;
        return PM_OK;
    }

    pm_status upload_coefficients() {
        drop_graphs();
        if (uniform) return PM_OK;
        if (precision != PM_PLAIN_F64) return upload_coefficients_f32();
        auto put = [&](DBuf& b, const void* src, size_t bytes) -> pm_status { return put_buf(b, src, bytes); };
        pm_status s;
        if ((s = put(dkx, kx.data(), kx.size() * 8)) != PM_OK) return s;
        if ((s = put(dky, ky.data(), ky.size() * 8)) != PM_OK) return s;
        if ((s = put(dkz, kz.data(), kz.size() * 8)) != PM_OK) return s;
        if ((s = put(dmob, mob.data(), mob.size() * 8)) != PM_OK) return s;
        if ((s = put(dcap, cap.data(), cap.size() * 8)) != PM_OK) return s;
        std::vector<uint32_t> w(n(), 0u);
        for (size_t c = 0; c < n(); ++c) w[c] = mat_of(c);
        if ((s = put(dwhich, w.data(), w.size() * 4)) != PM_OK) return s;
        std::vector<double> mk(mats.size()), me(mats.size());
        for (uint32_t m = 0; m < mats.size(); ++m) { mk[m] = mat_k(m); me[m] = mat_eps(m); }
        if ((s = put(dmatk, mk.data(), mk.size() * 8)) != PM_OK) return s;
        if ((s = put(dmateps, me.data(), me.size() * 8)) != PM_OK) return s;
        if ((s = upload_places()) != PM_OK) return s;
        // The gap table: per cell its entries in the pairs' order, which is the order the step adds
        // them (solid.rs:1866-1878 walks the pairs; each touches two cells).
        if (!gaps.empty()) {
            std::vector<std::vector<std::pair<size_t, int>>> per(n());  // (pair, this cell is its first)
            for (size_t q = 0; q < gaps.size(); ++q) {
                per[gaps[q].a].push_back({q, 1});
                per[gaps[q].b].push_back({q, 0});
            }
            std::vector<int> first(n(), -1);
            std::vector<HeatGapEntry> table;
            for (size_t c = 0; c < n(); ++c) {
                if (per[c].empty()) continue;
                first[c] = (int)table.size();
                for (size_t e = 0; e < per[c].size(); ++e) {
                    const Gap& g = gaps[per[c][e].first];
                    const int lower = per[c][e].second;
                    table.push_back(HeatGapEntry{(long long)(lower ? g.b : g.a), g.coefficient, lower,
                                                 e + 1 == per[c].size() ? 1 : 0});
                }
            }
            if ((s = put(dgap_of, first.data(), first.size() * 4)) != PM_OK) return s;
            if ((s = put(dgaps, table.data(), table.size() * sizeof(HeatGapEntry))) != PM_OK) return s;
        }
        return PM_OK;
    }

    // The sources (zeroed on void, where the step skips them: solid.rs:1857) and the void flags.
    pm_status upload_places() {
        pm_status s;
        if (!source.empty()) {
            std::vector<double> w(source);
            for (size_t c = 0; c < n(); ++c)
                if (is_void(c)) w[c] = 0.0;
            if ((s = put_buf(dsrc, w.data(), w.size() * 8)) != PM_OK) return s;
        }
        if (!vd.empty() && (s = put_buf(dvoid, vd.data(), vd.size())) != PM_OK) return s;
        return PM_OK;
    }

    HeatPlainArgs plain_args(int par, double dt) const {
        HeatPlainArgs a{};
        a.told = field[par].as<double>();
        a.tnew = field[par ^ 1].as<double>();
        a.uniform = uniform ? 1 : 0;
        if (!uniform) {
            a.kx = dkx.as<double>(); a.ky = dky.as<double>(); a.kz = dkz.as<double>();
            a.mob = dmob.as<double>(); a.cap = dcap.as<double>();
            a.which = dwhich.as<uint32_t>(); a.mat_k = dmatk.as<double>(); a.mat_eps = dmateps.as<double>();
            a.src = source.empty() ? nullptr : dsrc.as<double>();
            if (!gaps.empty()) { a.gap_of = dgap_of.as<int>(); a.gaps = dgaps.as<HeatGapEntry>(); }
        }
        a.kface = kface; a.mobility = mobility; a.capacity = capacity;
        a.k_cell = mat_k(0); a.eps_cell = mat_eps(0);
        a.nx = nx; a.ny = ny; a.nz = nz;
        a.dts = dt; a.dx = dx; a.reference = reference;
        a.films = films;
        a.films.dirichlet = 0;
        if (uniform) {  // solid.rs:1192-1219 at h = +inf: the film's series with the half cell, per face
            for (int f = 0; f < 6; ++f) {
                if (!((films.exposed >> f) & 1) || !(films.convection[f] == std::numeric_limits<double>::infinity())) continue;
                a.films.dirichlet |= 1 << f;
                a.films.g_inf[f] = host_series_with_half_cell(std::numeric_limits<double>::infinity(), mat_k(0),
                                                              films.share[f], dx);
            }
        }
        a.quads = uniform && nx % 4 == 0 && wide && quads64 ? 1 : 0;
        a.pairs = !a.quads && uniform && nx % 2 == 0 && wide ? 1 : 0;
        a.radiating = state_dependent() ? 1 : 0;
        a.static_rate = worst_rate;
        const unsigned w = wave_of(a.quads ? kHeatPlainQuad : a.pairs ? kHeatPlainPair : kHeatPlain);
        const int tx = a.quads ? nx / 4 : a.pairs ? nx / 2 : nx;  // the threads along a row
        a.tiles = make_tiles(tx, ny, nz, choose_zc(tx, ny, nz, w));
        a.nblocks = grid_for(a.tiles, w);
        a.st = state.as<DevState>();
        a.partials = partials.as<double>();
        return a;
    }

    bool tma_form() const {
        return precision == PM_FIELDS_F32 && uniform && wide && nx % 4 == 0 && tma_maps && !state_dependent();
    }
    // FP32 blocks of one material whose films radiate and that leave no gaps: the one-cell FP32
    // kernel, its limit following the state as the plain form's does
    bool radiating_f32() const { return precision == PM_FIELDS_F32 && uniform && gaps.empty() && radiating(); }

    HeatTmaArgs tma_args(int par, double dt) const {
        const HeatF32Args f = f32_args(par, dt);
        HeatTmaArgs a{};
        a.dnew = field[par ^ 1].as<float>();
        a.nx = nx; a.ny = ny; a.nz = nz;
        a.ntx = (unsigned)((nx + 31) / 32);
        a.nty = (unsigned)((ny + 7) / 8);
        a.ntz = (unsigned)((nz + kEnsTmaPlanes - 1) / kEnsTmaPlanes);
        a.cell.nx = nx; a.cell.ny = ny; a.cell.nz = nz; a.cell.pitch = nx;
        a.cell.exposed = f.exposed;
        a.cell.a = f.a;
        for (int q = 0; q < 6; ++q) { a.cell.b[q] = f.b[q]; a.cell.off[q] = f.off[q]; }
        a.capacity = capacity;
        a.st = state.as<DevState>();
        a.partials = partials.as<double>();
        const unsigned long long items = (unsigned long long)a.ntx * a.nty * a.ntz;
        a.nblocks = (unsigned)std::min<unsigned long long>(items, wave_of(kHeatTma));
        return a;
    }

    HeatF32Args f32_args(int par, double dt) const {
        HeatF32Args a{};
        a.dold = field[par].as<float>();
        a.dnew = field[par ^ 1].as<float>();
        a.nx = nx; a.ny = ny; a.nz = nz;
        const double dm = dt * mobility;
        a.a = (float)(dm * kface);
        a.exposed = films.exposed;
        for (int f = 0; f < 6; ++f) {
            double g = 0.0;
            if ((films.exposed >> f) & 1) {
                // The film's conductance with the half cell in series (solid.rs:1192-1219) at zero
                // emissivity, which does not depend on the temperature difference.
                g = host_series_with_half_cell(film_conv[f] * films.share[f], mat_k(0), films.share[f], dx);
            }
            a.b[f] = (float)(dm * g / dx);
            a.off[f] = (float)(reference - films.ambient[f]);
        }
        a.capacity = capacity;
        if (!uniform) {
            a.kx = dkx32.as<float>(); a.ky = dky32.as<float>(); a.kz = dkz32.as<float>();
            a.m = dm32.as<float>(); a.cap = dcap.as<double>();
            for (int f = 0; f < 6; ++f) a.film[f] = dfilm32.as<float>() + film_off[f];
            a.src = source.empty() ? nullptr : dsrc.as<double>();
        }
        a.dts = dt;
        a.quads = uniform && nx % 4 == 0 && wide && !state_dependent() ? 1 : 0;
        if (radiating_f32()) {  // the one-cell kernel, its face cells through the plain form's films
            a.radiating = 1;
            a.t0 = reference;
            a.rad = plain_args(par, dt);
        }
        const unsigned w = wave_of(a.quads ? kHeatF32Quad : kHeatF32);
        const int tx = a.quads ? nx / 4 : nx;  // the threads along a row
        a.tiles = make_tiles(tx, ny, nz, choose_zc(tx, ny, nz, w));
        a.nblocks = grid_for(a.tiles, w);
        a.st = state.as<DevState>();
        a.partials = partials.as<double>();
        return a;
    }

    // Small uniform plain f64 blocks in the pair form, films that do not radiate, more than one
    // step: every step of a launch-bound block in one cooperative launch per kPersistChunk steps.
    bool persistent(long long nsteps) const {
        const int width = precision == PM_PLAIN_F64 ? 2 : 4;  // the pair and the quad forms
        if (!uniform || !wide || nx % width != 0 || state_dependent() || nsteps < 2) return false;
        if (n() > kPersistMaxCells) return false;
        int coop = 0;
        return cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) == cudaSuccess && coop;
    }
    pm_status run_persistent(long long nsteps, double dt) {
        const size_t wait_bytes = kWaitWords * sizeof(unsigned);
        if (!dbarrier.p) PM_CUDA(dbarrier.alloc(wait_bytes));
        const bool plain = precision == PM_PLAIN_F64;
        // Blocks of 1024 threads (tiles of 32 rows) where the block has the rows for them, so that
        // fewer blocks meet at each step's wait; a grid of co-resident blocks, one of them keeping the
        // books, and tiles made as small as the others take.
        const int rows = ny >= 32 ? 32 : 8;
        const unsigned wave = wave_of(plain ? (rows == 32 ? kHeatPlainSteps32 : kHeatPlainSteps)
                                            : (rows == 32 ? kHeatF32QuadSteps32 : kHeatF32QuadSteps));
        if (wave < 2) return fail(PM_UNSUPPORTED, "the many-step heat kernel needs two co-resident blocks");
        const int tx = nx / (plain ? 2 : 4);
        int zc = 1;
        while (zc < nz && make_tiles(tx, ny, nz, zc, rows).ntiles > (long long)(wave - 1)) zc *= 2;
        const Tiles tiles = make_tiles(tx, ny, nz, zc, rows);
        const unsigned nblocks = 1u + (unsigned)std::min<long long>(tiles.ntiles, (long long)(wave - 1));
        int par = parity;
        for (long long done = 0; done < nsteps;) {
            const int chunk = (int)std::min<long long>(kPersistChunk, nsteps - done);
            PM_CUDA(cudaMemsetAsync(dbarrier.p, 0, wait_bytes, stream()));
            const HeatPersist p{dbarrier.as<unsigned>(), chunk, wait_budget};
            if (plain) {
                HeatPlainArgs a = plain_args(par, dt);
                a.tiles = tiles;
                a.nblocks = nblocks;
                PM_CUDA(launch_heat_plain_steps(a, p, stream()));
            } else {
                HeatF32Args a = f32_args(par, dt);
                a.tiles = tiles;
                a.nblocks = nblocks;
                PM_CUDA(launch_heat_f32_steps(a, p, stream()));
            }
            par ^= chunk & 1;
            done += chunk;
        }
        return PM_OK;
    }

    // solid.rs:1752-1765: the first step of a call takes the placeless heat handed in since the last
    // one, after its stability refusal, as a uniform rise over the solid cells. It is bus traffic,
    // not a change of the domain's own books, so the stored heat is re-measured and lost and
    // supplied kept; and since the refusal was made against the state before the rise, the rate
    // that state gave stays the one the step's own check reads.
    pm_status take_pending() {
        const double joules = pending;
        if (joules == 0.0) return PM_OK;
        pending = 0.0;
        const double rise = joules / cap_sum;  // solid.rs:1755
        PM_CUDA(launch_heat_rise(precision == PM_PLAIN_F64 ? field[parity].as<double>() : nullptr,
                                 precision == PM_PLAIN_F64 ? nullptr : field[parity].as<float>(), rise, n(),
                                 vd.empty() ? nullptr : dvoid.as<uint8_t>(), stream()));
        pm_status s = read_state();
        if (s != PM_OK) return s;
        const double lost = host_state->lost, supplied = host_state->supplied, rate = host_state->rate_now;
        s = measure();
        if (s != PM_OK) return s;
        host_state->lost = lost;
        host_state->supplied = supplied;
        host_state->rate_now = rate;
        return write_state();
    }

    pm_status measure() {  // the opening ledger of the present state
        HeatMeasureArgs m{};
        if (precision == PM_PLAIN_F64) m.t64 = field[parity].as<double>();
        else m.d32 = field[parity].as<float>();
        m.cap = uniform ? nullptr : dcap.as<double>();
        m.capacity = capacity;
        m.reference = reference;
        m.n = n();
        m.st = state.as<DevState>();
        m.partials = partials.as<double>();
        m.nblocks = kMeasureBlocks;
        PM_CUDA(precision == PM_PLAIN_F64 ? launch_heat_measure_plain(m, stream()) : launch_heat_measure_f32(m, stream()));
        pm_status s = read_state();
        if (s != PM_OK) return s;
        return refresh_rate();
    }
};

}  // namespace pm

using namespace pm;

#define HEAT_GUARD(h)                                          \
    do {                                                       \
        if (!(h)) return fail(PM_BAD_ARG, "null pm_heat");      \
        cudaSetDevice((h)->device);                            \
    } while (0)

extern "C" {

pm_status pm_heat_create(const pm_heat_desc* d, pm_heat** out) {
    if (!d || !out) return fail(PM_BAD_ARG, "null argument");
    *out = nullptr;
    if (d->precision != PM_PLAIN_F64 && d->precision != PM_FIELDS_F32) return fail(PM_BAD_ARG, "unknown precision");
    if (!(d->dx > 0.0)) return fail(PM_BAD_ARG, "dx must be positive");
    Heat* h = new (std::nothrow) Heat();
    if (!h) return fail(PM_OUT_OF_MEMORY, "host allocation");
    h->name = d->name ? d->name : "block";
    h->refusal_site = h->name + " (explicit 3D conduction)";
    h->nx = std::max(d->nx, 1); h->ny = std::max(d->ny, 1); h->nz = std::max(d->nz, 1);
    h->dx = d->dx;
    h->reference = d->initial_kelvin;
    h->precision = d->precision;
    h->mats.push_back(d->substance);
    h->resolve();
    pm_status s = h->init(d->device, 0);
    if (s != PM_OK) { delete h; return s; }
    for (auto& f : h->field) {
        cudaError_t e = f.alloc(h->n() * h->esize());
        if (e != cudaSuccess) { delete h; return cuda_fail(e, "cudaMalloc field"); }
    }
    // TMA maps of the FP32 deviations, where the rows hold a multiple of 4 cells (16-byte rows)
    if (h->precision == PM_FIELDS_F32 && h->nx % 4 == 0 && (size_t)h->nx * h->ny * h->nz < (size_t(1) << 31))
        h->tma_maps = heat_tma_map(&h->tmaps[0], h->field[0].p, h->nx, h->ny, h->nz) &&
                      heat_tma_map(&h->tmaps[1], h->field[1].p, h->nx, h->ny, h->nz);

    // Solid3D::new starts every cell at `initial`.
    std::vector<double> t(h->n(), d->initial_kelvin);
    *out = reinterpret_cast<pm_heat*>(h);
    s = pm_heat_upload(*out, t.data(), t.size());
    if (s != PM_OK) { delete h; *out = nullptr; return s; }
    return PM_OK;
}

pm_status pm_heat_fill(pm_heat* hp, const pm_substance* sub, const uint8_t* mask, size_t n) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!sub || !mask || n != h->n()) return fail(PM_BAD_ARG, "fill: substance, mask and a mask of one byte per cell");
    // solid.rs:524-530: reuse an equal substance, else append
    int id = -1;
    for (size_t q = 0; q < h->mats.size(); ++q) {
        const pm_substance& o = h->mats[q];
        if (o.density == sub->density && o.conductivity == sub->conductivity && o.specific_heat == sub->specific_heat &&
            o.emissivity == sub->emissivity && o.thermal == sub->thermal) { id = (int)q; break; }
    }
    if (id < 0) { h->mats.push_back(*sub); id = (int)h->mats.size() - 1; }
    if (h->which.empty()) h->which.assign(h->n(), 0u);
    for (size_t c = 0; c < n; ++c)
        if (mask[c]) h->which[c] = (uint32_t)id;
    h->resolve();
    pm_status s = h->upload_coefficients();
    if (s != PM_OK) return s;
    return h->measure();
}

pm_status pm_heat_empty(pm_heat* hp, const uint8_t* mask, size_t n) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!mask || n != h->n()) return fail(PM_BAD_ARG, "empty: a mask of one byte per cell");
    // solid.rs:986-1005: the cells the mask selects become nothing
    if (h->vd.empty()) h->vd.assign(h->n(), 0);
    for (size_t c = 0; c < n; ++c)
        if (mask[c]) h->vd[c] = 1;
    h->resolve();
    pm_status s = h->upload_coefficients();
    if (s != PM_OK) return s;
    return h->measure();
}

pm_status pm_heat_dissipating(pm_heat* hp, double watts, const uint8_t* mask, size_t n) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!mask || n != h->n()) return fail(PM_BAD_ARG, "dissipating: a mask of one byte per cell");
    // solid.rs:1045-1085: the watts spread evenly over the solid cells selected; none selected
    // generates nothing and is not an error
    size_t chosen = 0;
    for (size_t c = 0; c < n; ++c)
        if (!h->is_void(c) && mask[c]) ++chosen;
    if (chosen == 0) return PM_OK;
    const double each = watts / (double)chosen;
    if (h->source.empty()) h->source.assign(h->n(), 0.0);
    for (size_t c = 0; c < n; ++c)
        if (!h->is_void(c) && mask[c]) h->source[c] = each;
    h->resolve();
    pm_status s = h->upload_coefficients();
    if (s != PM_OK) return s;
    return h->measure();
}

pm_status pm_heat_generated(pm_heat* hp, double* watts, double* joules) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (watts) {  // solid.rs:1118-1121: summed over the cells
        double sum = -0.0;
        for (double w : h->source) sum += w;
        *watts = sum;
    }
    if (joules) {  // solid.rs:1123-1126: what the steps generated
        pm_status s = h->read_state();
        if (s != PM_OK) return s;
        *joules = h->host_state->supplied;
    }
    return PM_OK;
}

pm_status pm_heat_gaps(pm_heat* hp, long long* a, long long* b, double* coefficient, size_t capacity, size_t* count) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!count) return fail(PM_BAD_ARG, "null count");
    *count = h->gaps.size();
    for (size_t q = 0; q < h->gaps.size() && q < capacity; ++q) {
        if (a) a[q] = (long long)h->gaps[q].a;
        if (b) b[q] = (long long)h->gaps[q].b;
        if (coefficient) coefficient[q] = h->gaps[q].coefficient;
    }
    return PM_OK;
}

pm_status pm_heat_losing_from(pm_heat* hp, int face, double ambient, double convection, double area) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (face < 0 || face > 5) return fail(PM_BAD_ARG, "face must be 0..5");
    h->films.exposed |= 1 << face;
    h->films.ambient[face] = ambient;
    h->films.convection[face] = convection;
    h->film_conv[face] = convection;
    h->films.share[face] = area / (double)std::max<size_t>(h->cells_on(face), 1);  // solid.rs:1203
    h->resolve();
    h->drop_graphs();
    pm_status s = h->upload_films_f32();
    if (s != PM_OK) return s;
    return h->refresh_rate();
}

pm_status pm_heat_upload(pm_heat* hp, const double* kelvin, size_t n) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!kelvin || n != h->n()) return fail(PM_BAD_ARG, "upload: one value per cell");
    h->parity = 0;
    if (h->precision == PM_PLAIN_F64) {
        PM_CUDA(cudaMemcpyAsync(h->field[0].p, kelvin, n * 8, cudaMemcpyHostToDevice, h->stream()));
    } else {
        if (!h->stage.p || h->stage.bytes < n * 8) PM_CUDA(h->stage.alloc(n * 8));
        PM_CUDA(cudaMemcpyAsync(h->stage.p, kelvin, n * 8, cudaMemcpyHostToDevice, h->stream()));
        PM_CUDA(launch_heat_convert(h->stage.as<double>(), h->field[0].as<float>(), h->reference, n, 1, nullptr, h->stream()));
    }
    return h->measure();
}

pm_status pm_heat_download(pm_heat* hp, double* kelvin, size_t n) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!kelvin || n != h->n()) return fail(PM_BAD_ARG, "download: one value per cell");
    if (h->precision == PM_PLAIN_F64) {
        PM_CUDA(cudaMemcpyAsync(kelvin, h->field[h->parity].p, n * 8, cudaMemcpyDeviceToHost, h->stream()));
    } else {
        if (!h->stage.p || h->stage.bytes < n * 8) PM_CUDA(h->stage.alloc(n * 8));
        PM_CUDA(launch_heat_convert(nullptr, h->field[h->parity].as<float>(), h->reference, n, 0, h->stage.as<double>(), h->stream()));
        PM_CUDA(cudaMemcpyAsync(kelvin, h->stage.p, n * 8, cudaMemcpyDeviceToHost, h->stream()));
    }
    PM_CUDA(cudaStreamSynchronize(h->stream()));
    return PM_OK;
}

pm_status pm_heat_sample(pm_heat* hp, const double* lo, const double* hi, const int* samples, double* out, size_t n) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    SampleGrid g{};
    pm_status s = sample_grid_of(lo, hi, samples, out, n, g);
    if (s != PM_OK) return s;
    g.dx = h->dx;
    g.nx = h->nx; g.ny = h->ny; g.nz = h->nz;
    const uint8_t* vd = h->vd.empty() ? nullptr : h->dvoid.as<uint8_t>();
    return run_sample(h, out, n, [&](double* dev, cudaStream_t st) {
        return h->precision == PM_PLAIN_F64
                   ? launch_heat_sample<double>(g, h->field[h->parity].as<double>(), 0.0, vd, dev, st)
                   : launch_heat_sample<float>(g, h->field[h->parity].as<float>(), h->reference, vd, dev, st);
    });
}

pm_status pm_heat_max_stable_dt(pm_heat* hp, double* seconds) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!seconds) return fail(PM_BAD_ARG, "null output");
    double rate;
    if (h->state_dependent()) {
        if (h->precision != PM_PLAIN_F64 && !h->radiating_f32())
            return fail(PM_UNSUPPORTED, "radiative gaps, and radiating films on blocks of several materials, are on the plain f64 form only");
        pm_status s = h->read_state();  // the rate the last step (or the last change of state) left
        if (s != PM_OK) return s;
        rate = h->host_state->rate_now;
    } else {
        rate = h->worst_rate_now();
    }
    *seconds = std::isnan(rate) ? std::numeric_limits<double>::infinity() : 1.0 / rate;  // solid.rs:1709-1715
    return PM_OK;
}

pm_status pm_heat_set_tolerance(pm_heat* hp, double tol) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    h->tolerance = tol;
    return PM_OK;
}

pm_status pm_heat_step(pm_heat* hp, double dt, long long nsteps, pm_violation* out) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (nsteps < 0) return fail(PM_BAD_ARG, "nsteps must be >= 0");
    if (nsteps == 0) return PM_OK;
    double rate;
    if (h->state_dependent()) {
        // the limit follows the state: the first step is checked here against the present
        // state's rate, every later one on the device against the rate its own state gives
        if (h->precision != PM_PLAIN_F64 && !h->radiating_f32())
            return fail(PM_UNSUPPORTED, "radiative gaps, and radiating films on blocks of several materials, are on the plain f64 form only");
        pm_status rs = h->read_state();
        if (rs != PM_OK) return rs;
        rate = h->host_state->rate_now;
    } else {
        rate = h->worst_rate_now();
    }
    // solid.rs:1718-1738: the stability refusal, before anything moves.
    const double ratio = dt * rate;
    if (std::isnan(ratio)) {
        const double inf = std::numeric_limits<double>::infinity();
        fill_violation(out, "substance has no diffusivity", h->name, inf, inf, inf, 0.0, 1);
        set_error("substance has no diffusivity");
        return PM_VIOLATION;
    }
    if (ratio > 1.0 + 6e-12) {
        fill_violation(out, "Fourier number", h->name + " (explicit 3D conduction)", kStableFourier3D,
                       ratio * kStableFourier3D, kStableFourier3D, 1e-12, 1);
        set_error("Fourier number past the explicit limit");
        return PM_VIOLATION;
    }
    pm_status s = h->take_pending();
    if (s != PM_OK) return s;
    s = h->begin_call();
    if (s != PM_OK) return s;
    const long long before = h->host_state->steps;
    if (h->precision == PM_PLAIN_F64 && h->persistent(nsteps)) {
        s = h->run_persistent(nsteps, dt);
    } else if (h->precision == PM_PLAIN_F64) {
        s = h->run_steps(nsteps, dt, true, [h, dt](int par, cudaStream_t st) {
            return launch_heat_plain(h->plain_args(par, dt), st);
        });
    } else if (h->persistent(nsteps)) {
        s = h->run_persistent(nsteps, dt);
    } else if (h->tma_form()) {
        s = h->run_steps(nsteps, dt, true, [h, dt](int par, cudaStream_t st) {
            return launch_heat_tma(h->tma_args(par, dt), h->tmaps[par], st);
        });
    } else {
        if ((s = h->prepare_f32(dt)) != PM_OK) return s;
        s = h->run_steps(nsteps, dt, true, [h, dt](int par, cudaStream_t st) {
            return launch_heat_f32(h->f32_args(par, dt), st);
        });
    }
    if (s != PM_OK) return s;
    return h->finish_call(before, out, h->name + " (its own books, against what it moved on the bus)", h->name, true);
}

pm_status pm_heat_ledger(pm_heat* hp, pm_ledger* out) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!out) return fail(PM_BAD_ARG, "null output");
    pm_status s = h->read_state();
    if (s != PM_OK) return s;
    std::memset(out, 0, sizeof(*out));
    out->total = h->host_state->total;
    out->scale = h->host_state->scale;
    out->n_parts = 3;
    for (int q = 0; q < 3; ++q) out->parts[q] = h->host_state->part[q];
    out->steps = h->host_state->steps;
    return PM_OK;
}

pm_status pm_heat_absorb(pm_heat* hp, double joules) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    h->pending += joules;  // held, as the bus holds it, until the next step takes it
    return PM_OK;
}

pm_status pm_heat_checkpoint(pm_heat* hp) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    const size_t bytes = h->n() * h->esize();
    if (!h->saved.p) PM_CUDA(h->saved.alloc(bytes));
    PM_CUDA(cudaMemcpyAsync(h->saved.p, h->field[h->parity].p, bytes, cudaMemcpyDeviceToDevice, h->stream()));
    pm_status s = h->read_state();
    if (s != PM_OK) return s;
    h->saved_lost = h->host_state->lost;
    h->saved_supplied = h->host_state->supplied;
    h->has_saved = true;
    return PM_OK;
}

pm_status pm_heat_restore(pm_heat* hp) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!h->has_saved) return PM_OK;
    const size_t bytes = h->n() * h->esize();
    PM_CUDA(cudaMemcpyAsync(h->field[h->parity].p, h->saved.p, bytes, cudaMemcpyDeviceToDevice, h->stream()));
    pm_status s = h->read_state();
    if (s != PM_OK) return s;
    h->host_state->lost = h->saved_lost;
    h->host_state->supplied = h->saved_supplied;
    s = h->write_state();
    if (s != PM_OK) return s;
    return h->measure();
}

pm_status pm_heat_step_kernel(pm_heat* hp, long long nsteps, char* name, int cap, long long* launches) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    if (!name || cap < 1) return fail(PM_BAD_ARG, "step_kernel: a name buffer of one byte or more");
    const bool plain = h->precision == PM_PLAIN_F64;
    const bool filled = !h->uniform;
    std::string k;
    long long n = nsteps > 0 ? nsteps : 0;  // one launch a step, replayed from a graph or not
    if (nsteps < 1) {
        k = "none";
    } else if (h->persistent(nsteps)) {
        k = plain ? "heat_plain_pair_steps (cooperative, many steps a launch)"
                  : "heat_f32_quad_steps (cooperative, many steps a launch)";
        n = (nsteps + Heat::kPersistChunk - 1) / Heat::kPersistChunk;
    } else if (plain) {
        k = (!filled && h->nx % 4 == 0 && h->wide && h->quads64) ? "heat_plain_quad_step"
            : (!filled && h->nx % 2 == 0 && h->wide)               ? "heat_plain_pair_step"
                                                                    : "heat_plain_step";
    } else if (h->tma_form()) {
        k = "heat_tma_step (TMA-staged)";
    } else {
        k = filled ? "heat_f32_step<filled>"
            : (h->nx % 4 == 0 && h->wide && !h->state_dependent()) ? "heat_f32_quad_step"
                                                                   : "heat_f32_step";
    }
    std::snprintf(name, (size_t)cap, "%s", k.c_str());
    if (launches) *launches = n;
    return PM_OK;
}

pm_status pm_heat_set_cells_per_thread(pm_heat* hp, int cells) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    const bool plain = h->precision == PM_PLAIN_F64;
    if (plain ? (cells != 1 && cells != 2 && cells != 4) : (cells != 1 && cells != 4))
        return fail(PM_BAD_ARG, plain ? "cells per thread (plain f64): 1, 2 or 4" : "cells per thread (FP32): 1 or 4");
    const bool wide = cells != 1, quads64 = plain ? cells == 4 : h->quads64;
    if (wide != h->wide || quads64 != h->quads64) {
        PM_CUDA(cudaStreamSynchronize(h->stream()));
        h->drop_graphs();  // the captured launches hold the old tiling
        h->wide = wide;
        h->quads64 = quads64;
    }
    return PM_OK;
}

pm_status pm_heat_set_wait_budget(pm_heat* hp, unsigned polls) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    h->wait_budget = polls;
    return PM_OK;
}

pm_status pm_heat_set_stream(pm_heat* hp, void* stream) {
    Heat* h = reinterpret_cast<Heat*>(hp);
    HEAT_GUARD(h);
    PM_CUDA(cudaStreamSynchronize(h->stream()));
    h->user = static_cast<cudaStream_t>(stream);
    return PM_OK;
}

void pm_heat_destroy(pm_heat* hp) { delete reinterpret_cast<Heat*>(hp); }

}  // extern "C"
