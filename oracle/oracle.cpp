// ORACLE — TEST INFRASTRUCTURE ONLY. Never linked into, imported by, or called from the
// product library (pantometry_b200/). Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg use it, and only as the checker or as the timed CPU baseline.
//
// A CPU restatement, in C++17, of pantometry's 3D explicit staggered-grid path, written from
// the reference's Rust source with every operand order preserved. Built with
// `-O2 -ffp-contract=off -fno-fast-math` on x86-64 (SSE2 doubles), which gives the same IEEE
// results as rustc: Rust never contracts to FMA and the reference has no `mul_add` on this path.
//
// Parity pinning: the reference is pure Rust and no Rust toolchain exists here, so the reference
// cannot be built or run. The restatement is pinned against the reference's own known-answer
// tests (tests/test_oracle_*.py restate them): the pinned RNG digest
// (crates/pantometry-core/src/rng.rs:306-308), the exact discrete eigen-decay of Solid3D
// (crates/pantometry-thermal/tests/solid_closed_forms.rs:46-77), axis permutation (:84-112),
// insulated conservation (:156-194), the Hall invariant drift and startup order
// (crates/pantometry-acoustic/tests/hall_closed_forms.rs:132-181), the Cavity divergence
// identity (crates/pantometry-em/tests/against_closed_forms.rs:37-100), and the audit
// semantics (crates/pantometry-core/src/conserved.rs:376-460).
//
// Reference files below are cited by their path inside the pantometry project.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

namespace {

constexpr double STEFAN_BOLTZMANN = 5.670374419e-8;  // pantometry-units/src/lib.rs:899
constexpr double STABLE_FOURIER_3D = 1.0 / 6.0;       // pantometry-thermal/src/solid.rs:84
constexpr double EPSILON_0 = 8.8541878128e-12;        // pantometry-em/src/lib.rs:67
constexpr double MU_0 = 1.25663706212e-6;             // pantometry-em/src/lib.rs:69
constexpr double COURANT_3D = 0.5773502691896258;     // pantometry-em/src/cavity.rs:15
constexpr double INF = std::numeric_limits<double>::infinity();

// Rust `f64::powi` with a constant exponent lowers to binary-decomposition multiplies
// (LLVM ExpandPowI / compiler-rt __powidf2): x^3 = x*(x*x), x^4 = (x*x)*(x*x).
inline double powi3(double x) { return x * (x * x); }
inline double powi4(double x) { double s = x * x; return s * s; }

// Rust `f64::max`: NaN-ignoring.
inline double rmax(double a, double b) {
    if (std::isnan(a)) return b;
    if (std::isnan(b)) return a;
    return a > b ? a : b;
}

}  // namespace

extern "C" {

// Mirrors pantometry-core/src/conserved.rs:128-143 (`Violation`).
typedef struct {
    char quantity[32];
    char site[96];
    double before;
    double after;
    double scale;
    double tolerance;
} or_violation;

// One quantity's books (conserved.rs:37-41 `Entry`). Only "energy" lives on this path.
typedef struct {
    double total;
    double scale;
} or_entry;

}  // extern "C"

namespace {

void set_violation(or_violation* v, const std::string& q, const std::string& site, double before,
                   double after, double scale, double tol) {
    if (!v) return;
    std::memset(v, 0, sizeof(*v));
    std::snprintf(v->quantity, sizeof(v->quantity), "%s", q.c_str());
    std::snprintf(v->site, sizeof(v->site), "%s", site.c_str());
    v->before = before;
    v->after = after;
    v->scale = scale;
    v->tolerance = tol;
}

// conserved.rs:86-90 `Ledger::add`.
inline void ledger_add(or_entry& e, double x) {
    e.total += x;
    e.scale = rmax(e.scale, std::fabs(x));
}

// conserved.rs:323-363 `audit_with`, for the single quantity "energy".
bool audit_energy(const char* site, or_entry b, or_entry a, double tol, or_violation* out) {
    double scale = rmax(rmax(rmax(std::fabs(b.total), std::fabs(a.total)), b.scale), a.scale);
    if (scale < 1e-300) return true;
    if (std::fabs(a.total - b.total) / scale > tol) {
        set_violation(out, "energy", site, b.total, a.total, scale, tol);
        return false;
    }
    return true;
}

// sim.rs:1169-1223 `attribute` with no bus traffic (expected = 0).
bool attribute_energy(const std::string& name, or_entry b, or_entry a, double tol,
                      or_violation* out) {
    double expected = 0.0;
    double discrepancy = (a.total - b.total) - expected;
    double scale = rmax(rmax(rmax(rmax(std::fabs(b.total), std::fabs(a.total)), b.scale), a.scale),
                        std::fabs(expected));
    if (scale < 1e-300) return true;
    if (std::fabs(discrepancy) / scale > tol) {
        set_violation(out, "energy", name + " (its own books, against what it moved on the bus)",
                      b.total + expected, a.total, scale, tol);
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------------------------
// Solid3D — pantometry-thermal/src/solid.rs (uniform and filled one-phase blocks, films).
// ---------------------------------------------------------------------------------------------

struct Material {
    double density;
    double conductivity;
    double specific_heat;
    double emissivity;
    int thermal;  // 0 = `thermal: None`
};

struct Env {
    double ambient;
    double convection;
    double area;
};

struct Heat {
    std::string name;
    int nx, ny, nz;
    double dx;
    double reference;
    std::vector<Material> mats;
    std::vector<uint32_t> which;
    std::vector<double> cells, saved;
    std::vector<double> kx, ky, kz, mobility, capacity, face_sum;
    // solid.rs:238-266: void cells, the gap pairs across them (a, b, σA/(1/ε₁+1/ε₂−1)) and the
    // watts each cell generates
    std::vector<uint8_t> vd;
    struct Gap { size_t a, b; double coefficient; };
    std::vector<Gap> gaps;
    std::vector<double> source;
    double worst_rate = 0.0;
    bool exposed[6] = {false, false, false, false, false, false};
    Env env[6];
    double lost = 0.0, saved_lost = 0.0;
    double supplied = 0.0, saved_supplied = 0.0;
    double absorbed = 0.0;

    size_t n() const { return (size_t)nx * ny * nz; }

    // solid.rs:110-122
    static double series_with_half_cell(double film, double conductivity, double area, double dx) {
        if (film <= 0.0) return 0.0;
        double half = 2.0 * conductivity * area / dx;
        if (!std::isfinite(half)) return film;
        if (half <= 0.0) return 0.0;
        return 1.0 / (1.0 / film + 1.0 / half);
    }

    // solid.rs:1222-1229
    size_t cells_on(int face) const {
        switch (face) {
            case 0: case 1: return (size_t)ny * nz;
            case 2: case 3: return (size_t)nx * nz;
            default: return (size_t)nx * ny;
        }
    }

    // solid.rs:158-168
    bool holds(int face, int i, int j, int k) const {
        switch (face) {
            case 0: return i == 0;
            case 1: return i + 1 == nx;
            case 2: return j == 0;
            case 3: return j + 1 == ny;
            case 4: return k == 0;
            default: return k + 1 == nz;
        }
    }

    double mat_conductivity(size_t c) const {
        const Material& m = mats[which[c]];
        return m.thermal ? m.conductivity : INF;
    }
    double mat_emissivity(size_t c) const {
        const Material& m = mats[which[c]];
        return m.thermal ? m.emissivity : 0.0;
    }

    // solid.rs:588-784, one-phase: face conductivities, capacity, mobility, face_sum, worst_rate,
    // then the gaps (solid.rs:783).
    void resolve() {
        double volume = dx * dx * dx;
        size_t N = n();
        if (vd.size() != N) vd.assign(N, 0);
        if (source.size() != N) source.assign(N, 0.0);
        std::vector<double> kmix(N), cmix(N);
        for (size_t c = 0; c < N; ++c) {
            if (vd[c]) { kmix[c] = 0.0; cmix[c] = 0.0; continue; }  // solid.rs:689-694
            const Material& m = mats[which[c]];
            double k = m.thermal ? m.conductivity : NAN;
            // `heat_capacity(volume)` = (density * volume) * specific_heat (substance.rs:219-239)
            double cap = m.thermal ? (m.density * volume) * m.specific_heat : NAN;
            double phi = 0.0;  // one-phase: melted = 0 and liquid == solid
            kmix[c] = k + phi * (k - k);
            cmix[c] = cap + phi * (cap - cap);
        }
        auto series = [](double a, double b) {
            double sum = a + b;
            return sum > 0.0 ? 2.0 * a * b / sum : 0.0;
        };
        kx.assign((size_t)(nx + 1) * ny * nz, 0.0);
        ky.assign((size_t)nx * (ny + 1) * nz, 0.0);
        kz.assign((size_t)nx * ny * (nz + 1), 0.0);
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    size_t c = i + (size_t)nx * (j + (size_t)ny * k);
                    if (i > 0)
                        kx[i + (size_t)(nx + 1) * (j + (size_t)ny * k)] = series(kmix[c - 1], kmix[c]);
                    if (j > 0)
                        ky[i + (size_t)nx * (j + (size_t)(ny + 1) * k)] = series(kmix[c - nx], kmix[c]);
                    if (k > 0)
                        kz[i + (size_t)nx * (j + (size_t)ny * k)] =
                            series(kmix[c - (size_t)nx * ny], kmix[c]);
                }
        capacity.assign(N, 0.0);
        mobility.assign(N, 0.0);
        face_sum.assign(N, 0.0);
        worst_rate = 0.0;
        bool nowhere = false;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    size_t c = i + (size_t)nx * (j + (size_t)ny * k);
                    double cap = cmix[c];
                    capacity[c] = cap;
                    mobility[c] = vd[c] ? 0.0 : dx / cap;  // solid.rs:753-756
                    double sum = kx[i + (size_t)(nx + 1) * (j + (size_t)ny * k)] +
                                 kx[i + 1 + (size_t)(nx + 1) * (j + (size_t)ny * k)] +
                                 ky[i + (size_t)nx * (j + (size_t)(ny + 1) * k)] +
                                 ky[i + (size_t)nx * (j + 1 + (size_t)(ny + 1) * k)] +
                                 kz[i + (size_t)nx * (j + (size_t)ny * k)] +
                                 kz[i + (size_t)nx * (j + (size_t)ny * (k + 1))];
                    face_sum[c] = sum;
                    double rate = mobility[c] * sum;
                    if (std::isnan(rate))
                        nowhere = true;
                    else
                        worst_rate = rmax(worst_rate, rate);
                }
        if (nowhere) worst_rate = NAN;
        find_gaps();
    }

    // solid.rs:786-838 `find_gaps`: along every row, then every column, then every pillar, a run
    // of void with solid at both ends pairs the two end cells.
    void find_gaps() {
        gaps.clear();
        bool any = false;
        for (uint8_t v : vd) any = any || v;
        if (!any) return;
        const double area = dx * dx;
        auto walk = [&](size_t first, size_t stride, int len) {
            bool have_last = false, void_between = false;
            size_t last = 0;
            for (int q = 0; q < len; ++q) {
                const size_t c = first + stride * (size_t)q;
                if (vd[c]) { void_between = have_last; continue; }
                if (have_last && void_between) {
                    const double ea = mat_emissivity(last), eb = mat_emissivity(c);
                    if (ea > 0.0 && eb > 0.0) {
                        const double resistance = 1.0 / ea + 1.0 / eb - 1.0;
                        if (resistance > 0.0) gaps.push_back(Gap{last, c, STEFAN_BOLTZMANN * area / resistance});
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

    // solid.rs:1045-1085 `dissipating`: `watts` spread evenly over the solid cells the mask
    // selects, replacing what they generated before.
    void dissipating(double watts, const uint8_t* mask) {
        std::vector<size_t> chosen;
        for (size_t c = 0; c < n(); ++c)
            if (!vd[c] && mask[c]) chosen.push_back(c);
        if (chosen.empty()) return;
        const double each = watts / (double)chosen.size();
        for (size_t c : chosen) source[c] = each;
        resolve();
    }
    bool supplies() const {  // solid.rs:1110-1112
        for (double w : source) if (w != 0.0) return true;
        return false;
    }
    // solid.rs:1324-1335 `temperature_at`: not a number where there is nothing.
    double temperature_at(size_t c) const { return vd[c] ? NAN : cells[c]; }

    // solid.rs:1269-1288
    double loss_conductance_at(double at, int i, int j, int k, size_t c) const {
        double total = -0.0;  // Rust `Sum for f64` starts from -0.0
        for (int f = 0; f < 6; ++f) {
            if (!exposed[f] || !holds(f, i, j, k)) continue;
            double share = env[f].area / (double)std::max<size_t>(cells_on(f), 1);
            double emissivity = mat_emissivity(c);
            double hot = rmax(at, env[f].ambient);
            double h = env[f].convection + 4.0 * emissivity * STEFAN_BOLTZMANN * powi3(hot);
            total += series_with_half_cell(h * share, mat_conductivity(c), share, dx);
        }
        return total;
    }

    // solid.rs:1148-1185
    double worst_rate_now() const {
        bool any = false;
        for (int f = 0; f < 6; ++f) any = any || exposed[f];
        if ((!any && gaps.empty()) || std::isnan(worst_rate)) return worst_rate;
        double worst = worst_rate;
        for (const Gap& g : gaps) {
            const double hotter = rmax(cells[g.a], cells[g.b]);
            const double cond = 4.0 * g.coefficient * powi3(hotter);
            for (size_t c : {g.a, g.b})
                if (capacity[c] > 0.0) worst = rmax(worst, cond / capacity[c]);
        }
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    size_t c = i + (size_t)nx * (j + (size_t)ny * k);
                    double loss = loss_conductance_at(temperature_at(c), i, j, k, c);
                    if (loss == 0.0) continue;
                    worst = rmax(worst, mobility[c] * (face_sum[c] + loss / dx));
                }
        return worst;
    }

    // solid.rs:1192-1219 (reads `old`)
    double film_flux(const std::vector<double>& old, int i, int j, int k, size_t c) const {
        double emissivity = mat_emissivity(c);
        double conductivity = mat_conductivity(c);
        double here = old[c];
        double out = 0.0;
        for (int f = 0; f < 6; ++f) {
            if (!exposed[f] || !holds(f, i, j, k)) continue;
            double share = env[f].area / (double)std::max<size_t>(cells_on(f), 1);
            double gap = here - env[f].ambient;
            if (gap == 0.0) continue;
            // thermal/src/lib.rs:104-110 `Environment::loss_from` with area = share
            double convective = env[f].convection * share * (here - env[f].ambient);
            double radiative = emissivity * STEFAN_BOLTZMANN * share *
                               (powi4(here) - powi4(env[f].ambient));
            double bare = convective + radiative;
            double g = series_with_half_cell(bare / gap, conductivity, share, dx);
            out += g * gap / dx;
        }
        return out;
    }

    // solid.rs:1557-1561 + 1583-1598 (latent <= 0): Σ C·(T − reference) − 0.
    double stored_heat() const {
        double s = -0.0;
        for (size_t c = 0; c < n(); ++c) s += capacity[c] * (cells[c] - reference) - 0.0;
        return s;
    }

    // solid.rs:1904-1927
    or_entry ledger() const {
        or_entry e{0.0, 0.0};
        ledger_add(e, stored_heat());
        ledger_add(e, lost);
        ledger_add(e, -supplied);
        return e;
    }

    // solid.rs:1717-1901, one-phase, no gaps, no sources, empty bus.
    bool step(double dt, or_violation* out) {
        double ratio = dt * worst_rate_now();
        if (std::isnan(ratio)) {
            set_violation(out, "substance has no diffusivity", name, INF, INF, INF, 0.0);
            return false;
        }
        if (ratio > 1.0 + 6e-12) {
            set_violation(out, "Fourier number", name + " (explicit 3D conduction)",
                          STABLE_FOURIER_3D, ratio * STABLE_FOURIER_3D, STABLE_FOURIER_3D, 1e-12);
            return false;
        }
        take_pending();
        bool any = false;
        for (int f = 0; f < 6; ++f) any = any || exposed[f];
        std::vector<double> old = cells;
        double dts = dt;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    size_t c = i + (size_t)nx * (j + (size_t)ny * k);
                    double t = old[c];
                    size_t xr = (size_t)(nx + 1) * (j + (size_t)ny * k);
                    size_t yr = (size_t)nx * (j + (size_t)(ny + 1) * k);
                    size_t plane = (size_t)nx * ny;
                    double flux = 0.0;
                    if (i > 0) flux += kx[i + xr] * (old[c - 1] - t);
                    if (i + 1 < nx) flux += kx[i + 1 + xr] * (old[c + 1] - t);
                    if (j > 0) flux += ky[i + yr] * (old[c - nx] - t);
                    if (j + 1 < ny) flux += ky[i + nx + yr] * (old[c + nx] - t);
                    if (k > 0) flux += kz[c] * (old[c - plane] - t);
                    if (k + 1 < nz) flux += kz[c + plane] * (old[c + plane] - t);
                    double shed = any ? film_flux(old, i, j, k, c) : 0.0;
                    cells[c] += dts * mobility[c] * (flux - shed);  // add_kelvin, latent <= 0
                    if (shed != 0.0) lost += dts * mobility[c] * shed * capacity[c];
                }
        // solid.rs:1854-1864: heat that has a place, after the sweep
        if (supplies()) {
            for (size_t c = 0; c < n(); ++c) {
                if (source[c] == 0.0 || vd[c]) continue;
                const double joules = source[c] * dts;
                cells[c] += joules / capacity[c];
                supplied += joules;
            }
        }
        // solid.rs:1866-1878: what the gaps carry, read off `old`, in the pairs' order
        for (const Gap& g : gaps) {
            const double watts = g.coefficient * (powi4(old[g.a]) - powi4(old[g.b]));
            if (watts == 0.0) continue;
            const double joules = watts * dts;
            cells[g.a] += -joules / capacity[g.a];
            cells[g.b] += joules / capacity[g.b];
        }
        return true;
    }

    // Placeless heat handed in for the next step, as the bus's HEAT channel holds it: the step takes
    // it after its stability refusal (solid.rs:1718-1765), so a refused step leaves it pending.
    double pending = 0.0;
    void absorb(double gained) { pending += gained; }

    // solid.rs:1752-1765: the bus share, spread to a uniform rise through add_kelvin (as `deposit`,
    // 1368-1375, is).
    void take_pending() {
        const double gained = pending;
        pending = 0.0;
        if (gained == 0.0) return;
        absorbed += gained;
        double cap_sum = -0.0;
        for (double c : capacity) cap_sum += c;
        double rise = gained / cap_sum;
        for (size_t c = 0; c < n(); ++c)
            if (!vd[c]) cells[c] += rise;  // void takes no share (solid.rs:1756-1764)
    }
};

// ---------------------------------------------------------------------------------------------
// Hall — pantometry-acoustic/src/hall.rs, plus the point-source extension (not in the
// reference; its ledger term is this build's own derivation).
// ---------------------------------------------------------------------------------------------

inline double wall_weight(int k, int n) { return (k == 0 || k + 1 == n) ? 2.0 : 1.0; }  // hall.rs:675

struct Hall {
    std::string name;
    int nx, ny, nz;
    double dx, speed, density;
    std::vector<double> p, pp, vx, vy, vz;
    bool staggered = false;
    double offset = 0.0, datum = 0.0;
    // checkpoint (hall.rs:536-555)
    bool has_saved = false;
    std::vector<double> sp, svx, svy, svz;
    bool s_staggered = false;
    // Extension: a soft pressure source at one node, `wave[n]` Pa added after step n's update.
    long long source_node = -1;
    std::vector<double> wave;
    long long steps_taken = 0;
    double injected = 0.0;
    double last_delta = 0.0;
    // Extension: a sound speed per cubic block of `block` nodes a side (the heterogeneous
    // medium of the 1024³ configuration); `Hall` itself has one speed (hall.rs:82-83).
    int block = 0, nbx = 0, nby = 0;
    std::vector<double> speeds;

    size_t at(int i, int j, int k) const { return i + (size_t)nx * (j + (size_t)ny * k); }
    double speed_at(int i, int j, int k) const {
        if (block <= 0) return speed;
        return speeds[(size_t)(i / block) + (size_t)nbx * ((size_t)(j / block) + (size_t)nby * (k / block))];
    }
    double max_speed() const {
        double c = speed;
        if (block > 0) { c = speeds[0]; for (double v : speeds) c = v > c ? v : c; }
        return c;
    }

    // hall.rs:334-384
    double invariant_si() const {
        double volume = dx * dx * dx;
        double rc2 = density * speed * speed;
        if (block <= 0 && rc2 <= 0.0) return 0.0;
        double total = 0.0;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    double share = 1.0 / (wall_weight(i, nx) * wall_weight(j, ny) * wall_weight(k, nz));
                    size_t idx = at(i, j, k);
                    if (block > 0) {
                        double c = speed_at(i, j, k);
                        rc2 = density * c * c;
                    }
                    total += share * p[idx] * pp[idx] / (2.0 * rc2) * volume;
                }
        double half_rho = 0.5 * density;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx - 1; ++i) {
                    double v = vx[i + (size_t)(nx - 1) * (j + (size_t)ny * k)];
                    double share = 1.0 / (wall_weight(j, ny) * wall_weight(k, nz));
                    total += share * half_rho * v * v * volume;
                }
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny - 1; ++j)
                for (int i = 0; i < nx; ++i) {
                    double v = vy[i + (size_t)nx * (j + (size_t)(ny - 1) * k)];
                    double share = 1.0 / (wall_weight(i, nx) * wall_weight(k, nz));
                    total += share * half_rho * v * v * volume;
                }
        for (int k = 0; k < nz - 1; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    double v = vz[i + (size_t)nx * (j + (size_t)ny * k)];
                    double share = 1.0 / (wall_weight(i, nx) * wall_weight(j, ny));
                    total += share * half_rho * v * v * volume;
                }
        return total;
    }

    double courant(double dt) const { return max_speed() * dt * std::sqrt(3.0) / dx; }  // hall.rs:319

    // Source bookkeeping: adding δ at node s after the pressure update moves the discrete
    // invariant by share·δ·p_prev·V/(2ρc²) at once, and by share·δ·p·V/(2ρc²) one step later
    // (the consistency defect it leaves in the next leapfrog update). `injected` carries both,
    // so `invariant + offset − injected` is conserved to rounding.
    double node_weight(size_t idx) const {
        int i = (int)(idx % nx), j = (int)((idx / nx) % ny), k = (int)(idx / ((size_t)nx * ny));
        double share = 1.0 / (wall_weight(i, nx) * wall_weight(j, ny) * wall_weight(k, nz));
        double c = speed_at(i, j, k);
        double rc2 = density * c * c;
        return share * (dx * dx * dx) / (2.0 * rc2);
    }

    // hall.rs:408-530
    bool step(double dt, or_violation* out) {
        double c = courant(dt);
        if (c > 1.0 + 1e-12) {
            set_violation(out, "Courant number", name + " (three-dimensional wave equation)", 1.0, c,
                          1.0, 1e-12);
            return false;
        }
        double h = dt;
        if (h <= 0.0) return true;
        double rc2 = density * speed * speed;
        double vh = staggered ? h : 0.5 * h;
        bool starting = !staggered;
        staggered = true;
        double gain = vh / (density * dx);
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx - 1; ++i) {
                    double d = p[at(i + 1, j, k)] - p[at(i, j, k)];
                    vx[i + (size_t)(nx - 1) * (j + (size_t)ny * k)] -= gain * d;
                }
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny - 1; ++j)
                for (int i = 0; i < nx; ++i) {
                    double d = p[at(i, j + 1, k)] - p[at(i, j, k)];
                    vy[i + (size_t)nx * (j + (size_t)(ny - 1) * k)] -= gain * d;
                }
        for (int k = 0; k < nz - 1; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    double d = p[at(i, j, k + 1)] - p[at(i, j, k)];
                    vz[i + (size_t)nx * (j + (size_t)ny * k)] -= gain * d;
                }
        pp = p;
        double scale = h * rc2 / dx;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    double lo_x = i > 0 ? vx[i - 1 + (size_t)(nx - 1) * (j + (size_t)ny * k)] : 0.0;
                    double hi_x = i + 1 < nx ? vx[i + (size_t)(nx - 1) * (j + (size_t)ny * k)] : 0.0;
                    double lo_y = j > 0 ? vy[i + (size_t)nx * (j - 1 + (size_t)(ny - 1) * k)] : 0.0;
                    double hi_y = j + 1 < ny ? vy[i + (size_t)nx * (j + (size_t)(ny - 1) * k)] : 0.0;
                    double lo_z = k > 0 ? vz[i + (size_t)nx * (j + (size_t)ny * (k - 1))] : 0.0;
                    double hi_z = k + 1 < nz ? vz[i + (size_t)nx * (j + (size_t)ny * k)] : 0.0;
                    size_t idx = at(i, j, k);
                    if (block > 0) {
                        double c = speed_at(i, j, k);
                        scale = h * (density * c * c) / dx;
                    }
                    p[idx] -= scale * (wall_weight(i, nx) * (hi_x - lo_x) +
                                       wall_weight(j, ny) * (hi_y - lo_y) +
                                       wall_weight(k, nz) * (hi_z - lo_z));
                }
        double immediate = 0.0;
        if (source_node >= 0) {
            double delta = steps_taken < (long long)wave.size() ? wave[steps_taken] : 0.0;
            double w = node_weight((size_t)source_node);
            // deferred term of the previous injection (uses this step's p_prev), then this one's
            injected += w * (last_delta + delta) * pp[source_node];
            immediate = w * delta * pp[source_node];
            p[source_node] += delta;
            last_delta = delta;
        }
        steps_taken += 1;
        if (starting) {
            double invariant = invariant_si() - immediate;
            double off = datum - invariant;
            double sc = rmax(std::fabs(datum), std::fabs(invariant));
            if (sc > 0.0 && std::fabs(off) / sc > 0.25) {
                set_violation(out, "energy", name + " (starting the leapfrog)", datum, invariant, sc,
                              0.25);
                return false;
            }
            offset = off;
        }
        return true;
    }

    double energy() const { return invariant_si() + offset; }  // hall.rs:249-251

    // hall.rs:532-534, plus the source's injected work as an entry of its own, the way the
    // cavity books its source work (cavity.rs:1520-1524): the audit's scale then covers what the
    // source moved, not only the small net left after it.
    or_entry ledger() const {
        or_entry e{0.0, 0.0};
        ledger_add(e, energy());
        if (source_node >= 0) ledger_add(e, -injected);
        return e;
    }
};

// ---------------------------------------------------------------------------------------------
// Room — pantometry-acoustic/src/room.rs: the two-dimensional staggered scheme (pressure at the
// nodes, velocities on the faces between them, rigid walls, a depth for the volume).
// ---------------------------------------------------------------------------------------------

struct Room {
    std::string name;
    int nx, ny;
    double dx, speed, density, depth;
    std::vector<double> p, pp, vx, vy;
    bool staggered = false;
    double offset = 0.0, datum = 0.0;
    bool has_saved = false;  // room.rs:489-505
    std::vector<double> sp, svx, svy;
    bool s_staggered = false;

    // room.rs:243-281
    double invariant_si() const {
        double volume = dx * dx * depth;
        double rc2 = density * speed * speed;
        if (rc2 <= 0.0) return 0.0;
        double potential = 0.0;
        for (size_t k = 0; k < p.size(); ++k) {
            int i = (int)(k % nx), j = (int)(k / nx);
            double share = 1.0 / (wall_weight(i, nx) * wall_weight(j, ny));
            potential += share * p[k] * pp[k] / (2.0 * rc2) * volume;
        }
        double kinetic_x = 0.0;
        for (size_t k = 0; k < vx.size(); ++k) {
            double u = vx[k];
            kinetic_x += density * u * u / 2.0 * volume / wall_weight((int)(k / (nx - 1)), ny);
        }
        double kinetic_y = 0.0;
        for (size_t k = 0; k < vy.size(); ++k) {
            double u = vy[k];
            kinetic_y += density * u * u / 2.0 * volume / wall_weight((int)(k % nx), nx);
        }
        return potential + kinetic_x + kinetic_y;
    }

    double courant(double dt) const { return speed * dt * std::sqrt(2.0) / dx; }  // room.rs:336-338

    // room.rs:368-478
    bool step(double dt, or_violation* out) {
        double c = courant(dt);
        if (c > 1.0 + 1e-12) {
            set_violation(out, "Courant number", name + " (two-dimensional wave equation)", 1.0, c, 1.0, 1e-12);
            return false;
        }
        double h = dt;
        if (h <= 0.0) return true;
        double rc2 = density * speed * speed;
        double vh = staggered ? h : 0.5 * h;
        bool starting = !staggered;
        staggered = true;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx - 1; ++i) {
                size_t face = (size_t)j * (nx - 1) + i;
                vx[face] -= vh / (density * dx) * (p[(size_t)j * nx + i + 1] - p[(size_t)j * nx + i]);
            }
        for (int j = 0; j < ny - 1; ++j)
            for (int i = 0; i < nx; ++i) {
                size_t face = (size_t)j * nx + i;
                vy[face] -= vh / (density * dx) * (p[(size_t)(j + 1) * nx + i] - p[(size_t)j * nx + i]);
            }
        pp = p;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double left = i == 0 ? 0.0 : vx[(size_t)j * (nx - 1) + i - 1];
                double right = i == nx - 1 ? 0.0 : vx[(size_t)j * (nx - 1) + i];
                double below = j == 0 ? 0.0 : vy[(size_t)(j - 1) * nx + i];
                double above = j == ny - 1 ? 0.0 : vy[(size_t)j * nx + i];
                p[(size_t)j * nx + i] -= h * rc2 / dx * (wall_weight(i, nx) * (right - left) + wall_weight(j, ny) * (above - below));
            }
        if (starting) {
            double invariant = invariant_si();
            double off = datum - invariant;
            double sc = rmax(std::fabs(datum), std::fabs(invariant));
            if (sc > 0.0 && std::fabs(off) / sc > 0.25) {
                set_violation(out, "energy", name + " (starting the leapfrog)", datum, invariant, sc, 0.25);
                return false;
            }
            offset = off;
        }
        return true;
    }

    double energy() const { return invariant_si() + offset; }  // room.rs:226-228
    or_entry ledger() const {                                  // room.rs:480-482
        or_entry e{0.0, 0.0};
        ledger_add(e, energy());
        return e;
    }
};

// ---------------------------------------------------------------------------------------------
// Tube — pantometry-acoustic/src/lib.rs:107-560: the one-dimensional staggered scheme, pressure
// at the n samples, velocity on the n−1 faces, each end closed, open or matched to an impedance.
// ---------------------------------------------------------------------------------------------

struct Tube {
    std::string name;
    int n;
    double dx, speed, density, area;
    int end_kind[2] = {0, 0};  // 0 closed, 1 open, 2 matched (lib.rs:107-116)
    double end_z[2] = {0.0, 0.0};
    std::vector<double> p, pp, v;
    bool staggered = false;
    double offset = 0.0, datum = 0.0, radiated = 0.0;
    bool has_saved = false;  // lib.rs:539-556
    std::vector<double> sp, sv;
    bool s_staggered = false;

    double impedance() const { return density * speed; }  // lib.rs:255-257
    // lib.rs:301-327
    double invariant_si() const {
        double volume = area * dx;
        double rc2 = density * speed * speed;
        if (rc2 <= 0.0) return 0.0;
        int last = n - 1;
        double potential = 0.0;
        for (int i = 0; i < n; ++i) {
            double share = (i == 0 || i == last) ? 0.5 : 1.0;
            potential += share * p[i] * pp[i] / (2.0 * rc2) * volume;
        }
        double kinetic = 0.0;
        for (double u : v) kinetic += density * u * u / 2.0 * volume;
        return potential + kinetic;
    }
    // lib.rs:368-382
    double wall_velocity(int end, double boundary_pressure, double outward) const {
        if (end_kind[end] == 0) return 0.0;
        if (end_kind[end] == 1) return outward * boundary_pressure / impedance();
        double zz = end_z[end];
        if (zz <= 0.0) return outward * boundary_pressure / impedance();
        return outward * boundary_pressure / zz;
    }
    double courant(double dt) const { return speed * dt / dx; }  // lib.rs:358-360
    // lib.rs:386-463; returns the energy the ends published this step
    double advance(double dt) {
        double rc2 = density * speed * speed;
        double vh = staggered ? dt : 0.5 * dt;
        bool starting = !staggered;
        staggered = true;
        for (size_t i = 0; i < v.size(); ++i) v[i] -= vh / (density * dx) * (p[i + 1] - p[i]);
        double left_wall = wall_velocity(0, p[0], -1.0);
        double right_wall = wall_velocity(1, p[n - 1], 1.0);
        pp = p;
        double absorbed = 0.0;
        for (int i = 0; i < n; ++i) {
            double inflow = i == 0 ? left_wall : v[i - 1];
            double outflow = i == n - 1 ? right_wall : v[i];
            double share = (i == 0 || i == n - 1) ? 2.0 : 1.0;
            p[i] -= dt * rc2 / dx * share * (outflow - inflow);
        }
        absorbed += std::fabs(p[0] * left_wall) * area * dt;
        absorbed += std::fabs(p[n - 1] * right_wall) * area * dt;
        if (absorbed > 0.0) radiated += absorbed;
        if (starting) {
            double invariant = invariant_si();
            double off = datum - invariant;
            double sc = rmax(std::fabs(datum), std::fabs(invariant));
            if (sc > 0.0 && std::fabs(off) / sc <= 0.25) offset = off;
        }
        return absorbed > 0.0 ? absorbed : 0.0;
    }
    // lib.rs:516-533
    bool step(double dt, or_violation* out, double* published) {
        if (published) *published = 0.0;
        double c = courant(dt);
        if (c > 1.0 + 1e-12) {
            set_violation(out, "Courant number", name + " (explicit wave equation)", 1.0, c, 1.0, 1e-12);
            return false;
        }
        if (dt <= 0.0) return true;
        double pub = advance(dt);
        if (published) *published = pub;
        return true;
    }
    double energy() const { return invariant_si() + offset; }  // lib.rs:288-290
    or_entry ledger() const {                                  // lib.rs:535-537
        or_entry e{0.0, 0.0};
        ledger_add(e, energy());
        return e;
    }
};

// ---------------------------------------------------------------------------------------------
// Bar1D — pantometry-thermal/src/lib.rs:425-660: explicit conduction along a bar with insulated
// ends. The heat its step takes from the bus (lumped into the first cell, lib.rs:590-593; per
// cell over its exposed side, lib.rs:598-606) is handed in by the caller before the step.
// ---------------------------------------------------------------------------------------------

struct Bar {
    std::string name;
    int n;
    double dx, area, reference;
    double density, conductivity, specific_heat;
    int thermal;
    std::vector<double> cells, saved;
    double absorbed = 0.0;
    double lumped = 0.0;             // the next step's share of placeless heat
    std::vector<double> per_cell;    // the next step's heat per cell, empty: none

    // substance.rs:211-222 (mass_of: density·volume, substance.rs:237-239)
    double diffusivity() const { return thermal ? conductivity / (density * specific_heat) : NAN; }
    double cell_capacity() const {  // lib.rs:514-520
        double volume = area * dx;
        return thermal ? (density * volume) * specific_heat : INF;
    }
    double fourier_number(double dt) const {  // lib.rs:546-551
        if (!thermal) return INF;
        return diffusivity() * dt / (dx * dx);
    }
    double stored_heat() const {  // lib.rs:536-538
        double s = 0.0;
        for (double t : cells) s += t - reference;
        return cell_capacity() * s;
    }
    // lib.rs:571-627; `published` is what the step took from the bus
    bool step(double dt, or_violation* out, double* taken) {
        if (taken) *taken = 0.0;
        double f = fourier_number(dt);
        if (!std::isfinite(f)) {  // Violation::at (conserved.rs:149-158)
            set_violation(out, "substance has no diffusivity", name, f, f, std::fabs(f), 0.0);
            return false;
        }
        if (f > 0.5 + 1e-12) {
            set_violation(out, "Fourier number", name + " (explicit conduction)", 0.5, f, 0.5, 1e-12);
            return false;
        }
        double capacity = cell_capacity();
        double gained = lumped;
        lumped = 0.0;
        absorbed += gained;
        cells[0] += gained / capacity;
        double got = gained;
        if (!per_cell.empty()) {
            double total = 0.0;
            for (int i = 0; i < n; ++i) {
                cells[i] += per_cell[i] / capacity;
                total += per_cell[i];
            }
            absorbed += total;
            got += total;
            per_cell.clear();
        }
        std::vector<double> previous = cells;
        int last = n - 1;
        for (int i = 0; i <= last; ++i) {
            double left = previous[i > 0 ? i - 1 : 0];
            double right = previous[i + 1 < last ? i + 1 : last];
            cells[i] = previous[i] + f * (left - 2.0 * previous[i] + right);
        }
        if (taken) *taken = got;
        return true;
    }
    or_entry ledger() const {  // lib.rs:629-631
        or_entry e{0.0, 0.0};
        ledger_add(e, stored_heat());
        return e;
    }
};

// ---------------------------------------------------------------------------------------------
// Cavity — pantometry-em/src/cavity.rs (PEC / Magnetic / Open walls, per-cell media,
// obstruct), plus the soft dipole-current extension on one Ez edge.
// ---------------------------------------------------------------------------------------------

struct Medium {
    double eps_r, mu_r, sigma;
    double permittivity() const { return EPSILON_0 * eps_r; }
    double permeability() const { return MU_0 * mu_r; }
    double wave_speed() const { return 1.0 / std::sqrt(permittivity() * permeability()); }
};

enum { CONDUCTING = 0, MAGNETIC = 1, OPEN = 2 };

struct Cavity {
    std::string name;
    int nx, ny, nz;
    double dx;
    Medium medium;
    std::vector<double> ex, ey, ez, hx, hy, hz;
    int boundary[6] = {0, 0, 0, 0, 0, 0};
    std::vector<Medium> cells;
    std::vector<uint8_t> solid;
    bool any_solid = false;
    std::vector<double> eps[3], sigma[3], mu[3];
    bool has_prev = false;
    std::vector<double> pex, pey, pez;
    bool started = false;
    bool has_invariant = false;
    double invariant = 0.0;
    double dissipated = 0.0;
    // Extension: soft current density J(t) [A/m²] on the Ez edge `source_edge`, sampled at the
    // half step, with the work it does on the field kept beside the invariant.
    long long source_edge = -1;
    std::vector<double> current;
    long long steps_taken = 0;
    double source_work = 0.0;
    // The invariant of step n is taken before step n's electric update, so the work that
    // update does belongs against step n+1's invariant: the ledger books the work through the
    // previous step.
    double work_booked = 0.0;

    size_t iex(int i, int j, int k) const { return i + (size_t)nx * (j + (size_t)(ny + 1) * k); }
    size_t iey(int i, int j, int k) const { return i + (size_t)(nx + 1) * (j + (size_t)ny * k); }
    size_t iez(int i, int j, int k) const { return i + (size_t)(nx + 1) * (j + (size_t)(ny + 1) * k); }
    size_t ihx(int i, int j, int k) const { return i + (size_t)(nx + 1) * (j + (size_t)ny * k); }
    size_t ihy(int i, int j, int k) const { return i + (size_t)nx * (j + (size_t)(ny + 1) * k); }
    size_t ihz(int i, int j, int k) const { return i + (size_t)nx * (j + (size_t)ny * k); }

    // cavity.rs:348-458
    void refresh_media() {
        auto at = [&](long i, long j, long k) -> size_t {
            auto c = [](long v, long n) { return (size_t)std::min(std::max(v, 0L), n - 1); };
            return c(i, nx) + (size_t)nx * (c(j, ny) + (size_t)ny * c(k, nz));
        };
        auto mean4 = [&](const size_t* of, int which_prop) {
            double s = -0.0;
            for (int q = 0; q < 4; ++q) {
                const Medium& m = cells[of[q]];
                double v = which_prop == 0 ? m.permittivity() : std::max(m.sigma, 0.0);
                s += v;
            }
            return s / 4.0;
        };
        for (int q = 0; q < 3; ++q) { eps[q].clear(); sigma[q].clear(); mu[q].clear(); }
        eps[0].assign(ex.size(), 0.0); eps[1].assign(ey.size(), 0.0); eps[2].assign(ez.size(), 0.0);
        sigma[0] = eps[0]; sigma[1] = eps[1]; sigma[2] = eps[2];
        for (long k = 0; k <= nz; ++k)
            for (long j = 0; j <= ny; ++j)
                for (long i = 0; i <= nx; ++i) {
                    if (i < nx) {
                        size_t of[4] = {at(i, j - 1, k - 1), at(i, j, k - 1), at(i, j - 1, k), at(i, j, k)};
                        size_t idx = iex(i, j, k);
                        eps[0][idx] = mean4(of, 0);
                        sigma[0][idx] = mean4(of, 1);
                    }
                    if (j < ny) {
                        size_t of[4] = {at(i - 1, j, k - 1), at(i, j, k - 1), at(i - 1, j, k), at(i, j, k)};
                        size_t idx = iey(i, j, k);
                        eps[1][idx] = mean4(of, 0);
                        sigma[1][idx] = mean4(of, 1);
                    }
                    if (k < nz) {
                        size_t of[4] = {at(i - 1, j - 1, k), at(i, j - 1, k), at(i - 1, j, k), at(i, j, k)};
                        size_t idx = iez(i, j, k);
                        eps[2][idx] = mean4(of, 0);
                        sigma[2][idx] = mean4(of, 1);
                    }
                }
        mu[0].assign(hx.size(), 0.0); mu[1].assign(hy.size(), 0.0); mu[2].assign(hz.size(), 0.0);
        auto mean2 = [&](size_t a, size_t b) {
            double s = -0.0;
            s += cells[a].permeability();
            s += cells[b].permeability();
            return s / 2.0;
        };
        for (long k = 0; k < nz; ++k)
            for (long j = 0; j < ny; ++j)
                for (long i = 0; i < nx; ++i) {
                    mu[0][ihx(i, j, k)] = mean2(at(i - 1, j, k), at(i, j, k));
                    mu[1][ihy(i, j, k)] = mean2(at(i, j - 1, k), at(i, j, k));
                    mu[2][ihz(i, j, k)] = mean2(at(i, j, k - 1), at(i, j, k));
                }
        double fallback = medium.permeability();
        for (int q = 0; q < 3; ++q)
            for (double& v : mu[q])
                if (v <= 0.0) v = fallback;
    }

    // cavity.rs:304-331
    void enforce_solid() {
        if (!any_solid) return;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    if (!solid[i + (size_t)nx * (j + (size_t)ny * k)]) continue;
                    const int d[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
                    for (auto& q : d) ex[iex(i, j + q[0], k + q[1])] = 0.0;
                    for (auto& q : d) ey[iey(i + q[0], j, k + q[1])] = 0.0;
                    for (auto& q : d) ez[iez(i + q[0], j + q[1], k)] = 0.0;
                }
    }

    // cavity.rs:1239-1293
    void enforce_walls_where(int kind) {
        for (int w = 0; w < 6; ++w) {
            if (boundary[w] != kind) continue;
            if (w < 2) {
                int edge = w == 0 ? 0 : nx;
                for (int k = 0; k <= nz; ++k) for (int j = 0; j < ny; ++j) ey[iey(edge, j, k)] = 0.0;
                for (int k = 0; k < nz; ++k) for (int j = 0; j <= ny; ++j) ez[iez(edge, j, k)] = 0.0;
            } else if (w < 4) {
                int edge = w == 2 ? 0 : ny;
                for (int k = 0; k <= nz; ++k) for (int i = 0; i < nx; ++i) ex[iex(i, edge, k)] = 0.0;
                for (int k = 0; k < nz; ++k) for (int i = 0; i <= nx; ++i) ez[iez(i, edge, k)] = 0.0;
            } else {
                int edge = w == 4 ? 0 : nz;
                for (int j = 0; j <= ny; ++j) for (int i = 0; i < nx; ++i) ex[iex(i, j, edge)] = 0.0;
                for (int j = 0; j < ny; ++j) for (int i = 0; i <= nx; ++i) ey[iey(i, j, edge)] = 0.0;
            }
        }
    }

    // cavity.rs:1296-1343
    void enforce_walls() {
        for (int k = 0; k <= nz; ++k) for (int i = 0; i < nx; ++i) { ex[iex(i, 0, k)] = 0.0; ex[iex(i, ny, k)] = 0.0; }
        for (int j = 0; j <= ny; ++j) for (int i = 0; i < nx; ++i) { ex[iex(i, j, 0)] = 0.0; ex[iex(i, j, nz)] = 0.0; }
        for (int k = 0; k <= nz; ++k) for (int j = 0; j < ny; ++j) { ey[iey(0, j, k)] = 0.0; ey[iey(nx, j, k)] = 0.0; }
        for (int j = 0; j < ny; ++j) for (int i = 0; i <= nx; ++i) { ey[iey(i, j, 0)] = 0.0; ey[iey(i, j, nz)] = 0.0; }
        for (int k = 0; k < nz; ++k) for (int j = 0; j <= ny; ++j) { ez[iez(0, j, k)] = 0.0; ez[iez(nx, j, k)] = 0.0; }
        for (int k = 0; k < nz; ++k) for (int i = 0; i <= nx; ++i) { ez[iez(i, 0, k)] = 0.0; ez[iez(i, ny, k)] = 0.0; }
    }

    // cavity.rs:1170-1236
    void mirror_magnetic_walls() {
        for (int w = 0; w < 6; ++w) {
            if (boundary[w] != MAGNETIC) continue;
            if (w < 2) {
                int edge = w == 0 ? 0 : nx, inner = w == 0 ? 1 : nx - 1;
                for (int k = 0; k <= nz; ++k) for (int j = 0; j < ny; ++j) ey[iey(edge, j, k)] = ey[iey(inner, j, k)];
                for (int k = 0; k < nz; ++k) for (int j = 0; j <= ny; ++j) ez[iez(edge, j, k)] = ez[iez(inner, j, k)];
            } else if (w < 4) {
                int edge = w == 2 ? 0 : ny, inner = w == 2 ? 1 : ny - 1;
                for (int k = 0; k <= nz; ++k) for (int i = 0; i < nx; ++i) ex[iex(i, edge, k)] = ex[iex(i, inner, k)];
                for (int k = 0; k < nz; ++k) for (int i = 0; i <= nx; ++i) ez[iez(i, edge, k)] = ez[iez(i, inner, k)];
            } else {
                int edge = w == 4 ? 0 : nz, inner = w == 4 ? 1 : nz - 1;
                for (int j = 0; j <= ny; ++j) for (int i = 0; i < nx; ++i) ex[iex(i, j, edge)] = ex[iex(i, j, inner)];
                for (int j = 0; j < ny; ++j) for (int i = 0; i <= nx; ++i) ey[iey(i, j, edge)] = ey[iey(i, j, inner)];
            }
        }
    }

    // cavity.rs:588-591: Mur's coefficient (c·dt − dx)/(c·dt + dx)
    double mur_coefficient(double dt) const {
        const double c_dt = medium.wave_speed() * dt;
        return (c_dt - dx) / (c_dt + dx);
    }

    // cavity.rs:1074-1164
    void apply_boundaries(double dt) {
        double kk = mur_coefficient(dt);
        bool prev = has_prev;
        has_prev = false;
        enforce_walls_where(CONDUCTING);
        mirror_magnetic_walls();
        if (!prev) enforce_walls_where(OPEN);
        if (prev) {
            for (int w = 0; w < 6; ++w) {
                if (boundary[w] != OPEN) continue;
                if (w < 2) {
                    int edge = w == 0 ? 0 : nx, inner = w == 0 ? 1 : nx - 1;
                    for (int q = 0; q <= nz; ++q) for (int j = 0; j < ny; ++j) {
                        size_t a = iey(edge, j, q), b = iey(inner, j, q);
                        ey[a] = pey[b] + kk * (ey[b] - pey[a]);
                    }
                    for (int q = 0; q < nz; ++q) for (int j = 0; j <= ny; ++j) {
                        size_t a = iez(edge, j, q), b = iez(inner, j, q);
                        ez[a] = pez[b] + kk * (ez[b] - pez[a]);
                    }
                } else if (w < 4) {
                    int edge = w == 2 ? 0 : ny, inner = w == 2 ? 1 : ny - 1;
                    for (int q = 0; q <= nz; ++q) for (int i = 0; i < nx; ++i) {
                        size_t a = iex(i, edge, q), b = iex(i, inner, q);
                        ex[a] = pex[b] + kk * (ex[b] - pex[a]);
                    }
                    for (int q = 0; q < nz; ++q) for (int i = 0; i <= nx; ++i) {
                        size_t a = iez(i, edge, q), b = iez(i, inner, q);
                        ez[a] = pez[b] + kk * (ez[b] - pez[a]);
                    }
                } else {
                    int edge = w == 4 ? 0 : nz, inner = w == 4 ? 1 : nz - 1;
                    for (int j = 0; j <= ny; ++j) for (int i = 0; i < nx; ++i) {
                        size_t a = iex(i, j, edge), b = iex(i, j, inner);
                        ex[a] = pex[b] + kk * (ex[b] - pex[a]);
                    }
                    for (int j = 0; j < ny; ++j) for (int i = 0; i <= nx; ++i) {
                        size_t a = iey(i, j, edge), b = iey(i, j, inner);
                        ey[a] = pey[b] + kk * (ey[b] - pey[a]);
                    }
                }
            }
        }
        pex = ex; pey = ey; pez = ez;
        has_prev = true;
    }

    // cavity.rs:1346-1379
    void advance_magnetic(double dt) {
        double g = dt / dx;
        for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i <= nx; ++i) {
            double curl = (ez[iez(i, j + 1, k)] - ez[iez(i, j, k)]) - (ey[iey(i, j, k + 1)] - ey[iey(i, j, k)]);
            size_t idx = ihx(i, j, k);
            hx[idx] -= g / mu[0][idx] * curl;
        }
        for (int k = 0; k < nz; ++k) for (int j = 0; j <= ny; ++j) for (int i = 0; i < nx; ++i) {
            double curl = (ex[iex(i, j, k + 1)] - ex[iex(i, j, k)]) - (ez[iez(i + 1, j, k)] - ez[iez(i, j, k)]);
            size_t idx = ihy(i, j, k);
            hy[idx] -= g / mu[1][idx] * curl;
        }
        for (int k = 0; k <= nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
            double curl = (ey[iey(i + 1, j, k)] - ey[iey(i, j, k)]) - (ex[iex(i, j + 1, k)] - ex[iex(i, j, k)]);
            size_t idx = ihz(i, j, k);
            hz[idx] -= g / mu[2][idx] * curl;
        }
    }

    // cavity.rs:1383-1452, plus the soft current on one Ez edge (extension).
    double advance_electric(double dt, double current_density) {
        auto coefficients = [&](double e, double s, double& decay, double& gain) {
            double half = s * dt / (2.0 * e);
            decay = (1.0 - half) / (1.0 + half);
            gain = (dt / (e * dx)) / (1.0 + half);
        };
        double lost = 0.0;
        double volume = dx * (dx * dx);  // dx.powi(3)
        for (int k = 1; k < nz; ++k) for (int j = 1; j < ny; ++j) for (int i = 0; i < nx; ++i) {
            double curl = (hz[ihz(i, j, k)] - hz[ihz(i, j - 1, k)]) - (hy[ihy(i, j, k)] - hy[ihy(i, j, k - 1)]);
            size_t idx = iex(i, j, k);
            double e = eps[0][idx], s = sigma[0][idx], decay, gain;
            coefficients(e, s, decay, gain);
            double before = ex[idx];
            ex[idx] = decay * before + gain * curl;
            double mid = 0.5 * (before + ex[idx]);
            lost += s * mid * mid * dt * volume;
        }
        for (int k = 1; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 1; i < nx; ++i) {
            double curl = (hx[ihx(i, j, k)] - hx[ihx(i, j, k - 1)]) - (hz[ihz(i, j, k)] - hz[ihz(i - 1, j, k)]);
            size_t idx = iey(i, j, k);
            double e = eps[1][idx], s = sigma[1][idx], decay, gain;
            coefficients(e, s, decay, gain);
            double before = ey[idx];
            ey[idx] = decay * before + gain * curl;
            double mid = 0.5 * (before + ey[idx]);
            lost += s * mid * mid * dt * volume;
        }
        for (int k = 0; k < nz; ++k) for (int j = 1; j < ny; ++j) for (int i = 1; i < nx; ++i) {
            double curl = (hy[ihy(i, j, k)] - hy[ihy(i - 1, j, k)]) - (hx[ihx(i, j, k)] - hx[ihx(i, j - 1, k)]);
            size_t idx = iez(i, j, k);
            double e = eps[2][idx], s = sigma[2][idx], decay, gain;
            coefficients(e, s, decay, gain);
            double before = ez[idx];
            double after = decay * before + gain * curl;
            if ((long long)idx == source_edge) {
                // soft current: ε dE/dt = ∇×H − J, semi-implicit like the σ term
                after = after - (dt / e) / (1.0 + (s * dt / (2.0 * e))) * current_density;
                source_work += -(dt * volume) * current_density * (0.5 * (before + after));
            }
            ez[idx] = after;
            double mid = 0.5 * (before + ez[idx]);
            lost += s * mid * mid * dt * volume;
        }
        return std::max(lost, 0.0);
    }

    // cavity.rs:776-797 weighted_square_with, 766-772 weight
    static double wsq(const std::vector<double>& f, const std::vector<double>& m, int cx, int cy, int cz,
                      bool n0, bool n1, bool n2) {
        auto weight = [](int index, int last, bool node) { return (node && (index == 0 || index == last)) ? 0.5 : 1.0; };
        double total = 0.0;
        for (int k = 0; k < cz; ++k) for (int j = 0; j < cy; ++j) for (int i = 0; i < cx; ++i) {
            double w = weight(i, cx - 1, n0) * weight(j, cy - 1, n1) * weight(k, cz - 1, n2);
            size_t idx = i + (size_t)cx * (j + (size_t)cy * k);
            total += w * m[idx] * f[idx] * f[idx];
        }
        return total;
    }

    // cavity.rs:824-847
    double electric_energy() const {
        double v = dx * (dx * dx);
        double sum = wsq(ex, eps[0], nx, ny + 1, nz + 1, false, true, true) +
                     wsq(ey, eps[1], nx + 1, ny, nz + 1, true, false, true) +
                     wsq(ez, eps[2], nx + 1, ny + 1, nz, true, true, false);
        return 0.5 * sum * v;
    }

    // cavity.rs:919-940
    double magnetic_energy() const {
        double v = dx * (dx * dx);
        double sum = wsq(hx, mu[0], nx + 1, ny, nz, true, false, false) +
                     wsq(hy, mu[1], nx, ny + 1, nz, false, true, false) +
                     wsq(hz, mu[2], nx, ny, nz + 1, false, false, true);
        return 0.5 * sum * v;
    }

    // cavity.rs:854-905
    double paired_magnetic_energy(const std::vector<double>& bx, const std::vector<double>& by,
                                  const std::vector<double>& bz) const {
        double v = dx * (dx * dx);
        auto pair = [](const std::vector<double>& now, const std::vector<double>& was, const std::vector<double>& m,
                       int cx, int cy, int cz, bool e0, bool e1, bool e2) {
            double sum = 0.0;
            for (int k = 0; k < cz; ++k) for (int j = 0; j < cy; ++j) for (int i = 0; i < cx; ++i) {
                size_t at = i + (size_t)cx * (j + (size_t)cy * k);
                double w = 1.0;
                if (e0 && (i == 0 || i + 1 == cx)) w *= 0.5;
                if (e1 && (j == 0 || j + 1 == cy)) w *= 0.5;
                if (e2 && (k == 0 || k + 1 == cz)) w *= 0.5;
                sum += w * m[at] * now[at] * was[at];
            }
            return sum;
        };
        return 0.5 * v * (pair(hx, bx, mu[0], nx + 1, ny, nz, true, false, false) +
                          pair(hy, by, mu[1], nx, ny + 1, nz, false, true, false) +
                          pair(hz, bz, mu[2], nx, ny, nz + 1, false, false, true));
    }

    double energy() const { return electric_energy() + magnetic_energy(); }
    double invariant_energy() const { return has_invariant ? invariant : energy(); }

    double courant_limit() const { return COURANT_3D * dx / medium.wave_speed(); }

    // cavity.rs:559-563 with size() (639-647): f_c = (c/2)·√((m/a)² + (n/b)²), a = nx·dx, b = ny·dx
    double cutoff_frequency(int m, int n) const {
        const double a = (double)m / ((double)nx * dx), b = (double)n / ((double)ny * dx);
        return 0.5 * medium.wave_speed() * std::sqrt(a * a + b * b);
    }

    // cavity.rs:488-521: Ey from the envelope at its edges (i·dx, (j+½)·dx, k·dx), Hx = −envelope/η
    // at its faces with z moved on by c·dt/2 (the caller evaluates the envelope at both sets of
    // points, in the layouts of ey and hx), then the conducting walls' tangential E cleared; the
    // next step starts the leapfrog as already begun.
    void launch_along_z(const double* ey_env, const double* hx_env) {
        const double eta = std::sqrt(medium.permeability() / medium.permittivity());
        for (size_t c = 0; c < ey.size(); ++c) ey[c] = ey_env[c];
        for (size_t c = 0; c < hx.size(); ++c) hx[c] = -hx_env[c] / eta;
        enforce_walls_where(CONDUCTING);
        started = true;
    }

    // cavity.rs:537-548: a soft source, `add` (at (i·dx, (j+½)·dx), i fastest over nx+1, then j over
    // ny) added to Ey on the plane k = min(plane, nz), then the conducting walls' tangential E cleared.
    void impress(int plane, const double* add) {
        const int k = std::min(plane, nz);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i <= nx; ++i) ey[iey(i, j, k)] += add[i + (size_t)(nx + 1) * j];
        enforce_walls_where(CONDUCTING);
    }

    // cavity.rs:675-732
    void release_mode(int mm, int pm, double amplitude, double dt) {
        double m = (double)std::max(mm, 1), pp = (double)std::max(pm, 1);
        double sx = (double)nx * dx, sz = (double)nz * dx;
        double kxv = M_PI * m / sx, kzv = M_PI * pp / sz;
        std::fill(ex.begin(), ex.end(), 0.0); std::fill(ey.begin(), ey.end(), 0.0);
        std::fill(ez.begin(), ez.end(), 0.0); std::fill(hx.begin(), hx.end(), 0.0);
        std::fill(hy.begin(), hy.end(), 0.0); std::fill(hz.begin(), hz.end(), 0.0);
        for (int k = 0; k <= nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i <= nx; ++i) {
            double x = (double)i * dx, z = (double)k * dx;
            ey[iey(i, j, k)] = amplitude * std::sin(kxv * x) * std::sin(kzv * z);
        }
        enforce_walls();
        advance_magnetic(-0.5 * dt);
        enforce_walls();
        started = true;
        std::vector<double> kx_ = hx, ky_ = hy, kz_ = hz;
        advance_magnetic(dt);
        invariant = electric_energy() + paired_magnetic_energy(kx_, ky_, kz_);
        has_invariant = true;
        hx = kx_; hy = ky_; hz = kz_;
    }

    // cavity.rs:1468-1501
    bool step(double dt, or_violation* out) {
        double h = dt;
        double limit = courant_limit();
        if (h > limit) {
            set_violation(out, "Courant number", name, limit, h, limit, 0.0);
            return false;
        }
        if (!started) {
            advance_magnetic(0.5 * h);
            started = true;
        }
        std::vector<double> bx = hx, by = hy, bz = hz;
        advance_magnetic(h);
        invariant = electric_energy() + paired_magnetic_energy(bx, by, bz);
        has_invariant = true;
        double j = (source_edge >= 0 && steps_taken < (long long)current.size()) ? current[steps_taken] : 0.0;
        work_booked = source_work;
        dissipated += advance_electric(h, j);
        apply_boundaries(h);
        enforce_solid();
        steps_taken += 1;
        return true;
    }

    or_entry ledger() const {  // cavity.rs:1520-1524 (+ the source work, when a source is set)
        or_entry e{0.0, 0.0};
        ledger_add(e, invariant_energy());
        ledger_add(e, dissipated);
        if (source_edge >= 0) ledger_add(e, -work_booked);
        return e;
    }

    double peak_magnetic_divergence() const {  // cavity.rs:979-993
        double worst = 0.0;
        for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
            double d = (hx[ihx(i + 1, j, k)] - hx[ihx(i, j, k)]) + (hy[ihy(i, j + 1, k)] - hy[ihy(i, j, k)]) +
                       (hz[ihz(i, j, k + 1)] - hz[ihz(i, j, k)]);
            worst = rmax(worst, std::fabs(d));
        }
        return worst;
    }
};

// ---------------------------------------------------------------------------------------------
// Rng — pantometry-core/src/rng.rs:36-100
// ---------------------------------------------------------------------------------------------

inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

}  // namespace

// =============================================================================================
// C API (ctypes)
// =============================================================================================
extern "C" {

// ---- Rng ----
uint64_t or_rng_new(uint64_t seed) { return seed == 0 ? 0x9E3779B97F4A7C15ULL : seed; }
uint64_t or_rng_for_index(uint64_t seed, uint64_t index) { return or_rng_new(mix64(seed ^ mix64(index))); }
uint64_t or_rng_next_u64(uint64_t* state) {
    uint64_t x = *state;
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    *state = x;
    return x * 0x2545F4914F6CDD1DULL;
}
double or_rng_unit(uint64_t* state) { return (double)(or_rng_next_u64(state) >> 11) / (double)(1ULL << 53); }
double or_rng_range(uint64_t* state, double lo, double hi) { return lo + (hi - lo) * or_rng_unit(state); }
// rng.rs:296-308 digest of 10 000 draws
uint64_t or_rng_digest(uint64_t seed, int draws) {
    uint64_t s = or_rng_new(seed), hash = 0;
    for (int d = 0; d < draws; ++d) {
        uint64_t rot = (hash << 7) | (hash >> 57);
        hash = (rot * 0x100000001B3ULL) ^ (uint64_t)(or_rng_unit(&s) * (double)(1ULL << 53));
    }
    return hash;
}

// ---- Ledger / audit ----
int or_audit_energy(const char* site, double b_total, double b_scale, double a_total, double a_scale, double tol,
                    or_violation* out) {
    return audit_energy(site, or_entry{b_total, b_scale}, or_entry{a_total, a_scale}, tol, out) ? 0 : 1;
}

// ---- Solid3D ----
void* or_heat_new(const char* name, int nx, int ny, int nz, double dx, double density, double conductivity,
                  double specific_heat, double emissivity, int thermal, double initial) {
    Heat* h = new Heat();
    h->name = name ? name : "block";
    h->nx = std::max(nx, 1); h->ny = std::max(ny, 1); h->nz = std::max(nz, 1);
    h->dx = dx;
    h->reference = initial;
    h->mats.push_back(Material{density, conductivity, specific_heat, emissivity, thermal});
    h->which.assign(h->n(), 0);
    h->cells.assign(h->n(), initial);
    h->saved = h->cells;
    h->resolve();
    return h;
}
void or_heat_free(void* p) { delete (Heat*)p; }
void or_heat_losing_from(void* p, int face, double ambient, double convection, double area) {
    Heat* h = (Heat*)p;
    h->exposed[face] = true;
    h->env[face] = Env{ambient, convection, area};
    h->resolve();
}
// solid.rs:519-543 `fill`: cells where mask != 0 take the substance.
void or_heat_fill(void* p, double density, double conductivity, double specific_heat, double emissivity, int thermal,
                  const uint8_t* mask) {
    Heat* h = (Heat*)p;
    Material m{density, conductivity, specific_heat, emissivity, thermal};
    int id = -1;
    for (size_t q = 0; q < h->mats.size(); ++q) {
        const Material& o = h->mats[q];
        if (o.density == m.density && o.conductivity == m.conductivity && o.specific_heat == m.specific_heat &&
            o.emissivity == m.emissivity && o.thermal == m.thermal) { id = (int)q; break; }
    }
    if (id < 0) { h->mats.push_back(m); id = (int)h->mats.size() - 1; }
    for (size_t c = 0; c < h->n(); ++c)
        if (mask[c]) h->which[c] = (uint32_t)id;
    h->resolve();
}
// solid.rs:986-1005 `empty`: cells where mask != 0 become void.
void or_heat_empty(void* p, const uint8_t* mask) {
    Heat* h = (Heat*)p;
    for (size_t c = 0; c < h->n(); ++c)
        if (mask[c]) h->vd[c] = 1;
    h->resolve();
}
void or_heat_dissipating(void* p, double watts, const uint8_t* mask) { ((Heat*)p)->dissipating(watts, mask); }
// solid.rs:1118-1126: watts summed over the cells, and the joules generated over the run
double or_heat_generated_power(void* p) {
    double s = -0.0;
    for (double w : ((Heat*)p)->source) s += w;
    return s;
}
double or_heat_generated_energy(void* p) { return ((Heat*)p)->supplied; }
// The gap pairs in the reference's order: up to `cap` of them into a, b, coefficient; the count.
long long or_heat_gaps(void* p, long long* a, long long* b, double* coefficient, long long cap) {
    Heat* h = (Heat*)p;
    for (size_t q = 0; q < h->gaps.size() && (long long)q < cap; ++q) {
        a[q] = (long long)h->gaps[q].a;
        b[q] = (long long)h->gaps[q].b;
        coefficient[q] = h->gaps[q].coefficient;
    }
    return (long long)h->gaps.size();
}
void or_heat_set_cells(void* p, const double* t) { Heat* h = (Heat*)p; std::memcpy(h->cells.data(), t, h->n() * 8); }
void or_heat_get_cells(void* p, double* t) { Heat* h = (Heat*)p; std::memcpy(t, h->cells.data(), h->n() * 8); }
void or_heat_get_coefficients(void* p, double* kx, double* ky, double* kz, double* mobility, double* capacity) {
    Heat* h = (Heat*)p;
    if (kx) std::memcpy(kx, h->kx.data(), h->kx.size() * 8);
    if (ky) std::memcpy(ky, h->ky.data(), h->ky.size() * 8);
    if (kz) std::memcpy(kz, h->kz.data(), h->kz.size() * 8);
    if (mobility) std::memcpy(mobility, h->mobility.data(), h->mobility.size() * 8);
    if (capacity) std::memcpy(capacity, h->capacity.data(), h->capacity.size() * 8);
}
double or_heat_max_stable_dt(void* p) {
    double rate = ((Heat*)p)->worst_rate_now();
    if (std::isnan(rate)) return INF;
    return 1.0 / rate;
}
int or_heat_step(void* p, double dt, int nsteps, or_violation* out) {
    Heat* h = (Heat*)p;
    for (int s = 0; s < nsteps; ++s)
        if (!h->step(dt, out)) return 1;
    return 0;
}
void or_heat_ledger(void* p, double* total, double* scale, double* stored, double* lost) {
    Heat* h = (Heat*)p;
    or_entry e = h->ledger();
    if (total) *total = e.total;
    if (scale) *scale = e.scale;
    if (stored) *stored = h->stored_heat();
    if (lost) *lost = h->lost;
}
void or_heat_absorb(void* p, double joules) { ((Heat*)p)->absorb(joules); }
void or_heat_checkpoint(void* p) { Heat* h = (Heat*)p; h->saved = h->cells; h->saved_lost = h->lost; h->saved_supplied = h->supplied; }
void or_heat_restore(void* p) { Heat* h = (Heat*)p; h->cells = h->saved; h->lost = h->saved_lost; h->supplied = h->saved_supplied; }
// sim.rs:947-965 + 968-1111 with one books-balancing domain, Staggered schedule, empty bus.
int or_heat_advance(void* p, double dt, int nsteps, double tol, or_violation* out) {
    Heat* h = (Heat*)p;
    for (int s = 0; s < nsteps; ++s) {
        or_entry before = h->ledger();
        or_entry books = h->ledger();
        if (!h->step(dt, out)) return 1;
        if (!attribute_energy(h->name, books, h->ledger(), tol, out)) return 1;
        or_entry after = h->ledger();
        if (!audit_energy("simulation", before, after, tol, out)) return 1;
    }
    return 0;
}
// solid.rs:1478-1500 `release_mode`; 1508-1535 `mode_amplitude`; 1454-1472 amplification.
void or_heat_release_mode(void* p, int a, int b, int c, double mean, double amplitude) {
    Heat* h = (Heat*)p;
    auto phase = [](int m, int n, int i) { return n <= 1 ? 1.0 : std::cos((double)m * M_PI * ((double)i + 0.5) / (double)n); };
    for (int k = 0; k < h->nz; ++k) for (int j = 0; j < h->ny; ++j) for (int i = 0; i < h->nx; ++i) {
        size_t idx = i + (size_t)h->nx * (j + (size_t)h->ny * k);
        h->cells[idx] = mean + amplitude * phase(a, h->nx, i) * phase(b, h->ny, j) * phase(c, h->nz, k);
    }
    h->saved = h->cells;
}
double or_heat_mode_amplitude(void* p, int a, int b, int c) {
    Heat* h = (Heat*)p;
    auto phase = [](int m, int n, int i) { return n <= 1 ? 1.0 : std::cos((double)m * M_PI * ((double)i + 0.5) / (double)n); };
    int ms[3] = {a, b, c}, ns[3] = {h->nx, h->ny, h->nz};
    double norm = 1.0;
    for (int q = 0; q < 3; ++q) norm *= (ns[q] <= 1 || ms[q] == 0) ? 1.0 : 0.5;
    double sum = 0.0;
    for (int k = 0; k < h->nz; ++k) for (int j = 0; j < h->ny; ++j) for (int i = 0; i < h->nx; ++i) {
        size_t idx = i + (size_t)h->nx * (j + (size_t)h->ny * k);
        sum += h->cells[idx] * phase(a, h->nx, i) * phase(b, h->ny, j) * phase(c, h->nz, k);
    }
    return sum / ((double)h->n() * norm);
}
double or_heat_mode_amplification(void* p, int a, int b, int c, double dt) {
    Heat* h = (Heat*)p;
    const Material& m = h->mats[0];
    if (!m.thermal) return INF;
    double alpha = m.conductivity / (m.density * m.specific_heat);  // substance.rs:211-216
    double f = alpha * dt / (h->dx * h->dx);
    auto term = [](int mm, int n) {
        if (n <= 1) return 0.0;
        double s = std::sin((double)mm * M_PI / (2.0 * (double)n));
        return -4.0 * s * s;
    };
    return 1.0 + f * (term(a, h->nx) + term(b, h->ny) + term(c, h->nz));
}

// ---- Hall ----
void* or_hall_new(const char* name, double width, double height, double depth, int across, double speed,
                  double density) {
    Hall* h = new Hall();
    h->name = name ? name : "hall";
    int nx = std::max(across, 2);
    double dx = std::max(width / (double)(nx - 1), std::numeric_limits<double>::min());
    auto quantise = [&](double l) { return (int)std::max(std::round(l / dx), 0.0) + 1; };
    h->nx = nx; h->ny = quantise(height); h->nz = quantise(depth);
    h->dx = dx; h->speed = speed; h->density = density;
    size_t nodes = (size_t)h->nx * h->ny * h->nz;
    h->p.assign(nodes, 0.0); h->pp.assign(nodes, 0.0);
    h->vx.assign((size_t)(h->nx - 1) * h->ny * h->nz, 0.0);
    h->vy.assign((size_t)h->nx * (h->ny - 1) * h->nz, 0.0);
    h->vz.assign((size_t)h->nx * h->ny * (h->nz - 1), 0.0);
    return h;
}
void or_hall_free(void* p) { delete (Hall*)p; }
void or_hall_nodes(void* p, int* nx, int* ny, int* nz, double* dx) {
    Hall* h = (Hall*)p; *nx = h->nx; *ny = h->ny; *nz = h->nz; *dx = h->dx;
}
// hall.rs:166-184 `released_from`, with the profile already sampled at the nodes.
void or_hall_release(void* p, const double* pressure) {
    Hall* h = (Hall*)p;
    std::memcpy(h->p.data(), pressure, h->p.size() * 8);
    h->pp = h->p;
    std::fill(h->vx.begin(), h->vx.end(), 0.0);
    std::fill(h->vy.begin(), h->vy.end(), 0.0);
    std::fill(h->vz.begin(), h->vz.end(), 0.0);
    h->staggered = false;
    h->offset = 0.0;
    h->datum = h->invariant_si();
}
// hall.rs:190-210
void or_hall_release_mode(void* p, int a, int b, int c, double amplitude) {
    Hall* h = (Hall*)p;
    double lx = (double)(h->nx - 1) * h->dx, ly = (double)(h->ny - 1) * h->dx, lz = (double)(h->nz - 1) * h->dx;
    auto phase = [](int n, double x, double l) { return l > 0.0 ? std::cos((double)n * M_PI * x / l) : 1.0; };
    std::vector<double> prof(h->p.size());
    for (int k = 0; k < h->nz; ++k) for (int j = 0; j < h->ny; ++j) for (int i = 0; i < h->nx; ++i) {
        double x = (double)i * h->dx, y = (double)j * h->dx, z = (double)k * h->dx;
        prof[h->at(i, j, k)] = amplitude * phase(a, x, lx) * phase(b, y, ly) * phase(c, z, lz);
    }
    or_hall_release(p, prof.data());
}
void or_hall_set_source(void* p, long long node, const double* wave, long long n) {
    Hall* h = (Hall*)p;
    h->source_node = node;
    h->wave.assign(wave, wave + n);
}
int or_hall_step(void* p, double dt, int nsteps, or_violation* out) {
    Hall* h = (Hall*)p;
    for (int s = 0; s < nsteps; ++s)
        if (!h->step(dt, out)) return 1;
    return 0;
}
int or_hall_advance(void* p, double dt, int nsteps, double tol, or_violation* out) {
    Hall* h = (Hall*)p;
    for (int s = 0; s < nsteps; ++s) {
        or_entry before = h->ledger();
        or_entry books = h->ledger();
        if (!h->step(dt, out)) return 1;
        if (!attribute_energy(h->name, books, h->ledger(), tol, out)) return 1;
        or_entry after = h->ledger();
        if (!audit_energy("simulation", before, after, tol, out)) return 1;
    }
    return 0;
}
void or_hall_get(void* p, double* pr, double* pp, double* vx, double* vy, double* vz) {
    Hall* h = (Hall*)p;
    if (pr) std::memcpy(pr, h->p.data(), h->p.size() * 8);
    if (pp) std::memcpy(pp, h->pp.data(), h->pp.size() * 8);
    if (vx) std::memcpy(vx, h->vx.data(), h->vx.size() * 8);
    if (vy) std::memcpy(vy, h->vy.data(), h->vy.size() * 8);
    if (vz) std::memcpy(vz, h->vz.data(), h->vz.size() * 8);
}
void or_hall_ledger(void* p, double* total, double* scale, double* invariant, double* offset, double* injected) {
    Hall* h = (Hall*)p;
    or_entry e = h->ledger();
    if (total) *total = e.total;
    if (scale) *scale = e.scale;
    if (invariant) *invariant = h->invariant_si();
    if (offset) *offset = h->offset;
    if (injected) *injected = h->injected;
}
double or_hall_max_stable_dt(void* p) {
    Hall* h = (Hall*)p;
    const double c = h->max_speed();
    if (c <= 0.0) return INF;
    return h->dx / (c * std::sqrt(3.0));
}
// Extension: one speed per cubic block of `block` nodes a side, blocks in x-fastest order; the
// datum of the present state is re-taken under the new weights.
void or_hall_set_speed_blocks(void* p, int block, const double* speeds, long long n) {
    Hall* h = (Hall*)p;
    h->block = block;
    h->nbx = (h->nx + block - 1) / block;
    h->nby = (h->ny + block - 1) / block;
    h->speeds.assign(speeds, speeds + n);
    if (!h->staggered) h->datum = h->invariant_si();
}
void or_hall_checkpoint(void* p) {
    Hall* h = (Hall*)p;
    h->has_saved = true; h->sp = h->p; h->svx = h->vx; h->svy = h->vy; h->svz = h->vz; h->s_staggered = h->staggered;
}
void or_hall_restore(void* p) {
    Hall* h = (Hall*)p;
    if (!h->has_saved) return;
    h->pp = h->sp; h->p = h->sp; h->vx = h->svx; h->vy = h->svy; h->vz = h->svz; h->staggered = h->s_staggered;
}

// ---- Room ----
// room.rs:90-120: nx = max(across, 3), dx from the width, ny from the height, at least 3
void* or_room_new(const char* name, double width, double height, int across, double depth, double density,
                  double speed) {
    Room* r = new Room();
    r->name = name ? name : "room";
    r->nx = std::max(across, 3);
    r->dx = width / (double)(r->nx - 1);
    r->ny = std::max((int)std::round(height / r->dx) + 1, 3);
    r->speed = speed; r->density = density; r->depth = depth;
    size_t n = (size_t)r->nx * r->ny;
    r->p.assign(n, 0.0); r->pp.assign(n, 0.0);
    r->vx.assign((size_t)(r->nx - 1) * r->ny, 0.0);
    r->vy.assign((size_t)r->nx * (r->ny - 1), 0.0);
    return r;
}
void or_room_free(void* p) { delete (Room*)p; }
void or_room_cells(void* p, int* nx, int* ny, double* dx) {
    Room* r = (Room*)p; *nx = r->nx; *ny = r->ny; *dx = r->dx;
}
// room.rs:140-160 `released_from`, with the profile already sampled at the nodes.
void or_room_release(void* p, const double* pressure) {
    Room* r = (Room*)p;
    std::memcpy(r->p.data(), pressure, r->p.size() * 8);
    r->pp = r->p;
    std::fill(r->vx.begin(), r->vx.end(), 0.0);
    std::fill(r->vy.begin(), r->vy.end(), 0.0);
    r->staggered = false;
    r->offset = 0.0;
    r->datum = r->invariant_si();
}
int or_room_step(void* p, double dt, int nsteps, or_violation* out) {
    Room* r = (Room*)p;
    for (int s = 0; s < nsteps; ++s)
        if (!r->step(dt, out)) return 1;
    return 0;
}
int or_room_advance(void* p, double dt, int nsteps, double tol, or_violation* out) {
    Room* r = (Room*)p;
    for (int s = 0; s < nsteps; ++s) {
        or_entry before = r->ledger();
        or_entry books = r->ledger();
        if (!r->step(dt, out)) return 1;
        if (!attribute_energy(r->name, books, r->ledger(), tol, out)) return 1;
        or_entry after = r->ledger();
        if (!audit_energy("simulation", before, after, tol, out)) return 1;
    }
    return 0;
}
void or_room_get(void* p, double* pr, double* pp, double* vx, double* vy) {
    Room* r = (Room*)p;
    if (pr) std::memcpy(pr, r->p.data(), r->p.size() * 8);
    if (pp) std::memcpy(pp, r->pp.data(), r->pp.size() * 8);
    if (vx) std::memcpy(vx, r->vx.data(), r->vx.size() * 8);
    if (vy) std::memcpy(vy, r->vy.data(), r->vy.size() * 8);
}
void or_room_ledger(void* p, double* total, double* scale, double* invariant, double* offset) {
    Room* r = (Room*)p;
    or_entry e = r->ledger();
    if (total) *total = e.total;
    if (scale) *scale = e.scale;
    if (invariant) *invariant = r->invariant_si();
    if (offset) *offset = r->offset;
}
double or_room_max_stable_dt(void* p) {  // room.rs:361-366
    Room* r = (Room*)p;
    if (r->speed <= 0.0) return INF;
    return r->dx / (r->speed * std::sqrt(2.0));
}
void or_room_checkpoint(void* p) {
    Room* r = (Room*)p;
    r->has_saved = true; r->sp = r->p; r->svx = r->vx; r->svy = r->vy; r->s_staggered = r->staggered;
}
void or_room_restore(void* p) {  // room.rs:495-503: pressure_prev is set to the saved pressure
    Room* r = (Room*)p;
    if (!r->has_saved) return;
    r->pp = r->sp; r->p = r->sp; r->vx = r->svx; r->vy = r->svy; r->staggered = r->s_staggered;
}

// ---- Tube ----
// lib.rs:167-193: cells = max(cells, 3), dx = length/(cells-1), both ends closed
void* or_tube_new(const char* name, double length, int cells, double area, double density, double speed) {
    Tube* t = new Tube();
    t->name = name ? name : "tube";
    t->n = std::max(cells, 3);
    t->dx = length / (double)(t->n - 1);
    t->speed = speed; t->density = density; t->area = area;
    t->p.assign(t->n, 0.0); t->pp.assign(t->n, 0.0); t->v.assign(t->n - 1, 0.0);
    return t;
}
void or_tube_free(void* p) { delete (Tube*)p; }
double or_tube_dx(void* p) { return ((Tube*)p)->dx; }
int or_tube_cells(void* p) { return ((Tube*)p)->n; }
// lib.rs:211-215 `with_ends`: kind 0 closed, 1 open, 2 matched to z (z <= 0: the tube's own)
void or_tube_set_ends(void* p, int left, double zl, int right, double zr) {
    Tube* t = (Tube*)p;
    t->end_kind[0] = left; t->end_z[0] = zl; t->end_kind[1] = right; t->end_z[1] = zr;
}
// lib.rs:226-235 `released_from`, the profile sampled at the cells
void or_tube_release(void* p, const double* pressure) {
    Tube* t = (Tube*)p;
    std::memcpy(t->p.data(), pressure, t->p.size() * 8);
    t->pp = t->p;
    std::fill(t->v.begin(), t->v.end(), 0.0);
    t->staggered = false;
    t->offset = 0.0;
    t->datum = t->invariant_si();
}
int or_tube_step(void* p, double dt, int nsteps, or_violation* out) {
    Tube* t = (Tube*)p;
    for (int s = 0; s < nsteps; ++s)
        if (!t->step(dt, out, nullptr)) return 1;
    return 0;
}
// Simulation::advance over one tube with its books held against what it published
// (sim.rs:1169-1223, `attribute`): the energy plus the published total must hold.
int or_tube_advance(void* p, double dt, int nsteps, double tol, or_violation* out) {
    Tube* t = (Tube*)p;
    for (int s = 0; s < nsteps; ++s) {
        or_entry before = t->ledger();
        double published = 0.0;
        if (!t->step(dt, out, &published)) return 1;
        or_entry after = t->ledger();
        double expected = -published;
        double discrepancy = (after.total - before.total) - expected;
        double scale = rmax(rmax(rmax(rmax(std::fabs(before.total), std::fabs(after.total)), before.scale), after.scale),
                            std::fabs(expected));
        if (scale >= 1e-300 && std::fabs(discrepancy) / scale > tol) {
            set_violation(out, "energy", t->name + " (its own books, against what it moved on the bus)",
                          before.total + expected, after.total, scale, tol);
            return 1;
        }
    }
    return 0;
}
void or_tube_get(void* p, double* pr, double* pp, double* v) {
    Tube* t = (Tube*)p;
    if (pr) std::memcpy(pr, t->p.data(), t->p.size() * 8);
    if (pp) std::memcpy(pp, t->pp.data(), t->pp.size() * 8);
    if (v) std::memcpy(v, t->v.data(), t->v.size() * 8);
}
void or_tube_ledger(void* p, double* total, double* scale, double* invariant, double* offset, double* radiated) {
    Tube* t = (Tube*)p;
    or_entry e = t->ledger();
    if (total) *total = e.total;
    if (scale) *scale = e.scale;
    if (invariant) *invariant = t->invariant_si();
    if (offset) *offset = t->offset;
    if (radiated) *radiated = t->radiated;
}
// lib.rs:495-514
double or_tube_max_stable_dt(void* p) {
    Tube* t = (Tube*)p;
    if (t->speed <= 0.0) return INF;
    double wave = t->dx / t->speed;
    double rc2 = t->density * t->speed * t->speed;
    auto drain = [&](int e) {
        if (t->end_kind[e] == 0) return INF;
        if (t->end_kind[e] == 1) return t->dx * t->impedance() / (2.0 * rc2);
        double zz = t->end_z[e] > 0.0 ? t->end_z[e] : t->impedance();
        return t->dx * zz / (2.0 * rc2);
    };
    return std::min(std::min(wave, drain(0)), drain(1));
}
void or_tube_checkpoint(void* p) {
    Tube* t = (Tube*)p;
    t->has_saved = true; t->sp = t->p; t->sv = t->v; t->s_staggered = t->staggered;
}
void or_tube_restore(void* p) {  // lib.rs:547-554: pressure_prev is set to the saved pressure
    Tube* t = (Tube*)p;
    if (!t->has_saved) return;
    t->pp = t->sp; t->p = t->sp; t->v = t->sv; t->staggered = t->s_staggered;
}

// ---- Bar1D ----
// lib.rs:443-464: cells = max(cells, 2), every cell at `initial`, which is also the reference
void* or_bar_new(const char* name, int cells, double dx, double area, double density, double conductivity,
                 double specific_heat, int thermal, double initial) {
    Bar* b = new Bar();
    b->name = name ? name : "bar";
    b->n = std::max(cells, 2);
    b->dx = dx; b->area = area; b->reference = initial;
    b->density = density; b->conductivity = conductivity; b->specific_heat = specific_heat; b->thermal = thermal;
    b->cells.assign(b->n, initial);
    b->saved = b->cells;
    return b;
}
void or_bar_free(void* p) { delete (Bar*)p; }
int or_bar_cells(void* p) { return ((Bar*)p)->n; }
void or_bar_set(void* p, const double* t) { Bar* b = (Bar*)p; std::memcpy(b->cells.data(), t, b->cells.size() * 8); }
void or_bar_get(void* p, double* t) { Bar* b = (Bar*)p; std::memcpy(t, b->cells.data(), b->cells.size() * 8); }
// The bus's part: lumped heat for the next step's first cell, and heat per cell
void or_bar_absorb(void* p, double joules) { ((Bar*)p)->lumped += joules; }
void or_bar_deposit(void* p, const double* joules) {
    Bar* b = (Bar*)p;
    if (b->per_cell.empty()) b->per_cell.assign(b->n, 0.0);
    for (int i = 0; i < b->n; ++i) b->per_cell[i] += joules[i];
}
double or_bar_max_stable_dt(void* p) {  // lib.rs:564-569
    Bar* b = (Bar*)p;
    if (!b->thermal) return INF;
    return b->dx * b->dx / (2.0 * b->diffusivity());
}
double or_bar_fourier_number(void* p, double dt) { return ((Bar*)p)->fourier_number(dt); }
int or_bar_step(void* p, double dt, int nsteps, or_violation* out) {
    Bar* b = (Bar*)p;
    for (int s = 0; s < nsteps; ++s)
        if (!b->step(dt, out, nullptr)) return 1;
    return 0;
}
// Simulation::advance over one bar (books_balance, lib.rs:555-557): `attribute`
// (sim.rs:1169-1223) with the heat taken from the bus as the expected change.
int or_bar_advance(void* p, double dt, int nsteps, double tol, or_violation* out) {
    Bar* b = (Bar*)p;
    for (int s = 0; s < nsteps; ++s) {
        or_entry before = b->ledger();
        double taken = 0.0;
        if (!b->step(dt, out, &taken)) return 1;
        or_entry after = b->ledger();
        double discrepancy = (after.total - before.total) - taken;
        double scale = rmax(rmax(rmax(rmax(std::fabs(before.total), std::fabs(after.total)), before.scale), after.scale),
                            std::fabs(taken));
        if (scale >= 1e-300 && std::fabs(discrepancy) / scale > tol) {
            set_violation(out, "energy", b->name + " (its own books, against what it moved on the bus)",
                          before.total + taken, after.total, scale, tol);
            return 1;
        }
    }
    return 0;
}
void or_bar_ledger(void* p, double* total, double* scale, double* absorbed) {
    Bar* b = (Bar*)p;
    or_entry e = b->ledger();
    if (total) *total = e.total;
    if (scale) *scale = e.scale;
    if (absorbed) *absorbed = b->absorbed;
}
void or_bar_checkpoint(void* p) { Bar* b = (Bar*)p; b->saved = b->cells; }  // lib.rs:633-639
void or_bar_restore(void* p) { Bar* b = (Bar*)p; b->cells = b->saved; }

// ---- Cavity ----
void* or_yee_new(const char* name, int nx, int ny, int nz, double dx, double eps_r, double mu_r, double sigma) {
    Cavity* c = new Cavity();
    c->name = name ? name : "cavity";
    c->nx = std::max(nx, 1); c->ny = std::max(ny, 1); c->nz = std::max(nz, 1);
    c->dx = dx;
    c->medium = Medium{eps_r, mu_r, sigma};
    nx = c->nx; ny = c->ny; nz = c->nz;
    c->ex.assign((size_t)nx * (ny + 1) * (nz + 1), 0.0);
    c->ey.assign((size_t)(nx + 1) * ny * (nz + 1), 0.0);
    c->ez.assign((size_t)(nx + 1) * (ny + 1) * nz, 0.0);
    c->hx.assign((size_t)(nx + 1) * ny * nz, 0.0);
    c->hy.assign((size_t)nx * (ny + 1) * nz, 0.0);
    c->hz.assign((size_t)nx * ny * (nz + 1), 0.0);
    c->cells.assign((size_t)nx * ny * nz, c->medium);
    c->solid.assign((size_t)nx * ny * nz, 0);
    c->refresh_media();
    return c;
}
void or_yee_free(void* p) { delete (Cavity*)p; }
// cavity.rs:250-267 `fill`, once per cell: per-cell relative permittivity / permeability / σ.
void or_yee_set_cells(void* p, const double* eps_r, const double* mu_r, const double* sigma) {
    Cavity* c = (Cavity*)p;
    for (size_t q = 0; q < c->cells.size(); ++q) {
        if (eps_r) c->cells[q].eps_r = eps_r[q];
        if (mu_r) c->cells[q].mu_r = mu_r[q];
        if (sigma) c->cells[q].sigma = sigma[q];
    }
    c->refresh_media();
}
void or_yee_obstruct(void* p, const uint8_t* solid) {
    Cavity* c = (Cavity*)p;
    for (size_t q = 0; q < c->solid.size(); ++q)
        if (solid[q]) { c->solid[q] = 1; c->any_solid = true; }
    c->enforce_solid();
}
void or_yee_set_boundary(void* p, int wall, int kind) { ((Cavity*)p)->boundary[wall] = kind; }
double or_yee_mur_coefficient(void* p, double dt) { return ((Cavity*)p)->mur_coefficient(dt); }
double or_yee_cutoff_frequency(void* p, int m, int n) { return ((Cavity*)p)->cutoff_frequency(m, n); }
void or_yee_launch_along_z(void* p, const double* ey_env, const double* hx_env) {
    ((Cavity*)p)->launch_along_z(ey_env, hx_env);
}
void or_yee_impress(void* p, int plane, const double* add) { ((Cavity*)p)->impress(plane, add); }
void or_yee_release_mode(void* p, int m, int pm, double amplitude, double dt) { ((Cavity*)p)->release_mode(m, pm, amplitude, dt); }
void or_yee_set_source(void* p, long long edge, const double* current, long long n) {
    Cavity* c = (Cavity*)p;
    c->source_edge = edge;
    c->current.assign(current, current + n);
}
double or_yee_courant_limit(void* p) { return ((Cavity*)p)->courant_limit(); }
int or_yee_step(void* p, double dt, int nsteps, or_violation* out) {
    Cavity* c = (Cavity*)p;
    for (int s = 0; s < nsteps; ++s)
        if (!c->step(dt, out)) return 1;
    return 0;
}
int or_yee_advance(void* p, double dt, int nsteps, double tol, or_violation* out) {
    Cavity* c = (Cavity*)p;
    for (int s = 0; s < nsteps; ++s) {
        or_entry before = c->ledger();
        if (!c->step(dt, out)) return 1;
        or_entry after = c->ledger();
        if (!audit_energy("simulation", before, after, tol, out)) return 1;
    }
    return 0;
}
void or_yee_get(void* p, double* ex, double* ey, double* ez, double* hx, double* hy, double* hz) {
    Cavity* c = (Cavity*)p;
    if (ex) std::memcpy(ex, c->ex.data(), c->ex.size() * 8);
    if (ey) std::memcpy(ey, c->ey.data(), c->ey.size() * 8);
    if (ez) std::memcpy(ez, c->ez.data(), c->ez.size() * 8);
    if (hx) std::memcpy(hx, c->hx.data(), c->hx.size() * 8);
    if (hy) std::memcpy(hy, c->hy.data(), c->hy.size() * 8);
    if (hz) std::memcpy(hz, c->hz.data(), c->hz.size() * 8);
}
void or_yee_set(void* p, const double* ex, const double* ey, const double* ez, const double* hx, const double* hy,
                const double* hz, int started) {
    Cavity* c = (Cavity*)p;
    if (ex) std::memcpy(c->ex.data(), ex, c->ex.size() * 8);
    if (ey) std::memcpy(c->ey.data(), ey, c->ey.size() * 8);
    if (ez) std::memcpy(c->ez.data(), ez, c->ez.size() * 8);
    if (hx) std::memcpy(c->hx.data(), hx, c->hx.size() * 8);
    if (hy) std::memcpy(c->hy.data(), hy, c->hy.size() * 8);
    if (hz) std::memcpy(c->hz.data(), hz, c->hz.size() * 8);
    c->started = started != 0;
    // a new state starts fresh books and the source's clock (the reference has no setter)
    c->has_invariant = false;
    c->steps_taken = 0;
    c->dissipated = 0.0;
    c->source_work = 0.0;
    c->work_booked = 0.0;
}
void or_yee_get_media(void* p, double* eps, double* sigma, double* mu) {
    Cavity* c = (Cavity*)p;
    size_t off = 0;
    for (int q = 0; q < 3; ++q) {
        if (eps) std::memcpy(eps + off, c->eps[q].data(), c->eps[q].size() * 8);
        if (sigma) std::memcpy(sigma + off, c->sigma[q].data(), c->sigma[q].size() * 8);
        off += c->eps[q].size();
    }
    off = 0;
    for (int q = 0; q < 3; ++q) {
        if (mu) std::memcpy(mu + off, c->mu[q].data(), c->mu[q].size() * 8);
        off += c->mu[q].size();
    }
}
void or_yee_ledger(void* p, double* total, double* scale, double* invariant, double* dissipated, double* work) {
    Cavity* c = (Cavity*)p;
    or_entry e = c->ledger();
    if (total) *total = e.total;
    if (scale) *scale = e.scale;
    if (invariant) *invariant = c->invariant_energy();
    if (dissipated) *dissipated = c->dissipated;
    if (work) *work = c->source_work;
}
void or_yee_energies(void* p, double* electric, double* magnetic) {
    Cavity* c = (Cavity*)p;
    if (electric) *electric = c->electric_energy();
    if (magnetic) *magnetic = c->magnetic_energy();
}
double or_yee_peak_divergence(void* p) { return ((Cavity*)p)->peak_magnetic_divergence(); }
void or_yee_inject_divergence(void* p, int i, int j, int k, double amount) {  // cavity.rs:1000-1004
    Cavity* c = (Cavity*)p;
    size_t at = c->ihx(std::min(i, c->nx), std::min(j, c->ny - 1), std::min(k, c->nz - 1));
    c->hx[at] += amount;
}


}  // extern "C"

// ---- scene::capture's field sampling (crates/pantometry-scene/src/lib.rs:347-420): the extent's
// sample grid, x fastest; along an axis of n > 1 samples the point i / (n − 1) of the way from min
// to max, of one sample the middle (lib.rs:398-406); each point is `lo + (hi − lo) · f` per
// component, then the domain's own `ScalarField::at` there.
static double or_along(int i, int n) { return n > 1 ? (double)i / (double)(n - 1) : 0.5; }
template <typename At>
static void or_sample_grid(const double* lo, const double* hi, const int* n, double* out, At at) {
    size_t r = 0;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double f[3] = {or_along(i, n[0]), or_along(j, n[1]), or_along(k, n[2])};
                double q[3];
                for (int a = 0; a < 3; ++a) q[a] = lo[a] + (hi[a] - lo[a]) * f[a];
                out[r++] = at(q);
            }
}

extern "C" {

// Solid3D::at (solid.rs:2045-2104): trilinear between cell centres, clamped at the faces, NaN in
// a void cell, the weights renormalised over the solid corners.
void or_heat_sample(void* p, const double* lo, const double* hi, const int* n, double* out) {
    Heat* h = (Heat*)p;
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    auto is_void = [&](size_t c) { return !h->vd.empty() && h->vd[c] != 0; };
    or_sample_grid(lo, hi, n, out, [&](const double* pt) {
        const double q[3] = {pt[0] / h->dx - 0.5, pt[1] / h->dx - 0.5, pt[2] / h->dx - 0.5};
        if (std::isnan(q[0]) || std::isnan(q[1]) || std::isnan(q[2])) return std::nan("");
        auto axis = [](double v, int cnt, int& i, double& f) {
            const int last = cnt > 0 ? cnt - 1 : 0;
            if (v <= 0.0) { i = 0; f = 0.0; return; }
            if (v >= (double)last) { i = last; f = 0.0; return; }
            const double fl = std::floor(v);
            i = (int)fl;
            f = v - fl;
        };
        int i, j, k;
        double fx, fy, fz;
        axis(q[0], nx, i, fx);
        axis(q[1], ny, j, fy);
        axis(q[2], nz, k, fz);
        auto nearest = [](double v, int cnt) {
            double r = std::round(v);
            if (r < 0.0) r = 0.0;
            const int last = cnt > 0 ? cnt - 1 : 0;
            return std::min((int)r, last);
        };
        if (is_void((size_t)nearest(q[0], nx) + (size_t)nx * ((size_t)nearest(q[1], ny) + (size_t)ny * nearest(q[2], nz))))
            return std::nan("");
        const int i1 = std::min(i + 1, nx - 1), j1 = std::min(j + 1, ny - 1), k1 = std::min(k + 1, nz - 1);
        const int ai[2] = {i, i1}, bj[2] = {j, j1}, ck[2] = {k, k1};
        const double wa[2] = {1.0 - fx, fx}, wb[2] = {1.0 - fy, fy}, wc[2] = {1.0 - fz, fz};
        double sum = 0.0, weight = 0.0;
        for (int x = 0; x < 2; ++x)
            for (int y = 0; y < 2; ++y)
                for (int z = 0; z < 2; ++z) {
                    const double w = wa[x] * wb[y] * wc[z];
                    const size_t at = (size_t)ai[x] + (size_t)nx * ((size_t)bj[y] + (size_t)ny * ck[z]);
                    if (w > 0.0 && !is_void(at)) {
                        sum += w * h->cells[at];
                        weight += w;
                    }
                }
        return weight > 0.0 ? sum / weight : std::nan("");
    });
}

// Hall::at (hall.rs:591-613) with clamp_index (hall.rs:684-694): trilinear between nodes, clamped
// at the surfaces; a NaN point reads node 0.
void or_hall_sample(void* p, const double* lo, const double* hi, const int* n, double* out) {
    Hall* h = (Hall*)p;
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    or_sample_grid(lo, hi, n, out, [&](const double* pt) {
        const double q[3] = {pt[0] / h->dx, pt[1] / h->dx, pt[2] / h->dx};
        if (std::isnan(q[0]) || std::isnan(q[1]) || std::isnan(q[2])) return h->p[0];
        auto clamp_index = [](double v, int cnt, int& i, double& f) {
            if (std::isnan(v) || v <= 0.0) { i = 0; f = 0.0; return; }
            const double last = (double)(cnt - 1);
            if (v >= last) { i = cnt - 1; f = 0.0; return; }
            const double fl = std::floor(v);
            i = (int)fl;
            f = v - fl;
        };
        int i, j, k;
        double fx, fy, fz;
        clamp_index(q[0], nx, i, fx);
        clamp_index(q[1], ny, j, fy);
        clamp_index(q[2], nz, k, fz);
        const int i1 = std::min(i + 1, nx - 1), j1 = std::min(j + 1, ny - 1), k1 = std::min(k + 1, nz - 1);
        auto g = [&](int a, int b, int c) { return h->p[h->at(a, b, c)]; };
        auto lerp = [](double a, double b, double t) { return a * (1.0 - t) + b * t; };
        const double z0 = lerp(lerp(g(i, j, k), g(i1, j, k), fx), lerp(g(i, j1, k), g(i1, j1, k), fx), fy);
        const double z1 = lerp(lerp(g(i, j, k1), g(i1, j, k1), fx), lerp(g(i, j1, k1), g(i1, j1, k1), fx), fy);
        return lerp(z0, z1, fz);
    });
}

// Room::at (room.rs:587-601) with its clamp_index (room.rs:739-749): bilinear between the four nodes
// round (x, y), clamped at the walls; each coordinate is clamped on its own, a NaN one to node 0.
void or_room_sample(void* p, const double* lo, const double* hi, const int* n, double* out) {
    Room* r = (Room*)p;
    const int nx = r->nx, ny = r->ny;
    or_sample_grid(lo, hi, n, out, [&](const double* pt) {
        auto clamp_index = [](double q, int cnt, int& i, double& f) {
            if (std::isnan(q) || q <= 0.0) { i = 0; f = 0.0; return; }
            const double last = (double)(cnt - 1);
            if (q >= last) { i = cnt - 1; f = 0.0; return; }
            const double fl = std::floor(q);
            i = (int)fl;
            f = q - fl;
        };
        int i, j;
        double fx, fy;
        clamp_index(pt[0] / r->dx, nx, i, fx);
        clamp_index(pt[1] / r->dx, ny, j, fy);
        const int i1 = std::min(i + 1, nx - 1), j1 = std::min(j + 1, ny - 1);
        const double p00 = r->p[(size_t)j * nx + i], p10 = r->p[(size_t)j * nx + i1];
        const double p01 = r->p[(size_t)j1 * nx + i], p11 = r->p[(size_t)j1 * nx + i1];
        const double bottom = p00 * (1.0 - fx) + p10 * fx;
        const double top = p01 * (1.0 - fx) + p11 * fx;
        return bottom * (1.0 - fy) + top * fy;
    });
}

// Bar1D::at (crates/pantometry-thermal/src/lib.rs:736-751): linear between cell centres along x;
// the end cell's value beyond either centre and for a NaN x.
void or_bar_sample(void* p, const double* lo, const double* hi, const int* n, double* out) {
    Bar* b = (Bar*)p;
    const int last = (int)b->cells.size() - 1;
    or_sample_grid(lo, hi, n, out, [&](const double* pt) {
        const double u = pt[0] / b->dx - 0.5;
        if (std::isnan(u) || u <= 0.0) return b->cells[0];
        if (u >= (double)last) return b->cells[last];
        const double fl = std::floor(u);
        const int i = (int)fl;
        const double f = u - fl;
        return b->cells[i] * (1.0 - f) + b->cells[i + 1] * f;
    });
}

// Cavity::at (cavity.rs:197-206) over electric_at (cavity.rs:735-742): |E| of the edges of the cell
// the point falls in, nearest cell, clamped; NaN for a NaN point.
void or_yee_sample(void* p, const double* lo, const double* hi, const int* n, double* out) {
    Cavity* c = (Cavity*)p;
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    or_sample_grid(lo, hi, n, out, [&](const double* pt) {
        const double q[3] = {pt[0] / c->dx, pt[1] / c->dx, pt[2] / c->dx};
        if (std::isnan(q[0]) || std::isnan(q[1]) || std::isnan(q[2])) return std::nan("");
        auto pick = [](double v, int cnt) {
            double f = std::floor(v);
            if (f < 0.0) f = 0.0;
            return std::min((int)f, cnt > 0 ? cnt - 1 : 0);
        };
        const int i = pick(q[0], nx), j = pick(q[1], ny), k = pick(q[2], nz);
        const double x = c->ex[c->iex(std::min(i, nx - 1), std::min(j, ny), std::min(k, nz))];
        const double y = c->ey[c->iey(std::min(i, nx), std::min(j, ny - 1), std::min(k, nz))];
        const double z = c->ez[c->iez(std::min(i, nx), std::min(j, ny), std::min(k, nz - 1))];
        return std::sqrt((x * x + y * y) + z * z);  // DVec3::length: the dot product, then sqrt
    });
}

}  // extern "C"
