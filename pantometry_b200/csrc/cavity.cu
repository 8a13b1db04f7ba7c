// pm_cavity: the device form of `Cavity` (crates/pantometry-em/src/cavity.rs).
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <limits>
#include <new>

#include "runtime.h"

namespace pm {

namespace {
constexpr double kEpsilon0 = 8.8541878128e-12;  // crates/pantometry-em/src/lib.rs:67
constexpr double kMu0 = 1.25663706212e-6;       // crates/pantometry-em/src/lib.rs:69
constexpr double kCourant3D = 0.5773502691896258;  // cavity.rs:15
}  // namespace

struct Cavity : Handle {
    int nx = 1, ny = 1, nz = 1;
    double dx = 0.0;
    double eps_r = 1.0, mu_r = 1.0, sigma = 0.0;  // the constructor's `Medium`
    int boundary[6] = {0, 0, 0, 0, 0, 0};
    bool started = false;
    // media (cavity.rs:348-458)
    bool uniform = true;
    double eps_u = 0.0, sig_u = 0.0, mu_u = 0.0;
    std::vector<double> cell_eps, cell_mu, cell_sig;  // per cell, relative ε, μ and σ
    std::vector<double> eps[3], sig[3], mu[3];
    DBuf deps[3], dsig[3], dmu[3];
    // mixed media: the per-edge gain and decay and per-face g/μ of the step size coef_dt (in the
    // field type; the gains on the padded lattice when the cavity is TMA-staged), and what the
    // media leave uniform: σ = 0 on every edge (lossless, no decay array) and one μ on every face
    // (mu_one, no g/μ array)
    DBuf dgain[3], ddecay[3], dch[3];
    double coef_dt = NAN;
    bool lossless = true, mu_var = false;
    double mu_one = 0.0;
    std::vector<uint8_t> solid;
    bool any_solid = false;
    DBuf dsolid;
    // fields: ping-pong pairs, f[parity] holds the state
    DBuf f[2][6];  // ex ey ez hx hy hz
    DBuf keep[3];
    DBuf stage;
    DBuf energies;  // 2 doubles
    // source (extension)
    long long src = -1;
    DBuf current;
    long long ncurrent = 0;
    // checkpoint (cavity.rs:1566-1590)
    DBuf sf[6];
    bool s_started = false;
    double s_dissipated = 0.0;
    // the source extension's clock (which sample of the current comes next) and its work books,
    // so that steps retried after a restore drive the same pulse
    long long s_steps = 0;
    double s_work = 0.0, s_work_booked = 0.0;
    // FP32 cavities of one medium keep all six components on the padded lattice (row pitch L)
    // and step with the TMA-staged kernel (yee_tma.cuh); maps[par] describe parity par's fields
    bool tma = false;
    unsigned L = 0;
    YeeMaps maps[2];
    int yshape = 0;  // the TMA kernel's tile shape, an index of the present form's shape list
    bool wall_split_on = true;  // the TMA kernel's last column and row by its wall pass, where they split off
    // Mur's history (cavity.rs:141): E after the last step's walls. Normally the old buffer of the
    // ping-pong pair; after something rewrote E between steps it is a snapshot taken before that.
    bool has_prev = false;   // a step has run (cavity.rs:1087)
    bool use_stale = false;  // the next step's history is `stale`
    DBuf stale[3];
    // The source's near field in f64 (yee_near.cuh): the six components of a box of
    // kNearWidth³ lattice nodes around the source edge, one set per parity. Kept when the cavity
    // is TMA-staged FP32 with a source and the box, with the ring of edges on its high sides,
    // lies one node or more inside the walls (near_w = kNearWidth); otherwise near_w = 0.
    static constexpr int kNearWidth = 5;
    int near_x0 = 0, near_y0 = 0, near_z0 = 0, near_w = 0;
    DBuf dnear[2];
    bool near_dirty = true;  // the stored field changed outside a step: seed the box from it
    DBuf snear;              // the box of the checkpoint
    bool s_near = false;

    size_t count(int q) const {
        switch (q) {
            case 0: return (size_t)nx * (ny + 1) * (nz + 1);
            case 1: return (size_t)(nx + 1) * ny * (nz + 1);
            case 2: return (size_t)(nx + 1) * (ny + 1) * nz;
            case 3: return (size_t)(nx + 1) * ny * nz;
            case 4: return (size_t)nx * (ny + 1) * nz;
            default: return (size_t)nx * ny * (nz + 1);
        }
    }
    size_t cells() const { return (size_t)nx * ny * nz; }
    // elements held on the device per component
    size_t lattice() const { return (size_t)L * (ny + 1) * (nz + 1); }
    size_t dcount(int q) const { return tma ? lattice() : count(q); }
    void extents(int q, int& ex, int& ey, int& ez) const {
        ex = (q == 0 || q == 4 || q == 5) ? nx : nx + 1;
        ey = (q == 1 || q == 3 || q == 5) ? ny : ny + 1;
        ez = (q == 2 || q == 3 || q == 4) ? nz : nz + 1;
    }
    size_t esize() const { return precision == PM_PLAIN_F64 ? 8 : 4; }
    double volume() const { return dx * (dx * dx); }  // dx.powi(3)
    double permittivity() const { return kEpsilon0 * eps_r; }
    double permeability() const { return kMu0 * mu_r; }
    double wave_speed() const { return 1.0 / std::sqrt(permittivity() * permeability()); }
    double courant_limit() const { return kCourant3D * dx / wave_speed(); }

    // cavity.rs:348-458
    void refresh_media() {
        auto at = [&](long i, long j, long k) -> size_t {
            auto c = [](long v, long n) { return (size_t)std::min(std::max(v, 0L), n - 1); };
            return c(i, nx) + (size_t)nx * (c(j, ny) + (size_t)ny * c(k, nz));
        };
        auto perm = [&](size_t c) { return kEpsilon0 * cell_eps[c]; };
        auto cond = [&](size_t c) { return std::max(cell_sig[c], 0.0); };
        auto mean4 = [&](const size_t* of, bool conductivity) {
            double s = -0.0;
            for (int q = 0; q < 4; ++q) s += conductivity ? cond(of[q]) : perm(of[q]);
            return s / 4.0;
        };
        for (int q = 0; q < 3; ++q) {
            eps[q].assign(count(q), 0.0);
            sig[q].assign(count(q), 0.0);
            mu[q].assign(count(q + 3), 0.0);
        }
        for (long k = 0; k <= nz; ++k)
            for (long j = 0; j <= ny; ++j)
                for (long i = 0; i <= nx; ++i) {
                    if (i < nx) {
                        size_t of[4] = {at(i, j - 1, k - 1), at(i, j, k - 1), at(i, j - 1, k), at(i, j, k)};
                        size_t idx = i + (size_t)nx * (j + (size_t)(ny + 1) * k);
                        eps[0][idx] = mean4(of, false);
                        sig[0][idx] = mean4(of, true);
                    }
                    if (j < ny) {
                        size_t of[4] = {at(i - 1, j, k - 1), at(i, j, k - 1), at(i - 1, j, k), at(i, j, k)};
                        size_t idx = i + (size_t)(nx + 1) * (j + (size_t)ny * k);
                        eps[1][idx] = mean4(of, false);
                        sig[1][idx] = mean4(of, true);
                    }
                    if (k < nz) {
                        size_t of[4] = {at(i - 1, j - 1, k), at(i, j - 1, k), at(i - 1, j, k), at(i, j, k)};
                        size_t idx = i + (size_t)(nx + 1) * (j + (size_t)(ny + 1) * k);
                        eps[2][idx] = mean4(of, false);
                        sig[2][idx] = mean4(of, true);
                    }
                }
        auto mean2 = [&](size_t a, size_t b) {
            double s = -0.0;
            s += kMu0 * cell_mu[a];
            s += kMu0 * cell_mu[b];
            return s / 2.0;
        };
        for (long k = 0; k < nz; ++k)
            for (long j = 0; j < ny; ++j)
                for (long i = 0; i < nx; ++i) {
                    mu[0][i + (size_t)(nx + 1) * (j + (size_t)ny * k)] = mean2(at(i - 1, j, k), at(i, j, k));
                    mu[1][i + (size_t)nx * (j + (size_t)(ny + 1) * k)] = mean2(at(i, j - 1, k), at(i, j, k));
                    mu[2][i + (size_t)nx * (j + (size_t)ny * k)] = mean2(at(i, j, k - 1), at(i, j, k));
                }
        const double fallback = permeability();
        for (int q = 0; q < 3; ++q)
            for (double& v : mu[q])
                if (v <= 0.0) v = fallback;
        lossless = true;
        for (int q = 0; q < 3; ++q)
            for (double v : sig[q]) lossless = lossless && v == 0.0;
        mu_one = mu[0].empty() ? permeability() : mu[0][0];
        mu_var = false;
        for (int q = 0; q < 3; ++q)
            for (double v : mu[q]) mu_var = mu_var || v != mu_one;
    }

    // The uniform values every edge and face of a one-medium box holds (the same means).
    void uniform_media() {
        double s = -0.0;
        for (int q = 0; q < 4; ++q) s += permittivity();
        eps_u = s / 4.0;
        s = -0.0;
        for (int q = 0; q < 4; ++q) s += std::max(sigma, 0.0);
        sig_u = s / 4.0;
        s = -0.0;
        s += permeability();
        s += permeability();
        mu_u = s / 2.0;
        if (mu_u <= 0.0) mu_u = permeability();
    }

    template <typename Real>
    YeeHArgs<Real> hargs(double g, int energy) const {
        YeeHArgs<Real> a{};
        const DBuf* c = f[parity];
        a.ex = c[0].as<Real>(); a.ey = c[1].as<Real>(); a.ez = c[2].as<Real>();
        a.hx = c[3].as<Real>(); a.hy = c[4].as<Real>(); a.hz = c[5].as<Real>();
        a.nx = nx; a.ny = ny; a.nz = nz;
        a.g = g;
        a.uniform = uniform ? 1 : 0;
        a.ch = (Real)(g / mu_u);  // cavity.rs:1355: g / μ
        a.mu0 = dmu[0].as<double>(); a.mu1 = dmu[1].as<double>(); a.mu2 = dmu[2].as<double>();
        a.energy = energy;
        a.eps_u = eps_u; a.mu_u = mu_u;
        a.eps0 = deps[0].as<double>(); a.eps1 = deps[1].as<double>(); a.eps2 = deps[2].as<double>();
        a.volume = volume();
        const unsigned w = wave_of(sizeof(Real) == 8 ? kYeeHF64 : kYeeHF32);
        a.tiles = make_tiles(nx + 1, ny + 1, nz + 1, choose_zc(nx + 1, ny + 1, nz + 1, w));
        a.nblocks = grid_for(a.tiles, w);
        a.st = state.as<DevState>();
        a.partials = partials.as<double>();
        return a;
    }

    template <typename Real>
    YeeEArgs<Real> eargs(double dt) const {
        YeeEArgs<Real> a{};
        const DBuf* c = f[parity];
        a.ex = c[0].as<Real>(); a.ey = c[1].as<Real>(); a.ez = c[2].as<Real>();
        a.hx = c[3].as<Real>(); a.hy = c[4].as<Real>(); a.hz = c[5].as<Real>();
        a.nx = nx; a.ny = ny; a.nz = nz;
        a.dt = dt; a.dx = dx; a.volume = volume();
        a.uniform = uniform ? 1 : 0;
        // cavity.rs:1391-1397 at the uniform edge ε and σ
        const double half = sig_u * dt / (2.0 * eps_u);
        for (int q = 0; q < 3; ++q) {
            a.decay[q] = (Real)((1.0 - half) / (1.0 + half));
            a.gain[q] = (Real)((dt / (eps_u * dx)) / (1.0 + half));
            a.sigma_u[q] = sig_u;
        }
        a.eps0 = deps[0].as<double>(); a.eps1 = deps[1].as<double>(); a.eps2 = deps[2].as<double>();
        a.sig0 = dsig[0].as<double>(); a.sig1 = dsig[1].as<double>(); a.sig2 = dsig[2].as<double>();
        a.solid = any_solid ? dsolid.as<uint8_t>() : nullptr;
        a.src = src;
        a.current = current.as<double>();
        a.ncurrent = ncurrent;
        a.with_source = src >= 0 ? 1 : 0;
        if (src >= 0) {
            a.eps_src = uniform ? eps_u : eps[2][(size_t)src];
            a.sig_src = uniform ? sig_u : sig[2][(size_t)src];
        }
        const unsigned w = wave_of(sizeof(Real) == 8 ? kYeeEF64 : kYeeEF32);
        a.tiles = make_tiles(nx + 1, ny + 1, nz + 1, choose_zc(nx + 1, ny + 1, nz + 1, w));
        a.nblocks = grid_for(a.tiles, w);
        a.st = state.as<DevState>();
        a.partials = partials.as<double>();
        return a;
    }

    // The fused step from buffer set `par` into `par ^ 1`.
    template <typename Real>
    YeeStepArgs<Real> sargs(int par, double dt) const {
        YeeStepArgs<Real> a{};
        for (int q = 0; q < 6; ++q) {
            a.old[q] = f[par][q].as<Real>();
            a.neu[q] = f[par ^ 1][q].as<Real>();
        }
        a.pstride[0] = (unsigned)nx * (unsigned)(ny + 1);
        a.pstride[1] = (unsigned)(nx + 1) * (unsigned)ny;
        a.pstride[2] = (unsigned)(nx + 1) * (unsigned)(ny + 1);
        a.pstride[3] = (unsigned)(nx + 1) * (unsigned)ny;
        a.pstride[4] = (unsigned)nx * (unsigned)(ny + 1);
        a.pstride[5] = (unsigned)nx * (unsigned)ny;
        a.nx = nx; a.ny = ny; a.nz = nz;
        a.g = dt / dx;
        a.uniform = uniform ? 1 : 0;
        a.ch = (Real)(a.g / mu_u);  // cavity.rs:1355: g / μ
        a.mu0 = dmu[0].as<double>(); a.mu1 = dmu[1].as<double>(); a.mu2 = dmu[2].as<double>();
        a.mu_u = mu_u; a.eps_u = eps_u;
        a.dt = dt; a.dx = dx; a.volume = volume();
        const double half = sig_u * dt / (2.0 * eps_u);  // cavity.rs:1391-1397
        for (int q = 0; q < 3; ++q) {
            a.decay[q] = (Real)((1.0 - half) / (1.0 + half));
            a.gain[q] = (Real)((dt / (eps_u * dx)) / (1.0 + half));
            a.sigma_u[q] = sig_u;
        }
        a.eps0 = deps[0].as<double>(); a.eps1 = deps[1].as<double>(); a.eps2 = deps[2].as<double>();
        a.sig0 = dsig[0].as<double>(); a.sig1 = dsig[1].as<double>(); a.sig2 = dsig[2].as<double>();
        if (!uniform) {
            for (int q = 0; q < 3; ++q) {
                a.cgain[q] = dgain[q].as<Real>();
                a.cdecay[q] = lossless ? nullptr : ddecay[q].as<Real>();
                a.cch[q] = mu_var ? dch[q].as<Real>() : nullptr;
                if (lossless) { a.decay[q] = Real(1); a.sigma_u[q] = 0.0; }  // (1 − 0)/(1 + 0)
            }
            a.lossless = lossless ? 1 : 0;
            a.mu_var = mu_var ? 1 : 0;
            if (!mu_var) { a.mu_u = mu_one; a.ch = (Real)(a.g / mu_one); }
        }
        a.solid = any_solid ? dsolid.as<uint8_t>() : nullptr;
        a.src_i = a.src_j = a.src_k = -1;
        if (src >= 0) {
            a.src_i = (int)(src % (nx + 1));
            a.src_j = (int)((src / (nx + 1)) % (ny + 1));
            a.src_k = (int)(src / ((long long)(nx + 1) * (ny + 1)));
            a.eps_src = uniform ? eps_u : eps[2][(size_t)src];
            a.sig_src = uniform ? sig_u : sig[2][(size_t)src];
        }
        a.current = current.as<double>();
        a.ncurrent = ncurrent;
        const unsigned w = wave_of(sizeof(Real) == 8 ? kYeeStepF64 : kYeeStepF32);
        a.tiles = make_tiles(nx + 1, ny + 1, nz + 1, choose_zc(nx + 1, ny + 1, nz + 1, w));
        a.nblocks = grid_for(a.tiles, w);
        a.st = state.as<DevState>();
        a.partials = partials.as<double>();
        return a;
    }

    pm_status launch_h(double g, int energy, cudaStream_t s) const {
        if (precision == PM_PLAIN_F64) PM_CUDA(launch_yee_h<double>(hargs<double>(g, energy), s));
        else PM_CUDA(launch_yee_h<float>(hargs<float>(g, energy), s));
        return PM_OK;
    }

    pm_status put(int q, const double* src_host) {
        const size_t n = count(q);
        near_dirty = true;
        if (tma) {  // into the padded lattice, padding zero
            PM_CUDA(cudaMemsetAsync(f[parity][q].p, 0, lattice() * 4, stream()));
            if (!src_host) return PM_OK;
            if (!stage.p || stage.bytes < n * 8) PM_CUDA(stage.alloc(n * 8));
            PM_CUDA(cudaMemcpyAsync(stage.p, src_host, n * 8, cudaMemcpyHostToDevice, stream()));
            int ex, ey, ez;
            extents(q, ex, ey, ez);
            PM_CUDA(launch_yee_relayout(stage.p, true, f[parity][q].p, false, ex, ey, ez, L, ny + 1, 1, stream()));
            PM_CUDA(cudaStreamSynchronize(stream()));
            return PM_OK;
        }
        if (!src_host) {
            PM_CUDA(cudaMemsetAsync(f[parity][q].p, 0, n * esize(), stream()));
            return PM_OK;
        }
        if (precision == PM_PLAIN_F64) {
            PM_CUDA(cudaMemcpyAsync(f[parity][q].p, src_host, n * 8, cudaMemcpyHostToDevice, stream()));
        } else {
            if (!stage.p || stage.bytes < n * 8) PM_CUDA(stage.alloc(n * 8));
            PM_CUDA(cudaMemcpyAsync(stage.p, src_host, n * 8, cudaMemcpyHostToDevice, stream()));
            PM_CUDA(launch_to_f32(stage.as<double>(), f[parity][q].as<float>(), n, stream()));
            PM_CUDA(cudaStreamSynchronize(stream()));
        }
        return PM_OK;
    }
    pm_status get(int q, double* dst_host) {
        if (!dst_host) return PM_OK;
        const size_t n = count(q);
        if (tma) {
            if (!stage.p || stage.bytes < n * 8) PM_CUDA(stage.alloc(n * 8));
            int ex, ey, ez;
            extents(q, ex, ey, ez);
            PM_CUDA(launch_yee_relayout(f[parity][q].p, false, stage.p, true, ex, ey, ez, L, ny + 1, 0, stream()));
            PM_CUDA(cudaMemcpyAsync(dst_host, stage.p, n * 8, cudaMemcpyDeviceToHost, stream()));
            PM_CUDA(cudaStreamSynchronize(stream()));
            return PM_OK;
        }
        if (precision == PM_PLAIN_F64) {
            PM_CUDA(cudaMemcpyAsync(dst_host, f[parity][q].p, n * 8, cudaMemcpyDeviceToHost, stream()));
        } else {
            if (!stage.p || stage.bytes < n * 8) PM_CUDA(stage.alloc(n * 8));
            PM_CUDA(launch_to_f64(f[parity][q].as<float>(), stage.as<double>(), n, stream()));
            PM_CUDA(cudaMemcpyAsync(dst_host, stage.p, n * 8, cudaMemcpyDeviceToHost, stream()));
        }
        PM_CUDA(cudaStreamSynchronize(stream()));
        return PM_OK;
    }

    // Run `fn` on the present state in the reference layout. On a padded cavity the state is
    // gathered into the other ping-pong set (free between steps), `fn` sees that set as the
    // present one, and when `writes` the result is scattered back.
    template <typename F>
    pm_status with_reference_layout(bool writes, F fn) {
        if (!tma) return fn();
        const int home = parity;
        for (int q = 0; q < 6; ++q) {
            int ex, ey, ez;
            extents(q, ex, ey, ez);
            PM_CUDA(launch_yee_relayout(f[home][q].p, false, f[home ^ 1][q].p, false, ex, ey, ez, L, ny + 1, 0, stream()));
        }
        parity = home ^ 1;
        tma = false;
        pm_status s = fn();
        tma = true;
        parity = home;
        if (s != PM_OK) return s;
        if (writes) {
            near_dirty = true;
            for (int q = 0; q < 6; ++q) {
                int ex, ey, ez;
                extents(q, ex, ey, ez);
                PM_CUDA(cudaMemsetAsync(f[home][q].p, 0, lattice() * 4, stream()));
                PM_CUDA(launch_yee_relayout(f[home ^ 1][q].p, false, f[home][q].p, false, ex, ey, ez, L, ny + 1, 1, stream()));
            }
        }
        for (int q = 0; q < 6; ++q)  // the other set back to a zero-padded lattice
            PM_CUDA(cudaMemsetAsync(f[home ^ 1][q].p, 0, lattice() * 4, stream()));
        PM_CUDA(cudaStreamSynchronize(stream()));
        return PM_OK;
    }

    bool open_or_magnetic() const {
        for (int w = 0; w < 6; ++w)
            if (boundary[w] != 0) return true;
        return false;
    }
    // Obstacles with magnetic or open walls: the reference applies the walls, keeps E as Mur's
    // history, and only then zeroes the obstacles' edges (cavity.rs:1497-1499, 1159-1163). The
    // step kernels then leave those edges alone, the walls run, E is copied to `stale` (the history
    // lives there from then on) and yee_enforce_solid zeroes the edges.
    bool solid_after_walls() const { return any_solid && open_or_magnetic(); }
    pm_status ensure_stale() {
        for (int q = 0; q < 3; ++q) {
            const size_t bytes = dcount(q) * esize();
            if (stale[q].bytes < bytes) PM_CUDA(stale[q].alloc(bytes));
        }
        return PM_OK;
    }
    // Before E is rewritten between steps: keep the history the next step's open walls need.
    pm_status keep_history() {
        if (!has_prev || use_stale) return PM_OK;
        for (int q = 0; q < 3; ++q) {
            const size_t bytes = dcount(q) * esize();
            if (stale[q].bytes < bytes) PM_CUDA(stale[q].alloc(bytes));
            PM_CUDA(cudaMemcpyAsync(stale[q].p, f[parity][q].p, bytes, cudaMemcpyDeviceToDevice, stream()));
        }
        use_stale = true;
        return PM_OK;
    }
    // The walls after the step from `par` into `par ^ 1` (cavity.rs:1074-1164): magnetic mirrors,
    // then open walls by Mur (or held at zero before any history exists), one wall at a time.
    template <typename Real>
    YeeWallArgs<Real> wall_args(int par, bool stale_history) const {
        YeeWallArgs<Real> a{};
        for (int q = 0; q < 3; ++q) {
            a.e[q] = f[par ^ 1][q].as<Real>();
            a.pe[q] = stale_history ? stale[q].as<Real>() : f[par][q].as<Real>();
            int ex, ey, ez;
            extents(q, ex, ey, ez);
            a.rx[q] = tma ? L : (unsigned)ex;
            a.ry[q] = tma ? (unsigned)(ny + 1) : (unsigned)ey;
        }
        a.nx = nx; a.ny = ny; a.nz = nz;
        return a;
    }
    // After the walls of the step from `par`: E (before the obstacles are zeroed) becomes Mur's
    // history, then the obstacles' edges are zeroed.
    template <typename Real>
    cudaError_t solid_after(int par, cudaStream_t s) const {
        for (int q = 0; q < 3; ++q) {
            cudaError_t e = cudaMemcpyAsync(stale[q].p, f[par ^ 1][q].p, dcount(q) * esize(), cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return e;
        }
        return launch_yee_enforce_solid<Real>(wall_args<Real>(par, false), dsolid.as<uint8_t>(), s);
    }
    template <typename Real>
    cudaError_t walls(int par, bool prev, bool stale_history, double dt, cudaStream_t s) const {
        YeeWallArgs<Real> a = wall_args<Real>(par, stale_history);
        const double c_dt = wave_speed() * dt;
        a.k = (Real)((c_dt - dx) / (c_dt + dx));  // cavity.rs:1075-1078
        for (int w = 0; w < 6; ++w) {
            if (boundary[w] != 1) continue;
            a.wall = w;
            a.kind = 1;
            cudaError_t e = launch_yee_walls<Real>(a, s);
            if (e != cudaSuccess) return e;
        }
        for (int w = 0; w < 6; ++w) {
            if (boundary[w] != 2) continue;
            a.wall = w;
            a.kind = prev ? 2 : 3;
            cudaError_t e = launch_yee_walls<Real>(a, s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    // One step from `par`, its walls included.
    cudaError_t step_once(int par, double h, bool prev, bool stale_history, cudaStream_t s) const {
        cudaError_t e;
        const bool after = solid_after_walls();  // the obstacles' edges are zeroed after the walls
        if (precision == PM_PLAIN_F64) {
            YeeStepArgs<double> a = sargs<double>(par, h);
            if (after) a.solid = nullptr;
            e = launch_yee_step<double>(a, s);
        } else if (tma) {
            YeeStepArgs<float> t = targs(par, h);
            if (after) t.solid = nullptr;
            if (near_on()) {
                // the box's terms and the source are the step's last block's; it closes the books
                const YeeNearArgs n = nargs(par, h, t);
                t.nb_x0 = near_x0; t.nb_y0 = near_y0; t.nb_z0 = near_z0; t.nb_w = near_w;
                t.src_i = t.src_j = t.src_k = -1;
                e = launch_yee_tma(t, L, maps[par], yshape, s, n);
            } else {
                e = launch_yee_tma(t, L, maps[par], yshape, s);
            }
        } else {
            YeeStepArgs<float> a = sargs<float>(par, h);
            if (after) a.solid = nullptr;
            e = launch_yee_step<float>(a, s);
        }
        if (e != cudaSuccess || !open_or_magnetic()) return e;
        if (after) stale_history = prev;  // the history lives in `stale` once a step has run
        e = precision == PM_PLAIN_F64 ? walls<double>(par, prev, stale_history, h, s) : walls<float>(par, prev, stale_history, h, s);
        if (e != cudaSuccess || !after) return e;
        return precision == PM_PLAIN_F64 ? solid_after<double>(par, s) : solid_after<float>(par, s);
    }

    // Tensor maps of both parities' six components over the padded lattice.
    pm_status build_maps() {
        const unsigned P = (unsigned)yee_tma_shape(!uniform, yshape).planes;
        for (int q = 0; q < 2; ++q) {
            const int d0 = (int)L, d1 = ny + 1, d2 = nz + 1;
            if (!hall_tma_map(&maps[q].ex, f[q][0].p, d0, d1, d2, 36, 10, P + 1) ||
                !hall_tma_map(&maps[q].ey, f[q][1].p, d0, d1, d2, 40, 9, P + 1) ||
                !hall_tma_map(&maps[q].ez, f[q][2].p, d0, d1, d2, 40, 10, P) ||
                !hall_tma_map(&maps[q].hx, f[q][3].p, d0, d1, d2, 32, 9, P) ||
                !hall_tma_map(&maps[q].hy, f[q][4].p, d0, d1, d2, 36, 8, P) ||
                !hall_tma_map(&maps[q].hz, f[q][5].p, d0, d1, d2, 36, 9, P))
                return fail(PM_CUDA_ERROR, "cuTensorMapEncodeTiled refused a cavity field");
        }
        return PM_OK;
    }

    bool lossy_now() const { return uniform ? sig_u != 0.0 : !lossless; }
    // The near-field box is stepped: TMA-staged FP32, a source, a box inside the walls. A lossy
    // cavity with obstacles keeps the plain FP32 form: the Joule term of an edge is booked before
    // the obstacles zero it, and the ring's correction could not see that value.
    bool near_on() const {
        return tma && precision == PM_FIELDS_F32 && src >= 0 && near_w > 0 && !(any_solid && lossy_now());
    }
    // Place the box around the source edge's node, or turn it off where it would not fit.
    pm_status place_near() {
        near_w = 0;
        near_dirty = true;
        if (src < 0) return PM_OK;
        const int w = kNearWidth, r = w / 2;
        const int si = (int)(src % (nx + 1)), sj = (int)((src / (nx + 1)) % (ny + 1));
        const int sk = (int)(src / ((long long)(nx + 1) * (ny + 1)));
        const int x0 = si - r, y0 = sj - r, z0 = sk - r;
        // the box and the ring on its high sides at nodes 1 .. n−1: every component exists at
        // each of their nodes and every edge is interior
        if (x0 < 1 || y0 < 1 || z0 < 1 || x0 + w > nx - 1 || y0 + w > ny - 1 || z0 + w > nz - 1) return PM_OK;
        const size_t bytes = 6 * (size_t)w * w * w * sizeof(double);
        for (int par = 0; par < 2; ++par)
            if (dnear[par].bytes < bytes) PM_CUDA(dnear[par].alloc(bytes));
        near_x0 = x0; near_y0 = y0; near_z0 = z0; near_w = w;
        return PM_OK;
    }
    // Arguments of the box's kernel for the step from `par` with the TMA step's arguments `t`.
    YeeNearArgs nargs(int par, double h, const YeeStepArgs<float>& t) const {
        YeeNearArgs n{};
        for (int q = 0; q < 6; ++q) {
            n.old[q] = f[par][q].as<float>();
            n.neu[q] = f[par ^ 1][q].as<float>();
        }
        n.nold = dnear[par].as<double>();
        n.nneu = dnear[par ^ 1].as<double>();
        n.x0 = near_x0; n.y0 = near_y0; n.z0 = near_z0; n.w = near_w;
        n.L = L; n.ny1 = (unsigned)ny + 1;
        n.nx = nx; n.ny = ny; n.nz = nz;
        n.ch = t.g / t.mu_u;  // cavity.rs:1355 in f64
        if (uniform) {
            const double half = sig_u * h / (2.0 * eps_u);  // cavity.rs:1391-1397
            n.decay = (1.0 - half) / (1.0 + half);
            n.gain = (h / (eps_u * dx)) / (1.0 + half);
        } else {
            n.decay = 1.0;  // lossless mixed ε: each edge's own gain
            n.gain = 0.0;
            n.media = 1;
            for (int q = 0; q < 3; ++q) n.cgain[q] = dgain[q].as<float>();
        }
        n.chf = t.ch; n.gainf = t.gain[0]; n.decf = t.decay[0];
        n.lossy = t.sigma_u[0] != 0.0 ? 1 : 0;
        n.sig0 = t.sigma_u[0];
        n.solid = t.solid;
        n.src_i = t.src_i; n.src_j = t.src_j; n.src_k = t.src_k;
        n.current = t.current; n.ncurrent = t.ncurrent;
        n.eps_src = t.eps_src; n.sig_src = t.sig_src;
        n.dt = h; n.volume = t.volume; n.g = t.g; n.eps_u = t.eps_u; n.mu_u = t.mu_u;
        n.st = t.st;
        return n;
    }
    // The box's f64 values from the stored field of the present parity.
    pm_status seed_near() {
        if (!near_on()) return PM_OK;
        YeeNearArgs n{};
        for (int q = 0; q < 6; ++q) n.neu[q] = f[parity][q].as<float>();
        n.nneu = dnear[parity].as<double>();
        n.x0 = near_x0; n.y0 = near_y0; n.z0 = near_z0; n.w = near_w;
        n.L = L; n.ny1 = (unsigned)ny + 1;
        PM_CUDA(launch_yee_near_seed(n, stream()));
        near_dirty = false;
        return PM_OK;
    }

    // The mixed-ε form's gain boxes, the tile's own edges, 32 × 8 × P (both parities share the arrays).
    pm_status build_gain_maps() {
        if (uniform || !tma) return PM_OK;
        const unsigned P = (unsigned)yee_tma_shape(true, yshape).planes;
        for (int par = 0; par < 2; ++par)
            for (int q = 0; q < 3; ++q) {
                CUtensorMap* m = q == 0 ? &maps[par].gx : q == 1 ? &maps[par].gy : &maps[par].gz;
                if (!hall_tma_map(m, dgain[q].p, (int)L, ny + 1, nz + 1, 32, 8, P))
                    return fail(PM_CUDA_ERROR, "cuTensorMapEncodeTiled refused a cavity gain array");
            }
        return PM_OK;
    }
    pm_status set_shape(int sh) {
        if (sh < 0 || sh >= yee_tma_shape_count(!uniform)) return fail(PM_BAD_ARG, "cavity tile shape");
        if (!tma || sh == yshape) return PM_OK;
        PM_CUDA(cudaStreamSynchronize(stream()));
        yshape = sh;
        drop_graphs();
        pm_status s = build_maps();
        if (s != PM_OK) return s;
        return build_gain_maps();
    }
    // Time `trial` steps of every tile shape of the present form on the present state and keep the
    // fastest. Each trial step reads the present parity and writes the other one (free between
    // steps), so the fields are never touched; the books (the source's clock among them) are put back
    // after each trial. A grid shape timed once on a device is not timed again in the process.
    pm_status autotune(int trial) {
        if (!tma) return PM_OK;
        static std::mutex cache_mutex;
        static std::map<std::tuple<int, int, int, int, int, int>, int> cache;
        const auto key = std::make_tuple(nx, ny, nz, uniform ? 1 : 0, any_solid ? 1 : 0, device);
        {
            std::lock_guard<std::mutex> lock(cache_mutex);
            auto it = cache.find(key);
            if (it != cache.end()) return set_shape(it->second);
        }
        pm_status s = read_state();
        if (s != PM_OK) return s;
        const DevState books = *host_state;
        const double dt = 0.9 * courant_limit();
        if ((s = prepare_coefs(dt)) != PM_OK) return s;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        PM_CUDA(cudaEventCreate(&e0));
        PM_CUDA(cudaEventCreate(&e1));
        int best = yshape;
        float best_ms = 0.0f;
        for (int sh = 0; sh < yee_tma_shape_count(!uniform) && s == PM_OK; ++sh) {
            if ((s = set_shape(sh)) != PM_OK) break;
            host_state->tol = -1.0;  // no audit while timing
            if ((s = write_state()) != PM_OK) break;
            for (int q = 0; q < 2 + trial; ++q) {
                if (q == 2) PM_CUDA(cudaEventRecord(e0, stream()));
                PM_CUDA(launch_yee_tma(targs(parity, dt), L, maps[parity], yshape, stream()));
            }
            PM_CUDA(cudaEventRecord(e1, stream()));
            PM_CUDA(cudaEventSynchronize(e1));
            float ms = 0.0f;
            PM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (sh == 0 || ms < best_ms) { best = sh; best_ms = ms; }
            *host_state = books;
            s = write_state();
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (s != PM_OK) return s;
        {
            std::lock_guard<std::mutex> lock(cache_mutex);
            cache[key] = best;
        }
        return set_shape(best);
    }

    // The padded cavity back to the reference layout (before media with conductivity or per-cell
    // μ, which only the cp.async kernel reads). The state goes through the host once; a
    // checkpoint taken in the other layout is dropped.
    pm_status leave_tma() {
        if (!tma) return PM_OK;
        std::vector<double> v[6];
        pm_status s;
        for (int q = 0; q < 6; ++q) {
            v[q].resize(count(q));
            if ((s = get(q, v[q].data())) != PM_OK) return s;
        }
        tma = false;
        drop_graphs();
        has_saved = false;
        for (int q = 0; q < 6; ++q)
            if ((s = put(q, v[q].data())) != PM_OK) return s;
        PM_CUDA(cudaStreamSynchronize(stream()));
        return PM_OK;
    }

    // Step arguments of the TMA kernel: the cp.async kernel's, with its own tiling (chunks of
    // P·m − 1 planes, so a chunk and the plane below it fill whole stages).
    YeeStepArgs<float> targs(int par, double dt) const {
        YeeStepArgs<float> a = sargs<float>(par, dt);
        const unsigned w = wave_of(yee_tma_kernel_id(!uniform, yshape));
        const int P = yee_tma_shape(!uniform, yshape).planes;
        // the wall pass takes the last column and row when the tiles then cover the rest exactly;
        // a source on one of those edges stays with the tiles, which book its work
        const bool src_on_wall = a.src_i >= 0 && (a.src_i == nx || a.src_j == ny);
        a.wall_split = (wall_split_on && nx % 32 == 0 && ny % 8 == 0 && !src_on_wall) ? 1 : 0;
        const int X = a.wall_split ? nx : nx + 1, Y = a.wall_split ? ny : ny + 1, Z = nz + 1;
        int best = 2 * P - 1;
        double best_score = -1.0;
        for (int mlt : {2, 4, 8, 16}) {
            const int zc = P * mlt - 1;
            if (zc > Z && zc != 2 * P - 1) continue;
            const Tiles t = make_tiles(X, Y, Z, zc);
            const double per = (double)t.ntiles / w;
            const double rounds = per < 1.0 ? 1.0 : (double)((t.ntiles + w - 1) / w);
            const double balance = per < 1.0 ? per : per / rounds;
            const double score = balance * (1.0 - 1.0 / (2.0 * zc));
            if (score > best_score + 1e-9) { best_score = score; best = zc; }
        }
        a.tiles = make_tiles(X, Y, Z, best);
        a.nblocks = grid_for(a.tiles, w);
        return a;
    }

    // ½εE² and ½μH² of the present state.
    pm_status measure_naive(double* electric, double* magnetic) {
        if (tma) return with_reference_layout(false, [&]() { return measure_naive(electric, magnetic); });
        if (!energies.p) PM_CUDA(energies.alloc(2 * sizeof(double)));
        if (precision == PM_PLAIN_F64) PM_CUDA(launch_yee_measure<double>(hargs<double>(0.0, 0), energies.as<double>(), stream()));
        else PM_CUDA(launch_yee_measure<float>(hargs<float>(0.0, 0), energies.as<double>(), stream()));
        double e2[2];
        PM_CUDA(cudaMemcpyAsync(e2, energies.p, sizeof(e2), cudaMemcpyDeviceToHost, stream()));
        PM_CUDA(cudaStreamSynchronize(stream()));
        if (electric) *electric = e2[0];
        if (magnetic) *magnetic = e2[1];
        return PM_OK;
    }

    // The ledger as `Domain::ledger` reads it now (cavity.rs:1520-1524, 912-917), made the
    // audit's starting point.
    pm_status reset_ledger() {
        pm_status s = read_state();
        if (s != PM_OK) return s;
        DevState* st = host_state;
        double inv = st->invariant;
        if (!st->has_invariant) {
            double e = 0.0, m = 0.0;
            if ((s = measure_naive(&e, &m)) != PM_OK) return s;
            inv = e + m;
        }
        double total = 0.0, scale = 0.0;
        auto add = [&](double x) { total += x; scale = std::fmax(scale, std::fabs(x)); };  // Ledger::add
        add(inv);
        add(st->dissipated);
        if (src >= 0) add(-st->work_booked);
        st->total = total;
        st->scale = scale;
        st->part[0] = inv;
        st->part[1] = st->dissipated;
        st->part[2] = -st->work_booked;
        st->prev_total = total;
        st->prev_scale = scale;
        return write_state();
    }

    pm_status upload_media() {
        drop_graphs();
        if (uniform) return PM_OK;
        for (int q = 0; q < 3; ++q) {
            PM_CUDA(deps[q].alloc(eps[q].size() * 8));
            PM_CUDA(dsig[q].alloc(sig[q].size() * 8));
            PM_CUDA(dmu[q].alloc(mu[q].size() * 8));
            PM_CUDA(put_sync(deps[q].p, eps[q].data(), eps[q].size() * 8));
            PM_CUDA(put_sync(dsig[q].p, sig[q].data(), sig[q].size() * 8));
            PM_CUDA(put_sync(dmu[q].p, mu[q].data(), mu[q].size() * 8));
            PM_CUDA(dgain[q].alloc((tma ? dcount(q) : eps[q].size()) * esize()));
            if (lossless) ddecay[q].release();
            else PM_CUDA(ddecay[q].alloc(eps[q].size() * esize()));
            if (mu_var) PM_CUDA(dch[q].alloc(mu[q].size() * esize()));
            else dch[q].release();
        }
        if (tma) {
            yshape = 0;  // the mixed-ε form's own shape list
            pm_status ms = build_maps();
            if (ms != PM_OK) return ms;
            if ((ms = build_gain_maps()) != PM_OK) return ms;
        }
        coef_dt = NAN;
        return PM_OK;
    }

    // The mixed media's coefficients for step size h, once per change of h (or of the media).
    template <typename Real>
    YeeCoefArgs<Real> cargs(double h) const {
        YeeCoefArgs<Real> a{};
        for (int q = 0; q < 3; ++q) {
            a.eps[q] = deps[q].as<double>();
            a.sig[q] = dsig[q].as<double>();
            a.mu[q] = dmu[q].as<double>();
            a.gain[q] = dgain[q].as<Real>();
            a.decay[q] = lossless ? nullptr : ddecay[q].as<Real>();
            a.ch[q] = mu_var ? dch[q].as<Real>() : nullptr;
            a.ne[q] = count(q);
            a.nf[q] = count(q + 3);
        }
        a.dt = h; a.dx = dx; a.g = h / dx;
        if (tma) {
            a.L = L;
            a.ny1 = (unsigned)ny + 1;
            for (int q = 0; q < 3; ++q) {
                int ex, ey, ez;
                extents(q, ex, ey, ez);
                a.ext[q][0] = ex;
                a.ext[q][1] = ey;
            }
        }
        return a;
    }
    pm_status prepare_coefs(double h) {
        if (uniform || coef_dt == h) return PM_OK;
        if (precision == PM_PLAIN_F64) PM_CUDA(launch_yee_coefs<double>(cargs<double>(h), stream()));
        else PM_CUDA(launch_yee_coefs<float>(cargs<float>(h), stream()));
        coef_dt = h;
        return PM_OK;
    }
};

}  // namespace pm

using namespace pm;

#define CAV_GUARD(c)                                            \
    do {                                                        \
        if (!(c)) return fail(PM_BAD_ARG, "null pm_cavity");     \
        cudaSetDevice((c)->device);                             \
    } while (0)

extern "C" {

pm_status pm_cavity_create(const pm_cavity_desc* d, pm_cavity** out) {
    if (!d || !out) return fail(PM_BAD_ARG, "null argument");
    *out = nullptr;
    if (d->precision != PM_PLAIN_F64 && d->precision != PM_FIELDS_F32) return fail(PM_BAD_ARG, "unknown precision");
    if (!(d->dx > 0.0)) return fail(PM_BAD_ARG, "dx must be positive");
    Cavity* c = new (std::nothrow) Cavity();
    if (!c) return fail(PM_OUT_OF_MEMORY, "host allocation");
    c->name = d->name ? d->name : "cavity";
    c->precision = d->precision;
    c->nx = std::max(d->nx, 1); c->ny = std::max(d->ny, 1); c->nz = std::max(d->nz, 1);
    c->dx = d->dx;
    c->eps_r = d->eps_r; c->mu_r = d->mu_r; c->sigma = d->sigma;
    c->uniform_media();
    pm_status s = c->init(d->device, 0);
    if (s != PM_OK) { delete c; return s; }
    c->L = (unsigned)((c->nx + 1 + 3) & ~3);
    c->tma = c->precision == PM_FIELDS_F32 && c->lattice() < (1ull << 32);
    for (int attempt = 0; attempt < 2; ++attempt) {
        for (int par = 0; par < 2; ++par)
            for (int q = 0; q < 6; ++q) {
                cudaError_t e = c->f[par][q].alloc(c->dcount(q) * c->esize());
                if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaMalloc cavity fields"); }
                cudaMemset(c->f[par][q].p, 0, c->dcount(q) * c->esize());
            }
        // a shape the driver will not tile steps with the cp.async kernel on the reference layout
        if (!c->tma || c->build_maps() == PM_OK) break;
        c->tma = false;
    }
    *out = reinterpret_cast<pm_cavity*>(c);
    s = c->reset_ledger();
    if (s != PM_OK) { delete c; *out = nullptr; }
    return s;
}

pm_status pm_cavity_fill_cells(pm_cavity* cp, const double* eps_r, const double* mu_r, const double* sigma, size_t n) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (n != c->cells()) return fail(PM_BAD_ARG, "fill_cells: one value per cell");
    if (c->cell_eps.empty()) {
        c->cell_eps.assign(c->cells(), c->eps_r);
        c->cell_mu.assign(c->cells(), c->mu_r);
        c->cell_sig.assign(c->cells(), c->sigma);
    }
    for (size_t q = 0; q < n; ++q) {
        if (eps_r) c->cell_eps[q] = eps_r[q];
        if (mu_r) c->cell_mu[q] = mu_r[q];
        if (sigma) c->cell_sig[q] = sigma[q];
    }
    c->uniform = false;
    c->refresh_media();
    // the TMA-staged kernel steps per-cell ε with no conductivity and one μ on the padded layout;
    // other media go back to the reference layout and the cp.async kernel
    if (!(c->lossless && !c->mu_var)) {
        pm_status ls = c->leave_tma();
        if (ls != PM_OK) return ls;
    }
    pm_status s = c->upload_media();
    if (s != PM_OK) return s;
    return c->reset_ledger();
}

pm_status pm_cavity_obstruct(pm_cavity* cp, const uint8_t* mask, size_t n) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (!mask || n != c->cells()) return fail(PM_BAD_ARG, "obstruct: one byte per cell");
    if (c->solid.empty()) c->solid.assign(c->cells(), 0);
    for (size_t q = 0; q < n; ++q)
        if (mask[q]) { c->solid[q] = 1; c->any_solid = true; }
    if (!c->any_solid) return PM_OK;
    pm_status hs = c->keep_history();  // the edges it zeroes change E between steps
    if (hs != PM_OK) return hs;
    PM_CUDA(c->dsolid.alloc(c->cells()));
    PM_CUDA(c->put_sync(c->dsolid.p, c->solid.data(), c->cells()));
    c->drop_graphs();
    // cavity.rs:293 `enforce_solid` now, on the host copy of E
    std::vector<double> e[3];
    pm_status s;
    for (int q = 0; q < 3; ++q) {
        e[q].resize(c->count(q));
        if ((s = c->get(q, e[q].data())) != PM_OK) return s;
    }
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                if (!c->solid[i + (size_t)nx * (j + (size_t)ny * k)]) continue;
                const int d[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
                for (auto& q : d) e[0][(i) + (size_t)nx * ((j + q[0]) + (size_t)(ny + 1) * (k + q[1]))] = 0.0;
                for (auto& q : d) e[1][(i + q[0]) + (size_t)(nx + 1) * (j + (size_t)ny * (k + q[1]))] = 0.0;
                for (auto& q : d) e[2][(i + q[0]) + (size_t)(nx + 1) * ((j + q[1]) + (size_t)(ny + 1) * k)] = 0.0;
            }
    for (int q = 0; q < 3; ++q)
        if ((s = c->put(q, e[q].data())) != PM_OK) return s;
    PM_CUDA(cudaStreamSynchronize(c->stream()));
    return PM_OK;
}

pm_status pm_cavity_set_boundary(pm_cavity* cp, int wall, int kind) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (wall < 0 || wall > 5 || kind < 0 || kind > 2) return fail(PM_BAD_ARG, "wall 0..5, kind 0..2");
    c->boundary[wall] = kind;
    c->drop_graphs();
    return PM_OK;
}

pm_status pm_cavity_upload(pm_cavity* cp, const double* ex, const double* ey, const double* ez, const double* hx,
                           const double* hy, const double* hz, int started) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    const double* src[6] = {ex, ey, ez, hx, hy, hz};
    pm_status s = c->keep_history();  // the next step's open walls use the E of before the upload
    if (s != PM_OK) return s;
    c->parity = 0;
    for (int q = 0; q < 6; ++q)
        if ((s = c->put(q, src[q])) != PM_OK) return s;
    PM_CUDA(cudaStreamSynchronize(c->stream()));
    c->started = started != 0;
    if ((s = c->read_state()) != PM_OK) return s;
    // fresh books for a new state
    c->host_state->has_invariant = 0;
    c->host_state->steps = 0;
    c->host_state->violated = kRunning;
    c->host_state->dissipated = 0.0;
    c->host_state->work = 0.0;
    c->host_state->work_booked = 0.0;
    if ((s = c->write_state()) != PM_OK) return s;
    return c->reset_ledger();
}

pm_status pm_cavity_download(pm_cavity* cp, double* ex, double* ey, double* ez, double* hx, double* hy, double* hz) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    double* dst[6] = {ex, ey, ez, hx, hy, hz};
    pm_status s;
    for (int q = 0; q < 6; ++q)
        if ((s = c->get(q, dst[q])) != PM_OK) return s;
    return PM_OK;
}

pm_status pm_cavity_release_mode(pm_cavity* cp, int m_in, int p_in, double amplitude, double dt) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    // cavity.rs:675-732; the next step's open walls keep the history of before the release
    pm_status hs = c->keep_history();
    if (hs != PM_OK) return hs;
    const double m = (double)std::max(m_in, 1), p = (double)std::max(p_in, 1);
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const double sx = (double)nx * c->dx, sz = (double)nz * c->dx;
    const double kx = M_PI * m / sx, kz = M_PI * p / sz;
    std::vector<double> ey(c->count(1), 0.0);
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i <= nx; ++i) {
                const double x = (double)i * c->dx, z = (double)k * c->dx;
                ey[i + (size_t)(nx + 1) * (j + (size_t)ny * k)] = amplitude * std::sin(kx * x) * std::sin(kz * z);
            }
    // enforce_walls (cavity.rs:1296-1343): Ey is tangential to the x and z walls
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j < ny; ++j) {
            ey[0 + (size_t)(nx + 1) * (j + (size_t)ny * k)] = 0.0;
            ey[nx + (size_t)(nx + 1) * (j + (size_t)ny * k)] = 0.0;
        }
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i) {
            ey[i + (size_t)(nx + 1) * (j + (size_t)ny * 0)] = 0.0;
            ey[i + (size_t)(nx + 1) * (j + (size_t)ny * nz)] = 0.0;
        }
    pm_status s;
    if ((s = c->read_state()) != PM_OK) return s;
    c->host_state->violated = kRunning;
    c->host_state->has_invariant = 0;
    c->host_state->steps = 0;
    if ((s = c->write_state()) != PM_OK) return s;
    s = c->with_reference_layout(true, [&]() -> pm_status {
        pm_status r;
        for (int q = 0; q < 6; ++q)
            if ((r = c->put(q, q == 1 ? ey.data() : nullptr)) != PM_OK) return r;
        // H = +(dt/2μ)∇×E with the scheme's own stencil, then the invariant from a trial step
        if ((r = c->launch_h((-0.5 * dt) / c->dx, 0, c->stream())) != PM_OK) return r;
        for (int q = 0; q < 3; ++q) {
            const size_t bytes = c->count(q + 3) * c->esize();
            if (!c->keep[q].p) PM_CUDA(c->keep[q].alloc(bytes));
            PM_CUDA(cudaMemcpyAsync(c->keep[q].p, c->f[c->parity][q + 3].p, bytes, cudaMemcpyDeviceToDevice, c->stream()));
        }
        if ((r = c->launch_h(dt / c->dx, 1, c->stream())) != PM_OK) return r;
        for (int q = 0; q < 3; ++q)
            PM_CUDA(cudaMemcpyAsync(c->f[c->parity][q + 3].p, c->keep[q].p, c->count(q + 3) * c->esize(),
                                    cudaMemcpyDeviceToDevice, c->stream()));
        PM_CUDA(cudaStreamSynchronize(c->stream()));
        return PM_OK;
    });
    if (s != PM_OK) return s;
    c->started = true;
    return c->reset_ledger();
}

pm_status pm_cavity_set_source(pm_cavity* cp, long long edge, const double* cur, size_t n) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (edge < 0 || (size_t)edge >= c->count(2) || (!cur && n > 0)) return fail(PM_BAD_ARG, "source edge out of range");
    c->src = edge;
    c->ncurrent = (long long)n;
    if (n > 0) {
        PM_CUDA(c->current.alloc(n * 8));
        PM_CUDA(c->put_sync(c->current.p, cur, n * 8));
    }
    c->drop_graphs();
    pm_status ps = c->place_near();
    if (ps != PM_OK) return ps;
    return c->reset_ledger();
}

pm_status pm_cavity_courant_limit(pm_cavity* cp, double* seconds) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (!seconds) return fail(PM_BAD_ARG, "null output");
    *seconds = c->courant_limit();
    return PM_OK;
}

pm_status pm_cavity_set_tolerance(pm_cavity* cp, double tol) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    c->tolerance = tol;
    return PM_OK;
}

pm_status pm_cavity_step(pm_cavity* cp, double dt, long long nsteps, pm_violation* out) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (nsteps < 0) return fail(PM_BAD_ARG, "nsteps must be >= 0");
    if (nsteps == 0) return PM_OK;
    if (c->solid_after_walls()) {
        pm_status es = c->ensure_stale();
        if (es != PM_OK) return es;
        if (c->has_prev && !c->use_stale) {
            // the history the last step left, now kept in `stale` (stepped before these walls were
            // set: the field after its step, the obstacles' edges already zeroed)
            for (int q = 0; q < 3; ++q)
                PM_CUDA(cudaMemcpyAsync(c->stale[q].p, c->f[c->parity][q].p, c->dcount(q) * c->esize(), cudaMemcpyDeviceToDevice,
                                        c->stream()));
            c->use_stale = true;
        }
    }
    // cavity.rs:1469-1480
    const double h = dt, limit = c->courant_limit();
    if (h > limit) {
        fill_violation(out, "Courant number", c->name, limit, h, limit, 0.0, 1);
        set_error("Courant limit");
        return PM_VIOLATION;
    }
    pm_status s = c->begin_call();
    if (s != PM_OK) return s;
    if ((s = c->prepare_coefs(h)) != PM_OK) return s;
    const long long before = c->host_state->steps;
    if (!c->started) {  // cavity.rs:1486-1489
        s = c->with_reference_layout(true, [&]() { return c->launch_h((0.5 * h) / c->dx, 0, c->stream()); });
        if (s != PM_OK) return s;
        c->started = true;
    }
    if (c->near_dirty && (s = c->seed_near()) != PM_OK) return s;
    long long remaining = nsteps;
    if (!c->has_prev || c->use_stale) {
        // the first step after creation holds open walls at zero; the first after E was rewritten
        // takes its history from the snapshot: both run on their own, outside any graph
        PM_CUDA(c->step_once(c->parity, h, c->has_prev, c->use_stale, c->stream()));
        c->parity ^= 1;
        c->has_prev = true;
        c->use_stale = c->solid_after_walls();  // there the history stays in `stale`
        remaining -= 1;
    }
    s = c->run_steps(remaining, dt, true, [c, h](int par, cudaStream_t st) { return c->step_once(par, h, true, false, st); });
    if (s != PM_OK) return s;
    return c->finish_call(before, out, "simulation", "simulation", true);
}

pm_status pm_cavity_ledger(pm_cavity* cp, pm_ledger* out) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (!out) return fail(PM_BAD_ARG, "null output");
    pm_status s = c->read_state();
    if (s != PM_OK) return s;
    std::memset(out, 0, sizeof(*out));
    const DevState* st = c->host_state;
    out->total = st->total;
    out->scale = st->scale;
    out->n_parts = 3;
    out->parts[0] = st->part[0];
    out->parts[1] = st->part[1];
    out->parts[2] = st->part[2];
    out->steps = st->steps;
    return PM_OK;
}

pm_status pm_cavity_sample(pm_cavity* cp, const double* lo, const double* hi, const int* samples, double* out,
                           size_t n) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    SampleGrid g{};
    pm_status s = sample_grid_of(lo, hi, samples, out, n, g);
    if (s != PM_OK) return s;
    g.dx = c->dx;
    g.nx = c->nx; g.ny = c->ny; g.nz = c->nz;
    const unsigned nx = (unsigned)c->nx, ny = (unsigned)c->ny;
    // each E component's row pitch and rows per plane: its own extents, or the padded lattice
    const uint3 rx = c->tma ? make_uint3(c->L, c->L, c->L) : make_uint3(nx, nx + 1, nx + 1);
    const uint3 ry = c->tma ? make_uint3(ny + 1, ny + 1, ny + 1) : make_uint3(ny + 1, ny, ny + 1);
    const DBuf* f = c->f[c->parity];
    return run_sample(c, out, n, [&](double* dev, cudaStream_t st) {
        return c->precision == PM_PLAIN_F64
                   ? launch_yee_sample<double>(g, f[0].as<double>(), f[1].as<double>(), f[2].as<double>(), rx, ry, dev, st)
                   : launch_yee_sample<float>(g, f[0].as<float>(), f[1].as<float>(), f[2].as<float>(), rx, ry, dev, st);
    });
}

pm_status pm_cavity_energies(pm_cavity* cp, double* electric, double* magnetic) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    return c->measure_naive(electric, magnetic);
}

pm_status pm_cavity_checkpoint(pm_cavity* cp) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    for (int q = 0; q < 6; ++q) {
        const size_t bytes = c->dcount(q) * c->esize();
        if (!c->sf[q].p || c->sf[q].bytes < bytes) PM_CUDA(c->sf[q].alloc(bytes));
        PM_CUDA(cudaMemcpyAsync(c->sf[q].p, c->f[c->parity][q].p, bytes, cudaMemcpyDeviceToDevice, c->stream()));
    }
    c->s_near = false;
    if (c->near_on()) {  // the box's f64 values are part of the state
        pm_status ns = c->near_dirty ? c->seed_near() : PM_OK;
        if (ns != PM_OK) return ns;
        const size_t bytes = c->dnear[c->parity].bytes;
        if (c->snear.bytes < bytes) PM_CUDA(c->snear.alloc(bytes));
        PM_CUDA(cudaMemcpyAsync(c->snear.p, c->dnear[c->parity].p, bytes, cudaMemcpyDeviceToDevice, c->stream()));
        c->s_near = true;
    }
    pm_status s = c->read_state();
    if (s != PM_OK) return s;
    c->s_started = c->started;
    c->s_dissipated = c->host_state->dissipated;
    c->s_steps = c->host_state->steps;
    c->s_work = c->host_state->work;
    c->s_work_booked = c->host_state->work_booked;
    c->has_saved = true;
    return PM_OK;
}

pm_status pm_cavity_restore(pm_cavity* cp) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (!c->has_saved) return PM_OK;
    pm_status hs = c->keep_history();  // Mur's history is not part of the checkpoint (cavity.rs:1566-1590)
    if (hs != PM_OK) return hs;
    for (int q = 0; q < 6; ++q)
        PM_CUDA(cudaMemcpyAsync(c->f[c->parity][q].p, c->sf[q].p, c->dcount(q) * c->esize(), cudaMemcpyDeviceToDevice, c->stream()));
    c->near_dirty = true;
    if (c->s_near && c->near_on() && c->snear.bytes == c->dnear[c->parity].bytes) {
        PM_CUDA(cudaMemcpyAsync(c->dnear[c->parity].p, c->snear.p, c->snear.bytes, cudaMemcpyDeviceToDevice, c->stream()));
        c->near_dirty = false;
    }
    pm_status s = c->read_state();
    if (s != PM_OK) return s;
    c->started = c->s_started;
    c->host_state->dissipated = c->s_dissipated;
    if (c->src >= 0) {
        c->host_state->steps = c->s_steps;
        c->host_state->work = c->s_work;
        c->host_state->work_booked = c->s_work_booked;
    }
    if ((s = c->write_state()) != PM_OK) return s;
    c->has_saved = false;  // cavity.rs:1580 takes the checkpoint
    return c->reset_ledger();
}

pm_status pm_cavity_autotune(pm_cavity* cp, int trial_steps, int* planes, int* stages) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (trial_steps < 1) return fail(PM_BAD_ARG, "autotune: at least one trial step");
    pm_status s = c->autotune(trial_steps);
    if (s != PM_OK) return s;
    return pm_cavity_tile(cp, planes, stages);
}

pm_status pm_cavity_set_tile(pm_cavity* cp, int planes, int stages) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (!c->tma) return fail(PM_UNSUPPORTED, "tile shapes are those of the TMA-staged FP32 kernel");
    for (int q = 0; q < yee_tma_shape_count(!c->uniform); ++q) {
        const YeeTmaShape sh = yee_tma_shape(!c->uniform, q);
        if (sh.planes == planes && sh.stages == stages) return c->set_shape(q);
    }
    return fail(PM_BAD_ARG, c->uniform ? "cavity tile: planes x stages of 3x2, 4x2 or 3x3" : "cavity tile: planes x stages of 4x2 or 3x2");
}

pm_status pm_cavity_tile(pm_cavity* cp, int* planes, int* stages) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    const YeeTmaShape sh = yee_tma_shape(!c->uniform, c->yshape);
    if (planes) *planes = c->tma ? sh.planes : 0;
    if (stages) *stages = c->tma ? sh.stages : 0;
    return PM_OK;
}

pm_status pm_cavity_set_wall_split(pm_cavity* cp, int on) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (c->wall_split_on == (on != 0)) return PM_OK;
    PM_CUDA(cudaStreamSynchronize(c->stream()));
    c->wall_split_on = on != 0;
    c->drop_graphs();
    return PM_OK;
}

pm_status pm_cavity_wall_split(pm_cavity* cp, int* on) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    if (on) *on = (c->tma && c->targs(c->parity, c->courant_limit()).wall_split) ? 1 : 0;
    return PM_OK;
}

pm_status pm_cavity_set_stream(pm_cavity* cp, void* stream) {
    Cavity* c = reinterpret_cast<Cavity*>(cp);
    CAV_GUARD(c);
    PM_CUDA(cudaStreamSynchronize(c->stream()));
    c->user = static_cast<cudaStream_t>(stream);
    return PM_OK;
}

void pm_cavity_destroy(pm_cavity* cp) { delete reinterpret_cast<Cavity*>(cp); }

}  // extern "C"
