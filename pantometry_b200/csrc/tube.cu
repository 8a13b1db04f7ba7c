// pm_tube: the device form of `Tube` (crates/pantometry-acoustic/src/lib.rs:107-560).
#include <algorithm>
#include <limits>
#include <new>

#include "runtime.h"

namespace pm {

struct Tube : Handle {
    int n = 3;
    double dx = 0.0, speed = 0.0, density = 0.0, area = 0.0;
    int end_kind[2] = {0, 0};  // 0 closed, 1 open, 2 matched (lib.rs:107-116)
    double end_z[2] = {0.0, 0.0};
    bool staggered = false;
    DBuf p[2], v[2];
    DBuf stage;
    DBuf sp, sv;  // checkpoint (lib.rs:539-554)
    bool s_staggered = false;

    size_t nv() const { return (size_t)n - 1; }
    size_t esize() const { return precision == PM_PLAIN_F64 ? 8 : 4; }
    double rc2() const { return density * speed * speed; }
    double impedance() const { return density * speed; }  // lib.rs:255-257
    double volume() const { return area * dx; }
    double knode() const { return rc2() <= 0.0 ? 0.0 : volume() / (2.0 * rc2()); }
    double kface() const { return rc2() <= 0.0 ? 0.0 : 0.5 * density * volume(); }
    unsigned grid(KernelId id) const {
        const size_t need = ((size_t)n + 255) / 256;
        return (unsigned)std::max<size_t>(1, std::min<size_t>(need, wave_of(id)));
    }

    template <typename Real>
    TubeArgs<Real> args(int par, double h, bool starting) const {
        TubeArgs<Real> a{};
        a.p0 = p[par].as<Real>(); a.v0 = v[par].as<Real>();
        a.p1 = p[par ^ 1].as<Real>(); a.v1 = v[par ^ 1].as<Real>();
        a.n = n;
        const double vh = starting ? 0.5 * h : h;  // lib.rs:393-397
        a.gain = (Real)(vh / (density * dx));       // lib.rs:404
        a.coef = (Real)(h * rc2() / dx);            // lib.rs:432
        for (int e = 0; e < 2; ++e) {
            // lib.rs:368-382: closed ends hold still, the others move as outward·p/Z
            a.outward[e] = end_kind[e] == 0 ? 0.0 : (e == 0 ? -1.0 : 1.0);
            a.z[e] = (end_kind[e] == 2 && end_z[e] > 0.0) ? end_z[e] : impedance();
        }
        a.knode = knode();
        a.kface = kface();
        a.area = area;
        a.dt = h;
        a.starting = starting ? 1 : 0;
        a.nblocks = grid(sizeof(Real) == 8 ? kTubeF64 : kTubeF32);
        a.st = state.as<DevState>();
        a.partials = partials.as<double>();
        return a;
    }
    cudaError_t launch(int par, double h, bool starting, cudaStream_t s) const {
        if (precision == PM_PLAIN_F64) return launch_tube<double>(args<double>(par, h, starting), s);
        return launch_tube<float>(args<float>(par, h, starting), s);
    }

    pm_status measure(int par_p, int par_pp) {
        if (precision == PM_PLAIN_F64) {
            TubeMeasureArgs<double> m{};
            m.p = p[par_p].as<double>(); m.pp = p[par_pp].as<double>(); m.v = v[parity].as<double>();
            m.n = n; m.knode = knode(); m.kface = kface();
            m.st = state.as<DevState>(); m.partials = partials.as<double>(); m.nblocks = grid(kTubeF64);
            PM_CUDA(launch_tube_measure<double>(m, stream()));
        } else {
            TubeMeasureArgs<float> m{};
            m.p = p[par_p].as<float>(); m.pp = p[par_pp].as<float>(); m.v = v[parity].as<float>();
            m.n = n; m.knode = knode(); m.kface = kface();
            m.st = state.as<DevState>(); m.partials = partials.as<double>(); m.nblocks = grid(kTubeF32);
            PM_CUDA(launch_tube_measure<float>(m, stream()));
        }
        return read_state();
    }

    pm_status put(DBuf& dst, const double* src_host, size_t count) {
        if (precision == PM_PLAIN_F64) {
            PM_CUDA(cudaMemcpyAsync(dst.p, src_host, count * 8, cudaMemcpyHostToDevice, stream()));
        } else {
            if (!stage.p || stage.bytes < count * 8) PM_CUDA(stage.alloc(std::max<size_t>(count, 1) * 8));
            PM_CUDA(cudaMemcpyAsync(stage.p, src_host, count * 8, cudaMemcpyHostToDevice, stream()));
            PM_CUDA(launch_to_f32(stage.as<double>(), dst.as<float>(), count, stream()));
        }
        return PM_OK;
    }
    pm_status get(const DBuf& src_dev, double* dst_host, size_t count) {
        if (!dst_host || count == 0) return PM_OK;
        if (precision == PM_PLAIN_F64) {
            PM_CUDA(cudaMemcpyAsync(dst_host, src_dev.p, count * 8, cudaMemcpyDeviceToHost, stream()));
        } else {
            if (!stage.p || stage.bytes < count * 8) PM_CUDA(stage.alloc(std::max<size_t>(count, 1) * 8));
            PM_CUDA(launch_to_f64(src_dev.as<float>(), stage.as<double>(), count, stream()));
            PM_CUDA(cudaMemcpyAsync(dst_host, stage.p, count * 8, cudaMemcpyDeviceToHost, stream()));
        }
        PM_CUDA(cudaStreamSynchronize(stream()));
        return PM_OK;
    }
    // The books of the state in host_state: the energy, then the published total, the two
    // entries the step kernel books.
    void book_totals() {
        DevState* st = host_state;
        const double energy = st->invariant + st->offset;
        st->total = energy + st->injected;
        st->scale = std::fmax(std::fabs(energy), std::fabs(st->injected));
        st->part[0] = energy;
        st->part[1] = st->injected;
    }
};

}  // namespace pm

using namespace pm;

#define TUBE_GUARD(t)                                          \
    do {                                                       \
        if (!(t)) return fail(PM_BAD_ARG, "null pm_tube");      \
        cudaSetDevice((t)->device);                            \
    } while (0)

extern "C" {

pm_status pm_tube_create(const pm_tube_desc* d, pm_tube** out) {
    if (!d || !out) return fail(PM_BAD_ARG, "null argument");
    *out = nullptr;
    if (d->precision != PM_PLAIN_F64 && d->precision != PM_FIELDS_F32) return fail(PM_BAD_ARG, "unknown precision");
    Tube* t = new (std::nothrow) Tube();
    if (!t) return fail(PM_OUT_OF_MEMORY, "host allocation");
    t->name = d->name ? d->name : "tube";
    t->precision = d->precision;
    t->n = std::max(d->cells, 3);  // lib.rs:175
    t->dx = d->length / (double)(t->n - 1);
    t->speed = d->speed;
    t->density = d->density;
    t->area = d->area;
    pm_status s = t->init(d->device, 0);
    if (s != PM_OK) { delete t; return s; }
    for (int q = 0; q < 2; ++q) {
        cudaError_t e;
        if ((e = t->p[q].alloc((size_t)t->n * t->esize())) != cudaSuccess ||
            (e = t->v[q].alloc(t->nv() * t->esize())) != cudaSuccess) {
            delete t;
            return cuda_fail(e, "cudaMalloc tube fields");
        }
    }
    *out = reinterpret_cast<pm_tube*>(t);
    std::vector<double> zero((size_t)t->n, 0.0);
    s = pm_tube_release(*out, zero.data(), zero.size());  // Tube::new is at rest
    if (s != PM_OK) { delete t; *out = nullptr; }
    return s;
}

pm_status pm_tube_cells(pm_tube* tp, int* n, double* dx) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    if (n) *n = t->n;
    if (dx) *dx = t->dx;
    return PM_OK;
}

pm_status pm_tube_set_ends(pm_tube* tp, int left, double z_left, int right, double z_right) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    if (left < 0 || left > 2 || right < 0 || right > 2) return fail(PM_BAD_ARG, "end kind must be 0 closed, 1 open or 2 matched");
    t->end_kind[0] = left; t->end_z[0] = z_left;
    t->end_kind[1] = right; t->end_z[1] = z_right;
    t->drop_graphs();
    return PM_OK;
}

pm_status pm_tube_release(pm_tube* tp, const double* pressure, size_t n) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    if (!pressure || n != (size_t)t->n) return fail(PM_BAD_ARG, "release: one pressure per cell");
    // lib.rs:226-235: pressure from the profile, pressure_prev = pressure, v = 0, then the datum
    t->parity = 0;
    pm_status s;
    if ((s = t->put(t->p[0], pressure, n)) != PM_OK) return s;
    PM_CUDA(cudaMemcpyAsync(t->p[1].p, t->p[0].p, n * t->esize(), cudaMemcpyDeviceToDevice, t->stream()));
    for (int q = 0; q < 2; ++q) PM_CUDA(cudaMemsetAsync(t->v[q].p, 0, t->nv() * t->esize(), t->stream()));
    t->staggered = false;
    if ((s = t->measure(0, 1)) != PM_OK) return s;
    DevState* st = t->host_state;
    const double datum = st->invariant;
    std::memset(st, 0, sizeof(DevState));
    st->tol = t->tolerance;
    st->datum = datum;
    st->invariant = datum;
    st->offset = 0.0;
    t->book_totals();
    st->prev_total = st->total;
    st->prev_scale = st->scale;
    return t->write_state();
}

pm_status pm_tube_max_stable_dt(pm_tube* tp, double* seconds) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    if (!seconds) return fail(PM_BAD_ARG, "null output");
    const double inf = std::numeric_limits<double>::infinity();
    if (t->speed <= 0.0) { *seconds = inf; return PM_OK; }
    // lib.rs:495-514: the wave's dx/c, and each absorbing end's drain dx Z/(2ρc²)
    const double wave = t->dx / t->speed;
    const double rc2 = t->rc2();
    auto drain = [&](int e) {
        if (t->end_kind[e] == 0) return inf;
        if (t->end_kind[e] == 1) return t->dx * t->impedance() / (2.0 * rc2);
        const double zz = t->end_z[e] > 0.0 ? t->end_z[e] : t->impedance();
        return t->dx * zz / (2.0 * rc2);
    };
    *seconds = std::min(std::min(wave, drain(0)), drain(1));
    return PM_OK;
}

pm_status pm_tube_set_tolerance(pm_tube* tp, double tol) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    t->tolerance = tol;
    return PM_OK;
}

pm_status pm_tube_step(pm_tube* tp, double dt, long long nsteps, pm_violation* out) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    if (nsteps < 0) return fail(PM_BAD_ARG, "nsteps must be >= 0");
    if (nsteps == 0) return PM_OK;
    // lib.rs:517-527 (Tube::courant, lib.rs:358-360)
    const double courant = t->speed * dt / t->dx;
    if (courant > 1.0 + 1e-12) {
        fill_violation(out, "Courant number", t->name + " (explicit wave equation)", 1.0, courant, 1.0, 1e-12, 1);
        set_error("Courant number past the limit");
        return PM_VIOLATION;
    }
    if (dt <= 0.0) return PM_OK;  // lib.rs:528-530
    pm_status s;
    if ((s = t->begin_call()) != PM_OK) return s;
    const long long before = t->host_state->steps;
    long long remaining = nsteps;
    if (!t->staggered) {
        PM_CUDA(t->launch(t->parity, dt, true, t->stream()));
        t->parity ^= 1;
        t->staggered = true;
        remaining -= 1;
    }
    s = t->run_steps(remaining, dt, true, [t, dt](int par, cudaStream_t st) { return t->launch(par, dt, false, st); });
    if (s != PM_OK) return s;
    return t->finish_call(before, out, t->name + " (its own books, against what it moved on the bus)",
                          t->name + " (starting the leapfrog)", true);
}

pm_status pm_tube_ledger(pm_tube* tp, pm_ledger* out) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    if (!out) return fail(PM_BAD_ARG, "null output");
    pm_status s = t->read_state();
    if (s != PM_OK) return s;
    std::memset(out, 0, sizeof(*out));
    const DevState* st = t->host_state;
    out->total = st->part[0];  // Ledger::new().with(ENERGY, energy()) (lib.rs:535-537)
    out->scale = std::fabs(st->part[0]);
    out->n_parts = 3;
    out->parts[0] = st->part[0];
    out->parts[1] = st->injected;
    out->parts[2] = st->datum;
    out->steps = st->steps;
    return PM_OK;
}

pm_status pm_tube_download(pm_tube* tp, double* pr, double* pp, double* v) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    const int par = t->parity;
    pm_status s;
    if ((s = t->get(t->p[par], pr, (size_t)t->n)) != PM_OK) return s;
    if ((s = t->get(t->p[par ^ 1], pp, (size_t)t->n)) != PM_OK) return s;
    return t->get(t->v[par], v, t->nv());
}

pm_status pm_tube_checkpoint(pm_tube* tp) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    const int par = t->parity;
    auto save = [&](DBuf& dst, const DBuf& src, size_t count) -> pm_status {
        if (!dst.p) PM_CUDA(dst.alloc(std::max<size_t>(count, 1) * t->esize()));
        PM_CUDA(cudaMemcpyAsync(dst.p, src.p, count * t->esize(), cudaMemcpyDeviceToDevice, t->stream()));
        return PM_OK;
    };
    pm_status s;
    if ((s = save(t->sp, t->p[par], (size_t)t->n)) != PM_OK) return s;
    if ((s = save(t->sv, t->v[par], t->nv())) != PM_OK) return s;
    t->s_staggered = t->staggered;
    t->has_saved = true;
    PM_CUDA(cudaStreamSynchronize(t->stream()));
    return PM_OK;
}

pm_status pm_tube_restore(pm_tube* tp) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    if (!t->has_saved) return PM_OK;
    const int par = t->parity;
    const size_t e = t->esize();
    // lib.rs:547-554: pressure_prev = pressure = saved
    PM_CUDA(cudaMemcpyAsync(t->p[par].p, t->sp.p, (size_t)t->n * e, cudaMemcpyDeviceToDevice, t->stream()));
    PM_CUDA(cudaMemcpyAsync(t->p[par ^ 1].p, t->sp.p, (size_t)t->n * e, cudaMemcpyDeviceToDevice, t->stream()));
    PM_CUDA(cudaMemcpyAsync(t->v[par].p, t->sv.p, t->nv() * e, cudaMemcpyDeviceToDevice, t->stream()));
    t->staggered = t->s_staggered;
    pm_status s = t->measure(par, par ^ 1);
    if (s != PM_OK) return s;
    DevState* st = t->host_state;
    t->book_totals();
    st->prev_total = st->total;
    st->prev_scale = st->scale;
    return t->write_state();
}

pm_status pm_tube_set_stream(pm_tube* tp, void* stream) {
    Tube* t = reinterpret_cast<Tube*>(tp);
    TUBE_GUARD(t);
    PM_CUDA(cudaStreamSynchronize(t->stream()));
    t->user = static_cast<cudaStream_t>(stream);
    return PM_OK;
}

void pm_tube_destroy(pm_tube* tp) { delete reinterpret_cast<Tube*>(tp); }

}  // extern "C"
