// pm_room: the device form of `Room` (crates/pantometry-acoustic/src/room.rs).
#include <algorithm>
#include <limits>
#include <new>

#include "runtime.h"

namespace pm {

struct Room : Handle {
    int nx = 3, ny = 3;
    double dx = 0.0, speed = 0.0, density = 0.0, depth = 0.0;
    bool staggered = false;  // room.rs:74 `velocity_staggered`
    DBuf p[2], vx[2], vy[2];
    DBuf stage;
    DBuf sp, svx, svy;       // checkpoint (room.rs:484-505)
    bool s_staggered = false;

    size_t nodes() const { return (size_t)nx * ny; }
    size_t nvx() const { return (size_t)(nx - 1) * ny; }
    size_t nvy() const { return (size_t)nx * (ny - 1); }
    size_t esize() const { return precision == PM_PLAIN_F64 ? 8 : 4; }
    double rc2() const { return density * speed * speed; }
    double volume() const { return dx * dx * depth; }
    // room.rs:243-248: the invariant is zero for a medium with no stiffness
    double knode() const { return rc2() <= 0.0 ? 0.0 : volume() / (2.0 * rc2()); }
    double kface() const { return rc2() <= 0.0 ? 0.0 : 0.5 * density * volume(); }
    unsigned grid(KernelId id) const {
        const unsigned w = wave_of(id);
        const size_t need = (nodes() + 255) / 256;
        return (unsigned)std::max<size_t>(1, std::min<size_t>(need, w));
    }

    template <typename Real>
    RoomArgs<Real> args(int par, double h, bool starting) const {
        RoomArgs<Real> a{};
        a.p0 = p[par].as<Real>(); a.vx0 = vx[par].as<Real>(); a.vy0 = vy[par].as<Real>();
        a.p1 = p[par ^ 1].as<Real>(); a.vx1 = vx[par ^ 1].as<Real>(); a.vy1 = vy[par ^ 1].as<Real>();
        a.nx = nx; a.ny = ny;
        const double vh = starting ? 0.5 * h : h;  // room.rs:387
        a.gain = (Real)(vh / (density * dx));       // room.rs:407
        a.scale = (Real)(h * rc2() / dx);           // room.rs:443
        a.knode = knode();
        a.kface = kface();
        a.starting = starting ? 1 : 0;
        a.nblocks = grid(sizeof(Real) == 8 ? kRoomF64 : kRoomF32);
        a.st = state.as<DevState>();
        a.partials = partials.as<double>();
        return a;
    }
    cudaError_t launch(int par, double h, bool starting, cudaStream_t s) const {
        if (precision == PM_PLAIN_F64) return launch_room<double>(args<double>(par, h, starting), s);
        return launch_room<float>(args<float>(par, h, starting), s);
    }

    // The invariant of the present state (pressure of parity par_p against par_pp, the faces of
    // `parity`), into host_state->invariant.
    pm_status measure(int par_p, int par_pp) {
        if (precision == PM_PLAIN_F64) {
            RoomMeasureArgs<double> m{};
            m.p = p[par_p].as<double>(); m.pp = p[par_pp].as<double>();
            m.vx = vx[parity].as<double>(); m.vy = vy[parity].as<double>();
            m.nx = nx; m.ny = ny; m.knode = knode(); m.kface = kface();
            m.st = state.as<DevState>(); m.partials = partials.as<double>(); m.nblocks = grid(kRoomF64);
            PM_CUDA(launch_room_measure<double>(m, stream()));
        } else {
            RoomMeasureArgs<float> m{};
            m.p = p[par_p].as<float>(); m.pp = p[par_pp].as<float>();
            m.vx = vx[parity].as<float>(); m.vy = vy[parity].as<float>();
            m.nx = nx; m.ny = ny; m.knode = knode(); m.kface = kface();
            m.st = state.as<DevState>(); m.partials = partials.as<double>(); m.nblocks = grid(kRoomF32);
            PM_CUDA(launch_room_measure<float>(m, stream()));
        }
        return read_state();
    }

    // Host f64 → device field (converted to f32 on the device for the chosen form).
    pm_status put(DBuf& dst, const double* src_host, size_t n) {
        if (precision == PM_PLAIN_F64) {
            PM_CUDA(cudaMemcpyAsync(dst.p, src_host, n * 8, cudaMemcpyHostToDevice, stream()));
        } else {
            if (!stage.p || stage.bytes < n * 8) PM_CUDA(stage.alloc(std::max<size_t>(n, 1) * 8));
            PM_CUDA(cudaMemcpyAsync(stage.p, src_host, n * 8, cudaMemcpyHostToDevice, stream()));
            PM_CUDA(launch_to_f32(stage.as<double>(), dst.as<float>(), n, stream()));
        }
        return PM_OK;
    }
    pm_status get(const DBuf& src_dev, double* dst_host, size_t n) {
        if (!dst_host || n == 0) return PM_OK;
        if (precision == PM_PLAIN_F64) {
            PM_CUDA(cudaMemcpyAsync(dst_host, src_dev.p, n * 8, cudaMemcpyDeviceToHost, stream()));
        } else {
            if (!stage.p || stage.bytes < n * 8) PM_CUDA(stage.alloc(std::max<size_t>(n, 1) * 8));
            PM_CUDA(launch_to_f64(src_dev.as<float>(), stage.as<double>(), n, stream()));
            PM_CUDA(cudaMemcpyAsync(dst_host, stage.p, n * 8, cudaMemcpyDeviceToHost, stream()));
        }
        PM_CUDA(cudaStreamSynchronize(stream()));
        return PM_OK;
    }
    // The ledger of the state in host_state: the energy, invariant + startup offset.
    void book_totals() {
        DevState* st = host_state;
        st->total = st->invariant + st->offset;
        st->scale = std::fabs(st->total);
        st->part[0] = st->total;
    }
};

}  // namespace pm

using namespace pm;

#define ROOM_GUARD(r)                                          \
    do {                                                       \
        if (!(r)) return fail(PM_BAD_ARG, "null pm_room");      \
        cudaSetDevice((r)->device);                            \
    } while (0)

extern "C" {

pm_status pm_room_create(const pm_room_desc* d, pm_room** out) {
    if (!d || !out) return fail(PM_BAD_ARG, "null argument");
    *out = nullptr;
    if (d->precision != PM_PLAIN_F64 && d->precision != PM_FIELDS_F32) return fail(PM_BAD_ARG, "unknown precision");
    Room* r = new (std::nothrow) Room();
    if (!r) return fail(PM_OUT_OF_MEMORY, "host allocation");
    r->name = d->name ? d->name : "room";
    r->precision = d->precision;
    // room.rs:99-101
    r->nx = std::max(d->across, 3);
    r->dx = d->width / (double)(r->nx - 1);
    r->ny = std::max((int)std::round(d->height / r->dx) + 1, 3);
    r->speed = d->speed;
    r->density = d->density;
    r->depth = d->depth;
    pm_status s = r->init(d->device, 0);
    if (s != PM_OK) { delete r; return s; }
    for (int q = 0; q < 2; ++q) {
        cudaError_t e;
        if ((e = r->p[q].alloc(r->nodes() * r->esize())) != cudaSuccess ||
            (e = r->vx[q].alloc(r->nvx() * r->esize())) != cudaSuccess ||
            (e = r->vy[q].alloc(r->nvy() * r->esize())) != cudaSuccess) {
            delete r;
            return cuda_fail(e, "cudaMalloc room fields");
        }
    }
    *out = reinterpret_cast<pm_room*>(r);
    std::vector<double> zero(r->nodes(), 0.0);
    s = pm_room_release(*out, zero.data(), zero.size());  // Room::new is at rest
    if (s != PM_OK) { delete r; *out = nullptr; }
    return s;
}

pm_status pm_room_cells(pm_room* rp, int* nx, int* ny, double* dx) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    if (nx) *nx = r->nx;
    if (ny) *ny = r->ny;
    if (dx) *dx = r->dx;
    return PM_OK;
}

pm_status pm_room_release(pm_room* rp, const double* pressure, size_t n) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    if (!pressure || n != r->nodes()) return fail(PM_BAD_ARG, "release: one pressure per node");
    // room.rs:140-160: pressure from the profile, pressure_prev = pressure, v = 0, then the datum
    r->parity = 0;
    pm_status s;
    if ((s = r->put(r->p[0], pressure, n)) != PM_OK) return s;
    PM_CUDA(cudaMemcpyAsync(r->p[1].p, r->p[0].p, n * r->esize(), cudaMemcpyDeviceToDevice, r->stream()));
    for (int q = 0; q < 2; ++q) {
        PM_CUDA(cudaMemsetAsync(r->vx[q].p, 0, r->nvx() * r->esize(), r->stream()));
        PM_CUDA(cudaMemsetAsync(r->vy[q].p, 0, r->nvy() * r->esize(), r->stream()));
    }
    r->staggered = false;
    if ((s = r->measure(0, 1)) != PM_OK) return s;
    DevState* st = r->host_state;
    const double datum = st->invariant;
    std::memset(st, 0, sizeof(DevState));
    st->tol = r->tolerance;
    st->datum = datum;
    st->invariant = datum;
    st->offset = 0.0;
    r->book_totals();  // Ledger::new().with(ENERGY, energy()) with energy = invariant + 0
    st->prev_total = st->total;
    st->prev_scale = st->scale;
    return r->write_state();
}

pm_status pm_room_max_stable_dt(pm_room* rp, double* seconds) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    if (!seconds) return fail(PM_BAD_ARG, "null output");
    *seconds = r->speed <= 0.0 ? std::numeric_limits<double>::infinity() : r->dx / (r->speed * std::sqrt(2.0));
    return PM_OK;
}

pm_status pm_room_set_tolerance(pm_room* rp, double tol) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    r->tolerance = tol;
    return PM_OK;
}

pm_status pm_room_step(pm_room* rp, double dt, long long nsteps, pm_violation* out) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    if (nsteps < 0) return fail(PM_BAD_ARG, "nsteps must be >= 0");
    if (nsteps == 0) return PM_OK;
    // room.rs:369-380 (Room::courant, room.rs:336-338)
    const double courant = r->speed * dt * std::sqrt(2.0) / r->dx;
    if (courant > 1.0 + 1e-12) {
        fill_violation(out, "Courant number", r->name + " (two-dimensional wave equation)", 1.0, courant, 1.0, 1e-12, 1);
        set_error("Courant number past the limit");
        return PM_VIOLATION;
    }
    if (dt <= 0.0) return PM_OK;  // room.rs:381-384
    pm_status s;
    if ((s = r->begin_call()) != PM_OK) return s;
    const long long before = r->host_state->steps;
    long long remaining = nsteps;
    if (!r->staggered) {
        PM_CUDA(r->launch(r->parity, dt, true, r->stream()));
        r->parity ^= 1;
        r->staggered = true;
        remaining -= 1;
    }
    s = r->run_steps(remaining, dt, true, [r, dt](int par, cudaStream_t st) { return r->launch(par, dt, false, st); });
    if (s != PM_OK) return s;
    return r->finish_call(before, out, r->name + " (its own books, against what it moved on the bus)",
                          r->name + " (starting the leapfrog)", true);
}

pm_status pm_room_ledger(pm_room* rp, pm_ledger* out) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    if (!out) return fail(PM_BAD_ARG, "null output");
    pm_status s = r->read_state();
    if (s != PM_OK) return s;
    std::memset(out, 0, sizeof(*out));
    const DevState* st = r->host_state;
    out->total = st->total;
    out->scale = st->scale;
    out->n_parts = 3;
    out->parts[0] = st->invariant;
    out->parts[1] = st->offset;
    out->parts[2] = st->datum;
    out->steps = st->steps;
    return PM_OK;
}

pm_status pm_room_download(pm_room* rp, double* pr, double* pp, double* vx, double* vy) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    const int par = r->parity;
    pm_status s;
    if ((s = r->get(r->p[par], pr, r->nodes())) != PM_OK) return s;
    if ((s = r->get(r->p[par ^ 1], pp, r->nodes())) != PM_OK) return s;
    if ((s = r->get(r->vx[par], vx, r->nvx())) != PM_OK) return s;
    return r->get(r->vy[par], vy, r->nvy());
}

pm_status pm_room_sample(pm_room* rp, const double* lo, const double* hi, const int* samples, double* out, size_t n) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    SampleGrid g{};
    pm_status s = sample_grid_of(lo, hi, samples, out, n, g);
    if (s != PM_OK) return s;
    g.dx = r->dx;
    g.nx = r->nx; g.ny = r->ny; g.nz = 1;
    return run_sample(r, out, n, [&](double* dev, cudaStream_t st) {
        return r->precision == PM_PLAIN_F64 ? launch_room_sample<double>(g, r->p[r->parity].as<double>(), dev, st)
                                            : launch_room_sample<float>(g, r->p[r->parity].as<float>(), dev, st);
    });
}

pm_status pm_room_checkpoint(pm_room* rp) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    const int par = r->parity;
    auto save = [&](DBuf& dst, const DBuf& src, size_t n) -> pm_status {
        if (!dst.p) PM_CUDA(dst.alloc(std::max<size_t>(n, 1) * r->esize()));
        PM_CUDA(cudaMemcpyAsync(dst.p, src.p, n * r->esize(), cudaMemcpyDeviceToDevice, r->stream()));
        return PM_OK;
    };
    pm_status s;
    if ((s = save(r->sp, r->p[par], r->nodes())) != PM_OK) return s;
    if ((s = save(r->svx, r->vx[par], r->nvx())) != PM_OK) return s;
    if ((s = save(r->svy, r->vy[par], r->nvy())) != PM_OK) return s;
    r->s_staggered = r->staggered;
    r->has_saved = true;
    PM_CUDA(cudaStreamSynchronize(r->stream()));
    return PM_OK;
}

pm_status pm_room_restore(pm_room* rp) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    if (!r->has_saved) return PM_OK;
    const int par = r->parity;
    const size_t e = r->esize();
    // room.rs:493-503: pressure_prev = pressure = saved
    PM_CUDA(cudaMemcpyAsync(r->p[par].p, r->sp.p, r->nodes() * e, cudaMemcpyDeviceToDevice, r->stream()));
    PM_CUDA(cudaMemcpyAsync(r->p[par ^ 1].p, r->sp.p, r->nodes() * e, cudaMemcpyDeviceToDevice, r->stream()));
    PM_CUDA(cudaMemcpyAsync(r->vx[par].p, r->svx.p, r->nvx() * e, cudaMemcpyDeviceToDevice, r->stream()));
    PM_CUDA(cudaMemcpyAsync(r->vy[par].p, r->svy.p, r->nvy() * e, cudaMemcpyDeviceToDevice, r->stream()));
    r->staggered = r->s_staggered;
    pm_status s = r->measure(par, par ^ 1);
    if (s != PM_OK) return s;
    DevState* st = r->host_state;
    r->book_totals();
    st->prev_total = st->total;
    st->prev_scale = st->scale;
    return r->write_state();
}

pm_status pm_room_set_stream(pm_room* rp, void* stream) {
    Room* r = reinterpret_cast<Room*>(rp);
    ROOM_GUARD(r);
    PM_CUDA(cudaStreamSynchronize(r->stream()));
    r->user = static_cast<cudaStream_t>(stream);
    return PM_OK;
}

void pm_room_destroy(pm_room* rp) { delete reinterpret_cast<Room*>(rp); }

}  // extern "C"
