// pm_bar: the device form of `Bar1D` (crates/pantometry-thermal/src/lib.rs:425-660).
#include <algorithm>
#include <limits>
#include <new>

#include "runtime.h"

namespace pm {

struct Bar : Handle {
    int n = 2;
    double dx = 0.0, area = 0.0, reference = 0.0;
    pm_substance sub{};
    DBuf field[2];  // f64 kelvin (plain) or f32 T − T_ref
    DBuf stage, saved, dpending;
    // the heat the next step takes from the bus: lumped (into the first cell) and per cell
    double lumped = 0.0;
    std::vector<double> per_cell;

    size_t esize() const { return precision == PM_PLAIN_F64 ? 8 : 4; }
    // substance.rs:211-222, lib.rs:514-520 and 546-551
    double diffusivity() const {
        return sub.thermal ? sub.conductivity / (sub.density * sub.specific_heat) : std::numeric_limits<double>::quiet_NaN();
    }
    double cell_capacity() const {
        const double volume = area * dx;
        return sub.thermal ? (sub.density * volume) * sub.specific_heat : std::numeric_limits<double>::infinity();
    }
    double fourier_number(double dt) const {
        if (!sub.thermal) return std::numeric_limits<double>::infinity();
        return diffusivity() * dt / (dx * dx);
    }
    unsigned grid(KernelId id) const {
        const size_t need = ((size_t)n + 255) / 256;
        return (unsigned)std::max<size_t>(1, std::min<size_t>(need, wave_of(id)));
    }
    cudaError_t launch(int par, double f, cudaStream_t s) const {
        if (precision == PM_PLAIN_F64) {
            BarArgs<double> a{};
            a.told = field[par].as<double>(); a.tnew = field[par ^ 1].as<double>();
            a.n = n; a.f = f; a.capacity = cell_capacity(); a.reference = reference;
            a.st = state.as<DevState>(); a.partials = partials.as<double>(); a.nblocks = grid(kBarF64);
            return launch_bar<double>(a, s);
        }
        BarArgs<float> a{};
        a.told = field[par].as<float>(); a.tnew = field[par ^ 1].as<float>();
        a.n = n; a.f = (float)f; a.capacity = cell_capacity(); a.reference = 0.0;
        a.st = state.as<DevState>(); a.partials = partials.as<double>(); a.nblocks = grid(kBarF32);
        return launch_bar<float>(a, s);
    }
    // The stored heat of the present state and the books around it (stored − taken).
    pm_status measure() {
        HeatMeasureArgs m{};
        if (precision == PM_PLAIN_F64) m.t64 = field[parity].as<double>();
        else m.d32 = field[parity].as<float>();
        m.capacity = cell_capacity();
        m.reference = reference;
        m.n = (size_t)n;
        m.st = state.as<DevState>();
        m.partials = partials.as<double>();
        m.nblocks = kMeasureBlocks;
        PM_CUDA(precision == PM_PLAIN_F64 ? launch_heat_measure_plain(m, stream()) : launch_heat_measure_f32(m, stream()));
        pm_status s = read_state();
        if (s != PM_OK) return s;
        book_totals();
        return write_state();
    }
    void book_totals() {
        DevState* st = host_state;
        const double stored = st->part[0];
        double total = stored - st->injected;
        st->total = total;
        st->scale = std::fmax(std::fabs(stored), std::fabs(st->injected));
        st->part[1] = st->injected;
        st->prev_total = st->total;
        st->prev_scale = st->scale;
    }
};

}  // namespace pm

using namespace pm;

#define BAR_GUARD(b)                                          \
    do {                                                      \
        if (!(b)) return fail(PM_BAD_ARG, "null pm_bar");      \
        cudaSetDevice((b)->device);                           \
    } while (0)

extern "C" {

pm_status pm_bar_create(const pm_bar_desc* d, pm_bar** out) {
    if (!d || !out) return fail(PM_BAD_ARG, "null argument");
    *out = nullptr;
    if (d->precision != PM_PLAIN_F64 && d->precision != PM_FIELDS_F32) return fail(PM_BAD_ARG, "unknown precision");
    Bar* b = new (std::nothrow) Bar();
    if (!b) return fail(PM_OUT_OF_MEMORY, "host allocation");
    b->name = d->name ? d->name : "bar";
    b->precision = d->precision;
    b->n = std::max(d->cells, 2);  // lib.rs:451
    b->dx = d->dx;
    b->area = d->area;
    b->sub = d->substance;
    b->reference = d->initial_kelvin;
    pm_status s = b->init(d->device, 0);
    if (s != PM_OK) { delete b; return s; }
    for (auto& f : b->field) {
        cudaError_t e = f.alloc((size_t)b->n * b->esize());
        if (e != cudaSuccess) { delete b; return cuda_fail(e, "cudaMalloc bar cells"); }
    }
    *out = reinterpret_cast<pm_bar*>(b);
    std::vector<double> t((size_t)b->n, d->initial_kelvin);  // lib.rs:452
    s = pm_bar_upload(*out, t.data(), t.size());
    if (s != PM_OK) { delete b; *out = nullptr; }
    return s;
}

pm_status pm_bar_upload(pm_bar* bp, const double* kelvin, size_t n) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    if (!kelvin || n != (size_t)b->n) return fail(PM_BAD_ARG, "upload: one temperature per cell");
    b->parity = 0;
    if (b->precision == PM_PLAIN_F64) {
        PM_CUDA(cudaMemcpyAsync(b->field[0].p, kelvin, n * 8, cudaMemcpyHostToDevice, b->stream()));
    } else {
        if (!b->stage.p || b->stage.bytes < n * 8) PM_CUDA(b->stage.alloc(n * 8));
        PM_CUDA(cudaMemcpyAsync(b->stage.p, kelvin, n * 8, cudaMemcpyHostToDevice, b->stream()));
        PM_CUDA(launch_heat_convert(b->stage.as<double>(), b->field[0].as<float>(), b->reference, n, 1, nullptr, b->stream()));
    }
    return b->measure();
}

pm_status pm_bar_download(pm_bar* bp, double* kelvin, size_t n) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    if (!kelvin || n != (size_t)b->n) return fail(PM_BAD_ARG, "download: one temperature per cell");
    if (b->precision == PM_PLAIN_F64) {
        PM_CUDA(cudaMemcpyAsync(kelvin, b->field[b->parity].p, n * 8, cudaMemcpyDeviceToHost, b->stream()));
    } else {
        if (!b->stage.p || b->stage.bytes < n * 8) PM_CUDA(b->stage.alloc(n * 8));
        PM_CUDA(launch_heat_convert(nullptr, b->field[b->parity].as<float>(), b->reference, n, 0, b->stage.as<double>(), b->stream()));
        PM_CUDA(cudaMemcpyAsync(kelvin, b->stage.p, n * 8, cudaMemcpyDeviceToHost, b->stream()));
    }
    PM_CUDA(cudaStreamSynchronize(b->stream()));
    return PM_OK;
}

pm_status pm_bar_sample(pm_bar* bp, const double* lo, const double* hi, const int* samples, double* out, size_t n) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    SampleGrid g{};
    pm_status s = sample_grid_of(lo, hi, samples, out, n, g);
    if (s != PM_OK) return s;
    g.dx = b->dx;
    g.nx = b->n; g.ny = 1; g.nz = 1;
    return run_sample(b, out, n, [&](double* dev, cudaStream_t st) {
        return b->precision == PM_PLAIN_F64
                   ? launch_bar_sample<double>(g, b->field[b->parity].as<double>(), 0.0, dev, st)
                   : launch_bar_sample<float>(g, b->field[b->parity].as<float>(), b->reference, dev, st);
    });
}

pm_status pm_bar_absorb(pm_bar* bp, double joules) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    b->lumped += joules;
    return PM_OK;
}

pm_status pm_bar_deposit(pm_bar* bp, const double* joules, size_t n) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    if (!joules || n != (size_t)b->n) return fail(PM_BAD_ARG, "deposit: one amount per cell");
    if (b->per_cell.empty()) b->per_cell.assign((size_t)b->n, 0.0);
    for (size_t i = 0; i < n; ++i) b->per_cell[i] += joules[i];
    return PM_OK;
}

pm_status pm_bar_max_stable_dt(pm_bar* bp, double* seconds) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    if (!seconds) return fail(PM_BAD_ARG, "null output");
    // lib.rs:564-569
    *seconds = b->sub.thermal ? b->dx * b->dx / (2.0 * b->diffusivity()) : std::numeric_limits<double>::infinity();
    return PM_OK;
}

pm_status pm_bar_set_tolerance(pm_bar* bp, double tol) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    b->tolerance = tol;
    return PM_OK;
}

pm_status pm_bar_step(pm_bar* bp, double dt, long long nsteps, pm_violation* out) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    if (nsteps < 0) return fail(PM_BAD_ARG, "nsteps must be >= 0");
    if (nsteps == 0) return PM_OK;
    // lib.rs:571-589
    const double f = b->fourier_number(dt);
    if (!std::isfinite(f)) {  // Violation::at (conserved.rs:149-158)
        fill_violation(out, "substance has no diffusivity", b->name, f, f, std::fabs(f), 0.0, 1);
        set_error("substance has no diffusivity");
        return PM_VIOLATION;
    }
    if (f > 0.5 + 1e-12) {
        fill_violation(out, "Fourier number", b->name + " (explicit conduction)", 0.5, f, 0.5, 1e-12, 1);
        set_error("Fourier number past the explicit limit");
        return PM_VIOLATION;
    }
    pm_status s;
    if ((s = b->begin_call()) != PM_OK) return s;
    const long long before = b->host_state->steps;
    // lib.rs:590-606: the heat handed in since the last step, before it conducts; the books
    // take it as what came from the bus
    if (b->lumped != 0.0 || !b->per_cell.empty()) {
        double taken = b->lumped;
        const double* dev = nullptr;
        if (!b->per_cell.empty()) {
            if (!b->dpending.p || b->dpending.bytes < (size_t)b->n * 8) PM_CUDA(b->dpending.alloc((size_t)b->n * 8));
            PM_CUDA(b->put_sync(b->dpending.p, b->per_cell.data(), (size_t)b->n * 8));
            dev = b->dpending.as<double>();
            double total = 0.0;
            for (double j : b->per_cell) total += j;
            taken += total;
        }
        const double cap = b->cell_capacity();
        cudaError_t e = b->precision == PM_PLAIN_F64
                            ? launch_bar_deposit<double>(b->field[b->parity].as<double>(), dev, b->lumped, cap, b->n, b->stream())
                            : launch_bar_deposit<float>(b->field[b->parity].as<float>(), dev, b->lumped, cap, b->n, b->stream());
        PM_CUDA(e);
        b->host_state->injected += taken;
        if ((s = b->write_state()) != PM_OK) return s;
        b->lumped = 0.0;
        b->per_cell.clear();
    }
    s = b->run_steps(nsteps, dt, true, [b, f](int par, cudaStream_t st) { return b->launch(par, f, st); });
    if (s != PM_OK) return s;
    return b->finish_call(before, out, b->name + " (its own books, against what it moved on the bus)", b->name, true);
}

pm_status pm_bar_ledger(pm_bar* bp, pm_ledger* out) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    if (!out) return fail(PM_BAD_ARG, "null output");
    pm_status s = b->read_state();
    if (s != PM_OK) return s;
    std::memset(out, 0, sizeof(*out));
    const DevState* st = b->host_state;
    out->total = st->part[0];  // Ledger::new().with(ENERGY, stored_heat()) (lib.rs:629-631)
    out->scale = std::fabs(st->part[0]);
    out->n_parts = 2;
    out->parts[0] = st->part[0];
    out->parts[1] = st->injected;  // `absorbed_energy`
    out->steps = st->steps;
    return PM_OK;
}

pm_status pm_bar_checkpoint(pm_bar* bp) {  // lib.rs:633-635: the cells
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    if (!b->saved.p) PM_CUDA(b->saved.alloc((size_t)b->n * b->esize()));
    PM_CUDA(cudaMemcpyAsync(b->saved.p, b->field[b->parity].p, (size_t)b->n * b->esize(), cudaMemcpyDeviceToDevice, b->stream()));
    b->has_saved = true;
    PM_CUDA(cudaStreamSynchronize(b->stream()));
    return PM_OK;
}

pm_status pm_bar_restore(pm_bar* bp) {  // lib.rs:637-639
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    if (!b->has_saved) return PM_OK;
    PM_CUDA(cudaMemcpyAsync(b->field[b->parity].p, b->saved.p, (size_t)b->n * b->esize(), cudaMemcpyDeviceToDevice, b->stream()));
    return b->measure();
}

pm_status pm_bar_set_stream(pm_bar* bp, void* stream) {
    Bar* b = reinterpret_cast<Bar*>(bp);
    BAR_GUARD(b);
    PM_CUDA(cudaStreamSynchronize(b->stream()));
    b->user = static_cast<cudaStream_t>(stream);
    return PM_OK;
}

void pm_bar_destroy(pm_bar* bp) { delete reinterpret_cast<Bar*>(bp); }

}  // extern "C"
