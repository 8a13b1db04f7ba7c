// pm_hall: the device form of `Hall` (crates/pantometry-acoustic/src/hall.rs).
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <limits>
#include <new>

#include "runtime.h"

namespace pm {

struct Hall : Handle {
    int nx = 2, ny = 1, nz = 1;
    double dx = 0.0, speed = 0.0, density = 0.0;
    bool staggered = false;  // hall.rs:84-85 `velocity_staggered`
    DBuf p[2], vx[2], vy[2], vz[2];
    DBuf stage;
    // point source (extension)
    long long src = -1;
    DBuf wave;
    long long nwave = 0;
    double wsrc = 0.0;
    // heterogeneous speed (extension)
    int block = 0, nbx = 0, nby = 0, nbz = 0;
    DBuf bscale, bknode;
    std::vector<double> speeds;
    double max_speed = 0.0;
    double bscale_dt = NAN;
    // checkpoint (hall.rs:536-555)
    DBuf sp, svx, svy, svz;
    bool s_staggered = false;
    // FP32 halls whose x extent is a multiple of 4 keep the face arrays padded to the node grid
    // and step with the TMA-staged kernel (hall_tma.cuh); maps[par] describe the fields of parity par
    bool tma = false;
    HallMaps maps[2];
    int tshape = 0;  // the TMA kernel's tile shape, an index of kHallTmaShapes

    size_t nodes() const { return (size_t)nx * ny * nz; }
    size_t nvx() const { return (size_t)(nx - 1) * ny * nz; }
    size_t nvy() const { return (size_t)nx * (ny - 1) * nz; }
    size_t nvz() const { return (size_t)nx * ny * (nz - 1); }
    // elements held on the device per face array (the padded layout keeps one per node)
    size_t dvx() const { return tma ? nodes() : nvx(); }
    size_t dvy() const { return tma ? nodes() : nvy(); }
    size_t dvz() const { return tma ? nodes() : nvz(); }
    size_t esize() const { return precision == PM_PLAIN_F64 ? 8 : 4; }
    double rc2() const { return density * speed * speed; }
    double volume() const { return dx * dx * dx; }

    template <typename Real>
    HallArgs<Real> args(int par, double h, bool starting) const {
        HallArgs<Real> a{};
        a.p0 = p[par].as<Real>(); a.vx0 = vx[par].as<Real>(); a.vy0 = vy[par].as<Real>(); a.vz0 = vz[par].as<Real>();
        a.p1 = p[par ^ 1].as<Real>(); a.vx1 = vx[par ^ 1].as<Real>(); a.vy1 = vy[par ^ 1].as<Real>(); a.vz1 = vz[par ^ 1].as<Real>();
        a.nx = nx; a.ny = ny; a.nz = nz;
        const double vh = starting ? 0.5 * h : h;  // hall.rs:428
        a.gain = (Real)(vh / (density * dx));       // hall.rs:433
        a.scale = (Real)(h * rc2() / dx);           // hall.rs:464
        if (block > 0) {
            a.block_scale = bscale.as<Real>();
            a.block_knode = bknode.as<double>();
            a.block = block; a.nbx = nbx; a.nby = nby;
        }
        a.knode = volume() / (2.0 * rc2());
        a.kface = 0.5 * density * volume();
        a.src = src;
        a.src_i = a.src_j = a.src_k = -1;
        if (src >= 0) {
            a.src_i = (int)(src % nx);
            a.src_j = (int)((src / nx) % ny);
            a.src_k = (int)(src / ((long long)nx * ny));
        }
        a.wave = wave.as<double>();
        a.nwave = nwave;
        a.wsrc = wsrc;
        a.starting = starting ? 1 : 0;
        const unsigned w = wave_of(sizeof(Real) == 8 ? kHallF64 : (tma ? hall_tma_kernel_id(tshape) : kHallF32));
        a.tiles = make_tiles(nx, ny, nz, choose_zc(nx, ny, nz, w, (sizeof(Real) == 4 && tma) ? kHallTmaShapes[tshape].planes : 4));
        a.nblocks = grid_for(a.tiles, w);
        a.st = state.as<DevState>();
        a.partials = partials.as<double>();
        return a;
    }

    cudaError_t launch(int par, double h, bool starting, cudaStream_t s) const {
        if (precision == PM_PLAIN_F64) return launch_hall<double>(args<double>(par, h, starting), s);
        if (tma) return launch_hall_tma(args<float>(par, h, starting), maps[par], tshape, s);
        return launch_hall<float>(args<float>(par, h, starting), s);
    }
    pm_status launch_one(int par, double h, bool starting, cudaStream_t s) const {
        PM_CUDA(launch(par, h, starting, s));
        return PM_OK;
    }

    // Tensor maps of both parities' fields, with the boxes hall_tma_step loads.
    pm_status build_maps() {
        const unsigned P = (unsigned)kHallTmaShapes[tshape].planes;
        for (int q = 0; q < 2; ++q) {
            if (!hall_tma_map(&maps[q].p, p[q].p, nx, ny, nz, 40, 10, P + 2) ||
                !hall_tma_map(&maps[q].vx, vx[q].p, nx, ny, nz, 36, 8, P) ||
                !hall_tma_map(&maps[q].vy, vy[q].p, nx, ny, nz, 32, 9, P) ||
                !hall_tma_map(&maps[q].vz, vz[q].p, nx, ny, nz, 32, 8, P + 1))
                return fail(PM_CUDA_ERROR, "cuTensorMapEncodeTiled refused a hall field");
        }
        return PM_OK;
    }

    // Time `trial` steps of every TMA tile shape on the present state and keep the fastest. Each
    // trial step reads the present parity and writes the other one. The other parity's velocities
    // are free between steps; its pressure is the previous pressure the invariant reads (hall.rs
    // keeps `p_prev`), so it is copied aside first (on the device where there is room, else on the
    // host) and put back after the trials, as are the books (the source's clock among them). A grid
    // shape (nx, ny, nz, with or without speed blocks) timed once on a device is not timed again in
    // the process.
    pm_status autotune(int trial) {
        if (!tma) return PM_OK;
        static std::mutex cache_mutex;
        static std::map<std::tuple<int, int, int, int, int>, int> cache;
        const auto key = std::make_tuple(nx, ny, nz, block > 0 ? 1 : 0, device);
        {
            std::lock_guard<std::mutex> lock(cache_mutex);
            auto it = cache.find(key);
            if (it != cache.end()) return set_shape(it->second);
        }
        pm_status s = read_state();
        if (s != PM_OK) return s;
        const DevState books = *host_state;
        const size_t pbytes = nodes() * esize();
        DBuf aside;
        std::vector<unsigned char> aside_host;
        if (aside.alloc(pbytes) == cudaSuccess) {
            PM_CUDA(cudaMemcpyAsync(aside.p, p[parity ^ 1].p, pbytes, cudaMemcpyDeviceToDevice, stream()));
        } else {
            cudaGetLastError();  // the refused allocation is not an error of the stream
            aside_host.resize(pbytes);
            PM_CUDA(cudaMemcpyAsync(aside_host.data(), p[parity ^ 1].p, pbytes, cudaMemcpyDeviceToHost, stream()));
            PM_CUDA(cudaStreamSynchronize(stream()));
        }
        const double c = block > 0 ? max_speed : speed;
        const double dt = 0.5 * dx / (c * std::sqrt(3.0));
        if ((s = upload_block_scale(dt)) != PM_OK) return s;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        PM_CUDA(cudaEventCreate(&e0));
        PM_CUDA(cudaEventCreate(&e1));
        int best = tshape;
        float best_ms = 0.0f;
        for (int sh = 0; sh < kHallTmaShapeCount && s == PM_OK; ++sh) {
            if ((s = set_shape(sh)) != PM_OK) break;
            host_state->tol = -1.0;  // no audit while timing
            if ((s = write_state()) != PM_OK) break;
            for (int q = 0; q < 2 + trial; ++q) {
                if (q == 2) PM_CUDA(cudaEventRecord(e0, stream()));
                PM_CUDA(launch(parity, dt, false, stream()));
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
        PM_CUDA(cudaMemcpyAsync(p[parity ^ 1].p, aside.p ? aside.p : (void*)aside_host.data(), pbytes,
                                aside.p ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream()));
        PM_CUDA(cudaStreamSynchronize(stream()));
        {
            std::lock_guard<std::mutex> lock(cache_mutex);
            cache[key] = best;
        }
        return set_shape(best);
    }
    pm_status set_shape(int sh) {
        if (sh < 0 || sh >= kHallTmaShapeCount) return fail(PM_BAD_ARG, "hall tile shape");
        if (!tma || sh == tshape) return PM_OK;
        PM_CUDA(cudaStreamSynchronize(stream()));
        tshape = sh;
        drop_graphs();
        return build_maps();
    }

    // The ledger of the state in host_state: the energy, then the source's injected work as an
    // entry of its own, the same two entries the step kernel books.
    void book_totals() {
        DevState* st = host_state;
        const double energy = st->invariant + st->offset;
        st->total = energy - st->injected;
        st->scale = std::fmax(std::fabs(energy), std::fabs(st->injected));
        st->part[0] = st->total;
    }

    // The source node's share of the invariant, share · V/(2ρc²), at the speed of the source's
    // own block when the medium has blocks (whichever of the source and the blocks came first).
    void weigh_source() {
        if (src < 0) return;
        const int i = (int)(src % nx), j = (int)((src / nx) % ny), k = (int)(src / ((long long)nx * ny));
        auto w = [](int q, int m) { return (q == 0 || q + 1 == m) ? 2.0 : 1.0; };
        const double share = 1.0 / (w(i, nx) * w(j, ny) * w(k, nz));
        double r = rc2();
        if (block > 0) {
            const double c = speeds[(size_t)(i / block) + (size_t)nbx * ((size_t)(j / block) + (size_t)nby * (k / block))];
            r = density * c * c;
        }
        wsrc = share * (dx * dx * dx) / (2.0 * r);
    }

    // Per-block scale h·ρc_b²/dx (in the field type) and invariant weight V/(2ρc_b²).
    pm_status upload_block_scale(double h) {
        if (block <= 0 || bscale_dt == h) return PM_OK;
        const size_t nb = speeds.size();
        std::vector<double> kn(nb), sc64(nb);
        std::vector<float> sc32(nb);
        for (size_t b = 0; b < nb; ++b) {
            const double r = density * speeds[b] * speeds[b];
            kn[b] = volume() / (2.0 * r);
            sc64[b] = h * r / dx;
            sc32[b] = (float)sc64[b];
        }
        if (!bscale.p) PM_CUDA(bscale.alloc(nb * 8));
        if (!bknode.p) PM_CUDA(bknode.alloc(nb * 8));
        if (precision == PM_PLAIN_F64) PM_CUDA(put_sync(bscale.p, sc64.data(), nb * 8));
        else PM_CUDA(put_sync(bscale.p, sc32.data(), nb * 4));
        PM_CUDA(put_sync(bknode.p, kn.data(), nb * 8));
        bscale_dt = h;
        drop_graphs();
        return PM_OK;
    }

    // `invariant_si` of the present state (hall.rs:334-384), into host_state->invariant.
    pm_status measure(int par_p, int par_pp) {
        if (precision == PM_PLAIN_F64) {
            HallMeasureArgs<double> m{};
            m.p = p[par_p].as<double>(); m.pp = p[par_pp].as<double>();
            m.vx = vx[parity].as<double>(); m.vy = vy[parity].as<double>(); m.vz = vz[parity].as<double>();
            m.nx = nx; m.ny = ny; m.nz = nz;
            m.knode = volume() / (2.0 * rc2()); m.kface = 0.5 * density * volume();
            if (block > 0) { m.block_knode = bknode.as<double>(); m.block = block; m.nbx = nbx; m.nby = nby; }
            m.tiles = make_tiles(nx, ny, nz, choose_zc(nx, ny, nz, resident)); m.nblocks = grid_for(m.tiles, resident);
            m.st = state.as<DevState>(); m.partials = partials.as<double>();
            PM_CUDA(launch_hall_measure<double>(m, stream()));
        } else {
            HallMeasureArgs<float> m{};
            m.p = p[par_p].as<float>(); m.pp = p[par_pp].as<float>();
            m.vx = vx[parity].as<float>(); m.vy = vy[parity].as<float>(); m.vz = vz[parity].as<float>();
            m.nx = nx; m.ny = ny; m.nz = nz;
            m.knode = volume() / (2.0 * rc2()); m.kface = 0.5 * density * volume();
            if (block > 0) { m.block_knode = bknode.as<double>(); m.block = block; m.nbx = nbx; m.nby = nby; }
            m.padded = tma ? 1 : 0;
            m.tiles = make_tiles(nx, ny, nz, choose_zc(nx, ny, nz, resident)); m.nblocks = grid_for(m.tiles, resident);
            m.st = state.as<DevState>(); m.partials = partials.as<double>();
            PM_CUDA(launch_hall_measure<float>(m, stream()));
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
    // A face array to the host in the reference's layout (hall.rs:67-77): the padded layout
    // drops the high column (x), row (y) or plane (z) of each array.
    pm_status get_face(int axis, const DBuf& src_dev, double* dst_host) {
        if (!dst_host) return PM_OK;
        const size_t n = axis == 0 ? nvx() : axis == 1 ? nvy() : nvz();
        if (!tma) return get(src_dev, dst_host, n);
        if (n == 0) return PM_OK;
        if (!stage.p || stage.bytes < nodes() * 8) PM_CUDA(stage.alloc(nodes() * 8));
        PM_CUDA(launch_to_f64(src_dev.as<float>(), stage.as<double>(), nodes(), stream()));
        const size_t row = (size_t)nx * 8;
        if (axis == 0)
            PM_CUDA(cudaMemcpy2DAsync(dst_host, (nx - 1) * 8, stage.p, row, (nx - 1) * 8, (size_t)ny * nz,
                                      cudaMemcpyDeviceToHost, stream()));
        else if (axis == 1)
            PM_CUDA(cudaMemcpy2DAsync(dst_host, row * (ny - 1), stage.p, row * ny, row * (ny - 1), nz,
                                      cudaMemcpyDeviceToHost, stream()));
        else
            PM_CUDA(cudaMemcpyAsync(dst_host, stage.p, n * 8, cudaMemcpyDeviceToHost, stream()));
        PM_CUDA(cudaStreamSynchronize(stream()));
        return PM_OK;
    }
    pm_status get(const DBuf& src_dev, double* dst_host, size_t n) {
        if (!dst_host) return PM_OK;
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
};

}  // namespace pm

using namespace pm;

#define HALL_GUARD(h)                                          \
    do {                                                       \
        if (!(h)) return fail(PM_BAD_ARG, "null pm_hall");      \
        cudaSetDevice((h)->device);                            \
    } while (0)

extern "C" {

pm_status pm_hall_create(const pm_hall_desc* d, pm_hall** out) {
    if (!d || !out) return fail(PM_BAD_ARG, "null argument");
    *out = nullptr;
    if (d->precision != PM_PLAIN_F64 && d->precision != PM_FIELDS_F32) return fail(PM_BAD_ARG, "unknown precision");
    Hall* h = new (std::nothrow) Hall();
    if (!h) return fail(PM_OUT_OF_MEMORY, "host allocation");
    h->name = d->name ? d->name : "hall";
    h->precision = d->precision;
    // hall.rs:108-114
    h->nx = std::max(d->across, 2);
    h->dx = std::max(d->width / (double)(h->nx - 1), std::numeric_limits<double>::min());
    auto quantise = [&](double l) { return (int)std::max(std::round(l / h->dx), 0.0) + 1; };
    h->ny = quantise(d->height);
    h->nz = quantise(d->depth);
    h->speed = d->speed;
    h->density = d->density;
    h->max_speed = d->speed;
    pm_status s = h->init(d->device, 0);
    if (s != PM_OK) { delete h; return s; }
    h->tma = h->precision == PM_FIELDS_F32 && h->nx % 4 == 0 && h->nodes() < (1ull << 32);
    for (int attempt = 0; attempt < 2; ++attempt) {
        for (int q = 0; q < 2; ++q) {
            cudaError_t e;
            if ((e = h->p[q].alloc(h->nodes() * h->esize())) != cudaSuccess ||
                (e = h->vx[q].alloc(h->dvx() * h->esize())) != cudaSuccess ||
                (e = h->vy[q].alloc(h->dvy() * h->esize())) != cudaSuccess ||
                (e = h->vz[q].alloc(h->dvz() * h->esize())) != cudaSuccess) {
                delete h;
                return cuda_fail(e, "cudaMalloc hall fields");
            }
        }
        // a shape the driver will not tile steps with the cp.async kernel on the reference layout
        if (!h->tma || h->build_maps() == PM_OK) break;
        h->tma = false;
    }
    *out = reinterpret_cast<pm_hall*>(h);
    std::vector<double> zero(h->nodes(), 0.0);
    s = pm_hall_release(*out, zero.data(), zero.size());  // Hall::new is at rest
    if (s != PM_OK) { delete h; *out = nullptr; }
    return s;
}

pm_status pm_hall_nodes(pm_hall* hp, int* nx, int* ny, int* nz, double* dx) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (nx) *nx = h->nx;
    if (ny) *ny = h->ny;
    if (nz) *nz = h->nz;
    if (dx) *dx = h->dx;
    return PM_OK;
}

pm_status pm_hall_release(pm_hall* hp, const double* pressure, size_t n) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (!pressure || n != h->nodes()) return fail(PM_BAD_ARG, "release: one pressure per node");
    // hall.rs:166-184: pressure from the profile, pressure_prev = pressure, v = 0, then the datum
    h->parity = 0;
    pm_status s;
    if ((s = h->put(h->p[0], pressure, n)) != PM_OK) return s;
    PM_CUDA(cudaMemcpyAsync(h->p[1].p, h->p[0].p, n * h->esize(), cudaMemcpyDeviceToDevice, h->stream()));
    for (int q = 0; q < 2; ++q) {
        PM_CUDA(cudaMemsetAsync(h->vx[q].p, 0, h->dvx() * h->esize(), h->stream()));
        PM_CUDA(cudaMemsetAsync(h->vy[q].p, 0, h->dvy() * h->esize(), h->stream()));
        PM_CUDA(cudaMemsetAsync(h->vz[q].p, 0, h->dvz() * h->esize(), h->stream()));
    }
    h->staggered = false;
    if ((s = h->measure(0, 1)) != PM_OK) return s;
    DevState* st = h->host_state;
    const double datum = st->invariant;
    std::memset(st, 0, sizeof(DevState));
    st->tol = h->tolerance;
    st->datum = datum;
    st->invariant = datum;
    st->offset = 0.0;
    st->total = datum;  // Ledger::new().with(ENERGY, energy()) with energy = invariant + 0
    st->scale = std::fabs(datum);
    st->part[0] = datum;
    st->prev_total = st->total;
    st->prev_scale = st->scale;
    return h->write_state();
}

pm_status pm_hall_set_source(pm_hall* hp, long long node, const double* wave, size_t n) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (node < 0 || (size_t)node >= h->nodes() || (!wave && n > 0)) return fail(PM_BAD_ARG, "source node out of range");
    h->src = node;
    h->nwave = (long long)n;
    if (n > 0) {
        PM_CUDA(h->wave.alloc(n * 8));
        PM_CUDA(h->put_sync(h->wave.p, wave, n * 8));
    }
    h->weigh_source();
    h->drop_graphs();
    return PM_OK;
}

pm_status pm_hall_set_speed_blocks(pm_hall* hp, int block, const double* speeds, size_t n) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (block <= 0 || !speeds) return fail(PM_BAD_ARG, "block must be positive and speeds non-null");
    const int nbx = (h->nx + block - 1) / block, nby = (h->ny + block - 1) / block, nbz = (h->nz + block - 1) / block;
    if (n != (size_t)nbx * nby * nbz) return fail(PM_BAD_ARG, "speeds: one per block");
    h->block = block; h->nbx = nbx; h->nby = nby; h->nbz = nbz;
    h->speeds.assign(speeds, speeds + n);
    h->max_speed = *std::max_element(h->speeds.begin(), h->speeds.end());
    h->weigh_source();
    h->bscale_dt = NAN;
    h->bscale.release();
    h->bknode.release();
    h->drop_graphs();
    pm_status s = h->upload_block_scale(0.0);
    if (s != PM_OK) return s;
    h->bscale_dt = NAN;
    // the datum of the present state under the new weights
    const int par = h->parity;
    if ((s = h->measure(par, par ^ 1)) != PM_OK) return s;
    DevState* st = h->host_state;
    if (!h->staggered) {
        st->datum = st->invariant;
        h->book_totals();
        st->prev_total = st->total;
        st->prev_scale = st->scale;
    }
    return h->write_state();
}

pm_status pm_hall_max_stable_dt(pm_hall* hp, double* seconds) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (!seconds) return fail(PM_BAD_ARG, "null output");
    // hall.rs:401-406 (with the fastest block when the speed varies)
    const double c = h->block > 0 ? h->max_speed : h->speed;
    *seconds = c <= 0.0 ? std::numeric_limits<double>::infinity() : h->dx / (c * std::sqrt(3.0));
    return PM_OK;
}

pm_status pm_hall_set_tolerance(pm_hall* hp, double tol) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    h->tolerance = tol;
    return PM_OK;
}

pm_status pm_hall_step(pm_hall* hp, double dt, long long nsteps, pm_violation* out) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (nsteps < 0) return fail(PM_BAD_ARG, "nsteps must be >= 0");
    if (nsteps == 0) return PM_OK;
    // hall.rs:409-419
    const double c = h->block > 0 ? h->max_speed : h->speed;
    const double courant = c * dt * std::sqrt(3.0) / h->dx;
    if (courant > 1.0 + 1e-12) {
        fill_violation(out, "Courant number", h->name + " (three-dimensional wave equation)", 1.0, courant, 1.0, 1e-12, 1);
        set_error("Courant number past the limit");
        return PM_VIOLATION;
    }
    if (dt <= 0.0) return PM_OK;  // hall.rs:421-423
    pm_status s;
    if ((s = h->upload_block_scale(dt)) != PM_OK) return s;
    if ((s = h->begin_call()) != PM_OK) return s;
    const long long before = h->host_state->steps;
    long long remaining = nsteps;
    if (!h->staggered) {
        if ((s = h->launch_one(h->parity, dt, true, h->stream())) != PM_OK) return s;
        h->parity ^= 1;
        h->staggered = true;
        remaining -= 1;
    }
    s = h->run_steps(remaining, dt, true, [h, dt](int par, cudaStream_t st) { return h->launch(par, dt, false, st); });
    if (s != PM_OK) return s;
    return h->finish_call(before, out, h->name + " (its own books, against what it moved on the bus)",
                          h->name + " (starting the leapfrog)", true);
}

pm_status pm_hall_ledger(pm_hall* hp, pm_ledger* out) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (!out) return fail(PM_BAD_ARG, "null output");
    pm_status s = h->read_state();
    if (s != PM_OK) return s;
    std::memset(out, 0, sizeof(*out));
    const DevState* st = h->host_state;
    out->total = st->total;
    out->scale = st->scale;
    out->n_parts = 4;
    out->parts[0] = st->invariant;
    out->parts[1] = st->offset;
    out->parts[2] = -st->injected;
    out->parts[3] = st->datum;
    out->steps = st->steps;
    return PM_OK;
}

pm_status pm_hall_sample(pm_hall* hp, const double* lo, const double* hi, const int* samples, double* out, size_t n) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    SampleGrid g{};
    pm_status s = sample_grid_of(lo, hi, samples, out, n, g);
    if (s != PM_OK) return s;
    g.dx = h->dx;
    g.nx = h->nx; g.ny = h->ny; g.nz = h->nz;
    return run_sample(h, out, n, [&](double* dev, cudaStream_t st) {
        return h->precision == PM_PLAIN_F64 ? launch_hall_sample<double>(g, h->p[h->parity].as<double>(), dev, st)
                                            : launch_hall_sample<float>(g, h->p[h->parity].as<float>(), dev, st);
    });
}

pm_status pm_hall_download(pm_hall* hp, double* pr, double* pp, double* vx, double* vy, double* vz) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    const int par = h->parity;
    pm_status s;
    if ((s = h->get(h->p[par], pr, h->nodes())) != PM_OK) return s;
    if ((s = h->get(h->p[par ^ 1], pp, h->nodes())) != PM_OK) return s;
    if ((s = h->get_face(0, h->vx[par], vx)) != PM_OK) return s;
    if ((s = h->get_face(1, h->vy[par], vy)) != PM_OK) return s;
    return h->get_face(2, h->vz[par], vz);
}

pm_status pm_hall_checkpoint(pm_hall* hp) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    const int par = h->parity;
    auto save = [&](DBuf& dst, const DBuf& src, size_t n) -> pm_status {
        if (!dst.p) PM_CUDA(dst.alloc(std::max<size_t>(n, 1) * h->esize()));
        PM_CUDA(cudaMemcpyAsync(dst.p, src.p, n * h->esize(), cudaMemcpyDeviceToDevice, h->stream()));
        return PM_OK;
    };
    pm_status s;
    if ((s = save(h->sp, h->p[par], h->nodes())) != PM_OK) return s;
    if ((s = save(h->svx, h->vx[par], h->dvx())) != PM_OK) return s;
    if ((s = save(h->svy, h->vy[par], h->dvy())) != PM_OK) return s;
    if ((s = save(h->svz, h->vz[par], h->dvz())) != PM_OK) return s;
    h->s_staggered = h->staggered;
    h->has_saved = true;
    PM_CUDA(cudaStreamSynchronize(h->stream()));
    return PM_OK;
}

pm_status pm_hall_restore(pm_hall* hp) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (!h->has_saved) return PM_OK;
    const int par = h->parity;
    const size_t e = h->esize();
    // hall.rs:546-555: pressure_prev = pressure = saved
    PM_CUDA(cudaMemcpyAsync(h->p[par].p, h->sp.p, h->nodes() * e, cudaMemcpyDeviceToDevice, h->stream()));
    PM_CUDA(cudaMemcpyAsync(h->p[par ^ 1].p, h->sp.p, h->nodes() * e, cudaMemcpyDeviceToDevice, h->stream()));
    PM_CUDA(cudaMemcpyAsync(h->vx[par].p, h->svx.p, h->dvx() * e, cudaMemcpyDeviceToDevice, h->stream()));
    PM_CUDA(cudaMemcpyAsync(h->vy[par].p, h->svy.p, h->dvy() * e, cudaMemcpyDeviceToDevice, h->stream()));
    PM_CUDA(cudaMemcpyAsync(h->vz[par].p, h->svz.p, h->dvz() * e, cudaMemcpyDeviceToDevice, h->stream()));
    h->staggered = h->s_staggered;
    pm_status s = h->measure(par, par ^ 1);
    if (s != PM_OK) return s;
    DevState* st = h->host_state;
    h->book_totals();
    st->prev_total = st->total;
    st->prev_scale = st->scale;
    return h->write_state();
}

pm_status pm_hall_autotune(pm_hall* hp, int trial_steps, int* planes, int* stages) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (trial_steps < 1) return fail(PM_BAD_ARG, "autotune: at least one trial step");
    pm_status s = h->autotune(trial_steps);
    if (s != PM_OK) return s;
    if (planes) *planes = h->tma ? kHallTmaShapes[h->tshape].planes : 0;
    if (stages) *stages = h->tma ? kHallTmaShapes[h->tshape].stages : 0;
    return PM_OK;
}

pm_status pm_hall_set_tile(pm_hall* hp, int planes, int stages) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (!h->tma) return fail(PM_UNSUPPORTED, "tile shapes are those of the TMA-staged FP32 kernel (x extent a multiple of 4)");
    for (int q = 0; q < kHallTmaShapeCount; ++q)
        if (kHallTmaShapes[q].planes == planes && kHallTmaShapes[q].stages == stages) return h->set_shape(q);
    return fail(PM_BAD_ARG, "hall tile: planes x stages of 8x2, 6x2, 4x3 or 4x2");
}

pm_status pm_hall_tile(pm_hall* hp, int* planes, int* stages) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    if (planes) *planes = h->tma ? kHallTmaShapes[h->tshape].planes : 0;
    if (stages) *stages = h->tma ? kHallTmaShapes[h->tshape].stages : 0;
    return PM_OK;
}

pm_status pm_hall_set_stream(pm_hall* hp, void* stream) {
    Hall* h = reinterpret_cast<Hall*>(hp);
    HALL_GUARD(h);
    PM_CUDA(cudaStreamSynchronize(h->stream()));
    h->user = static_cast<cudaStream_t>(stream);
    return PM_OK;
}

void pm_hall_destroy(pm_hall* hp) { delete reinterpret_cast<Hall*>(hp); }

}  // extern "C"
