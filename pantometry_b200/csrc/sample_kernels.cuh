// scene::capture's field sampling on the device (crates/pantometry-scene/src/lib.rs:347-420): a
// domain's `ScalarField::at` evaluated at every point of an extent's sample grid, straight from the
// resident fields, so that only the samples come back to the host. Point r of a grid of n[0] × n[1]
// × n[2] samples (x fastest) lies `lo + (hi − lo) · f` per component, with f = i / (n − 1) along
// an axis of n > 1 samples and 1/2 along an axis of one (lib.rs:398-406). Compiled in the
// no-contraction unit, so the f64 forms give the reference's samples bit for bit; the FP32 forms
// read their f32 values (heat: T0 + deviation) in f64 and sample those.
#pragma once

#include <cstdint>

namespace pm {

struct SampleGrid {
    double lo[3], hi[3];
    int n[3];
    double dx;
    int nx, ny, nz;
};

__device__ __forceinline__ double sample_along(int i, int n) { return n > 1 ? (double)i / (double)(n - 1) : 0.5; }

__device__ __forceinline__ void sample_point(const SampleGrid& g, long long r, double (&pt)[3]) {
    const int i = (int)(r % g.n[0]);
    const long long rest = r / g.n[0];
    const int j = (int)(rest % g.n[1]), k = (int)(rest / g.n[1]);
    const double f[3] = {sample_along(i, g.n[0]), sample_along(j, g.n[1]), sample_along(k, g.n[2])};
#pragma unroll
    for (int a = 0; a < 3; ++a) pt[a] = g.lo[a] + (g.hi[a] - g.lo[a]) * f[a];
}

// Solid3D::at (solid.rs:2045-2104): trilinear between cell centres, clamped at the faces, NaN in a
// void cell (vd non-null), the weights renormalised over the solid corners. `t0` is added to each
// stored value (the FP32 form's deviations; 0 for kelvin).
template <typename Real>
static __global__ void heat_sample(const SampleGrid g, const Real* __restrict__ cells, double t0,
                                   const uint8_t* __restrict__ vd, double* __restrict__ out) {
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < total; r += (long long)gridDim.x * blockDim.x) {
        double pt[3];
        sample_point(g, r, pt);
        const double q[3] = {pt[0] / g.dx - 0.5, pt[1] / g.dx - 0.5, pt[2] / g.dx - 0.5};
        if (isnan(q[0]) || isnan(q[1]) || isnan(q[2])) {
            out[r] = nan("");
            continue;
        }
        int c[3];
        double fr[3];
        const int cnt[3] = {nx, ny, nz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int last = cnt[a] > 0 ? cnt[a] - 1 : 0;
            if (q[a] <= 0.0) { c[a] = 0; fr[a] = 0.0; }
            else if (q[a] >= (double)last) { c[a] = last; fr[a] = 0.0; }
            else { const double fl = floor(q[a]); c[a] = (int)fl; fr[a] = q[a] - fl; }
        }
        int near[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double rr = round(q[a]);
            if (rr < 0.0) rr = 0.0;
            near[a] = min((int)rr, cnt[a] > 0 ? cnt[a] - 1 : 0);
        }
        if (vd && vd[(size_t)near[0] + (size_t)nx * ((size_t)near[1] + (size_t)ny * near[2])]) {
            out[r] = nan("");
            continue;
        }
        const int ai[2] = {c[0], min(c[0] + 1, nx - 1)}, bj[2] = {c[1], min(c[1] + 1, ny - 1)},
                  ck[2] = {c[2], min(c[2] + 1, nz - 1)};
        const double wa[2] = {1.0 - fr[0], fr[0]}, wb[2] = {1.0 - fr[1], fr[1]}, wc[2] = {1.0 - fr[2], fr[2]};
        double sum = 0.0, weight = 0.0;
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
            for (int y = 0; y < 2; ++y)
#pragma unroll
                for (int z = 0; z < 2; ++z) {
                    const double w = wa[x] * wb[y] * wc[z];
                    const size_t at = (size_t)ai[x] + (size_t)nx * ((size_t)bj[y] + (size_t)ny * ck[z]);
                    if (w > 0.0 && !(vd && vd[at])) {
                        sum += w * ((double)cells[at] + t0);
                        weight += w;
                    }
                }
        out[r] = weight > 0.0 ? sum / weight : nan("");
    }
}

// Hall::at (hall.rs:591-613) with clamp_index (hall.rs:684-694): trilinear between nodes, clamped at
// the surfaces; a NaN point reads node 0.
template <typename Real>
static __global__ void hall_sample(const SampleGrid g, const Real* __restrict__ p, double* __restrict__ out) {
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < total; r += (long long)gridDim.x * blockDim.x) {
        double pt[3];
        sample_point(g, r, pt);
        const double q[3] = {pt[0] / g.dx, pt[1] / g.dx, pt[2] / g.dx};
        if (isnan(q[0]) || isnan(q[1]) || isnan(q[2])) {
            out[r] = (double)p[0];
            continue;
        }
        int c[3];
        double fr[3];
        const int cnt[3] = {nx, ny, nz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (q[a] <= 0.0) { c[a] = 0; fr[a] = 0.0; }
            else if (q[a] >= (double)(cnt[a] - 1)) { c[a] = cnt[a] - 1; fr[a] = 0.0; }
            else { const double fl = floor(q[a]); c[a] = (int)fl; fr[a] = q[a] - fl; }
        }
        const int i = c[0], j = c[1], k = c[2];
        const int i1 = min(i + 1, nx - 1), j1 = min(j + 1, ny - 1), k1 = min(k + 1, nz - 1);
        auto gv = [&](int a, int b, int cc) { return (double)p[(size_t)a + (size_t)nx * ((size_t)b + (size_t)ny * cc)]; };
        auto lerp = [](double a, double b, double t) { return a * (1.0 - t) + b * t; };
        const double z0 = lerp(lerp(gv(i, j, k), gv(i1, j, k), fr[0]), lerp(gv(i, j1, k), gv(i1, j1, k), fr[0]), fr[1]);
        const double z1 = lerp(lerp(gv(i, j, k1), gv(i1, j, k1), fr[0]), lerp(gv(i, j1, k1), gv(i1, j1, k1), fr[0]), fr[1]);
        out[r] = lerp(z0, z1, fr[2]);
    }
}

// Room::at (room.rs:587-601) with its clamp_index (room.rs:739-749): bilinear between the four nodes
// round the point's (x, y), clamped at the walls, a NaN coordinate reading node 0 along its axis;
// z is not read. Pressure sits at i + nx·j.
__device__ __forceinline__ void clamp_node(double q, int n, int& i, double& f) {
    if (isnan(q) || q <= 0.0) { i = 0; f = 0.0; }
    else if (q >= (double)(n - 1)) { i = n - 1; f = 0.0; }
    else { const double fl = floor(q); i = (int)fl; f = q - fl; }
}

template <typename Real>
static __global__ void room_sample(const SampleGrid g, const Real* __restrict__ p, double* __restrict__ out) {
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    const int nx = g.nx, ny = g.ny;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < total; r += (long long)gridDim.x * blockDim.x) {
        double pt[3];
        sample_point(g, r, pt);
        int i, j;
        double fx, fy;
        clamp_node(pt[0] / g.dx, nx, i, fx);
        clamp_node(pt[1] / g.dx, ny, j, fy);
        const int i1 = min(i + 1, nx - 1), j1 = min(j + 1, ny - 1);
        const double p00 = (double)p[(size_t)j * nx + i], p10 = (double)p[(size_t)j * nx + i1];
        const double p01 = (double)p[(size_t)j1 * nx + i], p11 = (double)p[(size_t)j1 * nx + i1];
        const double bottom = p00 * (1.0 - fx) + p10 * fx;
        const double top = p01 * (1.0 - fx) + p11 * fx;
        out[r] = bottom * (1.0 - fy) + top * fy;
    }
}

// Bar1D::at (crates/pantometry-thermal/src/lib.rs:736-751): linear between cell centres along x,
// the end cell's value beyond either centre and for a NaN x; y and z are not read. The FP32 form
// adds `t0` to its stored deviations; the f64 form reads kelvin as stored.
template <typename Real>
static __global__ void bar_sample(const SampleGrid g, const Real* __restrict__ cells, double t0, double* __restrict__ out) {
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    const int last = g.nx - 1;
    auto kelvin = [&](int c) {
        const double v = (double)cells[c];
        return sizeof(Real) == 8 ? v : v + t0;
    };
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < total; r += (long long)gridDim.x * blockDim.x) {
        double pt[3];
        sample_point(g, r, pt);
        const double u = pt[0] / g.dx - 0.5;
        if (isnan(u) || u <= 0.0) {
            out[r] = kelvin(0);
        } else if (u >= (double)last) {
            out[r] = kelvin(last);
        } else {
            const double fl = floor(u);
            const int i = (int)fl;
            const double f = u - fl;
            out[r] = kelvin(i) * (1.0 - f) + kelvin(i + 1) * f;
        }
    }
}

// Cavity::at (cavity.rs:197-206) over electric_at (cavity.rs:735-742): |E| of the edges of the cell
// the point falls in (nearest cell, clamped), NaN for a NaN point. Component q of E sits at
// i + rx[q]·(j + ry[q]·k): the reference layout's extents, or the padded lattice's pitch.
template <typename Real>
static __global__ void yee_sample(const SampleGrid g, const Real* __restrict__ ex, const Real* __restrict__ ey,
                                  const Real* __restrict__ ez, uint3 rx, uint3 ry, double* __restrict__ out) {
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < total; r += (long long)gridDim.x * blockDim.x) {
        double pt[3];
        sample_point(g, r, pt);
        const double q[3] = {pt[0] / g.dx, pt[1] / g.dx, pt[2] / g.dx};
        if (isnan(q[0]) || isnan(q[1]) || isnan(q[2])) {
            out[r] = nan("");
            continue;
        }
        int c[3];
        const int cnt[3] = {nx, ny, nz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double f = floor(q[a]);
            if (f < 0.0) f = 0.0;
            c[a] = min((int)f, cnt[a] > 0 ? cnt[a] - 1 : 0);
        }
        const int i = c[0], j = c[1], k = c[2];
        const double x = (double)ex[(size_t)min(i, nx - 1) + (size_t)rx.x * ((size_t)min(j, ny) + (size_t)ry.x * min(k, nz))];
        const double y = (double)ey[(size_t)min(i, nx) + (size_t)rx.y * ((size_t)min(j, ny - 1) + (size_t)ry.y * min(k, nz))];
        const double z = (double)ez[(size_t)min(i, nx) + (size_t)rx.z * ((size_t)min(j, ny) + (size_t)ry.z * min(k, nz - 1))];
        out[r] = sqrt((x * x + y * y) + z * z);  // DVec3::length: the dot product, then sqrt
    }
}

}  // namespace pm
