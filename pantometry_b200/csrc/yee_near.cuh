// The near field of an FP32 cavity's soft current, kept in f64.
//
// Why. A soft current drives the field at its edge up and down with every cycle of the pulse, and
// what flows in and out of the edge and its neighbours is many times the net work the source does.
// Stored in f32, those values are rounded on every step while that flow passes through them, and
// the ledger (invariant − work) ends a few 1e-6 of the injected energy away from the f64 run's. A
// numpy emulation of the scheme shows where it comes from: with the six components of a 5³ box of
// lattice nodes around the source kept in f64 (every stencil reading the stored values), the same
// run ends 1e-9 away, against 2e-6 with the whole field in f32.
//
// The rule, in one line: inside the box every value is f64, outside it f32, and every stencil reads
// what is stored. yee_tma_step steps every node in f32 from the stored values (the box's f32
// roundings included) but leaves the box's energy terms and the source out; its last block, once
// every other block's cells and sums are in, runs yee_near_body with the grid's four sums (before
// the walls, which run after the step). yee_near_body then
//   A. forms H⁺ of the box's faces in f64 from the box's f64 H and E (f32 values outside),
//   B. forms Eⁿ⁺¹ of the box's edges in f64 from those H⁺ (f32 H⁺ outside), with the source,
//   C. forms again, in f32, the edges just outside the box whose curl reads a box face, so they
//      read the f32 rounding of the box's f64 H⁺ (the value stored there) and not the f32 value
//      yee_tma_step formed,
//   D. adds the box's energy terms, Joule loss and source work in f64 and closes the books with
//      yee_tma_close, as yee_tma_step does for a cavity without a box.
// The box and the ring of C lie inside the walls (one node from them at least), so every
// component exists at every node they hold, every edge is interior and no wall kernel touches it.
//
// The arithmetic of A and B is cavity.rs:1346-1452 with the uniform medium's f64 coefficients (or
// each edge's own f32 gain with MEDIA, the coefficient the update and the energy weight use), the
// soft current as in yee_tma_step.
#pragma once

#include "yee_tma.cuh"

namespace pm {

__device__ __forceinline__ bool near_in(const YeeNearArgs& a, int i, int j, int k) {
    return (unsigned)(i - a.x0) < (unsigned)a.w && (unsigned)(j - a.y0) < (unsigned)a.w &&
           (unsigned)(k - a.z0) < (unsigned)a.w;
}
__device__ __forceinline__ size_t near_lat(const YeeNearArgs& a, int i, int j, int k) {
    return (size_t)i + (size_t)a.L * ((size_t)j + (size_t)a.ny1 * (size_t)k);
}
__device__ __forceinline__ size_t near_box(const YeeNearArgs& a, int q, int i, int j, int k) {
    const size_t w = (size_t)a.w;
    return (size_t)q * w * w * w + (size_t)(i - a.x0) + w * ((size_t)(j - a.y0) + w * (size_t)(k - a.z0));
}
// Component q's pointer of a lattice set, chosen by a switch: indexing the parameter block's array
// with a runtime index would copy the whole block to local memory.
__device__ __forceinline__ const float* near_comp(const float* const (&lat)[6], int q) {
    switch (q) {
        case 0: return lat[0];
        case 1: return lat[1];
        case 2: return lat[2];
        case 3: return lat[3];
        case 4: return lat[4];
        default: return lat[5];
    }
}
__device__ __forceinline__ float* near_comp(float* const (&lat)[6], int q) {
    switch (q) {
        case 0: return lat[0];
        case 1: return lat[1];
        case 2: return lat[2];
        case 3: return lat[3];
        case 4: return lat[4];
        default: return lat[5];
    }
}
__device__ __forceinline__ const float* near_comp(const float* const (&lat)[3], int q) {
    return q == 0 ? lat[0] : q == 1 ? lat[1] : lat[2];
}
// The stored value of component q at node (i, j, k): f64 in the box, f32 outside.
__device__ __forceinline__ double near_get(const YeeNearArgs& a, const double* box, const float* lat_q, int q, int i,
                                           int j, int k) {
    return near_in(a, i, j, k) ? box[near_box(a, q, i, j, k)] : (double)lat_q[near_lat(a, i, j, k)];
}

// Seed the box's f64 values from the stored f32 field (after the state was set from outside a step).
static __global__ void yee_near_seed(YeeNearArgs a) {
    const int w = a.w, w3 = w * w * w;
    for (int r = threadIdx.x; r < 6 * w3; r += blockDim.x) {
        const int q = r / w3, l = r - q * w3;
        const int i = a.x0 + l % w, j = a.y0 + (l / w) % w, k = a.z0 + l / (w * w);
        a.nneu[r] = (double)near_comp(a.neu, q)[near_lat(a, i, j, k)];
    }
}

// A load of the new field, written by the other blocks of the step: from L2, past this SM's L1.
__device__ __forceinline__ float near_ld_new(const float* p) { return __ldcg(p); }

// Run by the whole last block of yee_tma_step, once every other block's cells are in, with the
// grid's four sums (valid in thread 0): one work item per (component, node), 3 × w³ in phases A
// and B, 3 × (w+1)³ in phase C, strided over the block's threads.
template <bool SOLID>
__device__ void yee_near_body(const YeeNearArgs& a, const double (&tma)[4]) {
    DevState* st = a.st;
    const int nthreads = blockDim.x * blockDim.y * blockDim.z, tid0 = linear_tid();
    const int w = a.w, w3 = w * w * w;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long long step = st->steps;
    const double jsrc = (a.src_i >= 0 && step < a.ncurrent) ? a.current[step] : 0.0;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};

    // A. H⁺ of face component q at each box node (cavity.rs:1346-1379) with its term of ½μ H⁻·H⁺,
    // and the ½ε|Eⁿ|² term of edge component q there (half weights of node-centred boundary
    // samples, cavity.rs:766-772)
    for (int r = tid0; r < 3 * w3; r += nthreads) {
        const int q = r / w3, l = r - q * w3;
        const int i = a.x0 + l % w, j = a.y0 + (l / w) % w, k = a.z0 + l / (w * w);
        const double hi = (i == 0 || i == nx) ? 0.5 : 1.0, hj = (j == 0 || j == ny) ? 0.5 : 1.0,
                     hk = (k == 0 || k == nz) ? 0.5 : 1.0;
        const double was = a.nold[near_box(a, 3 + q, i, j, k)];
        double curl, wh;
        if (q == 0) {  // hx: (ez(j+1) − ez) − (ey(k+1) − ey)
            curl = (near_get(a, a.nold, a.old[2], 2, i, j + 1, k) - a.nold[near_box(a, 2, i, j, k)]) -
                   (near_get(a, a.nold, a.old[1], 1, i, j, k + 1) - a.nold[near_box(a, 1, i, j, k)]);
            wh = hi;
        } else if (q == 1) {  // hy: (ex(k+1) − ex) − (ez(i+1) − ez)
            curl = (near_get(a, a.nold, a.old[0], 0, i, j, k + 1) - a.nold[near_box(a, 0, i, j, k)]) -
                   (near_get(a, a.nold, a.old[2], 2, i + 1, j, k) - a.nold[near_box(a, 2, i, j, k)]);
            wh = hj;
        } else {  // hz: (ey(i+1) − ey) − (ex(j+1) − ex)
            curl = (near_get(a, a.nold, a.old[1], 1, i + 1, j, k) - a.nold[near_box(a, 1, i, j, k)]) -
                   (near_get(a, a.nold, a.old[0], 0, i, j + 1, k) - a.nold[near_box(a, 0, i, j, k)]);
            wh = hk;
        }
        const double hn = was - a.ch * curl;
        const size_t n = near_lat(a, i, j, k);
        a.nneu[near_box(a, 3 + q, i, j, k)] = hn;
        near_comp(a.neu, 3 + q)[n] = (float)hn;
        acc[1] += wh * (hn * was);
        const double e0 = a.nold[near_box(a, q, i, j, k)];
        const double we = q == 0 ? hj * hk : q == 1 ? hi * hk : hi * hj;
        if (a.media)  // weighted by 1/g, the ε the update uses
            acc[0] += we * (e0 * e0) / (double)near_comp(a.cgain, q)[n];
        else
            acc[0] += we * (e0 * e0);
    }
    __syncthreads();  // the box's H⁺, in both stores, before any edge reads it

    // B. Eⁿ⁺¹ of edge component q at each box node (cavity.rs:1383-1452), the soft current, Joule loss
    for (int r = tid0; r < 3 * w3; r += nthreads) {
        const int q = r / w3, l = r - q * w3;
        const int i = a.x0 + l % w, j = a.y0 + (l / w) % w, k = a.z0 + l / (w * w);
        const size_t n = near_lat(a, i, j, k);
        auto hp = [&](int c, int ii, int jj, int kk) {
            return near_in(a, ii, jj, kk) ? a.nneu[near_box(a, c, ii, jj, kk)]
                                          : (double)near_ld_new(near_comp(a.neu, c) + near_lat(a, ii, jj, kk));
        };
        double curl;
        if (q == 0) curl = (hp(5, i, j, k) - hp(5, i, j - 1, k)) - (hp(4, i, j, k) - hp(4, i, j, k - 1));
        else if (q == 1) curl = (hp(3, i, j, k) - hp(3, i, j, k - 1)) - (hp(5, i, j, k) - hp(5, i - 1, j, k));
        else curl = (hp(4, i, j, k) - hp(4, i - 1, j, k)) - (hp(3, i, j, k) - hp(3, i, j - 1, k));
        const double e0 = a.nold[near_box(a, q, i, j, k)];
        const double g = a.media ? (double)near_comp(a.cgain, q)[n] : a.gain;
        double v = a.decay * e0 + g * curl;
        if (q == 2 && i == a.src_i && j == a.src_j && k == a.src_k) {
            // soft current: ε dE/dt = ∇×H − J, with the σ term's semi-implicit divisor
            const double e = a.eps_src, ss = a.sig_src;
            v = v - (a.dt / e) / (1.0 + (ss * a.dt / (2.0 * e))) * jsrc;
            acc[3] += -(a.dt * a.volume) * jsrc * (0.5 * (e0 + v));
        }
        const bool ix = i >= 1 && i < nx, iy = j >= 1 && j < ny, iz = k >= 1 && k < nz;
        const bool interior = q == 0 ? (iy && iz) : q == 1 ? (ix && iz) : (ix && iy);
        v = interior ? v : 0.0;
        if (a.lossy && interior) {
            const double m = 0.5 * (e0 + v);
            acc[2] += a.sig0 * m * m * a.dt * a.volume;
        }
        if constexpr (SOLID) {
            const bool hit = q == 0   ? touches_solid(a.solid, nx, ny, nz, i, i, j - 1, j, k - 1, k)
                             : q == 1 ? touches_solid(a.solid, nx, ny, nz, i - 1, i, j, j, k - 1, k)
                                      : touches_solid(a.solid, nx, ny, nz, i - 1, i, j - 1, j, k, k);
            if (hit) v = 0.0;
        }
        a.nneu[near_box(a, q, i, j, k)] = v;
        near_comp(a.neu, q)[n] = (float)v;
    }

    // C. The edges just outside the box whose curl reads a box face: the nodes of the (w+1)³ cube
    // that are not in the box, on its high sides. Each is formed again in f32 from the stored H⁺
    // (the box's own faces now hold the roundings of their f64 values), as yee_tma_step forms it;
    // with a lossy medium the Joule term yee_tma_step booked for it is replaced by this value's.
    const int w1 = w + 1, ring = w1 * w1 * w1;
    for (int r = tid0; r < 3 * ring; r += nthreads) {
        const int q = r / ring, l = r - q * ring;
        const int i = a.x0 + l % w1, j = a.y0 + (l / w1) % w1, k = a.z0 + l / (w1 * w1);
        if (near_in(a, i, j, k)) continue;
        // which faces the curl of component q reads besides the node's own: x reads j−1 and
        // k−1, y reads k−1 and i−1, z reads i−1 and j−1
        const bool reads = q == 0   ? (near_in(a, i, j - 1, k) || near_in(a, i, j, k - 1))
                           : q == 1 ? (near_in(a, i, j, k - 1) || near_in(a, i - 1, j, k))
                                    : (near_in(a, i - 1, j, k) || near_in(a, i, j - 1, k));
        if (!reads) continue;
        const size_t n = near_lat(a, i, j, k);
        auto h = [&](int c, int ii, int jj, int kk) { return near_ld_new(near_comp(a.neu, c) + near_lat(a, ii, jj, kk)); };
        const float before = near_comp(a.old, q)[n];
        float curl;
        if (q == 0) curl = (h(5, i, j, k) - h(5, i, j - 1, k)) - (h(4, i, j, k) - h(4, i, j, k - 1));
        else if (q == 1) curl = (h(3, i, j, k) - h(3, i, j, k - 1)) - (h(5, i, j, k) - h(5, i - 1, j, k));
        else curl = (h(4, i, j, k) - h(4, i - 1, j, k)) - (h(3, i, j, k) - h(3, i, j - 1, k));
        const float gq = a.media ? near_comp(a.cgain, q)[n] : a.gainf;
        float v = a.decf * before + gq * curl;
        const bool ix = i >= 1 && i < nx, iy = j >= 1 && j < ny, iz = k >= 1 && k < nz;
        const bool interior = q == 0 ? (iy && iz) : q == 1 ? (ix && iz) : (ix && iy);
        v = interior ? v : 0.0f;
        float* out = near_comp(a.neu, q);
        if (a.lossy && interior) {
            const double mold = 0.5 * ((double)before + (double)near_ld_new(out + n));
            const double mnew = 0.5 * ((double)before + (double)v);
            acc[2] += a.sig0 * mnew * mnew * a.dt * a.volume - a.sig0 * mold * mold * a.dt * a.volume;
        }
        if constexpr (SOLID) {
            const bool hit = q == 0   ? touches_solid(a.solid, nx, ny, nz, i, i, j - 1, j, k - 1, k)
                             : q == 1 ? touches_solid(a.solid, nx, ny, nz, i - 1, i, j, j, k - 1, k)
                                      : touches_solid(a.solid, nx, ny, nz, i - 1, i, j - 1, j, k, k);
            if (hit) v = 0.0f;
        }
        out[n] = v;
    }

    // D. the box's sums in a fixed order, added to yee_tma_step's, and the books
    __shared__ double red[32 * 4];
    block_sum<4>(acc, red);
    if (tid0 == 0) {
        double total[4];
        for (int q = 0; q < 4; ++q) total[q] = tma[q] + acc[q];
        yee_tma_close(st, total, a.media != 0, a.g, a.eps_u, a.mu_u, a.volume, a.src_i >= 0);
    }
}

}  // namespace pm
