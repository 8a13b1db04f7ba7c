// Cavity step, FP32 form for one uniform medium, or (MEDIA) for per-cell ε with no conductivity
// and one μ, with or without obstacles, staged by the Tensor Memory Accelerator. The arithmetic
// per edge and face is yee_step's (cavity.rs:1346-1501): H⁺ from Eⁿ, the invariant
// ½ε|Eⁿ|² + ½μ H⁻·H⁺, then Eⁿ⁺¹ from H⁺. With MEDIA the stage also holds the gains
// g = Δt/(ε Δx) of the tile's own edges (yee_coefs, on the padded lattice), and each thread weighs
// its electric terms by 1/g, so the energy it books is ½ (Δt/Δx) Σ w E²/g V: ½ Σ w ε E² V with
// the ε the update itself used.
//
// Layout. The handle keeps all six components on the (nx+1) × (ny+1) × (nz+1) node lattice with
// one index n = i + L·(j + (ny+1)·k), L = nx+1 rounded up to a multiple of 4 (so every row pitch
// is a multiple of 16 bytes, as TMA requires). A component's lattice positions outside its own
// extent (cavity.rs:112-123) are padding: zero, never written.
//
// Walk. Tiles are 32 × 8 columns of the lattice over a z-chunk, taken by a persistent grid in
// order; a tile's chunk of planes k0 .. k1−1 is streamed from k0 − 1 (whose H⁺ the first plane's
// Eⁿ⁺¹ needs) P planes at a time. For a stage of planes kb .. kb+P−1 one thread issues six tiled
// TMA loads into a ring of S shared-memory stages (boxes start at x0 − 4 or x0, 16-byte aligned;
// the hardware fills outside the lattice with zeros):
//   ex  x0−4 .. x0+31, y0−1 .. y0+8, kb .. kb+P      ey  x0−4 .. x0+35, y0−1 .. y0+7, kb .. kb+P
//   ez  x0−4 .. x0+35, y0−1 .. y0+8, kb .. kb+P−1    hx  x0   .. x0+31, y0−1 .. y0+7, kb .. kb+P−1
//   hy  x0−4 .. x0+31, y0   .. y0+7, kb .. kb+P−1    hz  x0−4 .. x0+31, y0−1 .. y0+7, kb .. kb+P−1
// Per plane: H⁺ on the tile's own faces and on the x0−1 column / y0−1 row its edges need, into a
// double-buffered shared plane; one barrier; Eⁿ⁺¹ on the tile's own edges, with H⁺ of the plane
// below carried in registers. Completion of each stage is one mbarrier; every wait is bounded.
#pragma once

#include <cuda.h>

#include "hall_tma.cuh"
#include "yee_kernels.cuh"

namespace pm {

struct YeeMaps {
    CUtensorMap ex, ey, ez, hx, hy, hz;
    CUtensorMap gx, gy, gz;  // per-edge gains of a cavity of mixed ε (MEDIA)
};

// The tile shapes of each form: planes per stage, stages in the ring, resident blocks per SM the
// kernel is held to. Shape 0 of each is the one hand sweeps chose on B200 at 384³: one medium 3
// planes × 2 stages at three blocks per SM (61 KB of shared memory a block, 100 Gcell/s against 95
// for 4 × 2 at two), mixed ε 4 × 2 at two (95 KB with its gain boxes, 85 against 60 for 3 × 2 at
// three). The others are the runners-up, which pm_cavity_autotune times on a cavity's own grid.
// Every shape computes each edge and face with the same expressions, so they agree bit for bit.
struct YeeTmaShape {
    int planes, stages, min_blocks;
};
constexpr YeeTmaShape kYeeTmaUniformShapes[] = {{3, 2, 3}, {4, 2, 2}, {3, 3, 2}};
constexpr YeeTmaShape kYeeTmaMediaShapes[] = {{4, 2, 2}, {3, 2, 3}};
constexpr int kYeeTmaUniformShapeCount = 3, kYeeTmaMediaShapeCount = 2;
inline constexpr YeeTmaShape yee_tma_shape(bool media, int shape) {
    return media ? kYeeTmaMediaShapes[shape] : kYeeTmaUniformShapes[shape];
}
inline constexpr int yee_tma_shape_count(bool media) { return media ? kYeeTmaMediaShapeCount : kYeeTmaUniformShapeCount; }
constexpr int kYeeTmaStages = 2;
constexpr int kYeeTmaPlanesUniform = 3, kYeeTmaPlanesMedia = 4;

constexpr unsigned round128(unsigned b) { return (b + 127u) & ~127u; }

// Byte offsets of the six boxes inside one stage (each 128-byte aligned), and with MEDIA the
// three gain boxes of the tile's own edges, x0 .. x0+31, y0 .. y0+7, kb .. kb+P−1.
template <int P, bool MEDIA = false>
struct YeeTmaLayout {
    static constexpr unsigned EX_B = (P + 1) * 10 * 36 * 4, EY_B = (P + 1) * 9 * 40 * 4, EZ_B = P * 10 * 40 * 4,
                              HX_B = P * 9 * 32 * 4, HY_B = P * 8 * 36 * 4, HZ_B = P * 9 * 36 * 4,
                              G_B = MEDIA ? P * 8 * 32 * 4 : 0;
    static constexpr unsigned EX = 0, EY = round128(EX + EX_B), EZ = round128(EY + EY_B), HX = round128(EZ + EZ_B),
                              HY = round128(HX + HX_B), HZ = round128(HY + HY_B), GX = round128(HZ + HZ_B),
                              GY = round128(GX + G_B), GZ = round128(GY + G_B), BYTES = round128(GZ + G_B);
    // bytes the loads of one stage deliver
    static constexpr unsigned TX = EX_B + EY_B + EZ_B + HX_B + HY_B + HZ_B + 3 * G_B;
};

template <int P, bool MEDIA = false>
inline size_t yee_tma_smem_bytes_for(int S) {
    return (size_t)S * YeeTmaLayout<P, MEDIA>::BYTES + 2 * sizeof(YeeHp<float>) + 8 * (size_t)S;
}

struct YeeTmaCursor {
    unsigned t;
    int x0, y0, k0, k1, kb;
    bool valid;
};
__device__ __forceinline__ void yee_tma_at(YeeTmaCursor& c, const Tiles& T, unsigned t) {
    c.t = t;
    c.valid = t < (unsigned)T.ntiles;
    if (!c.valid) return;
    const unsigned r = t / (unsigned)T.ntx;
    const unsigned tz = r / (unsigned)T.nty;
    c.x0 = (int)(t - r * (unsigned)T.ntx) * 32;
    c.y0 = (int)(r - tz * (unsigned)T.nty) * 8;
    c.k0 = (int)tz * T.zc;
    c.k1 = min(T.nz, c.k0 + T.zc);  // T.nz = nz + 1 lattice planes
    c.kb = c.k0 > 0 ? c.k0 - 1 : 0;
}
__device__ __forceinline__ void yee_tma_next(YeeTmaCursor& c, const Tiles& T, int planes) {
    c.kb += planes;
    if (c.kb >= c.k1) yee_tma_at(c, T, c.t + gridDim.x);
}

template <int P, bool MEDIA>
__device__ __forceinline__ void yee_tma_issue(const YeeMaps& m, unsigned stage, unsigned bar, const YeeTmaCursor& c) {
    using Lay = YeeTmaLayout<P, MEDIA>;
    mbar_expect_tx(bar, Lay::TX);
    tma_load_3d(stage + Lay::EX, &m.ex, c.x0 - 4, c.y0 - 1, c.kb, bar);
    tma_load_3d(stage + Lay::EY, &m.ey, c.x0 - 4, c.y0 - 1, c.kb, bar);
    tma_load_3d(stage + Lay::EZ, &m.ez, c.x0 - 4, c.y0 - 1, c.kb, bar);
    tma_load_3d(stage + Lay::HX, &m.hx, c.x0, c.y0 - 1, c.kb, bar);
    tma_load_3d(stage + Lay::HY, &m.hy, c.x0 - 4, c.y0, c.kb, bar);
    tma_load_3d(stage + Lay::HZ, &m.hz, c.x0 - 4, c.y0 - 1, c.kb, bar);
    if constexpr (MEDIA) {
        tma_load_3d(stage + Lay::GX, &m.gx, c.x0, c.y0, c.kb, bar);
        tma_load_3d(stage + Lay::GY, &m.gy, c.x0, c.y0, c.kb, bar);
        tma_load_3d(stage + Lay::GZ, &m.gz, c.x0, c.y0, c.kb, bar);
    }
}

// The books of one FP32 cavity step from its four sums (Σ w|Eⁿ|² or, with MEDIA, Σ w|Eⁿ|²/g;
// Σ w H⁺·H⁻; Joule loss; source work): the invariant, the running books, the ledger
// (cavity.rs:1520-1524) and the audit. Run by one thread.
__device__ __forceinline__ void yee_tma_close(DevState* st, const double (&acc)[4], bool media, double g, double eps_u,
                                              double mu_u, double v, bool with_source) {
    // cavity.rs:846; with MEDIA the terms are already weighted by 1/g = ε Δx/Δt
    const double electric = media ? 0.5 * (g * acc[0]) * v : 0.5 * (eps_u * acc[0]) * v;
    const double paired = 0.5 * v * (mu_u * acc[1]);  // cavity.rs:885-904
    st->invariant = electric + paired;
    st->has_invariant = 1;
    st->dissipated += fmax(acc[2], 0.0);
    st->work_booked = st->work;
    st->work += acc[3];
    double total = 0.0, scale = 0.0;
    ledger_add(total, scale, st->invariant);
    ledger_add(total, scale, st->dissipated);
    if (with_source) ledger_add(total, scale, -st->work_booked);
    st->part[0] = st->invariant;
    st->part[1] = st->dissipated;
    st->part[2] = -st->work_booked;
    audit_and_commit(st, total, scale);
}

// The near field of a soft current, kept in f64 (yee_near.cuh): its arguments, and the last
// block's work on it after the grid's sums are in.
struct YeeNearArgs {
    const float* old[6];    // ex ey ez hx hy hz at step n, padded lattice
    float* neu[6];          // at n + 1, already stepped by yee_tma_step
    const double* nold;     // the box's f64 values at step n: [q][lk][lj][li], w³ per component
    double* nneu;           // at n + 1
    int x0, y0, z0, w;      // the box: w³ lattice nodes from (x0, y0, z0)
    unsigned L, ny1;        // lattice row pitch and rows per plane
    int nx, ny, nz;
    double ch, gain, decay;  // f64 coefficients of one medium: g/μ, edge gain and decay
    float chf, gainf, decf;  // the f32 ones yee_tma_step used (the ring's edges)
    const float* cgain[3];   // MEDIA: per-edge gains on the padded lattice
    int media, lossy;
    double sig0;
    const uint8_t* solid;
    int src_i, src_j, src_k;
    const double* current;
    long long ncurrent;
    double eps_src, sig_src, dt, volume, g, eps_u, mu_u;
    DevState* st;
};
template <bool SOLID>
__device__ void yee_near_body(const YeeNearArgs& a, const double (&tma)[4]);

// One face of H⁺ (cavity.rs:1346-1379): was − (g/μ)·((a₁ − a₀) − (b₁ − b₀)). The tiles and the
// wall pass below form every face through this one expression, so the two agree bit for bit.
__device__ __forceinline__ float yee_face_f32(float was, float ch, float a1, float a0, float b1, float b0) {
    return was - ch * ((a1 - a0) - (b1 - b0));
}

// The lattice's last column (i = nx, every j and k) and last row (j = ny, i < nx), when the tiles
// cover only [0, nx) × [0, ny) (a.wall_split: nx a multiple of 32 and ny of 8, so that no tile is
// there for one column or row alone). Every edge on these nodes is tangential to the x = nx or
// y = ny wall, so the step writes 0 to each (cavity.rs:1239-1293; open and magnetic walls are the
// wall kernel's, after the step), and the one face that moves is hx on x = nx and hy on y = ny.
// Each value and energy term is the one a tile would have formed there: neighbours beyond the
// lattice read 0, as the tensor maps' fill does, and a component's absent positions hold the
// padding's 0. The node is taken from the thread's index, `nthreads` apart.
template <bool MEDIA>
__device__ __forceinline__ void yee_tma_wall_pass(const YeeStepArgs<float>& a, unsigned L, long long first,
                                                  long long nthreads, float& es, float& ms) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const unsigned ny1 = (unsigned)ny + 1;
    const size_t plane = (size_t)L * ny1;
    const long long ncol = (long long)(ny + 1) * (nz + 1), nall = ncol + (long long)nx * (nz + 1);
    const float ch = a.ch, gain0 = a.gain[0];
    for (long long r = first; r < nall; r += nthreads) {
        int i, j, k;
        if (r < ncol) {
            i = nx;
            j = (int)(r % (ny + 1));
            k = (int)(r / (ny + 1));
        } else {
            const long long q = r - ncol;
            i = (int)(q % nx);
            j = ny;
            k = (int)(q / nx);
        }
        const size_t n = (size_t)i + L * ((size_t)j + (size_t)ny1 * (size_t)k);
        const bool zin = k < nz;
        const float hi = (i == 0 || i == nx) ? 0.5f : 1.0f, hj = (j == 0 || j == ny) ? 0.5f : 1.0f,
                    hk = (k == 0 || k == nz) ? 0.5f : 1.0f;
        const float ex0 = a.old[0][n], ey0 = a.old[1][n], ez0 = a.old[2][n];
        if (i == nx) {
            const float wx = a.old[3][n];
            const float hxn = yee_face_f32(wx, ch, j < ny ? a.old[2][n + L] : 0.0f, ez0, zin ? a.old[1][n + plane] : 0.0f, ey0);
            if (j < ny && zin) a.neu[3][n] = hxn;
            ms += hi * (hxn * wx);
            if (j < ny) a.neu[1][n] = 0.0f;
        } else {
            const float wy = a.old[4][n];
            const float hyn = yee_face_f32(wy, ch, zin ? a.old[0][n + plane] : 0.0f, ex0, a.old[2][n + 1], ez0);
            if (zin) a.neu[4][n] = hyn;
            ms += hj * (hyn * wy);
            a.neu[0][n] = 0.0f;
        }
        if (zin) a.neu[2][n] = 0.0f;
        if constexpr (MEDIA) {
            const float gx = i < nx ? a.cgain[0][n] : gain0, gy = j < ny ? a.cgain[1][n] : gain0,
                        gz = zin ? a.cgain[2][n] : gain0;
            es += __fdividef((hj * hk) * (ex0 * ex0), gx) + __fdividef((hi * hk) * (ey0 * ey0), gy) +
                  __fdividef((hi * hj) * (ez0 * ez0), gz);
        } else {
            es += (hj * hk) * (ex0 * ex0) + (hi * hk) * (ey0 * ey0) + (hi * hj) * (ez0 * ez0);
        }
    }
}

template <int P, int S, bool SOLID, bool MEDIA, int MINB, bool SPLIT>
static __global__ void __launch_bounds__(256, MINB) yee_tma_step(YeeStepArgs<float> a, unsigned L,
                                                             const __grid_constant__ YeeMaps m,
                                                             const __grid_constant__ YeeNearArgs nr) {
    DevState* st = a.st;
    if (st->violated) return;
    using Lay = YeeTmaLayout<P, MEDIA>;
    extern __shared__ __align__(128) unsigned char yee_tma_smem[];
    const unsigned ring_base = static_cast<unsigned>(__cvta_generic_to_shared(yee_tma_smem));
    YeeHp<float>* hp = reinterpret_cast<YeeHp<float>*>(yee_tma_smem + S * Lay::BYTES);
    const unsigned bar_base = ring_base + S * Lay::BYTES + 2 * (unsigned)sizeof(YeeHp<float>);
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
    const Tiles T = a.tiles;
    const long long step = st->steps;
    const double jsrc = (a.src_i >= 0 && step < a.ncurrent) ? a.current[step] : 0.0;
    const double dt = a.dt;
    const bool lossy = a.sigma_u[0] != 0.0;
    // Σ w|Eⁿ|², Σ w H⁺·H⁻ (the uniform ε and μ applied at the end), Joule loss, source work.
    // Each thread forms its cells' energy terms in f32 and sums them over a stage's planes; the
    // stage sums, the reduction over the grid and the ledger are FP64.
    double acc[4] = {0.0, 0.0, 0.0, 0.0};

    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(bar_base + 8 * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    YeeTmaCursor pf, cc;
    yee_tma_at(cc, T, blockIdx.x);
    int issued = 0;
    if (tid == 0) {
        yee_tma_at(pf, T, blockIdx.x);
        for (; issued < S - 1 && pf.valid; ++issued) {
            yee_tma_issue<P, MEDIA>(m, ring_base + issued * Lay::BYTES, bar_base + 8 * issued, pf);
            yee_tma_next(pf, T, P);
        }
    }
    const float ch = a.ch;
    const float dec0 = a.decay[0], gain0 = a.gain[0];
    const double sig0 = a.sigma_u[0];
    const unsigned ny1 = (unsigned)ny + 1;
    float hx_below = 0.0f, hy_below = 0.0f;  // H⁺ of this column at the plane below
    int hpar = 0;                            // which H⁺ plane buffer the present plane fills
    bool timed_out = false;
    int it = 0;
    while (cc.valid) {
        const int slot = it % S;
        const bool got = mbar_wait(bar_base + 8 * slot, (unsigned)((it / S) & 1));
        if (!__syncthreads_and(got)) {
            timed_out = true;
            break;
        }
        if (tid == 0 && pf.valid) {
            const int fill = (it + S - 1) % S;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            yee_tma_issue<P, MEDIA>(m, ring_base + fill * Lay::BYTES, bar_base + 8 * fill, pf);
            yee_tma_next(pf, T, P);
            ++issued;
        }
        const unsigned char* sb = yee_tma_smem + slot * Lay::BYTES;
        const float(*EX)[10][36] = reinterpret_cast<const float(*)[10][36]>(sb + Lay::EX);
        const float(*EY)[9][40] = reinterpret_cast<const float(*)[9][40]>(sb + Lay::EY);
        const float(*EZ)[10][40] = reinterpret_cast<const float(*)[10][40]>(sb + Lay::EZ);
        const float(*HX)[9][32] = reinterpret_cast<const float(*)[9][32]>(sb + Lay::HX);
        const float(*HY)[8][36] = reinterpret_cast<const float(*)[8][36]>(sb + Lay::HY);
        const float(*HZ)[9][36] = reinterpret_cast<const float(*)[9][36]>(sb + Lay::HZ);
        const float(*GX)[8][32] = reinterpret_cast<const float(*)[8][32]>(sb + Lay::GX);
        const float(*GY)[8][32] = reinterpret_cast<const float(*)[8][32]>(sb + Lay::GY);
        const float(*GZ)[8][32] = reinterpret_cast<const float(*)[8][32]>(sb + Lay::GZ);
        const int i = cc.x0 + tx, j = cc.y0 + ty;
        // whether the lattice position lies in each component's extent along x and y; with the wall
        // split (SPLIT: a.wall_split) the tiles hold i < nx and j < ny only, so every test is true
        const bool in_x = SPLIT || i <= nx, in_y = SPLIT || j <= ny, bx = SPLIT || i < nx, by = SPLIT || j < ny;
        // node-centred half weights of the boundary samples (cavity.rs:766-772)
        const float hi = (i == 0 || (!SPLIT && i == nx)) ? 0.5f : 1.0f, hj = (j == 0 || (!SPLIT && j == ny)) ? 0.5f : 1.0f;
        // the column crosses the f64 near-field box (nb_w = 0: no box, never)
        const bool box_xy = (unsigned)(i - a.nb_x0) < (unsigned)a.nb_w && (unsigned)(j - a.nb_y0) < (unsigned)a.nb_w;
        // this stage's energy products of the thread's cells per component, the z weight in each:
        // Σ hk ex², Σ hk ey², Σ ez² (with MEDIA each over its gain), Σ hx⁺hx⁻, Σ hy⁺hy⁻, Σ hk hz⁺hz⁻;
        // the x and y weights are applied once a stage
        float sx = 0.0f, sy = 0.0f, sz = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
        for (int h = 0; h < P; ++h) {
            const int k = cc.kb + h;
            if (k >= cc.k1) break;
            const bool compute = k >= cc.k0;  // else the plane below the chunk: H⁺ only
            const bool zin = k < nz;
            const float hk = (k == 0 || k == nz) ? 0.5f : 1.0f;
            // a node of the near-field box: its energy terms are the box kernel's, in f64
            const bool inbox = box_xy && (unsigned)(k - a.nb_z0) < (unsigned)a.nb_w;
            const unsigned n = (unsigned)i + L * ((unsigned)j + ny1 * (unsigned)k);
            // the gains of the thread's own edges; at a position the component does not have (the
            // padding, or the fill outside the lattice) the uniform gain, never read as a value
            float gx = gain0, gy = gain0, gz = gain0;
            if constexpr (MEDIA) {
                gx = (bx && in_y) ? GX[h][ty][tx] : gain0;
                gy = (in_x && by) ? GY[h][ty][tx] : gain0;
                gz = (in_x && in_y && zin) ? GZ[h][ty][tx] : gain0;
            }
            YeeHp<float>* hq = hp + hpar;
            // ---- 1. H⁺ (cavity.rs:1346-1379) on own faces
            const bool fx = in_x && by && zin, fy = bx && in_y && zin, fz = bx && by;
            const float wx = HX[h][ty + 1][tx], wy = HY[h][ty][tx + 4], wz = HZ[h][ty + 1][tx + 4];
            const float ex0 = EX[h][ty + 1][tx + 4], ey0 = EY[h][ty + 1][tx + 4], ez0 = EZ[h][ty + 1][tx + 4];
            const float hxn = yee_face_f32(wx, ch, EZ[h][ty + 2][tx + 4], ez0, EY[h + 1][ty + 1][tx + 4], ey0);
            const float hyn = yee_face_f32(wy, ch, EX[h + 1][ty + 1][tx + 4], ex0, EZ[h][ty + 1][tx + 5], ez0);
            const float hzn = yee_face_f32(wz, ch, EY[h][ty + 1][tx + 5], ey0, EX[h][ty + 2][tx + 4], ex0);
            hq->hx[ty + 1][tx] = hxn;
            hq->hy[ty][tx + 1] = hyn;
            hq->hz[ty + 1][tx + 1] = hzn;
            if (compute) {
                if (fx) a.neu[3][n] = hxn;
                if (fy) a.neu[4][n] = hyn;
                if (fz) a.neu[5][n] = hzn;
                // ½μ H⁻·H⁺ (cavity.rs:854-905) and ½εEⁿ² (cavity.rs:776-847), weights only. No
                // mask is needed: at a lattice position a component does not have, its old value
                // (padding, or the fill outside the lattice) is exactly zero, so its E term and
                // its H⁻·H⁺ term are zero.
                if (!inbox) {
                    mx = fmaf(hxn, wx, mx);
                    my = fmaf(hyn, wy, my);
                    mz = fmaf(hk * hzn, wz, mz);
                    if constexpr (MEDIA) {  // 1/g to within 2 ulp: the terms are f32 roundings already
                        sx += __fdividef((hk * ex0) * ex0, gx);
                        sy += __fdividef((hk * ey0) * ey0, gy);
                        sz += __fdividef(ez0 * ez0, gz);
                    } else {
                        sx = fmaf(hk * ex0, ex0, sx);
                        sy = fmaf(hk * ey0, ey0, sy);
                        sz = fmaf(ez0, ez0, sz);
                    }
                }
                // halo faces, one line per warp so the barrier waits on no warp doing twice the
                // work: the y0 − 1 row of hx (warp 7) and of hz (warp 6), the x0 − 1 column of hz
                // (warp 5, rows y0 − 1 .. y0 + 7) and of hy (warp 4, rows y0 .. y0 + 7)
                if (ty == 7) {
                    hq->hx[0][tx] = yee_face_f32(HX[h][0][tx], ch, EZ[h][1][tx + 4], EZ[h][0][tx + 4], EY[h + 1][0][tx + 4], EY[h][0][tx + 4]);
                } else if (ty == 6) {
                    hq->hz[0][tx + 1] = yee_face_f32(HZ[h][0][tx + 4], ch, EY[h][0][tx + 5], EY[h][0][tx + 4], EX[h][1][tx + 4], EX[h][0][tx + 4]);
                } else if (ty == 5 && tx < 9) {
                    const int r = tx;
                    hq->hz[r][0] = yee_face_f32(HZ[h][r][3], ch, EY[h][r][4], EY[h][r][3], EX[h][r + 1][3], EX[h][r][3]);
                } else if (ty == 4 && tx >= 1 && tx < 9) {
                    const int r = tx;
                    hq->hy[r - 1][0] = yee_face_f32(HY[h][r - 1][3], ch, EX[h + 1][r][3], EX[h][r][3], EZ[h][r][4], EZ[h][r][3]);
                }
            }
            __syncthreads();
            // ---- 2. Eⁿ⁺¹ on own edges (cavity.rs:1383-1452): interior by the semi-implicit update,
            // conducting walls 0 (cavity.rs:1239-1293), edges touching a solid cell 0 (cavity.rs:304-331)
            if (compute) {
                const bool ix = i >= 1 && bx, iy = j >= 1 && by, iz = k >= 1 && k < nz;
                const float cex = (hzn - hq->hz[ty][tx + 1]) - (hyn - hy_below);  // own H⁺ from registers
                const float cey = (hxn - hx_below) - (hzn - hq->hz[ty + 1][tx]);
                const float cez = (hyn - hq->hy[ty][tx]) - (hxn - hq->hx[ty][tx]);
                float vx = dec0 * ex0 + gx * cex;
                float vy = dec0 * ey0 + gy * cey;
                float vz = dec0 * ez0 + gz * cez;
                if (i == a.src_i && j == a.src_j && k == a.src_k) {
                    // soft current: ε dE/dt = ∇×H − J, with the σ term's semi-implicit divisor
                    const double e = a.eps_src, ss = a.sig_src;
                    vz = (float)((double)vz - (dt / e) / (1.0 + (ss * dt / (2.0 * e))) * jsrc);
                    acc[3] += -(dt * a.volume) * jsrc * (0.5 * ((double)ez0 + (double)vz));
                }
                const bool lx = iy && iz, ly = ix && iz, lz = ix && iy;  // interior edges
                vx = lx ? vx : 0.0f;
                vy = ly ? vy : 0.0f;
                vz = lz ? vz : 0.0f;
                if (lossy && !inbox) {
                    const double mx = 0.5 * ((double)ex0 + (double)vx), my = 0.5 * ((double)ey0 + (double)vy),
                                 mz = 0.5 * ((double)ez0 + (double)vz);
                    acc[2] += (lx && bx && in_y) ? sig0 * mx * mx * dt * a.volume : 0.0;
                    acc[2] += (ly && in_x && by) ? sig0 * my * my * dt * a.volume : 0.0;
                    acc[2] += (lz && in_x && in_y && zin) ? sig0 * mz * mz * dt * a.volume : 0.0;
                }
                if constexpr (SOLID) {
                    if (touches_solid(a.solid, nx, ny, nz, i, i, j - 1, j, k - 1, k)) vx = 0.0f;
                    if (touches_solid(a.solid, nx, ny, nz, i - 1, i, j, j, k - 1, k)) vy = 0.0f;
                    if (touches_solid(a.solid, nx, ny, nz, i - 1, i, j - 1, j, k, k)) vz = 0.0f;
                }
                if (bx && in_y) a.neu[0][n] = vx;
                if (in_x && by) a.neu[1][n] = vy;
                if (in_x && in_y && zin) a.neu[2][n] = vz;
            }
            hx_below = hxn;
            hy_below = hyn;
            hpar ^= 1;
        }
        acc[0] += (double)(hj * sx + hi * sy + (hi * hj) * sz);
        acc[1] += (double)(hi * mx + hj * my + mz);
        yee_tma_next(cc, T, P);
        ++it;
    }
    if (SPLIT && !timed_out) {
        float es = 0.0f, ms = 0.0f;
        yee_tma_wall_pass<MEDIA>(a, L, (long long)blockIdx.x * 256 + tid, (long long)gridDim.x * 256, es, ms);
        acc[0] += (double)es;
        acc[1] += (double)ms;
    }
    if (timed_out) {
        // stop every later kernel of the call, and let the copies still in flight land before
        // the block's shared memory is given up
        if (tid == 0) {
            st->violated = kDeviceTimeout;
            for (int q = it; q < issued; ++q) mbar_wait(bar_base + 8 * (q % S), (unsigned)((q / S) & 1));
        }
        return;
    }
    if (finish_blocks<4>(acc, a.partials, a.nblocks, &st->counter)) {
        // the last block: with a near-field box it steps the box, adds the box's terms and closes the
        // books (every other block's cells are in by now: each published its sums after them)
        if (a.nb_w > 0)
            yee_near_body<SOLID>(nr, acc);
        else if (linear_tid() == 0)
            yee_tma_close(st, acc, MEDIA, a.g, a.eps_u, a.mu_u, a.volume, a.src_i >= 0);
    }
}

// Between the reference layout of one component (extents ex × ey × ez, x fastest) and the
// padded lattice (row pitch L, ny1 rows per plane): to_padded = 1 scatters into the lattice
// (whose padding the caller has zeroed), 0 gathers back.
template <typename S, typename D>
static __global__ void yee_relayout(const S* __restrict__ src, D* __restrict__ dst, int ex, int ey, int ez, unsigned L,
                                    unsigned ny1, int to_padded) {
    const size_t n = (size_t)ex * ey * ez;
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
        const size_t i = r % (size_t)ex, rest = r / (size_t)ex;
        const size_t j = rest % (size_t)ey, k = rest / (size_t)ey;
        const size_t p = i + (size_t)L * (j + (size_t)ny1 * k);
        if (to_padded) dst[p] = (D)src[r];
        else dst[r] = (D)src[p];
    }
}

}  // namespace pm
