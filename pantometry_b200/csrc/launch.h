// Host-side launchers for the stepping kernels. The plain f64 forms are compiled in
// plain_f64.cu with --fmad=false (no contraction, so bit-exact with the reference); the f32
// forms in fields_f32.cu with the default contraction.
#pragma once

#include <cuda_runtime.h>

#include "heat_kernels.cuh"
#include "hall_kernels.cuh"
#include "yee_kernels.cuh"
#include "ensemble_kernels.cuh"
#include "hall_tma.cuh"
#include "yee_tma.cuh"
#include "room_kernels.cuh"
#include "ens_tma.cuh"
#include "yee_near.cuh"
#include "heat_tma.cuh"
#include "sample_kernels.cuh"

namespace pm {

// Launch geometry: 32 × 8 threads per block; a persistent grid of at most `resident` blocks
// (8 per SM at 256 threads) walking the tiles of make_tiles().
inline dim3 tile_block() { return dim3(32, 8, 1); }
constexpr int kBlocksPerSM = 8;
constexpr int kMeasureBlocks = 592;  // 4 × 148 SMs, for the flat element-wise kernels

// The z-chunk that spreads the tiles most evenly over `resident` blocks, preferring deeper
// chunks (fewer re-read planes) when the balance is equal.
// `lo`: the smallest chunk a kernel takes (a multiple of the planes it streams per stage).
inline int choose_zc(int nx, int ny, int nz, unsigned resident, int lo = 4) {
    int best = lo;
    double best_score = -1.0;
    for (int zc : {4, 8, 16, 32}) {
        if (zc < lo || (zc > nz && zc != lo)) continue;
        Tiles t = make_tiles(nx, ny, nz, zc);
        double per = (double)t.ntiles / resident;
        double rounds = per < 1.0 ? 1.0 : (double)((t.ntiles + resident - 1) / resident);
        double balance = per < 1.0 ? per : per / rounds;
        double score = balance * (1.0 - 1.0 / (2.0 * zc));
        if (score > best_score + 1e-9) { best_score = score; best = zc; }
    }
    return best;
}
inline unsigned grid_for(const Tiles& t, unsigned resident) {
    return (unsigned)(t.ntiles < (long long)resident ? t.ntiles : (long long)resident);
}

// Opt `kernel` in to `bytes` of dynamic shared memory on the current device. The attribute
// belongs to the function on one device, so the opt-in is recorded per (kernel, device) and made
// once for each, under a lock (handles on several devices and several host threads share it).
cudaError_t allow_smem_fn(const void* kernel, int bytes);
template <typename K>
inline cudaError_t allow_smem(K* kernel, int bytes) {
    return allow_smem_fn(reinterpret_cast<const void*>(kernel), bytes);
}
// Launch `kernel` with `smem` bytes of dynamic shared memory, opting it in first on this device.
template <typename... P, typename... A>
inline cudaError_t launch_smem(void (*kernel)(P...), dim3 grid, dim3 block, int smem, cudaStream_t s, const A&... args) {
    if (cudaError_t e = allow_smem(kernel, smem); e != cudaSuccess) return e;
    kernel<<<grid, block, smem, s>>>(args...);
    return cudaGetLastError();
}

// Resident blocks per SM of each step kernel at 256 threads (cudaOccupancyMaxActiveBlocksPer-
// Multiprocessor, asked once per kernel and device), so a persistent grid is exactly one full wave.
enum KernelId : int {
    kHeatPlain = 0, kHeatF32, kHallF64, kHallF32, kYeeHF64, kYeeHF32, kYeeEF64, kYeeEF32, kYeeStepF64, kYeeStepF32,
    kEnsF64, kEnsF32, kHallTma, kYeeTma, kYeeTmaMedia, kEnsTma, kRoomF64, kRoomF32, kTubeF64, kTubeF32, kBarF64, kBarF32, kHeatF32Quad, kEnsF32Quad, kHeatPlainPair, kEnsF64Pair, kHeatPlainSteps, kHeatF32QuadSteps, kHeatPlainSteps32, kHeatF32QuadSteps32, kHeatTma,
    kHallTmaShape1, kHallTmaShape2, kHallTmaShape3,  // kHallTma is shape 0
    kYeeTmaShape1, kYeeTmaShape2, kYeeTmaMediaShape1,  // kYeeTma and kYeeTmaMedia are shape 0 of each form
    kHeatPlainQuad,
    kKernelCount
};
int blocks_per_sm(KernelId id);

template <typename Real>
inline size_t yee_smem_bytes() { return sizeof(YeeStage<Real>) * YeeDepth<Real>::stages + sizeof(YeeHp<Real>); }
template <typename Real>
inline size_t hall_smem_bytes() { return sizeof(HallStage<Real>) * HallDepth<Real>::stages; }

cudaError_t launch_heat_plain(const HeatPlainArgs& a, cudaStream_t s);
// Many plain f64 pair-form steps of a small block in one cooperative launch (heat_plain_pair_steps).
cudaError_t launch_heat_plain_steps(const HeatPlainArgs& a, const HeatPersist& p, cudaStream_t s);
cudaError_t launch_heat_measure_plain(const HeatMeasureArgs& a, cudaStream_t s);
cudaError_t launch_heat_f32(const HeatF32Args& a, cudaStream_t s);
// Many FP32 quad-form steps of a small block in one cooperative launch (heat_f32_quad_steps).
cudaError_t launch_heat_f32_steps(const HeatF32Args& a, const HeatPersist& p, cudaStream_t s);
// One FP32 step of a uniform block whose rows hold a multiple of 4 cells, staged by TMA
// (heat_tma_step) from the old deviations `map` describes (heat_tma_map).
cudaError_t launch_heat_tma(const HeatTmaArgs& a, const CUtensorMap& map, cudaStream_t s);
bool heat_tma_map(CUtensorMap* map, void* base, int nx, int ny, int nz);
cudaError_t launch_heat_measure_f32(const HeatMeasureArgs& a, cudaStream_t s);
// scene::capture's sampling of a field over an extent's grid (sample_kernels.cuh), into `out` on
// the device: Solid3D and Bar1D (kelvin, or FP32 deviations with t0 added), Hall and Room
// pressure, Cavity |E|.
template <typename Real>
cudaError_t launch_heat_sample(const SampleGrid& g, const Real* cells, double t0, const uint8_t* vd, double* out,
                               cudaStream_t s);
template <typename Real>
cudaError_t launch_hall_sample(const SampleGrid& g, const Real* p, double* out, cudaStream_t s);
template <typename Real>
cudaError_t launch_room_sample(const SampleGrid& g, const Real* p, double* out, cudaStream_t s);
template <typename Real>
cudaError_t launch_bar_sample(const SampleGrid& g, const Real* cells, double t0, double* out, cudaStream_t s);
template <typename Real>
cudaError_t launch_yee_sample(const SampleGrid& g, const Real* ex, const Real* ey, const Real* ez, uint3 rx, uint3 ry,
                              double* out, cudaStream_t s);
cudaError_t launch_heat_convert(const double* t, float* d, double t0, size_t n, int to_dev, double* tout,
                                cudaStream_t s);
cudaError_t launch_heat_rise(double* t64, float* d32, double rise, size_t n, const uint8_t* vd, cudaStream_t s);

template <typename Real> cudaError_t launch_hall(const HallArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_hall_measure(const HallMeasureArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_yee_h(const YeeHArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_yee_e(const YeeEArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_yee_step(const YeeStepArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_yee_measure(const YeeHArgs<Real>& a, double* out2, cudaStream_t s);
template <typename Real> cudaError_t launch_yee_walls(const YeeWallArgs<Real>& a, cudaStream_t s);
template <typename Real>
cudaError_t launch_yee_enforce_solid(const YeeWallArgs<Real>& a, const uint8_t* solid, cudaStream_t s);
template <typename Real> cudaError_t launch_yee_coefs(const YeeCoefArgs<Real>& a, cudaStream_t s);
// The FP32 Hall step staged by TMA (padded face layout, nx a multiple of 4), in tile shape `shape`
// (an index of kHallTmaShapes).
cudaError_t launch_hall_tma(const HallArgs<float>& a, const HallMaps& m, int shape, cudaStream_t s);
template <int P, int S>
inline size_t hall_tma_smem_bytes_for() {
    return sizeof(HallTmaStage<P>) * S + 8 * S;
}
inline size_t hall_tma_smem_bytes(int shape = 0) {
    switch (shape) {
        case 1: return hall_tma_smem_bytes_for<6, 2>();
        case 2: return hall_tma_smem_bytes_for<4, 3>();
        case 3: return hall_tma_smem_bytes_for<4, 2>();
        default: return hall_tma_smem_bytes_for<8, 2>();
    }
}
inline KernelId hall_tma_kernel_id(int shape) {
    return shape == 1 ? kHallTmaShape1 : shape == 2 ? kHallTmaShape2 : shape == 3 ? kHallTmaShape3 : kHallTma;
}
// Encode the tensor map of one f32 field of an nx × ny × nz hall (row pitch nx·4 bytes) with the
// given box; false if the driver refuses it.
bool hall_tma_map(CUtensorMap* map, void* base, int nx, int ny, int nz, unsigned bx, unsigned by, unsigned bz);
// The FP32 uniform-medium cavity step staged by TMA (padded lattice of row pitch L).
// `shape` indexes the form's list (kYeeTmaUniformShapes, or kYeeTmaMediaShapes when !a.uniform).
// `n`: the near-field box the last block steps (n.w = 0 with none; then it is not read).
cudaError_t launch_yee_tma(const YeeStepArgs<float>& a, unsigned L, const YeeMaps& m, int shape, cudaStream_t s,
                           const YeeNearArgs& n = YeeNearArgs{});
inline size_t yee_tma_smem_bytes(bool media = false, int shape = 0) {
    const YeeTmaShape sh = yee_tma_shape(media, shape);
    if (media) return sh.planes == 4 ? yee_tma_smem_bytes_for<4, true>(sh.stages) : yee_tma_smem_bytes_for<3, true>(sh.stages);
    return sh.planes == 4 ? yee_tma_smem_bytes_for<4, false>(sh.stages) : yee_tma_smem_bytes_for<3, false>(sh.stages);
}
inline KernelId yee_tma_kernel_id(bool media, int shape) {
    if (media) return shape == 1 ? kYeeTmaMediaShape1 : kYeeTmaMedia;
    return shape == 1 ? kYeeTmaShape1 : shape == 2 ? kYeeTmaShape2 : kYeeTma;
}
// The FP32 cavity's near-field box in f64 after the TMA step (yee_near.cuh), and its seeding from
// the stored field.
cudaError_t launch_yee_near_seed(const YeeNearArgs& a, cudaStream_t s);
// One component between the reference layout and the padded lattice (see yee_relayout);
// src_f64 / dst_f64 select double or float for each side.
cudaError_t launch_yee_relayout(const void* src, bool src_f64, void* dst, bool dst_f64, int ex, int ey, int ez,
                                unsigned L, unsigned ny1, int to_padded, cudaStream_t s);
// One FP32 ensemble step over 32 × 8-column bricks, staged by TMA.
cudaError_t launch_ens_tma(const EnsTmaArgs& t, unsigned nblocks, cudaStream_t s);
// One block between kelvin on the host's layout and f32 deviations on padded rows.
cudaError_t launch_ens_relayout(const double* kelvin, float* dev, double* out, int nx, int ny, int nz, int pitch,
                                double t0, int to_dev, cudaStream_t s);
// One f64 block between the caller's dense layout and the device's rows of `pitch`.
cudaError_t launch_ens_relayout64(const double* dense, double* padded, double* out, int nx, int ny, int nz, int pitch,
                                  int to_dev, cudaStream_t s);
// One ensemble step (measure = false) or the opening ledgers (measure = true) over the brick list.
template <typename Real> cudaError_t launch_ens(const EnsArgs<Real>& a, bool measure, unsigned nblocks, cudaStream_t s);

// Element-wise conversions between the caller's f64 arrays and an f32 store.
template <typename Real> cudaError_t launch_room(const RoomArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_room_measure(const RoomMeasureArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_tube(const TubeArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_bar(const BarArgs<Real>& a, cudaStream_t s);
template <typename Real>
cudaError_t launch_bar_deposit(Real* t, const double* per_cell, double lumped, double capacity, int n, cudaStream_t s);
template <typename Real> cudaError_t launch_tube_measure(const TubeMeasureArgs<Real>& a, cudaStream_t s);
cudaError_t launch_to_f32(const double* src, float* dst, size_t n, cudaStream_t s);
cudaError_t launch_to_f64(const float* src, double* dst, size_t n, cudaStream_t s);

}  // namespace pm
