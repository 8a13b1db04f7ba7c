// Host-side launchers for the stepping kernels. The plain f64 forms are compiled in
// plain_f64.cu with --fmad=false (no contraction, so bit-exact with the reference); the f32
// forms in fields_f32.cu with the default contraction.
#pragma once

#include <cuda_runtime.h>

#include "heat_kernels.cuh"
#include "hall_kernels.cuh"
#include "yee_kernels.cuh"

namespace pm {

// Launch geometry shared by every per-node kernel: 32 × 8 threads per block, one z-plane (or
// z-chunk) per grid row.
inline dim3 plane_block() { return dim3(32, 8, 1); }
inline dim3 plane_grid(int nx, int ny, int nz) { return dim3((nx + 31) / 32, (ny + 7) / 8, nz); }
inline unsigned plane_blocks(int nx, int ny, int nz) {
    dim3 g = plane_grid(nx, ny, nz);
    return g.x * g.y * g.z;
}
constexpr int kMeasureBlocks = 592;  // 4 × 148 SMs

cudaError_t launch_heat_plain(const HeatPlainArgs& a, cudaStream_t s);
cudaError_t launch_heat_measure_plain(const HeatMeasureArgs& a, cudaStream_t s);
cudaError_t launch_heat_f32(const HeatF32Args& a, int zchunk, cudaStream_t s);
cudaError_t launch_heat_measure_f32(const HeatMeasureArgs& a, cudaStream_t s);
cudaError_t launch_heat_convert(const double* t, float* d, double t0, size_t n, int to_dev, double* tout,
                                cudaStream_t s);
cudaError_t launch_heat_rise(double* t64, float* d32, double rise, size_t n, cudaStream_t s);

template <typename Real> cudaError_t launch_hall(const HallArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_hall_measure(const HallMeasureArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_yee_h(const YeeHArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_yee_e(const YeeEArgs<Real>& a, cudaStream_t s);
template <typename Real> cudaError_t launch_yee_measure(const YeeHArgs<Real>& a, double* out2, cudaStream_t s);

// Element-wise conversions between the caller's f64 arrays and an f32 store.
cudaError_t launch_to_f32(const double* src, float* dst, size_t n, cudaStream_t s);
cudaError_t launch_to_f64(const float* src, double* dst, size_t n, cudaStream_t s);

}  // namespace pm
