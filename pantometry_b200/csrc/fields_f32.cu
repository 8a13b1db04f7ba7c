// The f32-field forms (the chosen precision): fields in f32, ledgers and audits in f64.
#include "launch.h"

namespace pm {

cudaError_t launch_heat_f32(const HeatF32Args& a, int zchunk, cudaStream_t s) {
    dim3 g((a.nx + 31) / 32, (a.ny + 7) / 8, (a.nz + zchunk - 1) / zchunk);
    heat_f32_step<<<g, plane_block(), 0, s>>>(a, zchunk);
    return cudaGetLastError();
}

cudaError_t launch_heat_measure_f32(const HeatMeasureArgs& a, cudaStream_t s) {
    heat_measure<<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_hall<float>(const HallArgs<float>& a, cudaStream_t s) {
    hall_step<float><<<plane_grid(a.nx, a.ny, a.nz), plane_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_hall_measure<float>(const HallMeasureArgs<float>& a, cudaStream_t s) {
    hall_measure<float><<<plane_grid(a.nx, a.ny, a.nz), plane_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_h<float>(const YeeHArgs<float>& a, cudaStream_t s) {
    yee_h<float><<<plane_grid(a.nx + 1, a.ny + 1, a.nz + 1), plane_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_e<float>(const YeeEArgs<float>& a, cudaStream_t s) {
    yee_e<float><<<plane_grid(a.nx + 1, a.ny + 1, a.nz + 1), plane_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_measure<float>(const YeeHArgs<float>& a, double* out2, cudaStream_t s) {
    yee_measure<float><<<plane_grid(a.nx + 1, a.ny + 1, a.nz + 1), plane_block(), 0, s>>>(a, out2);
    return cudaGetLastError();
}

__global__ void to_f32_kernel(const double* __restrict__ src, float* __restrict__ dst, size_t n) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        dst[c] = (float)src[c];
}
__global__ void to_f64_kernel(const float* __restrict__ src, double* __restrict__ dst, size_t n) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        dst[c] = (double)src[c];
}
cudaError_t launch_to_f32(const double* src, float* dst, size_t n, cudaStream_t s) {
    to_f32_kernel<<<kMeasureBlocks, 256, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}
cudaError_t launch_to_f64(const float* src, double* dst, size_t n, cudaStream_t s) {
    to_f64_kernel<<<kMeasureBlocks, 256, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}

}  // namespace pm
