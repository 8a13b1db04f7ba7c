// The f32-field forms (the chosen precision): fields in f32, ledgers and audits in f64.
#include "launch.h"

namespace pm {

cudaError_t launch_heat_f32(const HeatF32Args& a, cudaStream_t s) {
    heat_f32_step<<<a.nblocks, tile_block(), 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_heat_measure_f32(const HeatMeasureArgs& a, cudaStream_t s) {
    heat_measure<<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_hall<float>(const HallArgs<float>& a, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(hall_step<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hall_smem_bytes<float>());
        cudaFuncSetAttribute(hall_step<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hall_smem_bytes<float>());
        attr = true;
    }
    if (a.block_scale)
        hall_step<float, true><<<a.nblocks, tile_block(), hall_smem_bytes<float>(), s>>>(a);
    else
        hall_step<float, false><<<a.nblocks, tile_block(), hall_smem_bytes<float>(), s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_hall_measure<float>(const HallMeasureArgs<float>& a, cudaStream_t s) {
    hall_measure<float><<<a.nblocks, tile_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_h<float>(const YeeHArgs<float>& a, cudaStream_t s) {
    yee_h<float><<<a.nblocks, tile_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_e<float>(const YeeEArgs<float>& a, cudaStream_t s) {
    yee_e<float><<<a.nblocks, tile_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_step<float>(const YeeStepArgs<float>& a, cudaStream_t s) {
    static bool attr = false;
    const int smem = (int)yee_smem_bytes<float>();
    if (!attr) {
        cudaFuncSetAttribute(yee_step<float, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(yee_step<float, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(yee_step<float, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(yee_step<float, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr = true;
    }
    if (a.uniform) {
        if (a.solid) yee_step<float, true, true><<<a.nblocks, tile_block(), smem, s>>>(a);
        else yee_step<float, true, false><<<a.nblocks, tile_block(), smem, s>>>(a);
    } else {
        if (a.solid) yee_step<float, false, true><<<a.nblocks, tile_block(), smem, s>>>(a);
        else yee_step<float, false, false><<<a.nblocks, tile_block(), smem, s>>>(a);
    }
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_measure<float>(const YeeHArgs<float>& a, double* out2, cudaStream_t s) {
    yee_measure<float><<<a.nblocks, tile_block(), 0, s>>>(a, out2);
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


template <>
cudaError_t launch_ens<float>(const EnsArgs<float>& a, bool measure, unsigned nblocks, cudaStream_t s) {
    if (measure) ens_step<float, true><<<nblocks, 256, 0, s>>>(a);
    else ens_step<float, false><<<nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

int occupancy_f32(KernelId id) {
    int n = 0;
    cudaError_t e = cudaSuccess;
    switch (id) {
        case kHeatF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_f32_step, 256, 0); break;
        case kHallF32:
            cudaFuncSetAttribute(hall_step<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hall_smem_bytes<float>());
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, hall_step<float, false>, 256, hall_smem_bytes<float>());
            break;
        case kYeeHF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_h<float>, 256, 0); break;
        case kYeeEF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_e<float>, 256, 0); break;
        case kYeeStepF32:
            cudaFuncSetAttribute(yee_step<float, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)yee_smem_bytes<float>());
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_step<float, false, true>, 256, yee_smem_bytes<float>());
            break;
        case kEnsF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_step<float, false>, 256, 0); break;
        default: return -1;
    }
    return (e == cudaSuccess && n > 0) ? n : 1;
}

}  // namespace pm
