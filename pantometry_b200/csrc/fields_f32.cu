// The f32-field forms (the chosen precision): fields in f32, ledgers and audits in f64.
#include <algorithm>
#include <cudaTypedefs.h>

#include "launch.h"

namespace pm {

cudaError_t launch_heat_f32(const HeatF32Args& a, cudaStream_t s) {
    if (a.kx) heat_f32_step<true><<<a.nblocks, tile_block(), 0, s>>>(a);
    else if (a.quads) heat_f32_quad_step<<<a.nblocks, tile_block(), 0, s>>>(a);
    else heat_f32_step<false><<<a.nblocks, tile_block(), 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_heat_f32_steps(const HeatF32Args& a, const HeatPersist& p, cudaStream_t s) {
    HeatF32Args aa = a;
    HeatPersist pp = p;
    void* args[2] = {&aa, &pp};
    // the tiling's rows are the block's y extent: 8 (256 threads) or 32 (1024)
    if (a.tiles.rows == 32)
        return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(heat_f32_quad_steps<32>), dim3(a.nblocks),
                                           dim3(32, 32), args, 0, s);
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(heat_f32_quad_steps<8>), dim3(a.nblocks), tile_block(),
                                       args, 0, s);
}

cudaError_t launch_heat_measure_f32(const HeatMeasureArgs& a, cudaStream_t s) {
    heat_measure<<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_hall<float>(const HallArgs<float>& a, cudaStream_t s) {
    const int smem = (int)hall_smem_bytes<float>();
    return launch_smem(a.block_scale ? hall_step<float, true> : hall_step<float, false>, a.nblocks, tile_block(), smem, s, a);
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
    const int smem = (int)yee_smem_bytes<float>();
    auto k = a.uniform ? (a.solid ? yee_step<float, true, true> : yee_step<float, true, false>)
                       : (a.solid ? yee_step<float, false, true> : yee_step<float, false, false>);
    return launch_smem(k, a.nblocks, tile_block(), smem, s, a);
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
    if (a.wide) {
        if (measure) ens_step<float, true, true><<<nblocks, 256, 0, s>>>(a);
        else ens_step<float, false, true><<<nblocks, 256, 0, s>>>(a);
    } else {
        if (measure) ens_step<float, true><<<nblocks, 256, 0, s>>>(a);
        else ens_step<float, false><<<nblocks, 256, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <int P, int S, int MINB>
static cudaError_t launch_hall_tma_shape(const HallArgs<float>& a, const HallMaps& m, cudaStream_t s) {
    const int smem = (int)hall_tma_smem_bytes_for<P, S>();
    return launch_smem(a.block_scale ? hall_tma_step<P, S, true, MINB> : hall_tma_step<P, S, false, MINB>, a.nblocks,
                       tile_block(), smem, s, a, m);
}
cudaError_t launch_hall_tma(const HallArgs<float>& a, const HallMaps& m, int shape, cudaStream_t s) {
    static_assert(kHallTmaShapes[0].planes == 8 && kHallTmaShapes[1].planes == 6 && kHallTmaShapes[2].planes == 4 &&
                      kHallTmaShapes[3].planes == 4,
                  "the dispatch below instantiates kHallTmaShapes in order");
    switch (shape) {
        case 1: return launch_hall_tma_shape<6, 2, 3>(a, m, s);
        case 2: return launch_hall_tma_shape<4, 3, 3>(a, m, s);
        case 3: return launch_hall_tma_shape<4, 2, 4>(a, m, s);
        default: return launch_hall_tma_shape<8, 2, 2>(a, m, s);
    }
}
template <int P, int S, int MINB>
static int hall_tma_occupancy() {
    int n = 0;
    if (allow_smem(hall_tma_step<P, S, false, MINB>, (int)hall_tma_smem_bytes_for<P, S>()) != cudaSuccess) return 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, hall_tma_step<P, S, false, MINB>, 256,
                                                      hall_tma_smem_bytes_for<P, S>()) != cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

bool hall_tma_map(CUtensorMap* map, void* base, int nx, int ny, int nz, unsigned bx, unsigned by, unsigned bz) {
    // looked up once per process (the driver's entry point is the same for every device); a
    // function-local static is initialised exactly once even when threads race to it
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * 4, (cuuint64_t)nx * ny * 4};
    const cuuint32_t box[3] = {bx, by, bz};
    const cuuint32_t estr[3] = {1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int P, int S, bool MEDIA, int MINB>
static cudaError_t launch_yee_tma_shape(const YeeStepArgs<float>& a, unsigned L, const YeeMaps& m, const YeeNearArgs& n,
                                       cudaStream_t s) {
    const int smem = (int)yee_tma_smem_bytes_for<P, MEDIA>(S);
    auto k = a.solid ? (a.wall_split ? yee_tma_step<P, S, true, MEDIA, MINB, true> : yee_tma_step<P, S, true, MEDIA, MINB, false>)
                     : (a.wall_split ? yee_tma_step<P, S, false, MEDIA, MINB, true> : yee_tma_step<P, S, false, MEDIA, MINB, false>);
    return launch_smem(k, a.nblocks, tile_block(), smem, s, a, L, m, n);
}
cudaError_t launch_yee_tma(const YeeStepArgs<float>& a, unsigned L, const YeeMaps& m, int shape, cudaStream_t s,
                           const YeeNearArgs& n) {
    static_assert(kYeeTmaUniformShapes[0].planes == 3 && kYeeTmaUniformShapes[1].planes == 4 &&
                      kYeeTmaUniformShapes[2].stages == 3 && kYeeTmaMediaShapes[0].planes == 4 &&
                      kYeeTmaMediaShapes[1].planes == 3,
                  "the dispatch below instantiates the shape lists in order");
    if (!a.uniform) return shape == 1 ? launch_yee_tma_shape<3, 2, true, 3>(a, L, m, n, s) : launch_yee_tma_shape<4, 2, true, 2>(a, L, m, n, s);
    switch (shape) {
        case 1: return launch_yee_tma_shape<4, 2, false, 2>(a, L, m, n, s);
        case 2: return launch_yee_tma_shape<3, 3, false, 2>(a, L, m, n, s);
        default: return launch_yee_tma_shape<3, 2, false, 3>(a, L, m, n, s);
    }
}
template <int P, int S, bool MEDIA, int MINB>
static int yee_tma_occupancy() {
    int n = 0;
    const size_t smem = yee_tma_smem_bytes_for<P, MEDIA>(S);
    if (allow_smem(yee_tma_step<P, S, false, MEDIA, MINB, false>, (int)smem) != cudaSuccess) return 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_tma_step<P, S, false, MEDIA, MINB, false>, 256, smem) != cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

cudaError_t launch_yee_near_seed(const YeeNearArgs& a, cudaStream_t s) {
    yee_near_seed<<<1, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_yee_relayout(const void* src, bool src_f64, void* dst, bool dst_f64, int ex, int ey, int ez,
                                unsigned L, unsigned ny1, int to_padded, cudaStream_t s) {
    if (src_f64 && !dst_f64)
        yee_relayout<double, float><<<kMeasureBlocks, 256, 0, s>>>(static_cast<const double*>(src), static_cast<float*>(dst), ex, ey,
                                                                   ez, L, ny1, to_padded);
    else if (!src_f64 && dst_f64)
        yee_relayout<float, double><<<kMeasureBlocks, 256, 0, s>>>(static_cast<const float*>(src), static_cast<double*>(dst), ex, ey,
                                                                   ez, L, ny1, to_padded);
    else if (!src_f64 && !dst_f64)
        yee_relayout<float, float><<<kMeasureBlocks, 256, 0, s>>>(static_cast<const float*>(src), static_cast<float*>(dst), ex, ey,
                                                                  ez, L, ny1, to_padded);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_ens_tma(const EnsTmaArgs& t, unsigned nblocks, cudaStream_t s) {
    const int smem = (int)ens_tma_smem_bytes();
    cudaError_t e = launch_smem(ens_tma_step<kEnsTmaPlanes, kEnsTmaStages>, nblocks, kEnsConsumers + 32, smem, s, t);
    if (e != cudaSuccess) return e;
    ens_tma_books<<<(t.e.ngrids + 7) / 8, 256, 0, s>>>(t.e);
    return cudaGetLastError();
}

cudaError_t launch_heat_tma(const HeatTmaArgs& a, const CUtensorMap& map, cudaStream_t s) {
    return launch_smem(heat_tma_step<kEnsTmaPlanes, kEnsTmaStages>, a.nblocks, kEnsConsumers + 32,
                       (int)ens_tma_smem_bytes(), s, a, map);
}
bool heat_tma_map(CUtensorMap* map, void* base, int nx, int ny, int nz) {
    return hall_tma_map(map, base, nx, ny, nz, 40, 10, kEnsTmaPlanes + 2);
}

cudaError_t launch_ens_relayout(const double* kelvin, float* dev, double* out, int nx, int ny, int nz, int pitch,
                                double t0, int to_dev, cudaStream_t s) {
    ens_relayout<<<kMeasureBlocks, 256, 0, s>>>(kelvin, dev, out, nx, ny, nz, pitch, t0, to_dev);
    return cudaGetLastError();
}

template <>
cudaError_t launch_yee_enforce_solid<float>(const YeeWallArgs<float>& a, const uint8_t* solid, cudaStream_t s) {
    yee_enforce_solid<float><<<kMeasureBlocks, 256, 0, s>>>(a, solid);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_walls<float>(const YeeWallArgs<float>& a, cudaStream_t s) {
    yee_walls<float><<<kMeasureBlocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_coefs<float>(const YeeCoefArgs<float>& a, cudaStream_t s) {
    yee_coefs<float><<<kMeasureBlocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_room<float>(const RoomArgs<float>& a, cudaStream_t s) {
    room_step<float><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_room_measure<float>(const RoomMeasureArgs<float>& a, cudaStream_t s) {
    room_measure<float><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_tube<float>(const TubeArgs<float>& a, cudaStream_t s) {
    tube_step<float><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_tube_measure<float>(const TubeMeasureArgs<float>& a, cudaStream_t s) {
    tube_measure<float><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_bar<float>(const BarArgs<float>& a, cudaStream_t s) {
    bar_step<float><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_bar_deposit<float>(float* t, const double* per_cell, double lumped, double capacity, int n, cudaStream_t s) {
    bar_deposit<float><<<(unsigned)std::min(592, (n + 255) / 256), 256, 0, s>>>(t, per_cell, lumped, capacity, n);
    return cudaGetLastError();
}

int occupancy_f32(KernelId id) {
    int n = 0;
    cudaError_t e = cudaSuccess;
    switch (id) {
        case kHeatF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_f32_step<false>, 256, 0); break;
        case kHeatF32Quad: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_f32_quad_step, 256, 0); break;
        case kHeatF32QuadSteps: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_f32_quad_steps<8>, 256, 0); break;
        case kHeatF32QuadSteps32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_f32_quad_steps<32>, 1024, 0); break;
        case kHeatTma:
            e = allow_smem(heat_tma_step<kEnsTmaPlanes, kEnsTmaStages>, (int)ens_tma_smem_bytes());
            if (e != cudaSuccess) break;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_tma_step<kEnsTmaPlanes, kEnsTmaStages>,
                                                              kEnsConsumers + 32, ens_tma_smem_bytes());
            break;
        case kHallF32:
            e = allow_smem(hall_step<float, false>, (int)hall_smem_bytes<float>());
            if (e != cudaSuccess) break;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, hall_step<float, false>, 256, hall_smem_bytes<float>());
            break;
        case kYeeHF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_h<float>, 256, 0); break;
        case kYeeEF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_e<float>, 256, 0); break;
        case kYeeStepF32:
            e = allow_smem(yee_step<float, false, true>, (int)yee_smem_bytes<float>());
            if (e != cudaSuccess) break;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_step<float, false, true>, 256, yee_smem_bytes<float>());
            break;
        case kEnsF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_step<float, false>, 256, 0); break;
        case kEnsF32Quad: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_step<float, false, true>, 256, 0); break;
        case kEnsTma:
            e = allow_smem(ens_tma_step<kEnsTmaPlanes, kEnsTmaStages>, (int)ens_tma_smem_bytes());
            if (e != cudaSuccess) break;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_tma_step<kEnsTmaPlanes, kEnsTmaStages>,
                                                              kEnsConsumers + 32, ens_tma_smem_bytes());
            break;
        case kYeeTma: return yee_tma_occupancy<3, 2, false, 3>();
        case kYeeTmaShape1: return yee_tma_occupancy<4, 2, false, 2>();
        case kYeeTmaShape2: return yee_tma_occupancy<3, 3, false, 2>();
        case kYeeTmaMedia: return yee_tma_occupancy<4, 2, true, 2>();
        case kYeeTmaMediaShape1: return yee_tma_occupancy<3, 2, true, 3>();
        case kHallTma: return hall_tma_occupancy<8, 2, 2>();
        case kHallTmaShape1: return hall_tma_occupancy<6, 2, 3>();
        case kHallTmaShape2: return hall_tma_occupancy<4, 3, 3>();
        case kHallTmaShape3: return hall_tma_occupancy<4, 2, 4>();
        case kRoomF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, room_step<float>, 256, 0); break;
        case kTubeF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, tube_step<float>, 256, 0); break;
        case kBarF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bar_step<float>, 256, 0); break;
        default: return -1;
    }
    return (e == cudaSuccess && n > 0) ? n : 1;
}

}  // namespace pm
