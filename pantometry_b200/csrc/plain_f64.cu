// The plain f64 forms. This translation unit is compiled with --fmad=false: no multiply-add is
// contracted, so every value is formed by the reference's own expression, rounded per operation
// as rustc's f64 arithmetic rounds it.
#include <algorithm>
#include "launch.h"

namespace pm {

cudaError_t launch_heat_plain(const HeatPlainArgs& a, cudaStream_t s) {
    if (a.quads) heat_plain_quad_step<<<a.nblocks, tile_block(), 0, s>>>(a);
    else if (a.pairs) heat_plain_pair_step<<<a.nblocks, tile_block(), 0, s>>>(a);
    else heat_plain_step<<<a.nblocks, tile_block(), 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_heat_plain_steps(const HeatPlainArgs& a, const HeatPersist& p, cudaStream_t s) {
    HeatPlainArgs aa = a;
    HeatPersist pp = p;
    void* args[2] = {&aa, &pp};
    // the tiling's rows are the block's y extent: 8 (256 threads) or 32 (1024)
    if (a.tiles.rows == 32)
        return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(heat_plain_pair_steps<32>), dim3(a.nblocks),
                                           dim3(32, 32), args, 0, s);
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(heat_plain_pair_steps<8>), dim3(a.nblocks), tile_block(),
                                       args, 0, s);
}

cudaError_t launch_heat_measure_plain(const HeatMeasureArgs& a, cudaStream_t s) {
    heat_measure<<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_heat_convert(const double* t, float* d, double t0, size_t n, int to_dev, double* tout,
                                cudaStream_t s) {
    if (to_dev)
        heat_to_deviation<<<kMeasureBlocks, 256, 0, s>>>(t, d, t0, n);
    else
        heat_from_deviation<<<kMeasureBlocks, 256, 0, s>>>(d, tout, t0, n);
    return cudaGetLastError();
}

cudaError_t launch_heat_rise(double* t64, float* d32, double rise, size_t n, const uint8_t* vd, cudaStream_t s) {
    if (t64)
        heat_add_rise64<<<kMeasureBlocks, 256, 0, s>>>(t64, rise, n, vd);
    else
        heat_add_rise32<<<kMeasureBlocks, 256, 0, s>>>(d32, (float)rise, n, vd);
    return cudaGetLastError();
}

template <>
cudaError_t launch_hall<double>(const HallArgs<double>& a, cudaStream_t s) {
    const int smem = (int)hall_smem_bytes<double>();
    return launch_smem(a.block_scale ? hall_step<double, true> : hall_step<double, false>, a.nblocks, tile_block(), smem, s, a);
}
template <>
cudaError_t launch_hall_measure<double>(const HallMeasureArgs<double>& a, cudaStream_t s) {
    hall_measure<double><<<a.nblocks, tile_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_h<double>(const YeeHArgs<double>& a, cudaStream_t s) {
    yee_h<double><<<a.nblocks, tile_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_e<double>(const YeeEArgs<double>& a, cudaStream_t s) {
    yee_e<double><<<a.nblocks, tile_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_step<double>(const YeeStepArgs<double>& a, cudaStream_t s) {
    const int smem = (int)yee_smem_bytes<double>();
    auto k = a.uniform ? (a.solid ? yee_step<double, true, true> : yee_step<double, true, false>)
                       : (a.solid ? yee_step<double, false, true> : yee_step<double, false, false>);
    return launch_smem(k, a.nblocks, tile_block(), smem, s, a);
}
template <>
cudaError_t launch_yee_measure<double>(const YeeHArgs<double>& a, double* out2, cudaStream_t s) {
    yee_measure<double><<<a.nblocks, tile_block(), 0, s>>>(a, out2);
    return cudaGetLastError();
}
template <>
cudaError_t launch_ens<double>(const EnsArgs<double>& a, bool measure, unsigned nblocks, cudaStream_t s) {
    if (a.wide) {
        if (measure) ens_step<double, true, true><<<nblocks, 256, 0, s>>>(a);
        else ens_step<double, false, true><<<nblocks, 256, 0, s>>>(a);
    } else {
        if (measure) ens_step<double, true><<<nblocks, 256, 0, s>>>(a);
        else ens_step<double, false><<<nblocks, 256, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <>
cudaError_t launch_yee_enforce_solid<double>(const YeeWallArgs<double>& a, const uint8_t* solid, cudaStream_t s) {
    yee_enforce_solid<double><<<kMeasureBlocks, 256, 0, s>>>(a, solid);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_walls<double>(const YeeWallArgs<double>& a, cudaStream_t s) {
    yee_walls<double><<<kMeasureBlocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_coefs<double>(const YeeCoefArgs<double>& a, cudaStream_t s) {
    yee_coefs<double><<<kMeasureBlocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_room<double>(const RoomArgs<double>& a, cudaStream_t s) {
    room_step<double><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_room_measure<double>(const RoomMeasureArgs<double>& a, cudaStream_t s) {
    room_measure<double><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_tube<double>(const TubeArgs<double>& a, cudaStream_t s) {
    tube_step<double><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_tube_measure<double>(const TubeMeasureArgs<double>& a, cudaStream_t s) {
    tube_measure<double><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_bar<double>(const BarArgs<double>& a, cudaStream_t s) {
    bar_step<double><<<a.nblocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_bar_deposit<double>(double* t, const double* per_cell, double lumped, double capacity, int n, cudaStream_t s) {
    bar_deposit<double><<<(unsigned)std::min(592, (n + 255) / 256), 256, 0, s>>>(t, per_cell, lumped, capacity, n);
    return cudaGetLastError();
}

static unsigned sample_blocks(const SampleGrid& g) {
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    return (unsigned)std::max<long long>(1, std::min<long long>((total + 255) / 256, 592));
}
template <typename Real>
cudaError_t launch_heat_sample(const SampleGrid& g, const Real* cells, double t0, const uint8_t* vd, double* out,
                               cudaStream_t s) {
    heat_sample<Real><<<sample_blocks(g), 256, 0, s>>>(g, cells, t0, vd, out);
    return cudaGetLastError();
}
template <typename Real>
cudaError_t launch_hall_sample(const SampleGrid& g, const Real* p, double* out, cudaStream_t s) {
    hall_sample<Real><<<sample_blocks(g), 256, 0, s>>>(g, p, out);
    return cudaGetLastError();
}
template <typename Real>
cudaError_t launch_yee_sample(const SampleGrid& g, const Real* ex, const Real* ey, const Real* ez, uint3 rx, uint3 ry,
                              double* out, cudaStream_t s) {
    yee_sample<Real><<<sample_blocks(g), 256, 0, s>>>(g, ex, ey, ez, rx, ry, out);
    return cudaGetLastError();
}
template <typename Real>
cudaError_t launch_room_sample(const SampleGrid& g, const Real* p, double* out, cudaStream_t s) {
    room_sample<Real><<<sample_blocks(g), 256, 0, s>>>(g, p, out);
    return cudaGetLastError();
}
template <typename Real>
cudaError_t launch_bar_sample(const SampleGrid& g, const Real* cells, double t0, double* out, cudaStream_t s) {
    bar_sample<Real><<<sample_blocks(g), 256, 0, s>>>(g, cells, t0, out);
    return cudaGetLastError();
}
template cudaError_t launch_heat_sample<double>(const SampleGrid&, const double*, double, const uint8_t*, double*, cudaStream_t);
template cudaError_t launch_heat_sample<float>(const SampleGrid&, const float*, double, const uint8_t*, double*, cudaStream_t);
template cudaError_t launch_hall_sample<double>(const SampleGrid&, const double*, double*, cudaStream_t);
template cudaError_t launch_hall_sample<float>(const SampleGrid&, const float*, double*, cudaStream_t);
template cudaError_t launch_room_sample<double>(const SampleGrid&, const double*, double*, cudaStream_t);
template cudaError_t launch_room_sample<float>(const SampleGrid&, const float*, double*, cudaStream_t);
template cudaError_t launch_bar_sample<double>(const SampleGrid&, const double*, double, double*, cudaStream_t);
template cudaError_t launch_bar_sample<float>(const SampleGrid&, const float*, double, double*, cudaStream_t);
template cudaError_t launch_yee_sample<double>(const SampleGrid&, const double*, const double*, const double*, uint3, uint3,
                                               double*, cudaStream_t);
template cudaError_t launch_yee_sample<float>(const SampleGrid&, const float*, const float*, const float*, uint3, uint3,
                                              double*, cudaStream_t);

int occupancy_f64(KernelId id) {
    int n = 0;
    cudaError_t e = cudaSuccess;
    switch (id) {
        case kHeatPlain: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_plain_step, 256, 0); break;
        case kHeatPlainPair: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_plain_pair_step, 256, 0); break;
        case kHeatPlainQuad: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_plain_quad_step, 256, 0); break;
        case kHeatPlainSteps: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_plain_pair_steps<8>, 256, 0); break;
        case kHeatPlainSteps32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, heat_plain_pair_steps<32>, 1024, 0); break;
        case kHallF64:
            e = allow_smem(hall_step<double, false>, (int)hall_smem_bytes<double>());
            if (e != cudaSuccess) break;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, hall_step<double, false>, 256, hall_smem_bytes<double>());
            break;
        case kYeeHF64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_h<double>, 256, 0); break;
        case kYeeEF64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_e<double>, 256, 0); break;
        case kYeeStepF64:
            e = allow_smem(yee_step<double, false, true>, (int)yee_smem_bytes<double>());
            if (e != cudaSuccess) break;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, yee_step<double, false, true>, 256, yee_smem_bytes<double>());
            break;
        case kEnsF64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_step<double, false>, 256, 0); break;
        case kEnsF64Pair: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_step<double, false, true>, 256, 0); break;
        case kRoomF64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, room_step<double>, 256, 0); break;
        case kTubeF64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, tube_step<double>, 256, 0); break;
        case kBarF64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bar_step<double>, 256, 0); break;
        default: return -1;
    }
    return (e == cudaSuccess && n > 0) ? n : 1;
}

cudaError_t launch_ens_relayout64(const double* dense, double* padded, double* out, int nx, int ny, int nz, int pitch,
                                  int to_dev, cudaStream_t s) {
    ens_relayout64<<<kMeasureBlocks, 256, 0, s>>>(dense, padded, out, nx, ny, nz, pitch, to_dev);
    return cudaGetLastError();
}

}  // namespace pm
