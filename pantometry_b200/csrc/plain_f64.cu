// The plain f64 forms. This translation unit is compiled with --fmad=false: no multiply-add is
// contracted, so every value is formed by the reference's own expression, rounded per operation
// as rustc's f64 arithmetic rounds it.
#include "launch.h"

namespace pm {

cudaError_t launch_heat_plain(const HeatPlainArgs& a, cudaStream_t s) {
    heat_plain_step<<<plane_grid(a.nx, a.ny, a.nz), plane_block(), 0, s>>>(a);
    return cudaGetLastError();
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

cudaError_t launch_heat_rise(double* t64, float* d32, double rise, size_t n, cudaStream_t s) {
    if (t64)
        heat_add_rise64<<<kMeasureBlocks, 256, 0, s>>>(t64, rise, n);
    else
        heat_add_rise32<<<kMeasureBlocks, 256, 0, s>>>(d32, (float)rise, n);
    return cudaGetLastError();
}

template <>
cudaError_t launch_hall<double>(const HallArgs<double>& a, cudaStream_t s) {
    hall_step<double><<<plane_grid(a.nx, a.ny, a.nz), plane_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_hall_measure<double>(const HallMeasureArgs<double>& a, cudaStream_t s) {
    hall_measure<double><<<plane_grid(a.nx, a.ny, a.nz), plane_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_h<double>(const YeeHArgs<double>& a, cudaStream_t s) {
    yee_h<double><<<plane_grid(a.nx + 1, a.ny + 1, a.nz + 1), plane_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_e<double>(const YeeEArgs<double>& a, cudaStream_t s) {
    yee_e<double><<<plane_grid(a.nx + 1, a.ny + 1, a.nz + 1), plane_block(), 0, s>>>(a);
    return cudaGetLastError();
}
template <>
cudaError_t launch_yee_measure<double>(const YeeHArgs<double>& a, double* out2, cudaStream_t s) {
    yee_measure<double><<<plane_grid(a.nx + 1, a.ny + 1, a.nz + 1), plane_block(), 0, s>>>(a, out2);
    return cudaGetLastError();
}

}  // namespace pm
