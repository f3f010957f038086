// FP64 instantiation of the tile rasterizer (compiled with -fmad=false so the
// s, t, z and smoothed-normal arithmetic matches the reference bit for bit).
#include "raster_impl.cuh"

namespace shape {
void launch_raster_f64(const RasterArgs &a, cudaStream_t s) { launch_raster_t<double>(a, s); }
int raster_occupancy_f64(const RasterArgs &a) { return raster_occupancy_t<double>(a); }
cudaError_t configure_raster_f64() { return configure_raster_t<double>(); }
}  // namespace shape
