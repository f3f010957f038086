// FP32 instantiation of the tile rasterizer (batched FP32 form: FMA
// contraction allowed; vertex transforms arrive already rounded from FP64).
#include "raster_impl.cuh"

namespace shape {
void launch_raster_f32(const RasterArgs &a, cudaStream_t s) { launch_raster_t<float>(a, s); }
int raster_occupancy_f32(const RasterArgs &a) { return raster_occupancy_t<float>(a); }
cudaError_t configure_raster_f32() { return configure_raster_t<float>(); }
}  // namespace shape
