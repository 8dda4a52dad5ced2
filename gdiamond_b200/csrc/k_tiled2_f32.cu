// k_tiled2_f32.cu -- instances of the x-pair kernels (k_tiled2.cuh) for FP32 fields.
#include "k_tiled2.cuh"

namespace fdtd {

cudaError_t tiled2_launch_f32(const TiledConfig& c, const TiledArgs& a, dim3 grid,
                               cudaStream_t st) {
  return c.pairs32 ? launch_pairs32<float, float>(c.blt, c.rows, a, grid, st)
                   : launch_type2<float, float>(c, a, grid, st);
}

cudaError_t tiled2_batch_launch_f32(const TiledConfig& c, const BatchArgs& b, int ctas,
                                     cudaStream_t st) {
  return c.pairs32 ? launch_batch_pairs32<float, float>(c.blt, c.rows, b, ctas, st)
                   : launch_batch_type<float, float>(c, b, ctas, st);
}

size_t tiled2_batch_query_f32(const TiledConfig& c, bool occupancy) {
  return occupancy ? batch_query<float, float, true>(c) : batch_query<float, float, false>(c);
}

}  // namespace fdtd
