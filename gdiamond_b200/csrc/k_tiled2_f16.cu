// k_tiled2_f16.cu -- instances of the x-pair kernels (k_tiled2.cuh) for FP16 fields.
#include "k_tiled2.cuh"

namespace fdtd {

cudaError_t tiled2_launch_f16(const TiledConfig& c, const TiledArgs& a, dim3 grid,
                               cudaStream_t st) {
  return c.pairs32 ? launch_pairs32<__half, __half>(c.blt, c.rows, a, grid, st)
                   : launch_type2<__half, __half>(c, a, grid, st);
}

cudaError_t tiled2_batch_launch_f16(const TiledConfig& c, const BatchArgs& b, int ctas,
                                     cudaStream_t st) {
  return c.pairs32 ? launch_batch_pairs32<__half, __half>(c.blt, c.rows, b, ctas, st)
                   : launch_batch_type<__half, __half>(c, b, ctas, st);
}

size_t tiled2_batch_query_f16(const TiledConfig& c, bool occupancy) {
  return occupancy ? batch_query<__half, __half, true>(c) : batch_query<__half, __half, false>(c);
}

}  // namespace fdtd
