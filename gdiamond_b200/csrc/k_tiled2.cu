// k_tiled2.cu -- configuration checks, grid shape and storage dispatch of the x-pair kernels
// (k_tiled2.cuh); the kernel instances live in one translation unit per field storage.
#include "k_tiled2.cuh"

namespace fdtd {

namespace {

bool pairs32_supported(const TiledConfig& c) {
  return (c.esz == 4 || c.esz == 2) && c.width == 32 && c.min_blocks == 1 &&
         ((c.rows == 32 && c.blt >= 1 && c.blt <= 3) ||
          ((c.rows == 24 || c.rows == 48) && c.blt >= 1 && c.blt <= 2));
}

}  // namespace

bool tiled2_config_supported(const TiledConfig& c) {
  if (c.pairs32) return pairs32_supported(c) && c.z_chunks >= 1;
  if (c.esz != 4 && c.esz != 2) return false;
  if (c.rows != 8 && c.rows != 16 && c.rows != 20 && c.rows != 24 && c.rows != 32) return false;
  if (c.rows > 16 && c.esz != 4) return false;
  if (c.blt < 1 || c.blt > 4) return false;
  if ((c.rows == 8 || c.rows == 20) && c.blt > 3) return false;
  if ((c.rows == 24 || c.rows == 32) && c.blt > 2) return false;  // the pair state spills
  if (c.min_blocks > 1 && !(c.esz == 4 && c.blt == 2 &&
                            ((c.rows == 16 && c.min_blocks == 2) ||
                             (c.rows == 8 && c.min_blocks == 4))))
    return false;
  return c.z_chunks >= 1;
}

bool tiled2_batch_supported(const TiledConfig& c) {
  if (c.pairs32) return pairs32_supported(c);
  if (c.esz != 4 && c.esz != 2) return false;
  if (c.rows == 16) return c.blt >= 1 && c.blt <= 4;
  if (c.rows == 8) return c.blt >= 1 && c.blt <= 3;
  if (c.rows == 20) return c.esz == 4 && c.blt >= 1 && c.blt <= 3;
  if (c.rows == 24) return c.esz == 4 && c.blt >= 1 && c.blt <= 2;
  return false;
}

dim3 tiled2_grid(const TiledConfig& c, const Grid& g) {
  const int sx = tiled2_sx_w(c.pairs32 ? 32 : 64, c.blt), sy = tiled_sy(c.blt, c.rows);
  const int first = tiled2_xbase(c.blt) + c.blt;
  const int ntx = (g.nx - first + sx - 1) / sx;
  const int nty = (g.ny + sy - 1) / sy;
  const int zlen = (g.nz + c.z_chunks - 1) / c.z_chunks;
  const int nzc = (g.nz + zlen - 1) / zlen;
  return dim3(ntx, nty, nzc);
}

size_t tiled2_batch_smem(const TiledConfig& c) {
  switch (c.storage) {
    case 0: return tiled2_batch_query_f32(c, false);
    case 1: return tiled2_batch_query_f16(c, false);
    case 2: return tiled2_batch_query_bf16(c, false);
    case 4: return tiled2_batch_query_f16e(c, false);
  }
  return 0;
}

int tiled2_batch_ctas_per_sm(const TiledConfig& c) {
  switch (c.storage) {
    case 0: return (int)tiled2_batch_query_f32(c, true);
    case 1: return (int)tiled2_batch_query_f16(c, true);
    case 2: return (int)tiled2_batch_query_bf16(c, true);
    case 4: return (int)tiled2_batch_query_f16e(c, true);
  }
  return 1;
}

// storage: 0 FP32, 1 FP16, 2 BF16, 4 FP16 E with FP32 H.
cudaError_t launch_tiled2(const TiledConfig& c, const TiledArgs& a, const Grid& g,
                          cudaStream_t st) {
  if (!tiled2_config_supported(c)) return cudaErrorInvalidValue;
  const dim3 grid = tiled2_grid(c, g);
  switch (c.storage) {
    case 0: return tiled2_launch_f32(c, a, grid, st);
    case 1: return tiled2_launch_f16(c, a, grid, st);
    case 2: return tiled2_launch_bf16(c, a, grid, st);
    case 4: return tiled2_launch_f16e(c, a, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_tiled2_batch(const TiledConfig& c, const BatchArgs& b, int ctas,
                                cudaStream_t st) {
  if (!tiled2_batch_supported(c)) return cudaErrorInvalidValue;
  switch (c.storage) {
    case 0: return tiled2_batch_launch_f32(c, b, ctas, st);
    case 1: return tiled2_batch_launch_f16(c, b, ctas, st);
    case 2: return tiled2_batch_launch_bf16(c, b, ctas, st);
    case 4: return tiled2_batch_launch_f16e(c, b, ctas, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fdtd
