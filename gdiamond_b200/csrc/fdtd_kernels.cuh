// fdtd_kernels.cuh -- launcher interfaces between the C-ABI host code and the kernels.
#pragma once

#include <cuda.h>  // CUtensorMap (types only; the driver entry point is fetched at run time)
#include "fdtd_common.cuh"

namespace fdtd {

struct FieldPtrs {
  float* f[6];  // Ex Ey Ez Hx Hy Hz, pitched
};

// ---------------------------------------------------------------- naive kernels
cudaError_t launch_naive_step(const Grid& g, const FieldPtrs& F, const float* const* coef,
                              const uint16_t* mat, const Material* tab, const Sources& S,
                              const Monitors& M, long long t, float dx, cudaStream_t st,
                              int* launches);

// ---------------------------------------------------------------- tiled kernel
struct TiledArgs {
  CUtensorMap tm_src[6];  // 3-D maps of the source field set, box {width, rows, 1}
  CUtensorMap tm_mat;     // 3-D map of the uint16 material map, box {width + 8, rows, 1}
  Grid g;
  FieldPtrs dst;          // destination field set (pitched)
  const Material* table;
  Sources S;
  Monitors M;
  long long t0;           // global step index of the first of the BLT steps
  float dx;
  int zlen;               // output planes per z-chunk
  int* err;               // device error word
};

struct TiledConfig {
  int blt;        // time steps per launch
  int rows;       // tile rows (warps per CTA)
  int z_chunks;   // z-chunks per tile column
  int width = 32; // cells per warp row: 32 (k_tiled.cu) or 64 (k_tiled2.cu, x-pairs)
  int min_blocks = 1;  // register cap: CTAs per SM the compiler must fit (x-pair family)
};

// Tile geometry shared by the host (grid size, tensor-map boxes) and the kernel.
__host__ __device__ constexpr int tiled_sx(int blt) { return 4 * ((32 - 2 * blt) / 4); }
__host__ __device__ constexpr int tiled_xbase(int blt) { return -4 * ((blt + 3) / 4); }
__host__ __device__ constexpr int tiled_sy(int blt, int rows) { return rows - 2 * blt; }
constexpr int kTiledStages = 3;
constexpr int kMatBoxX = 40;  // material box is widened to start on an 8-element boundary

// Two-cells-per-thread family (k_tiled2.cu): 64-wide warp rows.
__host__ __device__ constexpr int tiled2_sx(int blt) { return 4 * ((64 - 2 * blt) / 4); }
constexpr int kTiled2Stages = 2;
constexpr int kMatBoxX2 = 72;  // 64 + 4 alignment offset, rounded to a 16-byte row
bool tiled2_config_supported(const TiledConfig& c);
dim3 tiled2_grid(const TiledConfig& c, const Grid& g);
cudaError_t launch_tiled2(const TiledConfig& c, const TiledArgs& args, const Grid& g,
                          cudaStream_t st);

bool tiled_config_supported(const TiledConfig& c);
size_t tiled_smem_bytes(const TiledConfig& c);
dim3 tiled_grid(const TiledConfig& c, const Grid& g);
// args.tm_* must have been encoded with box rows == c.rows.
cudaError_t launch_tiled(const TiledConfig& c, const TiledArgs& args, const Grid& g,
                         cudaStream_t st);

// ---------------------------------------------------------------- material dedup
struct DedupResult {
  int nmat;        // distinct 12-tuples (valid when ok)
  bool ok;         // false: more than 65536 materials, or a hash collision was detected
};
// coef12: 12 device arrays of nx*ny*nz floats (unpitched).  On success writes the pitched
// material map and the table (capacity 65536 entries).
cudaError_t build_material_map(const Grid& g, const float* const* coef12, uint16_t* mat,
                               Material* table, void* scratch, size_t scratch_bytes,
                               cudaStream_t st, DedupResult* out);
size_t material_scratch_bytes();

// Copies 12 unpitched arrays into 12 pitched ones (per-cell coefficient mode).
cudaError_t pitch_coefficients(const Grid& g, const float* const* src12, float* const* dst12,
                               cudaStream_t st);

}  // namespace fdtd
