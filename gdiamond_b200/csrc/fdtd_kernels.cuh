// fdtd_kernels.cuh -- launcher interfaces between the C-ABI host code and the kernels.
#pragma once

#include <cuda.h>  // CUtensorMap (types only; the driver entry point is fetched at run time)
#include "fdtd_common.cuh"

namespace fdtd {

struct FieldPtrs {
  float* f[6];  // Ex Ey Ez Hx Hy Hz, pitched
};

// ---------------------------------------------------------------- naive kernels
// fp64: fields are double (FP64 storage), else float.
cudaError_t launch_naive_step(const Grid& g, const FieldPtrs& F, const float* const* coef,
                              const uint16_t* mat, const Material* tab, const Sources& S,
                              const Monitors& M, long long t, float dx, cudaStream_t st,
                              int* launches, bool fp64);

// Running-DFT update of every monitor from the current FP32 fields at step t (one launch).
cudaError_t launch_naive_dft(const Grid& g, const FieldPtrs& F, const Monitors& M, long long t,
                             cudaStream_t st, int* launches);

// ---------------------------------------------------------------- CPML (cpml.cu)
// One axis of the CPML profiles: tables over the n positions of the axis, at the E positions
// (integer n: b, a, 1/kappa of the E updates' differences) and at the H positions (n + 1/2).
// slot_* >= 0 inside a layer (the position's slot in the axis' psi slabs), -1 outside.
struct CpmlAxis {
  const int *slot_e, *slot_h;
  const float *be, *ae, *ike;
  const float *bh, *ah, *ikh;
  int S;  // slots per axis
};
struct CpmlDev {
  CpmlAxis ax[3];
  // psi of the E updates: exy, exz, eyz, eyx, ezx, ezy; of the H updates: hxz, hxy, hyx, hyz,
  // hzy, hzx (component, axis of the difference).  The array of axis a is a slab array: slot s
  // of axis x at s + S*(j + ny*k); of y at i + nx*(s + S*k); of z at i + nx*(j + ny*s).
  float* psi_e[6];
  float* psi_h[6];
};
// One step of E then H with CPML layers (FP32 fields, in place), then the monitors.
cudaError_t launch_cpml_step(const Grid& g, const FieldPtrs& F, const float* const* coef,
                             const uint16_t* mat, const Material* tab, const Sources& S,
                             const Monitors& M, const CpmlDev& P, long long t, float dx,
                             cudaStream_t st, int* launches);

// One grid of a batch of CPML simulations (device-resident array, built by the host per batch
// step): fields are updated in place; monitor values go to the staging rings (dft_record) and
// are folded by launch_dft_fold_cpml_batch.  t0 = the grid's step counter at the start of the
// batch step.
struct CpmlSim {
  Grid g;
  FieldPtrs F;
  const float* coef[12];  // pitched per-cell arrays, or all null with a material map
  const uint16_t* mat;
  const Material* tab;
  Sources S;
  Monitors M;
  CpmlDev P;
  long long t0;
  float dx;
};
// Step t0 + t_offset of every grid: one E launch and one H launch over all grids (blockIdx.z =
// grid * max_nz + k; cells outside a smaller grid return at once).
cudaError_t launch_cpml_batch_step(const CpmlSim* sims, int nsims, int max_nx, int max_ny,
                                   int max_nz, long long t_offset, cudaStream_t st);
// The shell companion of the tiled kernel under CPML layers (cpml.cu): one half step (E, or
// H with h_half) of step t over the cells of `blocks` (int4 {x tile of 32 cells, y tile of 4
// rows, plane k, unused}) that lie outside the box `inner` ([lo, hi) per axis x, y, z).  Reads
// the fields of step t from Fi (and, for H, the new E from Fo), writes Fo; face cells are
// copied; the half step's monitor values are staged.  Material maps only.
struct CpmlBox {
  int lo[3], hi[3];
};
cudaError_t launch_cpml_region(bool h_half, const Grid& g, const FieldPtrs& Fi,
                               const FieldPtrs& Fo, const uint16_t* mat, const Material* tab,
                               const Sources& S, const Monitors& M, const CpmlDev& P,
                               long long t, float dx, const int4* blocks, int nblocks,
                               const CpmlBox& inner, cudaStream_t st);
// Deferred DFT of a CPML batch: like launch_dft_fold_batch over CpmlSim arguments.
cudaError_t launch_dft_fold_cpml_batch(const CpmlSim* sims, int nsims, long long max_np,
                                       int max_nf, long long t_offset, int n, cudaStream_t st);

// ---------------------------------------------------------------- storage conversion
// Pitched field array of `storage` (0 FP32, 1 FP16, 2 BF16, 3 FP64) <-> pitched FP32 / FP64.
cudaError_t convert_field_to_f32(const Grid& g, const void* src, int storage, float scale,
                                 float* dst, cudaStream_t st);
cudaError_t convert_field_from_f32(const Grid& g, const float* src, int storage, float inv_scale,
                                   void* dst, cudaStream_t st);
cudaError_t convert_field_to_f64(const Grid& g, const void* src, int storage, float scale,
                                 double* dst, cudaStream_t st);

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
  float scale[6];         // 16-bit storage: value = stored * scale (powers of two)
  float inv_scale[6];
  // Uniform-material path of the x-pair kernels: when lean != 0, material lean_id has
  // Ca = Da = 1 on all three axes, Cb = lean_cb and Db = lean_db on all three (an isotropic
  // lossless medium: vacuum or a dielectric).  A warp whose cells all carry that id (and lie
  // away from sources) updates them with paired FP32 adds and the two coefficients from the
  // parameters; 1*x == x, so the results are the general path's bit for bit.
  int lean;
  int lean_id;
  float lean_cb, lean_db;
  // Failure-path test hook (fdtd_debug_fail_copy): tile (fault_bx, fault_by, fault_bz) does not
  // issue the plane copy of its z-iteration fault_it (fault_bx = -1: no tile), and every bounded
  // wait gives up after wait_limit SM clocks (0: about a second).
  long long wait_limit;
  int fault_bx, fault_by, fault_bz, fault_it;
  // Uniform blocks for the lean-only z-march: ublk[(bz * uby + by) * ubx + bx] = 1 when every
  // cell of the block of kUniX x kUniY cells by kUniZ planes holds material lean_id (null: no
  // lean-only tiles).  A tile whose staged box touches only such blocks, and holds no source,
  // runs every iteration on the lean path without loading or testing material planes.
  const uint8_t* ublk;
  int ubx, uby, ubz;
  // Launch order of the tiles (single-grid launches): CTA q of the grid (x fastest) runs tile
  // tile_order[q] (linear index bx + ntx * (by + nty * bz)); null: CTA q runs tile q.  The host
  // puts the tiles that cannot take the lean-only march (sources, mixed materials) first, so
  // the slower CTAs start in the first wave instead of lengthening the last one.
  const int* tile_order;
};

// A batch of grids for the persistent kernel: per-grid arguments (tensor maps included) in
// device memory, and the (grid, bx, by, bz) work items pulled through an atomic counter.
struct BatchArgs {
  const TiledArgs* grids;  // [2][ngrids]: the arguments of each grid for both ping-pong parities
  int ngrids;
  int flip;                // parity of this launch: grids[flip * ngrids + g] is used
  long long t_offset;      // added to each grid's t0 (steps since the batch run started)
  const int4* items;       // (grid, bx, by, bz), longest z-march first
  int nitems;
  unsigned int* counter;   // zero before the launch
};

struct TiledConfig {
  int blt;        // time steps per launch
  int rows;       // tile rows (warps per CTA)
  int z_chunks;   // z-chunks per tile column
  int width = 32; // cells per warp row: 32 (k_tiled.cu) or 64 (k_tiled2.cu, x-pairs)
  int min_blocks = 1;  // register cap: CTAs per SM the compiler must fit (x-pair family)
  int storage = 0;     // 0 FP32, 1 FP16, 2 BF16, 4 FP16 E + FP32 H (x-pair family for all but 0)
  int esz = 4;         // bytes per stored field value (the narrower of E and H)
  bool pairs32 = false;  // x-pair kernel with 32-cell rows, two per warp (width must be 32)
};

// Tile geometry shared by the host (grid size, tensor-map boxes) and the kernel.
__host__ __device__ constexpr int tiled_sx(int blt) { return 4 * ((32 - 2 * blt) / 4); }
__host__ __device__ constexpr int tiled_xbase(int blt) { return -4 * ((blt + 3) / 4); }
__host__ __device__ constexpr int tiled_sy(int blt, int rows) { return rows - 2 * blt; }
constexpr int kTiledStages = 3;
constexpr int kMatBoxX = 40;  // material box is widened to start on an 8-element boundary

// Two-cells-per-thread family (k_tiled2.cu), w = 64 or 32 cells per warp row.  Tile x starts
// need no TMA alignment: every box (fields and material ids) starts at the tile start rounded
// down to 8 elements (16 bytes of any stored type) and is kTiled2BoxPad elements wider than the
// row, so a tile writes all w - 2*blt columns of its last level whatever the storage type.  Tile
// starts stay even so that the x-pairs' vector loads and stores stay aligned.
constexpr int kTiled2BoxPad = 8;
__host__ __device__ constexpr int tiled2_sx_w(int w, int blt) { return w - 2 * blt; }
__host__ __device__ constexpr int tiled2_xbase(int blt) { return -2 * ((blt + 1) / 2); }
constexpr int kTiled2Stages = 2;  // FP32; 16-bit storage uses one more
constexpr int kMatBoxX2 = 64 + kTiled2BoxPad;  // box width of 64-cell rows (fields and ids)
bool tiled2_config_supported(const TiledConfig& c);
dim3 tiled2_grid(const TiledConfig& c, const Grid& g);
cudaError_t launch_tiled2(const TiledConfig& c, const TiledArgs& args, const Grid& g,
                          cudaStream_t st);
// Persistent batch form.
bool tiled2_batch_supported(const TiledConfig& c);
size_t tiled2_batch_smem(const TiledConfig& c);
int tiled2_batch_ctas_per_sm(const TiledConfig& c);
cudaError_t launch_tiled2_batch(const TiledConfig& c, const BatchArgs& b, int ctas,
                                cudaStream_t st);

bool tiled_config_supported(const TiledConfig& c);
size_t tiled_smem_bytes(const TiledConfig& c);
dim3 tiled_grid(const TiledConfig& c, const Grid& g);
// args.tm_* must have been encoded with box rows == c.rows.
cudaError_t launch_tiled(const TiledConfig& c, const TiledArgs& args, const Grid& g,
                         cudaStream_t st);

// ---------------------------------------------------------------- deferred DFT (dft_fold.cu)
// Adds steps [t0, t0+n) (n <= kDftSlots) staged in the monitors' rings to their FP64 sums.
cudaError_t launch_dft_fold(const Monitors& M, const Grid& g, long long t0, int n,
                            cudaStream_t st);
// The same for every grid of a batch: grids[0..ngrids) (device memory) with their monitors; the
// window of grid i starts at grids[i].t0 + t_offset.  max_np / max_nf: the largest monitor
// plane (Nx*Ny) and frequency count over the batch (grid size of the launch).
cudaError_t launch_dft_fold_batch(const TiledArgs* grids, int ngrids, long long max_np,
                                  int max_nf, long long t_offset, int n, cudaStream_t st);

// ---------------------------------------------------------------- flux monitors (flux.cu)
// The six running DFTs of a flux monitor on the E plane k ([nf][ny][nx] FP64 each): Ex, Ey of
// plane k; Hx, Hy of planes k-1 (hx0, hy0) and k (hx1, hy1), phased at (t + 1/2) dt.
struct FluxPlanes {
  const double *ex_re, *ex_im, *ey_re, *ey_im;
  const double *hx0_re, *hx0_im, *hx1_re, *hx1_im;
  const double *hy0_re, *hy0_im, *hy1_re, *hy1_im;
};
// out_dev[f] = area * sum over the plane of Re[Ex conj(Hy) - Ey conj(Hx)], H averaged over the
// two planes; np = nx * ny.
cudaError_t launch_flux_reduce(const FluxPlanes& p, long long np, int nf, double area,
                               double* out_dev, cudaStream_t st);

// ---------------------------------------------------------------- coefficient builder
struct Coef12Out {
  float* c[12];  // pitched per-cell arrays Cax..Dbz
};
// gDiamond's coefficient formula per cell from a per-cell permittivity (eps_dev: unpitched
// nx*ny*nz floats, or nullptr for vacuum) and per-axis complex stretch factors (re, im).
cudaError_t build_coefficients(const Grid& g, const float* eps_dev, const float2* sx,
                               const float2* sy, const float2* sz, float omega0, float dt,
                               float dx, const Coef12Out& out, cudaStream_t st);

// ---------------------------------------------------------------- uniform blocks
constexpr int kUniX = 8, kUniY = 8, kUniZ = 16;
// out[(bz * nby + by) * nbx + bx] = 1 when every cell of the block holds material id `id`
// (nbx = ceil(nx / kUniX) etc.; mat is the pitched material map).
cudaError_t build_uniform_blocks(const Grid& g, const uint16_t* mat, int id, uint8_t* out,
                                 cudaStream_t st);

// ---------------------------------------------------------------- material dedup
struct DedupResult {
  int nmat;        // distinct 12-tuples (valid when ok)
  bool ok;         // false: more than 65536 materials, or a hash collision was detected
  int dominant;    // id held by the most cells (valid when ok)
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
