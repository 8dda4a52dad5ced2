// fdtd_capi.cu -- host side of the C-ABI declared in include/fdtd_capi.h.
//
// Owns the device state of one grid (two pitched field sets, coefficients as a material map or
// per-cell arrays, sources, monitors, the device error word), encodes the TMA tensor maps,
// runs the autotuner and dispatches the naive or tiled kernels.  Nothing here falls back to the
// CPU: every step runs a CUDA kernel or returns an error status.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fdtd_capi.h"
#include "fdtd_kernels.cuh"

using fdtd::Grid;
using fdtd::Material;

namespace {

constexpr int kMaxMaterials = 65536;
constexpr double kPiD = 3.14159265358979323846;

enum CoefMode { kCoefNone = 0, kCoefMaterial = 1, kCoefPerCell = 2 };

struct MonitorHost {
  int comp = 0;
  long long k = 0;
  int nf = 0;
  double scale = 1.0, dt = 0.0;
  double t_offset = 0.0;  // step t is phased at (t + t_offset) * dt (1/2 for a flux monitor's H)
  std::vector<double> freqs;
  double* re = nullptr;  // [nf][ny][nx]
  double* im = nullptr;
  double2* tab = nullptr;  // [tab_cap][nf]
  long long tab_cap = 0;
  float* stage = nullptr;  // [kDftSlots][ny][nx]: values the tiled kernels stage for the fold
};

// A flux monitor: six running DFTs (see flux.cu) and where its result goes.
constexpr int kMaxFlux = fdtd::kMaxMonitors / 6;
struct FluxHost {
  long long k = 0;
  int nf = 0;
  int mon[6] = {};  // Ex(k), Ey(k), Hx(k-1), Hx(k), Hy(k-1), Hy(k)
  double* out = nullptr;  // [nf] device result of the last reduction
};

std::string g_create_error;

PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Process-wide autotuning cache keyed by grid shape.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, long long>, fdtd::TiledConfig> g_tune_cache;

}  // namespace

struct fdtd_handle {
  fdtd_desc desc{};
  Grid g{};
  size_t cells = 0;  // pitched elements per field array
  cudaStream_t stream = nullptr;
  float* F[2][6] = {};
  int cur = 0;
  int coef_mode = kCoefNone;
  float* coef[12] = {};  // pitched per-cell arrays (staging / per-cell mode)
  uint16_t* mat = nullptr;
  Material* table = nullptr;
  int nmat = 0;
  void* scratch = nullptr;
  fdtd::SourceDev src[fdtd::kMaxSources] = {};
  int nsrc = 0;
  float* d_wave = nullptr;
  long long tw = 0;
  MonitorHost mon[fdtd::kMaxMonitors];
  int nmon = 0;
  FluxHost flux[kMaxFlux];
  int nflux = 0;
  long long t = 0;
  int* d_err = nullptr;
  fdtd::TiledConfig cfg{0, 0, 0};
  bool cfg_ready = false;
  CUtensorMap maps[2][6];
  CUtensorMap mat_map;
  int maps_key = 0;  // (field box width * 1000 + id box width) * 1000 + rows of the encoded boxes
  int last_kernel = 0, last_launches = 0;
  int last_folds = 0;  // DFT fold launches of the last fdtd_step
  int storage = FDTD_STORE_F32;
  int esz = 4;     // bytes per stored field value (F16E: the FP16 E components')
  int nsets = 2;   // field sets (1 for FP64: the naive kernel updates in place)
  float scale[6] = {1, 1, 1, 1, 1, 1}, inv_scale[6] = {1, 1, 1, 1, 1, 1};
  // Uniform-material fast path of the x-pair kernels (TiledArgs::lean): the dominant material
  // qualifies when Ca = Da = 1 and Cb, Db are the same on all three axes.
  // fdtd_debug_fail_copy: applied to the next tiled launch only
  int fault_tile[3] = {-1, -1, -1};
  int fault_it = 0;
  long long fault_wait = 0;
  // CPML layers (fdtd_set_cpml): per-axis tables in one device block, psi slab arrays
  bool cpml_on = false;
  fdtd_cpml_desc cpml{};
  void* cpml_tab = nullptr;
  float* cpml_psi[12] = {};
  std::vector<int> cpml_slot[3][2];      // host copies of the slot tables (E, H positions)
  std::vector<float> cpml_prof[3][2][3]; // host copies of b, a, 1/kappa
  fdtd::CpmlDev cpml_dev{};
  // Shell companion of the tiled kernel (cpml_companion): cpml_inner = per axis the [lo, hi)
  // range of positions whose E and H updates involve no layer, cpml_lo / cpml_hi = the axis has
  // a layer on that side; a third FP32 field set for the companion's intermediate steps; block
  // lists of the regions it updates, per depth r.
  int cpml_inner[3][2] = {};
  bool cpml_lo[3] = {}, cpml_hi[3] = {};
  float* cpml_scratch[6] = {};
  std::map<int, std::pair<int4*, int>> cpml_blocks;
  uint8_t* ublk = nullptr;  // uniform-block map of the lean material (fdtd::build_uniform_blocks)
  int ub[3] = {0, 0, 0};
  std::vector<uint8_t> ublk_host;  // its host copy (tile launch order)
  int* d_order = nullptr;          // tile launch order of the current configuration
  size_t order_cap = 0;
  std::vector<int> order_host;
  long long order_key = -1;
  int version = 0;                 // bumped when coefficients or sources change
  bool lean_ok = false;
  bool lean_enable = true;  // fdtd_set_fast_path
  int lean_id = 0;
  float lean_cb = 0.0f, lean_db = 0.0f;
  float* f32_stage = nullptr;   // pitched FP32 staging for field transfers of other storages
  double* f64_stage = nullptr;  // pitched FP64 staging for fdtd_get_field_f64
  std::string err;
};

namespace {

// Storage format of component c (0..5 = Ex Ey Ez Hx Hy Hz): F16E keeps E in FP16 and H in FP32.
int comp_storage(const fdtd_handle* h, int c) {
  if (h->storage == FDTD_STORE_F16E) return c < 3 ? FDTD_STORE_F16 : FDTD_STORE_F32;
  return h->storage;
}

int comp_esz(const fdtd_handle* h, int c) {
  const int s = comp_storage(h, c);
  return s == FDTD_STORE_F32 ? 4 : (s == FDTD_STORE_F64 ? 8 : 2);
}

fdtd_status fail(fdtd_handle* h, fdtd_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (h)
    h->err = buf;
  else
    g_create_error = buf;
  return s;
}

#define CUDA_TRY(h, call)                                                                    \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail((h), e_ == cudaErrorMemoryAllocation ? FDTD_ERR_OOM : FDTD_ERR_CUDA,       \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int now = -1;
    cudaGetDevice(&now);
    if (prev >= 0 && now != prev) cudaSetDevice(prev);
  }
};

cudaStream_t pick_stream(fdtd_handle* h, void* s) {
  return s ? static_cast<cudaStream_t>(s) : h->stream;
}

fdtd_status encode_map(fdtd_handle* h, CUtensorMap* m, void* base, CUtensorMapDataType dt,
                       int esz, int box_x, int box_y) {
  auto enc = get_encode_fn();
  if (!enc) return fail(h, FDTD_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  const cuuint64_t dims[3] = {(cuuint64_t)h->g.nx, (cuuint64_t)h->g.ny, (cuuint64_t)h->g.nz};
  const cuuint64_t strides[2] = {(cuuint64_t)h->g.pitch * esz, (cuuint64_t)h->g.plane * esz};
  const cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(m, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, FDTD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return FDTD_OK;
}

// Tensor maps of both field sets and of the material map for the boxes of kernel configuration
// c: {row width + 8, rows, 1} for fields and ids of the x-pair family (boxes start at the tile
// start rounded down to 8 elements); {32, rows, 1} for fields and {40, rows, 1} for ids of the
// one-cell 32-wide kernel (its tile starts are 16-byte aligned).
fdtd_status ensure_maps(fdtd_handle* h, const fdtd::TiledConfig& c) {
  const bool pairs = c.width == 64 || c.pairs32;
  const int width = pairs ? c.width + fdtd::kTiled2BoxPad : c.width;
  const int mat_box = pairs ? c.width + fdtd::kTiled2BoxPad : fdtd::kMatBoxX;
  const int rows = c.rows;
  const int key = (width * 1000 + mat_box) * 1000 + rows;
  if (h->maps_key == key) return FDTD_OK;
  for (int s = 0; s < 2; ++s)
    for (int c = 0; c < 6; ++c) {
      const int cs = comp_storage(h, c);
      const CUtensorMapDataType dt = cs == FDTD_STORE_F16    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                     : cs == FDTD_STORE_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                             : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
      fdtd_status st = encode_map(h, &h->maps[s][c], h->F[s][c], dt, comp_esz(h, c), width, rows);
      if (st != FDTD_OK) return st;
    }
  fdtd_status st = encode_map(h, &h->mat_map, h->mat, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2,
                              mat_box, rows);
  if (st != FDTD_OK) return st;
  h->maps_key = key;
  return FDTD_OK;
}

cudaError_t launch_any(const fdtd::TiledConfig& c, const fdtd::TiledArgs& a, const Grid& g,
                       cudaStream_t st) {
  return (c.width == 64 || c.pairs32) ? fdtd::launch_tiled2(c, a, g, st)
                                       : fdtd::launch_tiled(c, a, g, st);
}

bool config_supported(const fdtd::TiledConfig& c) {
  return (c.width == 64 || c.pairs32) ? fdtd::tiled2_config_supported(c)
                                       : fdtd::tiled_config_supported(c);
}

fdtd::Sources make_sources(const fdtd_handle* h) {
  fdtd::Sources S{};
  S.n = h->nsrc;
  for (int n = 0; n < h->nsrc; ++n) S.s[n] = h->src[n];
  S.wave = h->d_wave;
  S.tw = h->tw;
  return S;
}

fdtd::Monitors make_monitors(const fdtd_handle* h) {
  fdtd::Monitors M{};
  M.n = h->nmon;
  for (int m = 0; m < h->nmon; ++m) {
    const MonitorHost& mh = h->mon[m];
    M.m[m].comp = mh.comp;
    M.m[m].k = (int)mh.k;
    M.m[m].nf = mh.nf;
    M.m[m].scale = mh.scale;
    M.m[m].tab = mh.tab;
    M.m[m].re = mh.re;
    M.m[m].im = mh.im;
    M.m[m].stage = mh.stage;
  }
  return M;
}

// The cos/sin table must cover steps [0, upto).
fdtd_status ensure_tables(fdtd_handle* h, long long upto) {
  for (int m = 0; m < h->nmon; ++m) {
    MonitorHost& mh = h->mon[m];
    if (mh.tab_cap >= upto) continue;
    long long cap = std::max<long long>(upto, std::max<long long>(1024, mh.tab_cap * 2));
    std::vector<double2> host((size_t)cap * mh.nf);
    for (long long t = 0; t < cap; ++t) {
      const double tt = ((double)t + mh.t_offset) * mh.dt;
      for (int f = 0; f < mh.nf; ++f) {
        const double w = 2.0 * kPiD * mh.freqs[f];
        const double ph = w * tt;
        host[(size_t)t * mh.nf + f] = make_double2(std::cos(ph), std::sin(ph));
      }
    }
    double2* d = nullptr;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    CUDA_TRY(h, cudaMalloc(&d, host.size() * sizeof(double2)));
    CUDA_TRY(h, cudaMemcpy(d, host.data(), host.size() * sizeof(double2), cudaMemcpyHostToDevice));
    if (mh.tab) cudaFree(mh.tab);
    mh.tab = d;
    mh.tab_cap = cap;
  }
  return FDTD_OK;
}

fdtd::TiledArgs make_tiled_args(fdtd_handle* h, const fdtd::TiledConfig& c, long long t0,
                                bool with_io, int src_set = -1) {
  const int src = src_set < 0 ? h->cur : src_set;
  fdtd::TiledArgs a;
  memset(&a, 0, sizeof(a));
  for (int k = 0; k < 6; ++k) a.tm_src[k] = h->maps[src][k];
  a.tm_mat = h->mat_map;
  a.g = h->g;
  for (int k = 0; k < 6; ++k) a.dst.f[k] = h->F[src ^ 1][k];
  a.table = h->table;
  if (with_io) {
    a.S = make_sources(h);
    a.M = make_monitors(h);
  }
  a.t0 = t0;
  a.dx = h->desc.dx;
  a.zlen = (h->g.nz + c.z_chunks - 1) / c.z_chunks;
  a.err = h->d_err;
  for (int k = 0; k < 6; ++k) {
    a.scale[k] = h->scale[k];
    a.inv_scale[k] = h->inv_scale[k];
  }
  // the failure-path test hook applies to stepping launches only (not to autotuning)
  const bool hook = with_io && h->fault_tile[0] >= 0;
  a.fault_bx = hook ? h->fault_tile[0] : -1;
  a.fault_by = hook ? h->fault_tile[1] : -1;
  a.fault_bz = hook ? h->fault_tile[2] : -1;
  a.fault_it = h->fault_it;
  a.wait_limit = hook ? h->fault_wait : 0;
  a.lean = h->lean_ok && h->lean_enable ? 1 : 0;
  a.ublk = a.lean ? h->ublk : nullptr;
  a.ubx = h->ub[0];
  a.uby = h->ub[1];
  a.ubz = h->ub[2];
  a.lean_id = h->lean_id;
  a.lean_cb = h->lean_cb;
  a.lean_db = h->lean_db;
  return a;
}

// Candidate tiled configurations for the autotuner.
std::vector<fdtd::TiledConfig> candidates(const fdtd_handle* h) {
  std::vector<fdtd::TiledConfig> out;
  std::vector<int> blts = {1, 2, 3, 4, 5, 6}, rows_l = {8, 16, 20, 24, 32, 48};
  std::vector<int> zc = {1, 2, 4, 8};
  // kernel families: 0 one cell per thread (32-wide rows), 1 x-pairs in 64-wide rows,
  // 2 x-pairs in 32-wide rows (two per warp)
  std::vector<int> fams = {0, 1, 2};
  const bool half = h->esz == 2;
  if (half) {
    fams = {1, 2};
    rows_l = {8, 16, 24, 32, 48};
  }
  if (h->desc.blt > 0) blts = {h->desc.blt};
  if (h->desc.tile_rows > 0) rows_l = {h->desc.tile_rows};
  if (h->desc.z_chunks > 0) zc = {h->desc.z_chunks};
  if (h->desc.kernel == FDTD_KERNEL_TILED_W32) fams = {0};
  if (h->desc.kernel == FDTD_KERNEL_TILED_W64) fams = {1};
  if (h->desc.kernel == FDTD_KERNEL_TILED_W32P) fams = {2};
  const bool forced_z = h->desc.z_chunks > 0;
  for (int fam : fams)
    for (int rows : rows_l)
      for (int b : blts)
        for (int z : zc)
          for (int mb : {1, 2, 4}) {
            if (h->desc.min_blocks > 0 && mb != h->desc.min_blocks) continue;
            fdtd::TiledConfig c{b, rows, z, fam == 1 ? 64 : 32, mb, h->storage, h->esz};
            c.pairs32 = fam == 2;
            if (!config_supported(c)) continue;
            // A chunk shorter than its 2*BLT warm-up is only worth it when asked for.
            if (!forced_z && (h->g.nz + z - 1) / z < 2 * b) continue;
            out.push_back(c);
          }
  return out;
}

// Times every candidate on the current field set (source set -> scratch destination; sources
// and monitors off, so the simulation state is not changed) and keeps the fastest per step.
fdtd_status autotune(fdtd_handle* h, cudaStream_t st) {
  const auto key = std::make_tuple(h->g.nx, h->g.ny, h->g.nz,
                                   (h->cpml_on ? 10000000000LL : 0LL) +
                                       h->storage * 1000000000LL + h->desc.min_blocks * 100000000LL +
                                       h->desc.kernel * 1000000 + h->desc.blt * 10000 +
                                       h->desc.tile_rows * 100 + h->desc.z_chunks);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      h->cfg = it->second;
      h->cfg_ready = true;
      return FDTD_OK;
    }
  }
  std::vector<fdtd::TiledConfig> cands = candidates(h);
  if (h->cpml_on) {
    // With CPML layers the shell companion recomputes regions about 3 BLT cells deeper than
    // the layers after every launch, so its cost grows with BLT while the timing below sees the
    // tiled kernel alone: keep BLT <= 2 (by estimate the best total at 256^3 with 10-cell
    // layers; BLT 6 measured slower overall).
    std::vector<fdtd::TiledConfig> keep;
    for (const auto& c : cands)
      if (c.blt <= 2) keep.push_back(c);
    if (!keep.empty()) cands.swap(keep);
  }
  if (cands.empty()) return fail(h, FDTD_ERR_UNSUPPORTED, "no tiled configuration fits this grid");
  if (cands.size() == 1) {
    h->cfg = cands[0];
    h->cfg_ready = true;
    return FDTD_OK;
  }
  cudaEvent_t e0, e1;
  CUDA_TRY(h, cudaEventCreate(&e0));
  CUDA_TRY(h, cudaEventCreate(&e1));
  // Time one candidate: one untimed launch, then `reps` timed launches; ms per step.
  auto time_cfg = [&](const fdtd::TiledConfig& c, int reps, float* per_step) -> fdtd_status {
    fdtd_status s = ensure_maps(h, c);
    if (s != FDTD_OK) return s;
    const fdtd::TiledArgs a = make_tiled_args(h, c, 0, false);
    CUDA_TRY(h, launch_any(c, a, h->g, st));
    CUDA_TRY(h, cudaEventRecord(e0, st));
    for (int r = 0; r < reps; ++r) CUDA_TRY(h, launch_any(c, a, h->g, st));
    CUDA_TRY(h, cudaEventRecord(e1, st));
    CUDA_TRY(h, cudaEventSynchronize(e1));
    float ms = 0;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, e0, e1));
    *per_step = ms / (reps * c.blt);
    return FDTD_OK;
  };
  // Bring the SM clocks up before anything is compared (an idle GPU starts slow and would
  // penalise whichever candidates run first): launch the first candidate for ~50 ms.
  {
    float warm = 0, spent = 0;
    for (int r = 0; r < 64 && spent < 50.0f; ++r) {
      fdtd_status s = time_cfg(cands[0], 2, &warm);
      if (s != FDTD_OK) return s;
      spent += warm * 2 * cands[0].blt;
    }
  }
  std::vector<std::pair<float, size_t>> scored;
  for (size_t i = 0; i < cands.size(); ++i) {
    float per_step = 0;
    fdtd_status s = time_cfg(cands[i], 3, &per_step);
    if (s != FDTD_OK) return s;
    scored.emplace_back(per_step, i);
  }
  // Re-time the best few with more launches and keep the fastest.
  std::sort(scored.begin(), scored.end());
  float best = 1e30f;
  fdtd::TiledConfig best_c = cands[scored[0].second];
  for (size_t r = 0; r < std::min<size_t>(4, scored.size()); ++r) {
    const fdtd::TiledConfig& c = cands[scored[r].second];
    float per_step = 0;
    fdtd_status s = time_cfg(c, 8, &per_step);
    if (s != FDTD_OK) return s;
    if (per_step < best) {
      best = per_step;
      best_c = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->cfg = best_c;
  h->cfg_ready = true;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = best_c;
  return FDTD_OK;
}

fdtd_status check_device_error(fdtd_handle* h) {
  int e = 0;
  CUDA_TRY(h, cudaMemcpy(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e != fdtd::kErrNone) {
    cudaMemset(h->d_err, 0, sizeof(int));
    if (e & fdtd::kErrTimeout)
      return fail(h, FDTD_ERR_DEVICE_TIMEOUT,
                  "a device-side bounded wait expired (error word %d); results are invalid", e);
    return fail(h, FDTD_ERR_NUMERIC,
                "a field value stored in 16 bits overflowed to +-inf or became NaN (error word "
                "%d): the storage scale of that component is too small for the field; results "
                "are invalid", e);
  }
  return FDTD_OK;
}

// Releases the shell companion's field set and block lists (rebuilt on demand).
void cpml_release_companion(fdtd_handle* h) {
  for (int c = 0; c < 6; ++c) {
    cudaFree(h->cpml_scratch[c]);
    h->cpml_scratch[c] = nullptr;
  }
  for (auto& kv : h->cpml_blocks) cudaFree(kv.second.first);
  h->cpml_blocks.clear();
}

void free_all(fdtd_handle* h) {
  for (int s = 0; s < 2; ++s)
    for (int c = 0; c < 6; ++c) cudaFree(h->F[s][c]);
  for (int a = 0; a < 12; ++a) cudaFree(h->coef[a]);
  cudaFree(h->mat);
  cudaFree(h->table);
  cudaFree(h->scratch);
  cudaFree(h->d_wave);
  cudaFree(h->d_err);
  cudaFree(h->ublk);
  cudaFree(h->d_order);
  cudaFree(h->cpml_tab);
  for (int q = 0; q < 12; ++q) cudaFree(h->cpml_psi[q]);
  cpml_release_companion(h);
  cudaFree(h->f32_stage);
  cudaFree(h->f64_stage);
  for (int m = 0; m < h->nmon; ++m) {
    cudaFree(h->mon[m].re);
    cudaFree(h->mon[m].im);
    cudaFree(h->mon[m].tab);
    cudaFree(h->mon[m].stage);
  }
  for (int f = 0; f < h->nflux; ++f) cudaFree(h->flux[f].out);
  if (h->stream) cudaStreamDestroy(h->stream);
}

fdtd_status alloc_coef_staging(fdtd_handle* h) {
  const size_t bytes = h->cells * sizeof(float);
  for (int a = 0; a < 12; ++a)
    if (!h->coef[a]) {
      CUDA_TRY(h, cudaMalloc(&h->coef[a], bytes));
      CUDA_TRY(h, cudaMemsetAsync(h->coef[a], 0, bytes, h->stream));
    }
  return FDTD_OK;
}

fdtd_status compress_coefficients(fdtd_handle* h);

fdtd_status upload_coefficients(fdtd_handle* h, const float* const* src, cudaMemcpyKind kind) {
  for (int a = 0; a < 12; ++a)
    if (!src[a]) return fail(h, FDTD_ERR_INVALID_ARG, "coefficient array %d is NULL", a);
  fdtd_status s = alloc_coef_staging(h);
  if (s != FDTD_OK) return s;
  for (int a = 0; a < 12; ++a)
    CUDA_TRY(h, cudaMemcpy2DAsync(h->coef[a], (size_t)h->g.pitch * 4, src[a], (size_t)h->g.nx * 4,
                                  (size_t)h->g.nx * 4, (size_t)h->g.ny * h->g.nz, kind, h->stream));
  return compress_coefficients(h);
}

// One axis of graded stretch factors (gDiamond/utils.h:585-619), evaluated on the host with the
// C library's pow exactly as the reference does.
std::vector<float2> stretch_profile(int n, int t_pml, float sigma_max, float omega0) {
  std::vector<float2> out(n);
  for (int i = 0; i < n; ++i) {
    float dist = 0;
    if (i < t_pml) dist = (float)(1.0 - (double)((float)i / (float)t_pml));
    if (i + t_pml >= n) dist = (float)(1.0 - (double)((float)(n - i - 1) / (float)t_pml));
    const double d3 = std::pow((double)dist, 3.0);
    out[i] = make_float2((float)(1.0 + (double)2.0f * d3),
                         (float)((double)sigma_max * d3 / (double)(omega0 * 1.0f)));
  }
  return out;
}

fdtd_status compress_coefficients(fdtd_handle* h) {
  if (!h->mat) {
    CUDA_TRY(h, cudaMalloc(&h->mat, h->cells * sizeof(uint16_t)));
    CUDA_TRY(h, cudaMemsetAsync(h->mat, 0, h->cells * sizeof(uint16_t), h->stream));
    CUDA_TRY(h, cudaMalloc(&h->table, kMaxMaterials * sizeof(Material)));
    CUDA_TRY(h, cudaMalloc(&h->scratch, fdtd::material_scratch_bytes()));
  }
  fdtd::DedupResult r{};
  CUDA_TRY(h, fdtd::build_material_map(h->g, h->coef, h->mat, h->table, h->scratch,
                                       fdtd::material_scratch_bytes(), h->stream, &r));
  h->lean_ok = false;
  h->ublk_host.clear();
  h->version += 1;
  if (r.ok) {
    h->coef_mode = kCoefMaterial;
    h->nmat = r.nmat;
    // Does the material held by the most cells qualify for the fast path?
    Material m;
    CUDA_TRY(h, cudaMemcpy(&m, h->table + r.dominant, sizeof(m), cudaMemcpyDeviceToHost));
    // {Cax, Cbx, Cay, Cby}, {Caz, Cbz, Dax, Dbx}, {Day, Dby, Daz, Dbz}
    const bool unit_a = m.a.x == 1.0f && m.a.z == 1.0f && m.b.x == 1.0f && m.b.z == 1.0f &&
                        m.c.x == 1.0f && m.c.z == 1.0f;
    const bool iso_b = m.a.y == m.a.w && m.a.y == m.b.y && m.b.w == m.c.y && m.b.w == m.c.w;
    h->lean_ok = unit_a && iso_b;
    h->lean_id = r.dominant;
    h->lean_cb = m.a.y;
    h->lean_db = m.b.w;
    if (h->lean_ok) {  // which blocks hold the lean material only (lean-only tiles)
      h->ub[0] = (h->g.nx + fdtd::kUniX - 1) / fdtd::kUniX;
      h->ub[1] = (h->g.ny + fdtd::kUniY - 1) / fdtd::kUniY;
      h->ub[2] = (h->g.nz + fdtd::kUniZ - 1) / fdtd::kUniZ;
      if (!h->ublk)
        CUDA_TRY(h, cudaMalloc(&h->ublk, (size_t)h->ub[0] * h->ub[1] * h->ub[2]));
      CUDA_TRY(h, fdtd::build_uniform_blocks(h->g, h->mat, r.dominant, h->ublk, h->stream));
      h->ublk_host.resize((size_t)h->ub[0] * h->ub[1] * h->ub[2]);
      CUDA_TRY(h, cudaMemcpyAsync(h->ublk_host.data(), h->ublk, h->ublk_host.size(),
                                  cudaMemcpyDeviceToHost, h->stream));
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
  } else {
    h->coef_mode = kCoefPerCell;
    h->nmat = 0;
  }
  return FDTD_OK;
}

}  // namespace

// ============================================================================== C-ABI

namespace {

// Adds one running-DFT monitor (fdtd_add_dft_monitor; a flux monitor adds six).
fdtd_status add_monitor(fdtd_handle* h, int32_t component, int64_t k, const double* freqs,
                        int32_t nf, double scale, double dt, double t_offset,
                        int32_t* monitor_id) {
  if (!h) return FDTD_ERR_INVALID_ARG;
  if (h->nmon >= fdtd::kMaxMonitors)
    return fail(h, FDTD_ERR_UNSUPPORTED, "at most %d monitors", fdtd::kMaxMonitors);
  if (component < 0 || component > 5) return fail(h, FDTD_ERR_INVALID_ARG, "bad component");
  if (k < 0 || k >= h->g.nz) return fail(h, FDTD_ERR_INVALID_ARG, "monitor plane outside grid");
  if (!freqs || nf < 1 || nf > fdtd::kMaxFreqs)
    return fail(h, FDTD_ERR_INVALID_ARG, "nf must be 1..%d", fdtd::kMaxFreqs);
  DeviceGuard dg(h->desc.device);
  MonitorHost& m = h->mon[h->nmon];
  m = MonitorHost();
  m.comp = component;
  m.k = k;
  m.nf = nf;
  m.scale = scale;
  m.dt = dt;
  m.t_offset = t_offset;
  m.freqs.assign(freqs, freqs + nf);
  const size_t bytes = (size_t)nf * h->g.nx * h->g.ny * sizeof(double);
  const size_t stage_bytes = (size_t)fdtd::kDftSlots * h->g.nx * h->g.ny * sizeof(float);
  cudaError_t e = cudaMalloc(&m.re, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&m.im, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&m.stage, stage_bytes);
  if (e == cudaSuccess) e = cudaMemsetAsync(m.re, 0, bytes, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m.im, 0, bytes, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m.stage, 0, stage_bytes, h->stream);
  if (e != cudaSuccess) {  // the monitor is not added: release what it had
    cudaFree(m.re);
    cudaFree(m.im);
    cudaFree(m.stage);
    m = MonitorHost();
    return fail(h, e == cudaErrorMemoryAllocation ? FDTD_ERR_OOM : FDTD_ERR_CUDA,
                "monitor allocation failed: %s", cudaGetErrorString(e));
  }
  if (monitor_id) *monitor_id = h->nmon;
  h->nmon += 1;
  return FDTD_OK;
}

// Axis of the difference behind psi q (0..5: E exy exz eyz eyx ezx ezy; 6..11: H hxz hxy hyx
// hyz hzy hzx).
int cpml_psi_axis(int q) {
  static const int ax[12] = {1, 2, 2, 0, 0, 1, 2, 1, 0, 2, 1, 0};
  return ax[q];
}

size_t cpml_psi_bytes(const fdtd_handle* h, int q) {
  const int a = cpml_psi_axis(q);
  const size_t n[3] = {(size_t)h->g.nx, (size_t)h->g.ny, (size_t)h->g.nz};
  const size_t S = 2 * (size_t)h->cpml.thickness + 1;
  return S * n[(a + 1) % 3] * n[(a + 2) % 3] * sizeof(float);
}

// Profile of one axis at E positions (half = false: x = n) or H positions (x = n + 1/2).
void cpml_profile(const fdtd_cpml_desc& d, int n, bool lo, bool hi, double dx, bool half,
                  std::vector<int>* slot, std::vector<float>* b, std::vector<float>* a,
                  std::vector<float>* ik) {
  const int L = d.thickness;
  const double m = d.order;
  const double sigma_max = -(m + 1.0) * std::log((double)d.reflection) / (2.0 * L * dx);
  slot->assign(n, -1);
  b->assign(n, 1.0f);
  a->assign(n, 0.0f);
  ik->assign(n, 1.0f);
  for (int p = 0; p < n; ++p) {
    const double x = p + (half ? 0.5 : 0.0);
    double rho = 0.0;
    int s = -1;
    if (lo && x < L) {
      rho = (L - x) / L;
      s = p;
    }
    if (hi && x > n - 1 - L) {
      rho = (x - (n - 1 - L)) / L;
      s = L + (p - (n - 1 - L));
    }
    if (!(rho > 0.0)) continue;
    rho = std::min(rho, 1.0);
    const double rm = std::pow(rho, m);
    const double sigma = sigma_max * rm;
    const double kappa = 1.0 + ((double)d.kappa_max - 1.0) * rm;
    const double alpha = (double)d.alpha_max * (1.0 - rho);
    const double bb = std::exp(-(sigma / kappa + alpha) * (double)d.dt);
    const double den = sigma * kappa + kappa * kappa * alpha;
    (*slot)[p] = s;
    (*b)[p] = (float)bb;
    (*a)[p] = den > 0.0 ? (float)(sigma / den * (bb - 1.0)) : 0.0f;
    (*ik)[p] = (float)(1.0 / kappa);
  }
}

// Launch order of the tiles of x-pair configuration c (TiledArgs::tile_order): the tiles that
// will run the mixed z-march (a source or a non-uniform block in their staged box; the device
// test is tile_uniform in k_tiled2.cuh) first, then the lean-only ones.  Null when there is
// nothing to reorder.
// Whether tile (bx, by, bz) of h under config c (z-chunks of zlen planes) can run the lean-only
// z-march: no source in or next to its staged box and every cell of the box in a uniform block
// of the lean material -- the device's tile_uniform, decided on the host for launch order.
bool tile_is_lean(const fdtd_handle* h, const fdtd::TiledConfig& c, int bx, int by, int bz,
                  int zlen) {
  if (!(c.width == 64 || c.pairs32) || h->ublk_host.empty() || !h->lean_enable) return false;
  const Grid& g = h->g;
  const int W = c.pairs32 ? 32 : c.width, B = c.blt;
  const int SX = fdtd::tiled2_sx_w(W, B), SY = fdtd::tiled_sy(B, c.rows);
  const int XB = fdtd::tiled2_xbase(B), WB = W + fdtd::kTiled2BoxPad;
  const int z0 = bz * zlen, X8 = (bx * SX + XB) & ~7, Y = by * SY - B;
  const int za = std::max(0, z0 - B), zb = std::min(g.nz, std::min(g.nz, z0 + zlen) + B);
  const int xa = std::max(0, X8), xb = std::min(g.nx, X8 + WB);
  const int ya = std::max(0, Y), yb = std::min(g.ny, Y + c.rows);
  for (int n = 0; n < h->nsrc; ++n) {
    const fdtd::SourceDev& sd = h->src[n];
    const bool in_z = sd.k >= za - 1 && sd.k <= zb;
    if (in_z && (sd.kind != 0 || (sd.i >= xa && sd.i < xb && sd.j >= ya && sd.j < yb)))
      return false;
  }
  if (!(xa < xb && ya < yb)) return false;
  for (int kz = za / fdtd::kUniZ; kz <= (zb - 1) / fdtd::kUniZ; ++kz)
    for (int ky = ya / fdtd::kUniY; ky <= (yb - 1) / fdtd::kUniY; ++ky)
      for (int kx = xa / fdtd::kUniX; kx <= (xb - 1) / fdtd::kUniX; ++kx)
        if (h->ublk_host[((size_t)kz * h->ub[1] + ky) * h->ub[0] + kx] == 0) return false;
  return true;
}

const int* tile_order(fdtd_handle* h, const fdtd::TiledConfig& c) {
  if (!(c.width == 64 || c.pairs32) || h->ublk_host.empty() || !h->lean_enable) return nullptr;
  const long long key = ((((long long)h->version * 8 + c.blt) * 64 + c.rows) * 64 + c.z_chunks) *
                            2 + (c.pairs32 ? 1 : 0) + 4LL * c.width;
  if (key == h->order_key) return h->d_order;
  const Grid& g = h->g;
  const int zlen = (g.nz + c.z_chunks - 1) / c.z_chunks;
  const dim3 gd = fdtd::tiled2_grid(c, g);
  const int ntile = (int)(gd.x * gd.y * gd.z);
  std::vector<int> mixed, lean;
  for (int q = 0; q < ntile; ++q) {
    const int bx = q % gd.x, by = (q / gd.x) % gd.y, bz = q / (gd.x * gd.y);
    (tile_is_lean(h, c, bx, by, bz, zlen) ? lean : mixed).push_back(q);
  }
  h->order_key = key;
  if (mixed.empty() || lean.empty()) {
    h->order_host.clear();
    return nullptr;
  }
  h->order_host = mixed;
  h->order_host.insert(h->order_host.end(), lean.begin(), lean.end());
  if (h->order_cap < (size_t)ntile) {
    cudaFree(h->d_order);
    h->d_order = nullptr;
    h->order_cap = 0;
    if (cudaMalloc(&h->d_order, (size_t)ntile * sizeof(int)) != cudaSuccess) return nullptr;
    h->order_cap = ntile;
  }
  if (cudaMemcpy(h->d_order, h->order_host.data(), (size_t)ntile * sizeof(int),
                 cudaMemcpyHostToDevice) != cudaSuccess)
    return nullptr;
  return h->d_order;
}

// Removes the monitors from index `first` on (a flux monitor whose later parts failed).
void drop_monitors(fdtd_handle* h, int first) {
  for (int m = first; m < h->nmon; ++m) {
    cudaFree(h->mon[m].re);
    cudaFree(h->mon[m].im);
    cudaFree(h->mon[m].tab);
    cudaFree(h->mon[m].stage);
    h->mon[m] = MonitorHost();
  }
  h->nmon = first;
}

// ------------------------------------------------------------ CPML shell companion
// With CPML layers the tiled kernel advances the whole grid by k steps with the plain update;
// its results are right wherever the layers cannot reach within k steps.  One step moves
// information by at most one cell along each axis (E reads H at i and i-1, H reads E at i and
// i+1), so after k steps the tiled kernel is wrong only within k cells of the shell (the cells
// whose own update involves a layer).  The companion recomputes those cells: from the fields
// of the launch's start (set A) it runs the k steps with the CPML update over regions that
// shrink towards the shell, the intermediate steps in a third field set, the last into the
// tiled kernel's output (set B).  W_r = the cells within r of the shell = outside the inner
// box shrunk by r on every side with a layer.  Step j updates E on W_{e_j}, H on W_{e_j - 1},
// e_j = 3k - 2(j - 1): each half step needs the previous one on a region one cell deeper, and
// the last step covers W_{k+2} (E) and W_{k+1} (H), beyond what the tiled kernel got wrong.
// psi is updated by the companion alone, once per cell and step; monitor values of the
// recomputed cells are staged again over the tiled kernel's.

// The inner box shrunk by r cells on every side that has a layer.
fdtd::CpmlBox cpml_inner_box(const fdtd_handle* h, int r) {
  const int n[3] = {h->g.nx, h->g.ny, h->g.nz};
  fdtd::CpmlBox b;
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = h->cpml_lo[a] ? h->cpml_inner[a][0] + r : 0;
    b.hi[a] = h->cpml_hi[a] ? h->cpml_inner[a][1] - r : n[a];
    if (b.hi[a] < b.lo[a]) b.hi[a] = b.lo[a];
  }
  return b;
}

// The companion pays off when the inner box of its deepest region still holds most cells.
bool cpml_companion_fits(const fdtd_handle* h, int k) {
  const fdtd::CpmlBox b = cpml_inner_box(h, 3 * k);
  double inner = 1.0;
  for (int a = 0; a < 3; ++a) inner *= (double)(b.hi[a] - b.lo[a]);
  return inner >= 0.4 * (double)h->g.nx * h->g.ny * h->g.nz;
}

// Device list of the 32 x 4-cell blocks (x tile, y tile, plane) that hold cells of W_r.
fdtd_status cpml_region_blocks(fdtd_handle* h, int r, std::pair<int4*, int>* out) {
  auto it = h->cpml_blocks.find(r);
  if (it != h->cpml_blocks.end()) {
    *out = it->second;
    return FDTD_OK;
  }
  const fdtd::CpmlBox b = cpml_inner_box(h, r);
  const int ntx = (h->g.nx + 31) / 32, nty = (h->g.ny + 3) / 4;
  std::vector<int4> v;
  for (int k = 0; k < h->g.nz; ++k) {
    const bool zin = k >= b.lo[2] && k < b.hi[2];
    for (int ty = 0; ty < nty; ++ty)
      for (int tx = 0; tx < ntx; ++tx) {
        const bool inside = zin && 32 * tx >= b.lo[0] && 32 * tx + 32 <= b.hi[0] &&
                            4 * ty >= b.lo[1] && 4 * ty + 4 <= b.hi[1];
        if (!inside) v.push_back(make_int4(tx, ty, k, 0));
      }
  }
  int4* d = nullptr;
  CUDA_TRY(h, cudaMalloc(&d, std::max<size_t>(v.size(), 1) * sizeof(int4)));
  const cudaError_t e = cudaMemcpy(d, v.data(), v.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    return fail(h, FDTD_ERR_CUDA, "CPML block list upload failed: %s", cudaGetErrorString(e));
  }
  h->cpml_blocks[r] = {d, (int)v.size()};
  *out = h->cpml_blocks[r];
  return FDTD_OK;
}

// The companion of one tiled launch of k steps from field set `src` (step t) to `dst`.
fdtd_status cpml_companion(fdtd_handle* h, int k, int src, int dst, long long t,
                           const fdtd::Sources& S, const fdtd::Monitors& M, cudaStream_t st,
                           int* launches) {
  if (k > 1 && !h->cpml_scratch[0]) {  // all six or none
    for (int c = 0; c < 6; ++c)
      if (cudaMalloc(&h->cpml_scratch[c], h->cells * sizeof(float)) != cudaSuccess) {
        for (int q = 0; q < 6; ++q) {
          cudaFree(h->cpml_scratch[q]);
          h->cpml_scratch[q] = nullptr;
        }
        cudaGetLastError();
        return fail(h, FDTD_ERR_OOM, "CPML companion field set allocation failed");
      }
  }
  fdtd::FieldPtrs A, B, C;
  for (int c = 0; c < 6; ++c) {
    A.f[c] = h->F[src][c];
    B.f[c] = h->F[dst][c];
    C.f[c] = h->cpml_scratch[c];
  }
  for (int j = 1; j <= k; ++j) {
    const fdtd::FieldPtrs& Fi = j == 1 ? A : C;
    const fdtd::FieldPtrs& Fo = j == k ? B : C;
    const int re = 3 * k - 2 * (j - 1), rh = re - 1;
    std::pair<int4*, int> le, lh;
    fdtd_status s = cpml_region_blocks(h, re, &le);
    if (s == FDTD_OK) s = cpml_region_blocks(h, rh, &lh);
    if (s != FDTD_OK) return s;
    const long long tj = t + j - 1;
    CUDA_TRY(h, fdtd::launch_cpml_region(false, h->g, Fi, Fo, h->mat, h->table, S, M,
                                         h->cpml_dev, tj, h->desc.dx, le.first, le.second,
                                         cpml_inner_box(h, re), st));
    CUDA_TRY(h, fdtd::launch_cpml_region(true, h->g, Fi, Fo, h->mat, h->table, S, M,
                                         h->cpml_dev, tj, h->desc.dx, lh.first, lh.second,
                                         cpml_inner_box(h, rh), st));
    *launches += 2;
  }
  return FDTD_OK;
}

}  // namespace

extern "C" {

const char* fdtd_version(void) { return "gdiamond_b200 0.1 (sm_100a)"; }

const char* fdtd_status_string(fdtd_status s) {
  switch (s) {
    case FDTD_OK: return "ok";
    case FDTD_ERR_INVALID_ARG: return "invalid argument";
    case FDTD_ERR_OOM: return "out of device memory";
    case FDTD_ERR_CUDA: return "CUDA error";
    case FDTD_ERR_UNSUPPORTED: return "unsupported configuration";
    case FDTD_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case FDTD_ERR_NUMERIC: return "numeric check failed";
  }
  return "unknown status";
}

const char* fdtd_last_error(const fdtd_handle* h) {
  return h ? h->err.c_str() : g_create_error.c_str();
}

fdtd_status fdtd_create(const fdtd_desc* d, fdtd_handle** out) {
  if (!d || !out) return fail(nullptr, FDTD_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  if (d->nx < 3 || d->ny < 3 || d->nz < 3)
    return fail(nullptr, FDTD_ERR_INVALID_ARG, "grid must be at least 3 cells per axis");
  if (d->nx > (1 << 24) || d->ny > (1 << 24) || d->nz > (1 << 24))
    return fail(nullptr, FDTD_ERR_INVALID_ARG, "grid axis too large");
  if (d->storage < FDTD_STORE_F32 || d->storage > FDTD_STORE_F16E)
    return fail(nullptr, FDTD_ERR_INVALID_ARG, "unknown storage %d", d->storage);
  if (d->kernel < FDTD_KERNEL_AUTO || d->kernel > FDTD_KERNEL_TILED_W32P)
    return fail(nullptr, FDTD_ERR_INVALID_ARG, "unknown kernel %d", d->kernel);
  if ((d->storage == FDTD_STORE_F16 || d->storage == FDTD_STORE_BF16 ||
       d->storage == FDTD_STORE_F16E) &&
      (d->kernel == FDTD_KERNEL_NAIVE || d->kernel == FDTD_KERNEL_TILED_W32))
    return fail(nullptr, FDTD_ERR_UNSUPPORTED,
                "16-bit field storage runs the tiled x-pair kernel only");
  if (d->storage == FDTD_STORE_F64 && d->kernel != FDTD_KERNEL_AUTO &&
      d->kernel != FDTD_KERNEL_NAIVE)
    return fail(nullptr, FDTD_ERR_UNSUPPORTED, "FP64 field storage runs the naive kernel only");
  if (d->blt < 0 || d->blt > 6) return fail(nullptr, FDTD_ERR_INVALID_ARG, "blt must be 0..6");
  if (d->tile_rows != 0 && d->tile_rows != 8 && d->tile_rows != 16 && d->tile_rows != 20 &&
      d->tile_rows != 24 && d->tile_rows != 32 && d->tile_rows != 48)
    return fail(nullptr, FDTD_ERR_INVALID_ARG, "tile_rows must be 0, 8, 16, 20, 24, 32 or 48");
  if (d->z_chunks < 0) return fail(nullptr, FDTD_ERR_INVALID_ARG, "z_chunks must be >= 0");
  if (d->min_blocks != 0 && d->min_blocks != 1 && d->min_blocks != 2 && d->min_blocks != 4)
    return fail(nullptr, FDTD_ERR_INVALID_ARG, "min_blocks must be 0, 1, 2 or 4");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, FDTD_ERR_CUDA, "no CUDA device available");
  if (d->device < 0 || d->device >= ndev)
    return fail(nullptr, FDTD_ERR_INVALID_ARG, "device %d out of range", d->device);
  DeviceGuard dg(d->device);
  fdtd_handle* h = new fdtd_handle();
  h->desc = *d;
  h->g.nx = (int)d->nx;
  h->g.ny = (int)d->ny;
  h->g.nz = (int)d->nz;
  h->g.pitch = (int)((d->nx + 7) / 8 * 8);
  h->g.plane = (long long)h->g.pitch * d->ny;
  h->cells = (size_t)h->g.plane * d->nz;
  h->storage = d->storage;
  h->esz = d->storage == FDTD_STORE_F32 ? 4 : (d->storage == FDTD_STORE_F64 ? 8 : 2);
  h->nsets = d->storage == FDTD_STORE_F64 ? 1 : 2;
  auto bail = [&](fdtd_status s) {
    g_create_error = h->err;
    free_all(h);
    delete h;
    return s;
  };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(h, FDTD_ERR_CUDA, "cudaStreamCreate failed"));
  for (int s = 0; s < h->nsets; ++s)
    for (int c = 0; c < 6; ++c) {
      const size_t bytes = h->cells * (size_t)comp_esz(h, c);
      cudaError_t e = cudaMalloc(&h->F[s][c], bytes);
      if (e != cudaSuccess)
        return bail(fail(h, FDTD_ERR_OOM, "cudaMalloc of %zu field bytes failed: %s", bytes,
                         cudaGetErrorString(e)));
      cudaMemsetAsync(h->F[s][c], 0, bytes, h->stream);
    }
  if (cudaMalloc(&h->d_err, sizeof(int)) != cudaSuccess)
    return bail(fail(h, FDTD_ERR_OOM, "cudaMalloc failed"));
  cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess)
    return bail(fail(h, FDTD_ERR_CUDA, "initialisation failed"));
  *out = h;
  return FDTD_OK;
}

fdtd_status fdtd_destroy(fdtd_handle* h) {
  if (!h) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return FDTD_OK;
}

fdtd_status fdtd_set_coefficients(fdtd_handle* h, const float* const* coef12) {
  if (!h || !coef12) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  return upload_coefficients(h, coef12, cudaMemcpyHostToDevice);
}

fdtd_status fdtd_set_coefficients_device(fdtd_handle* h, const float* const* coef12_dev) {
  if (!h || !coef12_dev) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  return upload_coefficients(h, coef12_dev, cudaMemcpyDeviceToDevice);
}

fdtd_status fdtd_set_permittivity(fdtd_handle* h, const float* eps_re, int32_t t_pml, float dt,
                                  float omega0) {
  if (!h || t_pml < 0 || !(dt > 0) || !(omega0 > 0)) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  fdtd_status s = alloc_coef_staging(h);
  if (s != FDTD_OK) return s;
  const float dx = h->desc.dx;
  const float denom = 2 * 1.0f * (float)t_pml * dx;
  // t_pml = 0: no graded layer (e.g. under CPML layers): every stretch factor is 1
  const float sigma_max =
      t_pml > 0 ? (float)((double)(-4) * std::log(1e-5) / (double)denom) : 0.0f;
  std::vector<float2> prof[3] = {stretch_profile(h->g.nx, t_pml, sigma_max, omega0),
                                 stretch_profile(h->g.ny, t_pml, sigma_max, omega0),
                                 stretch_profile(h->g.nz, t_pml, sigma_max, omega0)};
  const size_t n = (size_t)h->g.nx * h->g.ny * h->g.nz;
  float2* d_prof = nullptr;
  float* d_eps = nullptr;
  const size_t np = prof[0].size() + prof[1].size() + prof[2].size();
  CUDA_TRY(h, cudaMalloc(&d_prof, np * sizeof(float2)));
  CUDA_TRY(h, cudaMemcpyAsync(d_prof, prof[0].data(), prof[0].size() * 8, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(d_prof + prof[0].size(), prof[1].data(), prof[1].size() * 8,
                              cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(d_prof + prof[0].size() + prof[1].size(), prof[2].data(),
                              prof[2].size() * 8, cudaMemcpyHostToDevice, h->stream));
  if (eps_re) {
    CUDA_TRY(h, cudaMalloc(&d_eps, n * sizeof(float)));
    CUDA_TRY(h, cudaMemcpyAsync(d_eps, eps_re, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  }
  fdtd::Coef12Out out;
  for (int a = 0; a < 12; ++a) out.c[a] = h->coef[a];
  CUDA_TRY(h, fdtd::build_coefficients(h->g, d_eps, d_prof, d_prof + prof[0].size(),
                                       d_prof + prof[0].size() + prof[1].size(), omega0, dt, dx,
                                       out, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  cudaFree(d_prof);
  cudaFree(d_eps);
  return compress_coefficients(h);
}

fdtd_status fdtd_get_coefficients(fdtd_handle* h, float* const* out12) {
  if (!h || !out12) return FDTD_ERR_INVALID_ARG;
  if (!h->coef[0]) return fail(h, FDTD_ERR_INVALID_ARG, "coefficients are not set");
  DeviceGuard dg(h->desc.device);
  for (int a = 0; a < 12; ++a) {
    if (!out12[a]) return FDTD_ERR_INVALID_ARG;
    CUDA_TRY(h, cudaMemcpy2DAsync(out12[a], (size_t)h->g.nx * 4, h->coef[a], (size_t)h->g.pitch * 4,
                                  (size_t)h->g.nx * 4, (size_t)h->g.ny * h->g.nz,
                                  cudaMemcpyDeviceToHost, h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return FDTD_OK;
}

fdtd_status fdtd_material_count(const fdtd_handle* h, int32_t* nmat) {
  if (!h || !nmat) return FDTD_ERR_INVALID_ARG;
  *nmat = h->coef_mode == kCoefMaterial ? h->nmat : 0;
  return FDTD_OK;
}

fdtd_status fdtd_set_sources(fdtd_handle* h, const fdtd_source* sources, int32_t nsrc,
                             const float* waveforms, int64_t T_wave) {
  if (!h) return FDTD_ERR_INVALID_ARG;
  if (nsrc < 0 || nsrc > fdtd::kMaxSources)
    return fail(h, FDTD_ERR_INVALID_ARG, "nsrc must be 0..%d", fdtd::kMaxSources);
  if (nsrc > 0 && (!sources || !waveforms || T_wave <= 0))
    return fail(h, FDTD_ERR_INVALID_ARG, "sources need a waveform table");
  DeviceGuard dg(h->desc.device);
  for (int n = 0; n < nsrc; ++n) {
    const fdtd_source& s = sources[n];
    if (s.component < 0 || s.component > 5)
      return fail(h, FDTD_ERR_INVALID_ARG, "source %d: bad component %d", n, s.component);
    if (s.kind != FDTD_SRC_POINT && s.kind != FDTD_SRC_PLANE_Z)
      return fail(h, FDTD_ERR_INVALID_ARG, "source %d: bad kind %d", n, s.kind);
    if (s.k < 0 || s.k >= h->g.nz ||
        (s.kind == FDTD_SRC_POINT && (s.i < 0 || s.i >= h->g.nx || s.j < 0 || s.j >= h->g.ny)))
      return fail(h, FDTD_ERR_INVALID_ARG, "source %d outside the grid", n);
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  cudaFree(h->d_wave);
  h->d_wave = nullptr;
  h->nsrc = 0;
  h->tw = 0;
  if (nsrc > 0) {
    const size_t bytes = (size_t)nsrc * T_wave * sizeof(float);
    CUDA_TRY(h, cudaMalloc(&h->d_wave, bytes));
    CUDA_TRY(h, cudaMemcpy(h->d_wave, waveforms, bytes, cudaMemcpyHostToDevice));
  }
  for (int n = 0; n < nsrc; ++n) {
    h->src[n].comp = sources[n].component;
    h->src[n].kind = sources[n].kind;
    h->src[n].i = (int)sources[n].i;
    h->src[n].j = (int)sources[n].j;
    h->src[n].k = (int)sources[n].k;
  }
  h->nsrc = nsrc;
  h->tw = T_wave;
  h->version += 1;
  return FDTD_OK;
}

fdtd_status fdtd_add_dft_monitor(fdtd_handle* h, int32_t component, int64_t k,
                                 const double* freqs, int32_t nf, double scale, double dt,
                                 int32_t* monitor_id) {
  return add_monitor(h, component, k, freqs, nf, scale, dt, 0.0, monitor_id);
}

fdtd_status fdtd_add_flux_monitor(fdtd_handle* h, int64_t k, const double* freqs, int32_t nf,
                                  double dt, int32_t* flux_id) {
  if (!h) return FDTD_ERR_INVALID_ARG;
  if (h->nflux >= kMaxFlux)
    return fail(h, FDTD_ERR_UNSUPPORTED, "at most %d flux monitors", kMaxFlux);
  if (k < 1 || k > h->g.nz - 2)
    return fail(h, FDTD_ERR_INVALID_ARG, "flux plane must be an interior plane 1..Nz-2");
  if (h->nmon + 6 > fdtd::kMaxMonitors)
    return fail(h, FDTD_ERR_UNSUPPORTED, "a flux monitor needs 6 of the %d monitor slots",
                fdtd::kMaxMonitors);
  FluxHost fx;
  fx.k = k;
  fx.nf = nf;
  const int comps[6] = {FDTD_EX, FDTD_EY, FDTD_HX, FDTD_HX, FDTD_HY, FDTD_HY};
  const int64_t planes[6] = {k, k, k - 1, k, k - 1, k};
  const int first = h->nmon;
  for (int q = 0; q < 6; ++q) {
    fdtd_status s = add_monitor(h, comps[q], planes[q], freqs, nf, 1.0, dt,
                                comps[q] >= FDTD_HX ? 0.5 : 0.0, &fx.mon[q]);
    if (s != FDTD_OK) {
      drop_monitors(h, first);
      return s;
    }
  }
  DeviceGuard dg(h->desc.device);
  if (cudaMalloc(&fx.out, (size_t)nf * sizeof(double)) != cudaSuccess) {
    drop_monitors(h, first);
    return fail(h, FDTD_ERR_OOM, "flux result allocation failed");
  }
  h->flux[h->nflux] = fx;
  if (flux_id) *flux_id = h->nflux;
  h->nflux += 1;
  return FDTD_OK;
}

fdtd_status fdtd_get_flux_device(fdtd_handle* h, int32_t flux_id, double* flux_dev,
                                 void* stream) {
  if (!h || !flux_dev || flux_id < 0 || flux_id >= h->nflux) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  cudaStream_t st = pick_stream(h, stream);
  const FluxHost& fx = h->flux[flux_id];
  auto M = [&](int q) { return &h->mon[fx.mon[q]]; };
  fdtd::FluxPlanes p{M(0)->re, M(0)->im, M(1)->re, M(1)->im, M(2)->re, M(2)->im,
                     M(3)->re, M(3)->im, M(4)->re, M(4)->im, M(5)->re, M(5)->im};
  const double dx = (double)h->desc.dx;
  CUDA_TRY(h, fdtd::launch_flux_reduce(p, (long long)h->g.nx * h->g.ny, fx.nf, dx * dx,
                                       flux_dev, st));
  return FDTD_OK;
}

fdtd_status fdtd_get_flux(fdtd_handle* h, int32_t flux_id, double* flux_out) {
  if (!h || !flux_out || flux_id < 0 || flux_id >= h->nflux) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  FluxHost& fx = h->flux[flux_id];
  fdtd_status s = fdtd_get_flux_device(h, flux_id, fx.out, nullptr);
  if (s != FDTD_OK) return s;
  CUDA_TRY(h, cudaMemcpyAsync(flux_out, fx.out, (size_t)fx.nf * sizeof(double),
                              cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return check_device_error(h);
}

fdtd_status fdtd_flux_monitor_ids(const fdtd_handle* h, int32_t flux_id, int32_t* ids6) {
  if (!h || !ids6 || flux_id < 0 || flux_id >= h->nflux) return FDTD_ERR_INVALID_ARG;
  for (int q = 0; q < 6; ++q) ids6[q] = h->flux[flux_id].mon[q];
  return FDTD_OK;
}

fdtd_status fdtd_reset(fdtd_handle* h) {
  if (!h) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  for (int s = 0; s < h->nsets; ++s)
    for (int c = 0; c < 6; ++c)
      CUDA_TRY(h, cudaMemsetAsync(h->F[s][c], 0, h->cells * comp_esz(h, c), h->stream));
  for (int m = 0; m < h->nmon; ++m) {
    const size_t bytes = (size_t)h->mon[m].nf * h->g.nx * h->g.ny * sizeof(double);
    CUDA_TRY(h, cudaMemsetAsync(h->mon[m].re, 0, bytes, h->stream));
    CUDA_TRY(h, cudaMemsetAsync(h->mon[m].im, 0, bytes, h->stream));
  }
  if (h->cpml_on) {
    for (int q = 0; q < 12; ++q)
      CUDA_TRY(h, cudaMemsetAsync(h->cpml_psi[q], 0, cpml_psi_bytes(h, q), h->stream));
  }
  h->t = 0;
  h->cur = 0;
  return FDTD_OK;
}

fdtd_status fdtd_step(fdtd_handle* h, int64_t T, void* stream) {
  if (!h || T < 0) return FDTD_ERR_INVALID_ARG;
  if (h->coef_mode == kCoefNone)
    return fail(h, FDTD_ERR_INVALID_ARG, "coefficients are not set");
  if (T == 0) return FDTD_OK;
  DeviceGuard dg(h->desc.device);
  cudaStream_t st = pick_stream(h, stream);
  if (st != h->stream) {
    // Order the caller's stream after any work queued on the handle's own stream.
    cudaEvent_t ev;
    CUDA_TRY(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventRecord(ev, h->stream));
    CUDA_TRY(h, cudaStreamWaitEvent(st, ev, 0));
    cudaEventDestroy(ev);
  }
  fdtd_status s = ensure_tables(h, h->t + T);
  if (s != FDTD_OK) return s;
  // CPML layers: the tiled kernel with the shell companion when the grid is large enough for
  // it (and the caller did not ask for the naive kernel), else one E and one H kernel per step
  // over the whole grid, monitors per step.
  bool companion = false;
  if (h->cpml_on) {
    if (h->storage != FDTD_STORE_F32)
      return fail(h, FDTD_ERR_UNSUPPORTED, "CPML layers need FP32 field storage");
    if (h->desc.kernel != FDTD_KERNEL_NAIVE && h->coef_mode == kCoefMaterial &&
        cpml_companion_fits(h, 1)) {
      if (!h->cfg_ready && (s = autotune(h, st)) != FDTD_OK) return s;
      companion = cpml_companion_fits(h, h->cfg.blt);
    }
  }
  if (h->cpml_on && !companion) {
    fdtd::FieldPtrs F;
    for (int c = 0; c < 6; ++c) F.f[c] = h->F[h->cur][c];
    const bool matm = h->coef_mode == kCoefMaterial;
    const fdtd::Sources S = make_sources(h);
    const fdtd::Monitors M = make_monitors(h);
    int launches = 0;
    for (int64_t q = 0; q < T; ++q) {
      CUDA_TRY(h, fdtd::launch_cpml_step(h->g, F, matm ? nullptr : h->coef,
                                         matm ? h->mat : nullptr, h->table, S, M, h->cpml_dev,
                                         h->t, h->desc.dx, st, &launches));
      h->t += 1;
    }
    h->last_kernel = 6;  // reported by fdtd_get_config: the per-step CPML kernels
    h->last_launches = launches;
    h->last_folds = 0;
    if (st != h->stream) {
      cudaEvent_t ev;
      CUDA_TRY(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      CUDA_TRY(h, cudaEventRecord(ev, st));
      CUDA_TRY(h, cudaStreamWaitEvent(h->stream, ev, 0));
      cudaEventDestroy(ev);
    }
    return FDTD_OK;
  }
  int kernel = h->desc.kernel;
  if (kernel == FDTD_KERNEL_AUTO)
    kernel = (h->coef_mode == kCoefMaterial && h->storage != FDTD_STORE_F64) ? FDTD_KERNEL_TILED
                                                                            : FDTD_KERNEL_NAIVE;
  if (kernel == FDTD_KERNEL_NAIVE && h->esz == 2)
    return fail(h, FDTD_ERR_UNSUPPORTED, "16-bit field storage needs the tiled kernel");
  if (kernel != FDTD_KERNEL_NAIVE && h->coef_mode != kCoefMaterial)
    return fail(h, FDTD_ERR_UNSUPPORTED,
                "the tiled kernel needs a material map (more than %d distinct coefficient "
                "tuples were given)", kMaxMaterials);
  int launches = 0, folds = 0;
  const fdtd::Sources S = make_sources(h);
  const fdtd::Monitors M = make_monitors(h);
  if (kernel == FDTD_KERNEL_NAIVE) {
    fdtd::FieldPtrs F;
    for (int c = 0; c < 6; ++c) F.f[c] = h->F[h->cur][c];
    const bool matm = h->coef_mode == kCoefMaterial;
    for (int64_t n = 0; n < T; ++n) {
      CUDA_TRY(h, fdtd::launch_naive_step(h->g, F, matm ? nullptr : h->coef, matm ? h->mat : nullptr,
                                          h->table, S, M, h->t, h->desc.dx, st, &launches,
                                          h->storage == FDTD_STORE_F64));
      h->t += 1;
    }
    h->last_kernel = FDTD_KERNEL_NAIVE;
  } else {
    if (!h->cfg_ready) {
      s = autotune(h, st);
      if (s != FDTD_OK) return s;
    }
    fdtd::TiledConfig c = h->cfg;
    c.storage = h->storage;  // the kernel instance must match this handle's field storage
    c.esz = h->esz;
    s = ensure_maps(h, c);
    if (s != FDTD_OK) return s;
    // The tiled kernels stage monitor-plane values in a ring of kDftSlots steps; a fold adds
    // them to the sums before the ring would wrap and once more at the end, so the sums are
    // complete whenever fdtd_step returns.
    long long t_fold = h->t;
    int64_t left = T;
    const int* order = tile_order(h, c);
    while (left > 0) {
      fdtd::TiledConfig cc = c;
      if (left < c.blt) {  // a shorter final pass (plain register allocation)
        cc.blt = (int)left;
        cc.min_blocks = 1;
      }
      if (M.n > 0 && h->t + cc.blt - t_fold > fdtd::kDftSlots) {
        CUDA_TRY(h, fdtd::launch_dft_fold(M, h->g, t_fold, (int)(h->t - t_fold), st));
        ++folds;
        t_fold = h->t;
      }
      fdtd::TiledArgs a = make_tiled_args(h, cc, h->t, true);
      a.tile_order = cc.blt == c.blt ? order : nullptr;
      h->fault_tile[0] = h->fault_tile[1] = h->fault_tile[2] = -1;  // the hook fires once
      CUDA_TRY(h, launch_any(cc, a, h->g, st));
      ++launches;
      if (companion &&
          (s = cpml_companion(h, cc.blt, h->cur, h->cur ^ 1, h->t, S, M, st, &launches)) !=
              FDTD_OK)
        return s;
      h->cur ^= 1;
      h->t += cc.blt;
      left -= cc.blt;
    }
    if (M.n > 0 && h->t > t_fold) {
      CUDA_TRY(h, fdtd::launch_dft_fold(M, h->g, t_fold, (int)(h->t - t_fold), st));
      ++folds;
    }
    h->last_kernel = c.pairs32 ? FDTD_KERNEL_TILED_W32P
                               : (c.width == 64 ? FDTD_KERNEL_TILED_W64 : FDTD_KERNEL_TILED_W32);
  }
  h->last_launches = launches;
  h->last_folds = folds;
  if (st != h->stream) {
    cudaEvent_t ev;
    CUDA_TRY(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventRecord(ev, st));
    CUDA_TRY(h, cudaStreamWaitEvent(h->stream, ev, 0));
    cudaEventDestroy(ev);
  }
  return FDTD_OK;
}

fdtd_status fdtd_sync(fdtd_handle* h) {
  if (!h) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return check_device_error(h);
}

fdtd_status fdtd_set_step(fdtd_handle* h, int64_t t) {
  if (!h || t < 0) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->t = t;
  return FDTD_OK;
}

fdtd_status fdtd_set_dft(fdtd_handle* h, int32_t monitor_id, const double* re, const double* im) {
  if (!h || monitor_id < 0 || monitor_id >= h->nmon || !re || !im) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  const MonitorHost& m = h->mon[monitor_id];
  const size_t bytes = (size_t)m.nf * h->g.nx * h->g.ny * sizeof(double);
  CUDA_TRY(h, cudaMemcpyAsync(m.re, re, bytes, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(m.im, im, bytes, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return FDTD_OK;
}

fdtd_status fdtd_get_step(const fdtd_handle* h, int64_t* t) {
  if (!h || !t) return FDTD_ERR_INVALID_ARG;
  *t = h->t;
  return FDTD_OK;
}

// Pitched FP32 view of a field component: the field itself for FP32 storage, else the
// component converted into the FP32 staging buffer (asynchronous on st).
fdtd_status f32_view(fdtd_handle* h, int32_t component, cudaStream_t st, const float** out) {
  if (comp_storage(h, component) == FDTD_STORE_F32) {
    *out = h->F[h->cur][component];
    return FDTD_OK;
  }
  if (!h->f32_stage) CUDA_TRY(h, cudaMalloc(&h->f32_stage, h->cells * sizeof(float)));
  CUDA_TRY(h, fdtd::convert_field_to_f32(h->g, h->F[h->cur][component], comp_storage(h, component),
                                         h->scale[component], h->f32_stage, st));
  *out = h->f32_stage;
  return FDTD_OK;
}

fdtd_status fdtd_get_field(fdtd_handle* h, int32_t component, float* host_out) {
  if (!h || !host_out || component < 0 || component > 5) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  const float* src = nullptr;
  fdtd_status s = f32_view(h, component, h->stream, &src);
  if (s != FDTD_OK) return s;
  CUDA_TRY(h, cudaMemcpy2DAsync(host_out, (size_t)h->g.nx * 4, src, (size_t)h->g.pitch * 4,
                                (size_t)h->g.nx * 4, (size_t)h->g.ny * h->g.nz,
                                cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return check_device_error(h);
}

fdtd_status fdtd_get_field_f64(fdtd_handle* h, int32_t component, double* host_out) {
  if (!h || !host_out || component < 0 || component > 5) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  if (!h->f64_stage) CUDA_TRY(h, cudaMalloc(&h->f64_stage, h->cells * sizeof(double)));
  CUDA_TRY(h, fdtd::convert_field_to_f64(h->g, h->F[h->cur][component],
                                         comp_storage(h, component), h->scale[component],
                                         h->f64_stage, h->stream));
  CUDA_TRY(h, cudaMemcpy2DAsync(host_out, (size_t)h->g.nx * 8, h->f64_stage,
                                (size_t)h->g.pitch * 8, (size_t)h->g.nx * 8,
                                (size_t)h->g.ny * h->g.nz, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return check_device_error(h);
}

fdtd_status fdtd_get_field_device(fdtd_handle* h, int32_t component, float* dev_out,
                                  void* stream) {
  if (!h || !dev_out || component < 0 || component > 5) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  cudaStream_t st = pick_stream(h, stream);
  const float* src = nullptr;
  fdtd_status s = f32_view(h, component, st, &src);
  if (s != FDTD_OK) return s;
  CUDA_TRY(h, cudaMemcpy2DAsync(dev_out, (size_t)h->g.nx * 4, src, (size_t)h->g.pitch * 4,
                                (size_t)h->g.nx * 4, (size_t)h->g.ny * h->g.nz,
                                cudaMemcpyDeviceToDevice, st));
  return FDTD_OK;
}

fdtd_status fdtd_set_field(fdtd_handle* h, int32_t component, const float* host_in) {
  if (!h || !host_in || component < 0 || component > 5) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  if (comp_storage(h, component) == FDTD_STORE_F32) {
    CUDA_TRY(h, cudaMemcpy2DAsync(h->F[h->cur][component], (size_t)h->g.pitch * 4, host_in,
                                  (size_t)h->g.nx * 4, (size_t)h->g.nx * 4,
                                  (size_t)h->g.ny * h->g.nz, cudaMemcpyHostToDevice, h->stream));
  } else {
    if (!h->f32_stage) {
      CUDA_TRY(h, cudaMalloc(&h->f32_stage, h->cells * sizeof(float)));
      CUDA_TRY(h, cudaMemsetAsync(h->f32_stage, 0, h->cells * sizeof(float), h->stream));
    }
    CUDA_TRY(h, cudaMemcpy2DAsync(h->f32_stage, (size_t)h->g.pitch * 4, host_in,
                                  (size_t)h->g.nx * 4, (size_t)h->g.nx * 4,
                                  (size_t)h->g.ny * h->g.nz, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, fdtd::convert_field_from_f32(h->g, h->f32_stage, comp_storage(h, component),
                                             h->inv_scale[component], h->F[h->cur][component],
                                             h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return FDTD_OK;
}

fdtd_status fdtd_get_dft(fdtd_handle* h, int32_t monitor_id, double* re, double* im) {
  if (!h || monitor_id < 0 || monitor_id >= h->nmon || !re || !im) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  const MonitorHost& m = h->mon[monitor_id];
  const size_t bytes = (size_t)m.nf * h->g.nx * h->g.ny * sizeof(double);
  CUDA_TRY(h, cudaMemcpyAsync(re, m.re, bytes, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(im, m.im, bytes, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return check_device_error(h);
}

fdtd_status fdtd_get_dft_device(fdtd_handle* h, int32_t monitor_id, double* re_dev,
                                double* im_dev, void* stream) {
  if (!h || monitor_id < 0 || monitor_id >= h->nmon || !re_dev || !im_dev)
    return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  cudaStream_t st = pick_stream(h, stream);
  const MonitorHost& m = h->mon[monitor_id];
  const size_t bytes = (size_t)m.nf * h->g.nx * h->g.ny * sizeof(double);
  CUDA_TRY(h, cudaMemcpyAsync(re_dev, m.re, bytes, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(h, cudaMemcpyAsync(im_dev, m.im, bytes, cudaMemcpyDeviceToDevice, st));
  return FDTD_OK;
}

// Raw (storage-format) copies of z-planes [k0, k0+nk) of one component of the current field
// set: the halo exchange of z-slab decomposition.
fdtd_status plane_copy(fdtd_handle* h, int32_t comp, int64_t k0, int64_t nk, void* dev,
                       void* stream, bool to_handle) {
  if (!h || !dev || comp < 0 || comp > 5 || k0 < 0 || nk < 1 || k0 + nk > h->g.nz)
    return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  cudaStream_t st = pick_stream(h, stream);
  const size_t esz = (size_t)comp_esz(h, comp);
  char* field = reinterpret_cast<char*>(h->F[h->cur][comp]) + (size_t)k0 * h->g.plane * esz;
  char* packed = static_cast<char*>(dev);
  const size_t row = (size_t)h->g.nx * esz, pitch = (size_t)h->g.pitch * esz;
  const size_t rows = (size_t)h->g.ny * (size_t)nk;
  if (to_handle)
    CUDA_TRY(h, cudaMemcpy2DAsync(field, pitch, packed, row, row, rows, cudaMemcpyDeviceToDevice, st));
  else
    CUDA_TRY(h, cudaMemcpy2DAsync(packed, row, field, pitch, row, rows, cudaMemcpyDeviceToDevice, st));
  return FDTD_OK;
}

fdtd_status fdtd_get_planes_device(fdtd_handle* h, int32_t component, int64_t k0, int64_t nk,
                                   void* dev_out, void* stream) {
  return plane_copy(h, component, k0, nk, dev_out, stream, false);
}

fdtd_status fdtd_set_planes_device(fdtd_handle* h, int32_t component, int64_t k0, int64_t nk,
                                   const void* dev_in, void* stream) {
  return plane_copy(h, component, k0, nk, const_cast<void*>(dev_in), stream, true);
}

fdtd_status fdtd_storage_bytes(const fdtd_handle* h, int32_t* esz) {
  if (!h || !esz) return FDTD_ERR_INVALID_ARG;
  *esz = h->esz;
  return FDTD_OK;
}

fdtd_status fdtd_component_bytes(const fdtd_handle* h, int32_t component, int32_t* esz) {
  if (!h || !esz || component < 0 || component > 5) return FDTD_ERR_INVALID_ARG;
  *esz = comp_esz(h, component);
  return FDTD_OK;
}

fdtd_status fdtd_set_storage_scale(fdtd_handle* h, const float* scale6) {
  if (!h || !scale6) return FDTD_ERR_INVALID_ARG;
  for (int c = 0; c < 6; ++c)
    if (!(scale6[c] > 0.0f) || !std::isfinite(scale6[c]))
      return fail(h, FDTD_ERR_INVALID_ARG, "storage scale %d must be positive and finite", c);
  for (int c = 0; c < 6; ++c) {
    if (comp_esz(h, c) != 2) continue;  // FP32 / FP64 components are unscaled
    const int e = (int)std::lround(std::log2((double)scale6[c]));
    if (e < -100 || e > 100) return fail(h, FDTD_ERR_INVALID_ARG, "storage scale out of range");
    h->scale[c] = std::ldexp(1.0f, e);
    h->inv_scale[c] = std::ldexp(1.0f, -e);
  }
  return FDTD_OK;
}

fdtd_status fdtd_debug_fail_copy(fdtd_handle* h, int32_t bx, int32_t by, int32_t bz,
                                  int32_t iteration, int64_t wait_cycles) {
  if (!h || bx < 0 || by < 0 || bz < 0 || iteration < 0 || wait_cycles < 1)
    return FDTD_ERR_INVALID_ARG;
  h->fault_tile[0] = bx;
  h->fault_tile[1] = by;
  h->fault_tile[2] = bz;
  h->fault_it = iteration;
  h->fault_wait = wait_cycles;
  return FDTD_OK;
}

fdtd_status fdtd_set_cpml(fdtd_handle* h, const fdtd_cpml_desc* d) {
  if (!h) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  cudaStreamSynchronize(h->stream);
  cudaFree(h->cpml_tab);
  h->cpml_tab = nullptr;
  for (int q = 0; q < 12; ++q) {
    cudaFree(h->cpml_psi[q]);
    h->cpml_psi[q] = nullptr;
  }
  cpml_release_companion(h);
  h->cpml_on = false;
  if (!d) return FDTD_OK;
  if (d->thickness < 1 || !(d->order >= 0) || !(d->reflection > 0 && d->reflection < 1) ||
      !(d->kappa_max >= 1) || !(d->alpha_max >= 0) || !(d->dt > 0) || (d->faces & ~63))
    return fail(h, FDTD_ERR_INVALID_ARG, "bad CPML description");
  if (h->storage != FDTD_STORE_F32)
    return fail(h, FDTD_ERR_UNSUPPORTED, "CPML layers need FP32 field storage");
  const int n[3] = {h->g.nx, h->g.ny, h->g.nz};
  for (int a = 0; a < 3; ++a)
    if ((d->faces >> (2 * a) & 3) && n[a] < 2 * d->thickness + 2)
      return fail(h, FDTD_ERR_INVALID_ARG, "axis %d has %d cells, CPML needs >= %d", a, n[a],
                  2 * d->thickness + 2);
  h->cpml = *d;
  // tables: per axis and position kind, int slot[n] then b, a, 1/kappa [n] each
  size_t bytes = 0;
  for (int a = 0; a < 3; ++a) bytes += 2 * (size_t)n[a] * 16;
  CUDA_TRY(h, cudaMalloc(&h->cpml_tab, bytes));
  char* base = static_cast<char*>(h->cpml_tab);
  size_t off = 0;
  for (int a = 0; a < 3; ++a) {
    fdtd::CpmlAxis& ax = h->cpml_dev.ax[a];
    ax.S = 2 * d->thickness + 1;
    for (int k = 0; k < 2; ++k) {
      const bool lo = d->faces >> (2 * a) & 1, hi = d->faces >> (2 * a + 1) & 1;
      auto& sl = h->cpml_slot[a][k];
      auto* pr = h->cpml_prof[a][k];
      cpml_profile(*d, n[a], lo, hi, (double)h->desc.dx, k == 1, &sl, &pr[0], &pr[1], &pr[2]);
      int* d_slot = reinterpret_cast<int*>(base + off);
      float* d_f = reinterpret_cast<float*>(base + off + (size_t)n[a] * 4);
      CUDA_TRY(h, cudaMemcpy(d_slot, sl.data(), (size_t)n[a] * 4, cudaMemcpyHostToDevice));
      for (int q = 0; q < 3; ++q)
        CUDA_TRY(h, cudaMemcpy(d_f + (size_t)q * n[a], pr[q].data(), (size_t)n[a] * 4,
                               cudaMemcpyHostToDevice));
      if (k == 0) {
        ax.slot_e = d_slot;
        ax.be = d_f;
        ax.ae = d_f + n[a];
        ax.ike = d_f + 2 * (size_t)n[a];
      } else {
        ax.slot_h = d_slot;
        ax.bh = d_f;
        ax.ah = d_f + n[a];
        ax.ikh = d_f + 2 * (size_t)n[a];
      }
      off += (size_t)n[a] * 16;
    }
  }
  for (int q = 0; q < 12; ++q) {
    const size_t pb = cpml_psi_bytes(h, q);
    if (cudaMalloc(&h->cpml_psi[q], pb) != cudaSuccess) {
      fdtd_set_cpml(h, nullptr);
      return fail(h, FDTD_ERR_OOM, "CPML psi allocation failed");
    }
    CUDA_TRY(h, cudaMemset(h->cpml_psi[q], 0, pb));
    (q < 6 ? h->cpml_dev.psi_e[q] : h->cpml_dev.psi_h[q - 6]) = h->cpml_psi[q];
  }
  // positions whose updates involve no layer, per axis (the shell companion's inner box)
  for (int a = 0; a < 3; ++a) {
    int lo = 0, hi = n[a];
    for (int p = 0; p < n[a]; ++p) {
      const bool in = h->cpml_slot[a][0][p] >= 0 || h->cpml_slot[a][1][p] >= 0;
      if (!in) continue;
      if (2 * p < n[a]) lo = std::max(lo, p + 1);
      else hi = std::min(hi, p);
    }
    h->cpml_inner[a][0] = lo;
    h->cpml_inner[a][1] = hi;
    h->cpml_lo[a] = lo > 0;
    h->cpml_hi[a] = hi < n[a];
  }
  h->cpml_on = true;
  return FDTD_OK;
}

fdtd_status fdtd_get_cpml_profile(const fdtd_handle* h, int32_t axis, int32_t h_positions,
                                  float* b, float* a, float* inv_kappa, int32_t* slot) {
  if (!h || axis < 0 || axis > 2 || !h->cpml_on) return FDTD_ERR_INVALID_ARG;
  const int k = h_positions ? 1 : 0;
  const auto& pr = h->cpml_prof[axis][k];
  const size_t n = pr[0].size();
  if (b) std::copy(pr[0].begin(), pr[0].end(), b);
  if (a) std::copy(pr[1].begin(), pr[1].end(), a);
  if (inv_kappa) std::copy(pr[2].begin(), pr[2].end(), inv_kappa);
  if (slot) std::copy(h->cpml_slot[axis][k].begin(), h->cpml_slot[axis][k].end(), slot);
  (void)n;
  return FDTD_OK;
}

fdtd_status fdtd_cpml_psi_bytes(const fdtd_handle* h, int32_t q, int64_t* bytes) {
  if (!h || !bytes || q < 0 || q > 11 || !h->cpml_on) return FDTD_ERR_INVALID_ARG;
  *bytes = (int64_t)cpml_psi_bytes(h, q);
  return FDTD_OK;
}

fdtd_status fdtd_get_cpml_psi(fdtd_handle* h, int32_t q, void* host_out) {
  if (!h || !host_out || q < 0 || q > 11 || !h->cpml_on) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  CUDA_TRY(h, cudaMemcpy(host_out, h->cpml_psi[q], cpml_psi_bytes(h, q), cudaMemcpyDeviceToHost));
  return FDTD_OK;
}

fdtd_status fdtd_set_cpml_psi(fdtd_handle* h, int32_t q, const void* host_in) {
  if (!h || !host_in || q < 0 || q > 11 || !h->cpml_on) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(h->desc.device);
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  CUDA_TRY(h, cudaMemcpy(h->cpml_psi[q], host_in, cpml_psi_bytes(h, q), cudaMemcpyHostToDevice));
  return FDTD_OK;
}

fdtd_status fdtd_set_fast_path(fdtd_handle* h, int32_t enable) {
  if (!h) return FDTD_ERR_INVALID_ARG;
  h->lean_enable = enable != 0;
  return FDTD_OK;
}

fdtd_status fdtd_fast_path(const fdtd_handle* h, int32_t* active) {
  if (!h || !active) return FDTD_ERR_INVALID_ARG;
  *active = h->coef_mode == kCoefMaterial && h->lean_ok && h->lean_enable ? 1 : 0;
  return FDTD_OK;
}

fdtd_status fdtd_dft_folds(const fdtd_handle* h, int32_t* n) {
  if (!h || !n) return FDTD_ERR_INVALID_ARG;
  *n = h->last_folds;
  return FDTD_OK;
}

fdtd_status fdtd_get_config(const fdtd_handle* h, int32_t* out6) {
  if (!h || !out6) return FDTD_ERR_INVALID_ARG;
  out6[0] = h->last_kernel;
  out6[1] = h->cfg.blt;
  out6[2] = h->cfg.rows;
  out6[3] = h->cfg.z_chunks;
  out6[4] = h->last_launches;
  out6[5] = h->cfg.min_blocks;
  return FDTD_OK;
}

}  // extern "C"

// ============================================================================== batches

struct fdtd_batch {
  std::vector<fdtd_handle*> sims;
  int device = 0;
  cudaStream_t stream = nullptr;
  int storage = 0, esz = 4;
  fdtd::TiledConfig cfg{0, 0, 1, 64};
  int zlen = 0;  // target z-chunk length of a work item (0: whole columns)
  bool cfg_ready = false;
  fdtd::TiledArgs* d_args = nullptr;  // [2][n]
  fdtd::TiledArgs* h_args = nullptr;  // pinned staging [2][n]
  // Recorded after each step's launches: the copy of h_args (a graph node or an asynchronous
  // copy) has run once it completes, so the next step may refill h_args.
  cudaEvent_t args_read = nullptr;
  bool args_pending = false;
  std::map<int, std::pair<int4*, int>> items;  // per BLT: device work items, count
  unsigned int* d_counters = nullptr;
  int counters_cap = 0;
  int ctas = 0;
  cudaGraphExec_t gexec = nullptr;
  std::vector<long long> gkey;
  int gfolds = 0;  // DFT fold launches in the captured graph
  int last_launches = 0, last_graph = 0, last_folds = 0;
  // CPML batches (every simulation has CPML layers): per-grid arguments of the per-step kernels
  fdtd::CpmlSim* d_cpml = nullptr;
  fdtd::CpmlSim* h_cpml = nullptr;  // pinned staging, copied to d_cpml at the head of a step
  std::string err;
};

namespace {

fdtd_status bfail(fdtd_batch* b, fdtd_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (b) b->err = buf; else g_create_error = buf;
  return s;
}

#define BCUDA(b, call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return bfail((b), e_ == cudaErrorMemoryAllocation ? FDTD_ERR_OOM : FDTD_ERR_CUDA,   \
                   "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,       \
                   __LINE__);                                                             \
  } while (0)

fdtd::TiledConfig batch_cfg(const fdtd_batch* b, int blt, int rows, bool pairs32 = false) {
  fdtd::TiledConfig c{blt, rows, 1, pairs32 ? 32 : 64, 1, b->storage, b->esz};
  c.pairs32 = pairs32;
  return c;
}

// Key of a batch's work-item list: z-chunk length and the tile configuration.
int items_key(int zlen, const fdtd::TiledConfig& c) {
  return ((zlen * 10 + c.blt) * 100 + c.rows) * 2 + (c.pairs32 ? 1 : 0);
}

// z-chunks of one simulation for a target chunk length (0: one chunk per column).
int sim_chunks(const Grid& g, int zlen) { return zlen <= 0 ? 1 : std::max(1, (g.nz + zlen - 1) / zlen); }

// Work items of one (BLT, rows, chunk length): every z-chunk of every tile column of every
// simulation, longest z-march first so the queue's tail is short.
fdtd_status batch_items(fdtd_batch* b, const fdtd::TiledConfig& c, std::pair<int4*, int>* out) {
  const int key = items_key(b->zlen, c);
  auto it = b->items.find(key);
  if (it != b->items.end()) {
    *out = it->second;
    return FDTD_OK;
  }
  // longest items first; at equal length the tiles that run the slower mixed march first
  std::vector<std::pair<int, int4>> v;  // {2 * length + (lean-only ? 0 : 1), item}
  for (size_t i = 0; i < b->sims.size(); ++i) {
    const fdtd_handle* h = b->sims[i];
    const Grid& g = h->g;
    fdtd::TiledConfig ci = c;
    ci.z_chunks = sim_chunks(g, b->zlen);
    const dim3 gd = fdtd::tiled2_grid(ci, g);
    const int zl = (g.nz + ci.z_chunks - 1) / ci.z_chunks;
    const int len = zl + 2 * c.blt;
    for (unsigned bz = 0; bz < gd.z; ++bz)
      for (unsigned by = 0; by < gd.y; ++by)
        for (unsigned bx = 0; bx < gd.x; ++bx) {
          const bool lean = tile_is_lean(h, ci, (int)bx, (int)by, (int)bz, zl);
          v.push_back({2 * len + (lean ? 0 : 1), make_int4((int)i, (int)bx, (int)by, (int)bz)});
        }
  }
  std::stable_sort(v.begin(), v.end(),
                   [](const std::pair<int, int4>& a, const std::pair<int, int4>& b2) {
                     return a.first > b2.first;
                   });
  std::vector<int4> host(v.size());
  for (size_t i = 0; i < v.size(); ++i) host[i] = v[i].second;
  int4* d = nullptr;
  BCUDA(b, cudaMalloc(&d, host.size() * sizeof(int4)));
  BCUDA(b, cudaMemcpy(d, host.data(), host.size() * sizeof(int4), cudaMemcpyHostToDevice));
  b->items[key] = {d, (int)host.size()};
  *out = b->items[key];
  return FDTD_OK;
}

fdtd_status batch_maps(fdtd_batch* b, const fdtd::TiledConfig& c) {
  for (fdtd_handle* h : b->sims) {
    fdtd_status s = ensure_maps(h, c);
    if (s != FDTD_OK) return bfail(b, s, "sim: %s", h->err.c_str());
  }
  return FDTD_OK;
}

// Fills h_args [2][n] for config c: parity p reads field set (cur ^ p) of each simulation.
void batch_fill_args(fdtd_batch* b, const fdtd::TiledConfig& c, bool with_io) {
  const size_t n = b->sims.size();
  for (size_t i = 0; i < n; ++i) {
    fdtd_handle* h = b->sims[i];
    fdtd::TiledConfig ci = c;
    ci.z_chunks = sim_chunks(h->g, b->zlen);
    for (int p = 0; p < 2; ++p) {
      b->h_args[p * n + i] = make_tiled_args(h, ci, h->t, with_io, h->cur ^ p);
      b->h_args[p * n + i].fault_bx = -1;  // the test hook is for single-grid steps
      b->h_args[p * n + i].wait_limit = 0;
    }
  }
}

fdtd_status batch_counters(fdtd_batch* b, int need) {
  if (need <= b->counters_cap) return FDTD_OK;
  if (b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
    b->gkey.clear();
  }
  cudaFree(b->d_counters);
  b->d_counters = nullptr;
  const int cap = std::max(need, 2 * b->counters_cap);
  BCUDA(b, cudaMalloc(&b->d_counters, cap * sizeof(unsigned int)));
  b->counters_cap = cap;
  return FDTD_OK;
}

fdtd_status batch_launch(fdtd_batch* b, const fdtd::TiledConfig& c, int flip, long long t_off,
                         unsigned int* counter, cudaStream_t st) {
  std::pair<int4*, int> it;
  fdtd_status s = batch_items(b, c, &it);
  if (s != FDTD_OK) return s;
  fdtd::BatchArgs a;
  a.grids = b->d_args;
  a.ngrids = (int)b->sims.size();
  a.flip = flip;
  a.t_offset = t_off;
  a.items = it.first;
  a.nitems = it.second;
  a.counter = counter;
  BCUDA(b, fdtd::launch_tiled2_batch(c, a, b->ctas, st));
  return FDTD_OK;
}

fdtd_status batch_autotune(fdtd_batch* b, cudaStream_t st) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
  // A BLT or tile-row count that every simulation of the batch asks for (fdtd_desc) is kept;
  // otherwise both are tuned.
  int want_blt = b->sims[0]->desc.blt, want_rows = b->sims[0]->desc.tile_rows;
  for (const fdtd_handle* h : b->sims) {
    if (h->desc.blt != want_blt) want_blt = 0;
    if (h->desc.tile_rows != want_rows) want_rows = 0;
  }
  std::vector<fdtd::TiledConfig> cands;
  for (int pairs32 = 0; pairs32 < 2; ++pairs32)
    for (int rows : {16, 8, 20, 24, 32, 48})
      for (int blt = 1; blt <= 4; ++blt) {
        if ((want_blt > 0 && blt != want_blt) || (want_rows > 0 && rows != want_rows)) continue;
        fdtd::TiledConfig c = batch_cfg(b, blt, rows, pairs32 != 0);
        if (fdtd::tiled2_batch_supported(c)) cands.push_back(c);
      }
  if (cands.empty())
    return bfail(b, FDTD_ERR_UNSUPPORTED, "no batched configuration for blt %d, tile_rows %d",
                 want_blt, want_rows);
  fdtd_status s = batch_counters(b, 4);
  if (s != FDTD_OK) return s;
  cudaEvent_t e0, e1;
  BCUDA(b, cudaEventCreate(&e0));
  BCUDA(b, cudaEventCreate(&e1));
  float best = 1e30f;
  fdtd::TiledConfig best_c = cands[0];
  int best_ctas = nsm, best_zlen = 0;
  for (int pass = 0; pass < 2; ++pass)  // the first pass also brings the clocks up
    for (const auto& c : cands)
    for (int zl : {0, 64, 32}) {
      b->zlen = zl;
      if ((s = batch_maps(b, c)) != FDTD_OK) return s;
      b->ctas = nsm * fdtd::tiled2_batch_ctas_per_sm(c);
      batch_fill_args(b, c, false);
      BCUDA(b, cudaMemcpyAsync(b->d_args, b->h_args, 2 * b->sims.size() * sizeof(fdtd::TiledArgs),
                               cudaMemcpyHostToDevice, st));
      BCUDA(b, cudaMemsetAsync(b->d_counters, 0, 3 * sizeof(unsigned int), st));
      if ((s = batch_launch(b, c, 0, 0, b->d_counters, st)) != FDTD_OK) return s;
      BCUDA(b, cudaEventRecord(e0, st));
      for (int r = 1; r < 3; ++r)
        if ((s = batch_launch(b, c, 0, 0, b->d_counters + r, st)) != FDTD_OK) return s;
      BCUDA(b, cudaEventRecord(e1, st));
      BCUDA(b, cudaEventSynchronize(e1));
      float ms = 0;
      BCUDA(b, cudaEventElapsedTime(&ms, e0, e1));
      const float per_step = ms / (2 * c.blt);
      if (pass == 1 && per_step < best) {
        best = per_step;
        best_c = c;
        best_ctas = b->ctas;
        best_zlen = zl;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->cfg = best_c;
  b->ctas = best_ctas;
  b->zlen = best_zlen;
  b->cfg_ready = true;
  return FDTD_OK;
}

// Makes `waiter` wait for everything queued on `on`.
fdtd_status stream_after(fdtd_batch* b, cudaStream_t waiter, cudaStream_t on) {
  if (waiter == on) return FDTD_OK;
  cudaEvent_t ev;
  BCUDA(b, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  BCUDA(b, cudaEventRecord(ev, on));
  BCUDA(b, cudaStreamWaitEvent(waiter, ev, 0));
  cudaEventDestroy(ev);
  return FDTD_OK;
}

// A batch whose simulations have CPML layers: per step one E and one H launch over every grid
// (in place, FP32), monitor values staged in the rings and folded before a ring would wrap and
// at the end, as in the tiled batches.  With use_graph the T steps are captured once and
// replayed; the argument table is refreshed by the copy at the head of the sequence, so the
// graph only depends on T and the batch's extents.
fdtd_status batch_step_cpml(fdtd_batch* b, int64_t T, int32_t use_graph, cudaStream_t st) {
  const int n = (int)b->sims.size();
  if (!b->h_cpml) {
    BCUDA(b, cudaMalloc(&b->d_cpml, n * sizeof(fdtd::CpmlSim)));
    BCUDA(b, cudaMallocHost(&b->h_cpml, n * sizeof(fdtd::CpmlSim)));
  }
  int max_nx = 0, max_ny = 0, max_nz = 0, max_nf = 0;
  long long max_np = 0;
  for (int i = 0; i < n; ++i) {
    const fdtd_handle* h = b->sims[i];
    if (h->storage != FDTD_STORE_F32)
      return bfail(b, FDTD_ERR_UNSUPPORTED, "CPML layers need FP32 field storage");
    fdtd::CpmlSim& a = b->h_cpml[i];
    a = fdtd::CpmlSim{};
    a.g = h->g;
    for (int c = 0; c < 6; ++c) a.F.f[c] = h->F[h->cur][c];
    a.mat = h->mat;  // batches hold material maps only
    a.tab = h->table;
    a.S = make_sources(h);
    a.M = make_monitors(h);
    a.P = h->cpml_dev;
    a.t0 = h->t;
    a.dx = h->desc.dx;
    max_nx = std::max(max_nx, h->g.nx);
    max_ny = std::max(max_ny, h->g.ny);
    max_nz = std::max(max_nz, h->g.nz);
    for (int m = 0; m < h->nmon; ++m) {
      max_np = std::max<long long>(max_np, (long long)h->g.nx * h->g.ny);
      max_nf = std::max(max_nf, h->mon[m].nf);
    }
  }
  int folds = 0;
  auto record = [&](cudaStream_t rs) -> fdtd_status {
    BCUDA(b, cudaMemcpyAsync(b->d_cpml, b->h_cpml, n * sizeof(fdtd::CpmlSim),
                             cudaMemcpyHostToDevice, rs));
    long long folded = 0;
    folds = 0;
    for (long long q = 0; q < T; ++q) {
      if (max_nf > 0 && q + 1 - folded > fdtd::kDftSlots) {
        BCUDA(b, fdtd::launch_dft_fold_cpml_batch(b->d_cpml, n, max_np, max_nf, folded,
                                                  (int)(q - folded), rs));
        ++folds;
        folded = q;
      }
      BCUDA(b, fdtd::launch_cpml_batch_step(b->d_cpml, n, max_nx, max_ny, max_nz, q, rs));
    }
    if (max_nf > 0 && T > folded) {
      BCUDA(b, fdtd::launch_dft_fold_cpml_batch(b->d_cpml, n, max_np, max_nf, folded,
                                                (int)(T - folded), rs));
      ++folds;
    }
    return FDTD_OK;
  };
  b->last_graph = 0;
  if (use_graph) {
    const std::vector<long long> key = {-1, T, n, max_nx, max_ny, max_nz, max_np, max_nf};
    if (!b->gexec || key != b->gkey) {
      if (b->gexec) {
        cudaGraphExecDestroy(b->gexec);
        b->gexec = nullptr;
      }
      cudaGraph_t graph;
      BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
      fdtd_status r = record(b->stream);
      cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
      if (r != FDTD_OK) return r;
      if (ce != cudaSuccess) return bfail(b, FDTD_ERR_CUDA, "graph capture failed: %s",
                                          cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&b->gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return bfail(b, FDTD_ERR_CUDA, "graph instantiation failed: %s",
                                          cudaGetErrorString(ce));
      b->gkey = key;
      b->gfolds = folds;
    } else {
      b->last_graph = 1;
      folds = b->gfolds;
    }
    BCUDA(b, cudaGraphLaunch(b->gexec, st));
  } else {
    fdtd_status r = record(st);
    if (r != FDTD_OK) return r;
  }
  if (!b->args_read) BCUDA(b, cudaEventCreateWithFlags(&b->args_read, cudaEventDisableTiming));
  BCUDA(b, cudaEventRecord(b->args_read, st));
  b->args_pending = true;
  const int per = 65535 / std::max(max_nz, 1);
  const int launches = (int)(2 * T * ((n + per - 1) / per));
  for (fdtd_handle* h : b->sims) {
    h->t += T;
    h->last_kernel = 6;  // the per-step CPML kernels
    h->last_launches = launches;
    h->last_folds = folds;
    fdtd_status r = stream_after(b, h->stream, st);
    if (r != FDTD_OK) return r;
  }
  b->last_launches = launches;
  b->last_folds = folds;
  return FDTD_OK;
}

}  // namespace

extern "C" {

const char* fdtd_batch_last_error(const fdtd_batch* b) {
  return b ? b->err.c_str() : g_create_error.c_str();
}

fdtd_status fdtd_batch_create(fdtd_handle* const* sims, int32_t n, fdtd_batch** out) {
  if (!sims || !out || n < 1) return bfail(nullptr, FDTD_ERR_INVALID_ARG, "empty batch");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    const fdtd_handle* h = sims[i];
    if (!h) return bfail(nullptr, FDTD_ERR_INVALID_ARG, "simulation %d is NULL", i);
    if (h->desc.device != sims[0]->desc.device || h->storage != sims[0]->storage)
      return bfail(nullptr, FDTD_ERR_INVALID_ARG, "simulations must share device and storage");
    if (h->storage == FDTD_STORE_F64)
      return bfail(nullptr, FDTD_ERR_UNSUPPORTED, "FP64 storage has no batched kernel");
    if (h->coef_mode != kCoefMaterial)
      return bfail(nullptr, FDTD_ERR_UNSUPPORTED,
                   "simulation %d has no material map (coefficients not set or too many)", i);
    if (h->cpml_on != sims[0]->cpml_on)
      return bfail(nullptr, FDTD_ERR_INVALID_ARG,
                   "simulations must all have CPML layers or all have none");
  }
  fdtd_batch* b = new fdtd_batch();
  b->sims.assign(sims, sims + n);
  b->device = sims[0]->desc.device;
  b->storage = sims[0]->storage;
  b->esz = sims[0]->esz;
  DeviceGuard dg(b->device);
  const size_t bytes = 2 * (size_t)n * sizeof(fdtd::TiledArgs);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&b->d_args, bytes) != cudaSuccess ||
      cudaMallocHost(&b->h_args, bytes) != cudaSuccess) {
    fdtd_batch_destroy(b);
    return bfail(nullptr, FDTD_ERR_OOM, "batch allocation failed");
  }
  *out = b;
  return FDTD_OK;
}

fdtd_status fdtd_batch_destroy(fdtd_batch* b) {
  if (!b) return FDTD_ERR_INVALID_ARG;
  DeviceGuard dg(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  for (auto& kv : b->items) cudaFree(kv.second.first);
  cudaFree(b->d_counters);
  cudaFree(b->d_args);
  if (b->h_args) cudaFreeHost(b->h_args);
  cudaFree(b->d_cpml);
  if (b->h_cpml) cudaFreeHost(b->h_cpml);
  if (b->args_read) cudaEventDestroy(b->args_read);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return FDTD_OK;
}

fdtd_status fdtd_batch_step(fdtd_batch* b, int64_t T, int32_t use_graph, void* stream) {
  if (!b || T < 0) return FDTD_ERR_INVALID_ARG;
  if (T == 0) return FDTD_OK;
  DeviceGuard dg(b->device);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  fdtd_status s;
  if (b->args_pending) {  // the previous step's copy of h_args must have run before a refill
    BCUDA(b, cudaEventSynchronize(b->args_read));
    b->args_pending = false;
  }
  for (fdtd_handle* h : b->sims) {
    if ((s = ensure_tables(h, h->t + T)) != FDTD_OK) return bfail(b, s, "%s", h->err.c_str());
    if ((s = stream_after(b, st, h->stream)) != FDTD_OK) return s;
  }
  for (const fdtd_handle* h : b->sims)  // layers may have been set after the batch was made
    if (h->cpml_on != b->sims[0]->cpml_on)
      return bfail(b, FDTD_ERR_INVALID_ARG,
                   "simulations must all have CPML layers or all have none");
  if (b->sims[0]->cpml_on) return batch_step_cpml(b, T, use_graph, st);
  if (!b->cfg_ready && (s = batch_autotune(b, st)) != FDTD_OK) return s;
  const fdtd::TiledConfig c = b->cfg;
  const long long nfull = T / c.blt;
  const int rem = (int)(T % c.blt);
  const int nl = (int)nfull + (rem ? 1 : 0);
  if ((s = batch_maps(b, c)) != FDTD_OK) return s;
  if ((s = batch_counters(b, nl)) != FDTD_OK) return s;
  std::pair<int4*, int> tmp;
  if ((s = batch_items(b, c, &tmp)) != FDTD_OK) return s;
  if (rem && (s = batch_items(b, batch_cfg(b, rem, c.rows, c.pairs32), &tmp)) != FDTD_OK)
    return s;
  batch_fill_args(b, c, true);
  // Deferred DFT: the largest monitor plane and frequency count size the fold launches.
  long long max_np = 0;
  int max_nf = 0;
  for (fdtd_handle* h : b->sims)
    for (int m = 0; m < h->nmon; ++m) {
      max_np = std::max<long long>(max_np, (long long)h->g.nx * h->g.ny);
      max_nf = std::max(max_nf, h->mon[m].nf);
    }
  int folds = 0;

  // Monitor values staged by the batched kernel are folded into the sums before a ring of
  // kDftSlots steps would wrap and at the end (the grids' t0 in d_args parity 0 is their step
  // counter at the start of this call).
  auto record = [&](cudaStream_t rs) -> fdtd_status {
    BCUDA(b, cudaMemcpyAsync(b->d_args, b->h_args,
                             2 * b->sims.size() * sizeof(fdtd::TiledArgs),
                             cudaMemcpyHostToDevice, rs));
    BCUDA(b, cudaMemsetAsync(b->d_counters, 0, nl * sizeof(unsigned int), rs));
    const int ng = (int)b->sims.size();
    long long folded = 0;
    folds = 0;
    for (int k = 0; k < nl; ++k) {
      const fdtd::TiledConfig ck = (k < nfull) ? c : batch_cfg(b, rem, c.rows, c.pairs32);
      const long long off = (long long)k * c.blt;
      if (max_nf > 0 && off + ck.blt - folded > fdtd::kDftSlots) {
        BCUDA(b, fdtd::launch_dft_fold_batch(b->d_args, ng, max_np, max_nf, folded,
                                             (int)(off - folded), rs));
        ++folds;
        folded = off;
      }
      fdtd_status r = batch_launch(b, ck, k & 1, off, b->d_counters + k, rs);
      if (r != FDTD_OK) return r;
    }
    if (max_nf > 0 && T > folded) {
      BCUDA(b, fdtd::launch_dft_fold_batch(b->d_args, ng, max_np, max_nf, folded,
                                           (int)(T - folded), rs));
      ++folds;
    }
    return FDTD_OK;
  };

  b->last_graph = 0;
  if (use_graph) {
    std::vector<long long> key = {T, c.blt, c.rows, b->ctas, b->zlen, max_np, max_nf};
    for (fdtd_handle* h : b->sims) {
      key.push_back(h->t);
      key.push_back(h->cur);
    }
    if (!b->gexec || key != b->gkey) {
      if (b->gexec) {
        cudaGraphExecDestroy(b->gexec);
        b->gexec = nullptr;
      }
      cudaGraph_t graph;
      BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
      fdtd_status r = record(b->stream);
      cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
      if (r != FDTD_OK) return r;
      if (ce != cudaSuccess) return bfail(b, FDTD_ERR_CUDA, "graph capture failed: %s",
                                          cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&b->gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return bfail(b, FDTD_ERR_CUDA, "graph instantiation failed: %s",
                                          cudaGetErrorString(ce));
      b->gkey = key;
      b->gfolds = folds;
    } else {
      b->last_graph = 1;
      folds = b->gfolds;
    }
    BCUDA(b, cudaGraphLaunch(b->gexec, st));
  } else {
    if ((s = record(st)) != FDTD_OK) return s;
  }
  if (!b->args_read) BCUDA(b, cudaEventCreateWithFlags(&b->args_read, cudaEventDisableTiming));
  BCUDA(b, cudaEventRecord(b->args_read, st));
  b->args_pending = true;
  for (fdtd_handle* h : b->sims) {
    h->t += T;
    h->cur ^= (nl & 1);
    h->last_kernel = c.pairs32 ? FDTD_KERNEL_TILED_W32P : FDTD_KERNEL_TILED_W64;
    h->last_launches = nl;
    h->last_folds = folds;
    if ((s = stream_after(b, h->stream, st)) != FDTD_OK) return s;
  }
  b->last_launches = nl;
  b->last_folds = folds;
  return FDTD_OK;
}

fdtd_status fdtd_batch_get_config(const fdtd_batch* b, int32_t* out6) {
  if (!b || !out6) return FDTD_ERR_INVALID_ARG;
  out6[0] = b->cfg.blt;
  out6[1] = b->cfg.rows;
  out6[2] = b->ctas;
  auto it = b->items.find(items_key(b->zlen, b->cfg));
  out6[3] = it == b->items.end() ? 0 : it->second.second;
  out6[4] = b->last_launches;
  out6[5] = b->last_graph;
  return FDTD_OK;
}

}  // extern "C"
