// materials_noalloc.cu -- material-map construction that allocates nothing.
//
// A variant of the material deduplication in materials.cu for callers that cannot allocate
// device memory when they need the map: a host application that owns all device memory
// through its own pool (a cudaMalloc from a plug-in would fail or fragment it), a loop where
// cudaMalloc's implicit synchronisation is not acceptable, or code that must not grow its
// footprint after start-up.  The caller passes the 12 coefficient arrays and the output
// buffers; the hash-table scratch lives in a file-scope __device__ array of fixed size.
//
// Limits and behaviour:
//  * The scratch is a 65536-slot table (about 1.25 MB).  Every GPU that loads this library
//    keeps it until the process exits.  At most kMaxNoAllocMaterials = 4096 distinct
//    coefficient 12-tuples are supported (load factor <= 1/16, so probes stay short).
//  * Every call shares the one table and leaves the last call's contents in it; each call
//    clears it first.  Calls that overlap on the GPU (two streams, or two host threads) race on
//    the table and must be serialised by the caller.
//  * In host code the array's name is only a host-side stand-in.  The first call on each
//    device, with that device current, resolves its device address with cudaGetSymbolAddress
//    (cached per device afterwards).
//  * No cudaMalloc, cudaFree or allocating library routine is called.  The call synchronises
//    the given stream twice to read the table's counters into host variables, so it cannot be
//    made on a stream that is being captured into a CUDA graph.
//  * Ids are handed out in table-slot order by an atomic counter, so the numbering of the
//    materials may differ from one call to the next; map and table are always consistent.
//  * Data with more distinct tuples than the caller's table holds is rejected early: inserting
//    threads stop once the count of distinct tuples passes max_materials.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fdtd_capi.h"
#include "fdtd_common.cuh"

namespace fdtd {
namespace {

constexpr int kNaSlotBits = 16;
constexpr uint32_t kNaSlots = 1u << kNaSlotBits;
constexpr int kMaxNoAllocMaterials = 4096;
constexpr unsigned long long kNaEmpty = ~0ull;
constexpr int kNaMaxProbe = 4096;
constexpr int kNaMaxDevices = 64;

struct NaTable {
  unsigned long long keys[kNaSlots];
  unsigned long long rep[kNaSlots];
  uint32_t ids[kNaSlots];
  unsigned int nuniq;  // keys inserted
  unsigned int nid;    // ids handed out
  unsigned int flags;  // 1 = probe overflow, 2 = hash collision
};

// The scratch: one per device, for the life of the process.
static __device__ __align__(256) NaTable g_noalloc_table;

struct NaCoef {
  const float* c[12];
};

__device__ __forceinline__ unsigned long long na_hash(const uint32_t* w) {
  unsigned long long h = 0x243F6A8885A308D3ull;
#pragma unroll
  for (int a = 0; a < 12; ++a) {
    h ^= (unsigned long long)w[a] + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    h *= 0xC2B2AE3D27D4EB4Full;
    h ^= h >> 29;
  }
  return h == kNaEmpty ? 0ull : h;
}

__global__ void na_clear(NaTable* s) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < kNaSlots) {
    s->keys[q] = kNaEmpty;
    s->rep[q] = kNaEmpty;
    s->ids[q] = 0xFFFFFFFFu;
  }
  if (q == 0) s->nuniq = s->nid = s->flags = 0;
}

// Inserts every cell's tuple; gives up (the call is rejected anyway) once more than
// max_materials distinct tuples are in the table, checked before each cell and every 32 probes,
// so data with many distinct tuples costs a short pass rather than full-table probes.
__global__ void na_insert(NaCoef C, NaTable* s, long long n, int max_materials) {
  const volatile unsigned int* nuniq = &s->nuniq;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (*nuniq > (unsigned)max_materials) return;
    uint32_t w[12];
#pragma unroll
    for (int a = 0; a < 12; ++a) w[a] = __float_as_uint(C.c[a][i]);
    const unsigned long long h = na_hash(w);
    uint32_t slot = (uint32_t)h & (kNaSlots - 1);
    bool done = false;
    for (int probe = 0; probe < kNaMaxProbe && !done; ++probe) {
      const unsigned long long cur = *((volatile unsigned long long*)&s->keys[slot]);
      if (cur == h) break;
      if (cur == kNaEmpty) {
        const unsigned long long old = atomicCAS(&s->keys[slot], kNaEmpty, h);
        if (old == kNaEmpty) {
          s->rep[slot] = (unsigned long long)i;
          atomicAdd(&s->nuniq, 1u);
          done = true;
          break;
        }
        if (old == h) break;
      }
      slot = (slot + 1) & (kNaSlots - 1);
      if ((probe & 31) == 31 && *nuniq > (unsigned)max_materials) return;
      if (probe == kNaMaxProbe - 1) atomicOr(&s->flags, 1u);
    }
  }
}

__global__ void na_assign(NaCoef C, NaTable* s, float* table, int max_materials) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kNaSlots || s->keys[q] == kNaEmpty) return;
  const unsigned int id = atomicAdd(&s->nid, 1u);
  s->ids[q] = id;
  if (id >= (unsigned)max_materials) return;
  const long long r = (long long)s->rep[q];
#pragma unroll
  for (int a = 0; a < 12; ++a) table[(long long)id * 12 + a] = C.c[a][r];
}

__global__ void na_map(NaCoef C, NaTable* s, const float* table, uint16_t* mat, long long n,
                       int max_materials) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    uint32_t w[12];
#pragma unroll
    for (int a = 0; a < 12; ++a) w[a] = __float_as_uint(C.c[a][i]);
    const unsigned long long h = na_hash(w);
    uint32_t slot = (uint32_t)h & (kNaSlots - 1);
    int probe = 0;
    while (probe < kNaMaxProbe && s->keys[slot] != h) {
      slot = (slot + 1) & (kNaSlots - 1);
      ++probe;
    }
    if (probe == kNaMaxProbe) {
      atomicOr(&s->flags, 1u);
      continue;
    }
    const uint32_t id = s->ids[slot];
    if (id >= (uint32_t)max_materials) continue;
    bool same = true;
#pragma unroll
    for (int a = 0; a < 12; ++a) same = same && (__float_as_uint(table[(long long)id * 12 + a]) == w[a]);
    if (!same) atomicOr(&s->flags, 2u);
    mat[i] = (uint16_t)id;
  }
}

// Device address of g_noalloc_table on the current device, resolved once per device.
cudaError_t table_address(NaTable** out) {
  static NaTable* addr[kNaMaxDevices] = {};
  static std::mutex mu;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNaMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_table);
    if (e != cudaSuccess) return e;
    addr[dev] = static_cast<NaTable*>(p);
  }
  *out = addr[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace fdtd

extern "C" fdtd_status fdtd_build_material_map_noalloc(const float* const* coef12_dev,
                                                       int64_t nx, int64_t ny, int64_t nz,
                                                       uint16_t* mat_dev, float* table_dev,
                                                       int32_t max_materials, int32_t* nmat_out,
                                                       void* stream) {
  using namespace fdtd;
  if (!coef12_dev || !mat_dev || !table_dev || !nmat_out) return FDTD_ERR_INVALID_ARG;
  if (nx < 1 || ny < 1 || nz < 1) return FDTD_ERR_INVALID_ARG;
  if (max_materials < 1 || max_materials > kMaxNoAllocMaterials) return FDTD_ERR_INVALID_ARG;
  for (int a = 0; a < 12; ++a)
    if (!coef12_dev[a]) return FDTD_ERR_INVALID_ARG;
  *nmat_out = 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  NaTable* s = nullptr;
  if (table_address(&s) != cudaSuccess) return FDTD_ERR_CUDA;
  NaCoef C;
  for (int a = 0; a < 12; ++a) C.c[a] = coef12_dev[a];
  const long long n = (long long)nx * ny * nz;
  const int threads = 256, blocks = 148 * 8;
  // A launch that fails leaves the table as the previous call left it, so its counters are
  // only read after both launches of a pair were accepted.
  na_clear<<<(kNaSlots + threads - 1) / threads, threads, 0, st>>>(s);
  na_insert<<<blocks, threads, 0, st>>>(C, s, n, max_materials);
  if (cudaPeekAtLastError() != cudaSuccess) return FDTD_ERR_CUDA;
  unsigned int hdr[3] = {0, 0, 0};
  if (cudaMemcpyAsync(hdr, &s->nuniq, sizeof(hdr), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return FDTD_ERR_CUDA;
  if (hdr[2] != 0 || hdr[0] > (unsigned)max_materials) {
    *nmat_out = (int32_t)hdr[0];
    return FDTD_ERR_UNSUPPORTED;  // more distinct tuples than the table holds
  }
  na_assign<<<(kNaSlots + threads - 1) / threads, threads, 0, st>>>(C, s, table_dev,
                                                                     max_materials);
  na_map<<<blocks, threads, 0, st>>>(C, s, table_dev, mat_dev, n, max_materials);
  if (cudaPeekAtLastError() != cudaSuccess) return FDTD_ERR_CUDA;
  if (cudaMemcpyAsync(hdr, &s->nuniq, sizeof(hdr), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return FDTD_ERR_CUDA;
  *nmat_out = (int32_t)hdr[0];
  return hdr[2] == 0 ? FDTD_OK : FDTD_ERR_UNSUPPORTED;
}
