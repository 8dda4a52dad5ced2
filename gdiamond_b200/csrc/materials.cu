// materials.cu -- compress 12 per-cell coefficient arrays into a material map on the GPU.
//
// The reference keeps Ca/Cb/Da/Db as 12 per-cell FP32 arrays (gDiamond/gdiamond.hpp:891-904,
// filled by set_FDTD_matrices_3D_structure, gDiamond/utils.h:542-690) and re-reads all 48
// bytes per cell in every step.  Real grids hold few distinct 12-tuples (vacuum, a handful of
// dielectrics, the graded PML shell), so the solver stores a uint16 id per cell plus a table
// of distinct tuples.  This file builds that map on the device:
//   1. insert: hash each cell's 12 words (bitwise) into an open-addressing table of 2^20
//      64-bit keys; the thread that inserts a key records its cell as the representative;
//   2. assign: number the occupied slots and copy each representative tuple into the table;
//   3. map: write each cell's id and compare its 12 words with the table entry, so a 64-bit
//      hash collision is detected (the map is then rejected) instead of silently merged; count
//      the cells of each id and report the id held by the most cells (the kernels' fast path
//      keeps that material's coefficients in registers).
// Probing is bounded; overflow or more than 65536 tuples reject the map (the per-cell arrays
// and the naive kernel are used instead).
#include "fdtd_kernels.cuh"

namespace fdtd {

namespace {

constexpr int kSlotBits = 20;
constexpr uint32_t kSlots = 1u << kSlotBits;
constexpr unsigned long long kEmpty = ~0ull;
constexpr int kMaxProbe = 4096;
constexpr int kMaxMaterials = 65536;

struct Scratch {
  unsigned long long keys[kSlots];
  unsigned long long rep[kSlots];
  uint32_t ids[kSlots];
  unsigned int nuniq;  // keys inserted
  unsigned int nid;    // ids handed out
  unsigned int flags;  // 1 = probe overflow, 2 = hash collision
  unsigned int mode;   // id held by the most cells (the lowest such id on a tie)
  unsigned int count[kMaxMaterials];  // cells per id
};

struct Coef12 {
  const float* c[12];  // pitched
};

__device__ __forceinline__ unsigned long long hash12(const uint32_t* w) {
  unsigned long long h = 0x9E3779B97F4A7C15ull;
#pragma unroll
  for (int a = 0; a < 12; ++a) {
    h ^= (unsigned long long)w[a] + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
    h *= 0xFF51AFD7ED558CCDull;
    h ^= h >> 33;
  }
  return h == kEmpty ? 0ull : h;
}

__device__ __forceinline__ void load12(const Coef12& C, long long idx, uint32_t* w) {
#pragma unroll
  for (int a = 0; a < 12; ++a) w[a] = __float_as_uint(C.c[a][idx]);
}

__device__ __forceinline__ long long cell_index(const Grid& g, long long lin) {
  const long long i = lin % g.nx, r = lin / g.nx;
  const long long j = r % g.ny, k = r / g.ny;
  return i + j * g.pitch + k * g.plane;
}

__global__ void k_reset(Scratch* s) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < kSlots) {
    s->keys[q] = kEmpty;
    s->rep[q] = kEmpty;
    s->ids[q] = 0xFFFFFFFFu;
  }
  if (q < (uint32_t)kMaxMaterials) s->count[q] = 0;
  if (q == 0) s->nuniq = s->nid = s->flags = s->mode = 0;
}

__global__ void k_insert(Grid g, Coef12 C, Scratch* s, long long n) {
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < n;
       lin += (long long)gridDim.x * blockDim.x) {
    const long long idx = cell_index(g, lin);
    uint32_t w[12];
    load12(C, idx, w);
    const unsigned long long h = hash12(w);
    uint32_t slot = (uint32_t)h & (kSlots - 1);
    bool done = false;
    for (int probe = 0; probe < kMaxProbe && !done; ++probe) {
      const unsigned long long cur = *((volatile unsigned long long*)&s->keys[slot]);
      if (cur == h) { done = true; break; }
      if (cur == kEmpty) {
        const unsigned long long old = atomicCAS(&s->keys[slot], kEmpty, h);
        if (old == kEmpty) {
          s->rep[slot] = (unsigned long long)idx;
          atomicAdd(&s->nuniq, 1u);
          done = true;
          break;
        }
        if (old == h) { done = true; break; }
      }
      slot = (slot + 1) & (kSlots - 1);
    }
    if (!done) atomicOr(&s->flags, 1u);
  }
}

__global__ void k_assign(Coef12 C, Scratch* s, Material* table) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kSlots || s->keys[q] == kEmpty) return;
  const unsigned int id = atomicAdd(&s->nid, 1u);
  s->ids[q] = id;
  if (id >= (unsigned)kMaxMaterials) return;
  const long long r = (long long)s->rep[q];
  float v[12];
#pragma unroll
  for (int a = 0; a < 12; ++a) v[a] = C.c[a][r];
  // {Cax, Cbx, Cay, Cby}, {Caz, Cbz, Dax, Dbx}, {Day, Dby, Daz, Dbz}
  Material m;
  m.a = make_float4(v[0], v[3], v[1], v[4]);
  m.b = make_float4(v[2], v[5], v[6], v[9]);
  m.c = make_float4(v[7], v[10], v[8], v[11]);
  table[id] = m;
}

__global__ void k_map(Grid g, Coef12 C, Scratch* s, const Material* table, uint16_t* mat,
                      long long n) {
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < n;
       lin += (long long)gridDim.x * blockDim.x) {
    const long long idx = cell_index(g, lin);
    uint32_t w[12];
    load12(C, idx, w);
    const unsigned long long h = hash12(w);
    uint32_t slot = (uint32_t)h & (kSlots - 1);
    int probe = 0;
    while (probe < kMaxProbe && s->keys[slot] != h) {
      slot = (slot + 1) & (kSlots - 1);
      ++probe;
    }
    if (probe == kMaxProbe) { atomicOr(&s->flags, 1u); continue; }
    const uint32_t id = s->ids[slot];
    if (id >= (uint32_t)kMaxMaterials) continue;  // rejected on the host
    const Material m = table[id];
    const uint32_t t[12] = {__float_as_uint(m.a.x), __float_as_uint(m.a.z),
                            __float_as_uint(m.b.x), __float_as_uint(m.a.y),
                            __float_as_uint(m.a.w), __float_as_uint(m.b.y),
                            __float_as_uint(m.b.z), __float_as_uint(m.c.x),
                            __float_as_uint(m.c.z), __float_as_uint(m.b.w),
                            __float_as_uint(m.c.y), __float_as_uint(m.c.w)};
    bool same = true;
#pragma unroll
    for (int a = 0; a < 12; ++a) same = same && (t[a] == w[a]);
    if (!same) atomicOr(&s->flags, 2u);
    mat[idx] = (uint16_t)id;
    // cells per id: one atomic per group of lanes holding the same id
    const unsigned peers = __match_any_sync(__activemask(), id);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicAdd(&s->count[id], __popc(peers));
  }
}

// The id with the most cells (lowest id on a tie): one CTA of 1024 threads.
__global__ void k_mode(Scratch* s, int nmat) {
  __shared__ unsigned long long best[32];
  unsigned long long b = 0;  // (count << 32) | (0xFFFFFFFF - id): max picks most cells, lowest id
  for (int q = threadIdx.x; q < nmat; q += blockDim.x)
    b = max(b, ((unsigned long long)s->count[q] << 32) | (0xFFFFFFFFu - (unsigned)q));
  for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
  if ((threadIdx.x & 31) == 0) best[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x < 32) {
    b = best[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    if (threadIdx.x == 0) s->mode = 0xFFFFFFFFu - (unsigned)(b & 0xFFFFFFFFu);
  }
}

}  // namespace

namespace {

// One warp per block of kUniX x kUniY x kUniZ cells: each lane tests 32 of its 1024 cells.
__global__ void k_uniform_blocks(Grid g, const uint16_t* mat, int id, uint8_t* out, int nbx,
                                 int nby, long long nblk) {
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
  const int lane = threadIdx.x & 31;
  if (w >= nblk) return;  // warp-uniform
  const int bx = (int)(w % nbx), by = (int)((w / nbx) % nby), bz = (int)(w / ((long long)nbx * nby));
  bool ok = true;
  for (int q = lane; q < kUniX * kUniY * kUniZ; q += 32) {
    const int i = bx * kUniX + q % kUniX, j = by * kUniY + (q / kUniX) % kUniY;
    const int k = bz * kUniZ + q / (kUniX * kUniY);
    if (i < g.nx && j < g.ny && k < g.nz)
      ok = ok && mat[i + (long long)j * g.pitch + (long long)k * g.plane] == (uint16_t)id;
  }
  ok = __all_sync(0xffffffffu, ok);
  if (lane == 0) out[w] = ok ? 1 : 0;
}

}  // namespace

cudaError_t build_uniform_blocks(const Grid& g, const uint16_t* mat, int id, uint8_t* out,
                                 cudaStream_t st) {
  const int nbx = (g.nx + kUniX - 1) / kUniX, nby = (g.ny + kUniY - 1) / kUniY;
  const int nbz = (g.nz + kUniZ - 1) / kUniZ;
  const long long nblk = (long long)nbx * nby * nbz;
  const int threads = 256;
  const long long blocks = (nblk * 32 + threads - 1) / threads;
  k_uniform_blocks<<<(unsigned)blocks, threads, 0, st>>>(g, mat, id, out, nbx, nby, nblk);
  return cudaGetLastError();
}

size_t material_scratch_bytes() { return sizeof(Scratch); }

cudaError_t build_material_map(const Grid& g, const float* const* coef12, uint16_t* mat,
                               Material* table, void* scratch, size_t scratch_bytes,
                               cudaStream_t st, DedupResult* out) {
  out->ok = false;
  out->nmat = 0;
  if (scratch_bytes < sizeof(Scratch)) return cudaErrorInvalidValue;
  Scratch* s = static_cast<Scratch*>(scratch);
  Coef12 C;
  for (int a = 0; a < 12; ++a) C.c[a] = coef12[a];
  const long long n = (long long)g.nx * g.ny * g.nz;
  const int threads = 256;
  const int blocks = 148 * 16;
  k_reset<<<(kSlots + threads - 1) / threads, threads, 0, st>>>(s);
  k_insert<<<blocks, threads, 0, st>>>(g, C, s, n);
  unsigned int hdr[3];
  cudaError_t e = cudaMemcpyAsync(hdr, &s->nuniq, sizeof(hdr), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  if (hdr[2] != 0 || hdr[0] > (unsigned)kMaxMaterials) return cudaGetLastError();
  k_assign<<<(kSlots + threads - 1) / threads, threads, 0, st>>>(C, s, table);
  k_map<<<blocks, threads, 0, st>>>(g, C, s, table, mat, n);
  k_mode<<<1, 1024, 0, st>>>(s, (int)hdr[0]);
  unsigned int hdr4[4];
  if ((e = cudaMemcpyAsync(hdr4, &s->nuniq, sizeof(hdr4), cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  out->nmat = (int)hdr4[0];
  out->ok = hdr4[2] == 0 && hdr4[0] <= (unsigned)kMaxMaterials;
  out->dominant = (int)hdr4[3];
  return cudaGetLastError();
}

}  // namespace fdtd
