// mlp_tc.cu -- the surrogate MLP's GEMMs on the 5th-generation tensor cores (tcgen05 + TMEM).
//
// C[M][N] = sum_k opA(m,k) opB(n,k) with BF16 operands and an FP32 accumulator held in tensor
// memory, followed by the fused epilogues of mlp.cuh.  One CTA = 4 warps computes a 128 x BN
// tile (BN = 64 or 128) for one ensemble member (blockIdx.z):
//   - K advances in 64-wide steps through two shared-memory stages.  All 128 threads load a
//     step's A (128 x 64) and B (BN x 64) tiles from global memory into registers one step
//     ahead, then write them, transposing where the operand is stored k-major, into the
//     no-swizzle K-major "core matrix" layout the tensor core reads (8 rows x 16 bytes
//     contiguous; the two 8-element halves of a K=16 slice 128 B apart, 8-row groups 1024 B
//     apart).
//   - One thread issues four tcgen05.mma (M=128, N=BN, K=16 each) per step and commits them to
//     the stage's mbarrier; the next step's staging overlaps them, and a stage is refilled only
//     after its commit arrives.
//   - The accumulator (BN FP32 columns x 128 lanes) is allocated in TMEM by warp 0 and read back
//     with tcgen05.ld (warp w owns lanes 32w..32w+31 = tile rows), 32 columns at a time, and
//     transposed through shared memory so the epilogue's stores are row-contiguous.
// Every mbarrier wait is bounded; on expiry the kernel records an error word, stops issuing
// (decided block-wide with __syncthreads_or), waits (bounded) for what it issued, skips the
// epilogue, frees its TMEM and returns.
#include <atomic>

#include "fdtd_common.cuh"
#include "mlp.cuh"

namespace fdtd {
namespace mlp {
namespace {

constexpr int TBM = 128, TBK = 64;
constexpr long long kTcWaitLimit = 2000000000LL;  // SM clocks, ~1 s

// Byte offset of element (r, k) of an R x 64 tile in the core-matrix layout.
__device__ __forceinline__ uint32_t cm_off(int r, int k) {
  return (uint32_t)(((((r >> 3) * (TBK / 8)) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// Shared-memory matrix descriptor: start address, leading byte offset (between the K halves:
// 128 B), stride byte offset (between 8-row groups: 1024 B), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  const uint64_t lbo = 128 >> 4, sbo = ((TBK / 8) * 128) >> 4;
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, N, M=128.
template <int BN>
__host__ __device__ constexpr uint32_t instr_desc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(TBM >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                          uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
        "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
        "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// One thread's share of an R x 64 tile of op(X): R*8/128 chunks of 8 BF16 values.
template <int R>
struct Chunks {
  uint4 v[R * 8 / 128];
};

// Chunk `it` of thread `tid`: (row, k) of its first element.  !T: 8 consecutive k of one row,
// so a warp covers 4 whole core matrices (512 contiguous shared bytes).  T: 8 consecutive rows
// at one k (contiguous in global memory).
template <bool T, int R>
__device__ __forceinline__ void chunk_coords(int id, int* r, int* k) {
  if (!T) {
    *r = (id >> 6) * 8 + (id & 7);
    *k = ((id >> 3) & 7) * 8;
  } else {
    *r = (id % (R / 8)) * 8;
    *k = id / (R / 8);
  }
}

// Loads rows [r0, r0+R) x k [k0, k0+64) of op(X) into registers (zeros outside R_tot x K).
template <bool T, int R>
__device__ __forceinline__ void load_tile(Chunks<R>& c, const Operand& X,
                                          const __nv_bfloat16* base, int R_tot, int K, int r0,
                                          int k0) {
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
#pragma unroll
  for (int it = 0; it < R * 8 / 128; ++it) {
    int r, k;
    chunk_coords<T, R>(threadIdx.x + it * 128, &r, &k);
    const int gr = r0 + r, gk = k0 + k;
    __nv_bfloat16 e[8];
    if (!T) {
      if (X.vec && gr < R_tot && gk + 8 <= K) {
        c.v[it] = *reinterpret_cast<const uint4*>(base + (long long)gr * X.ld + gk);
        continue;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q)
        e[q] = (gr < R_tot && gk + q < K) ? base[(long long)gr * X.ld + gk + q] : zero;
    } else {
      if (X.vec && gk < K && gr + 8 <= R_tot) {
        c.v[it] = *reinterpret_cast<const uint4*>(base + (long long)gk * X.ld + gr);
        continue;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q)
        e[q] = (gk < K && gr + q < R_tot) ? base[(long long)gk * X.ld + gr + q] : zero;
    }
    memcpy(&c.v[it], e, 16);
  }
}

// Writes the registers of load_tile into the core-matrix tile at s.
template <bool T, int R>
__device__ __forceinline__ void store_tile(uint8_t* s, const Chunks<R>& c) {
#pragma unroll
  for (int it = 0; it < R * 8 / 128; ++it) {
    int r, k;
    chunk_coords<T, R>(threadIdx.x + it * 128, &r, &k);
    if (!T) {
      *reinterpret_cast<uint4*>(s + cm_off(r, k)) = c.v[it];
    } else {
      __nv_bfloat16 e[8];
      memcpy(e, &c.v[it], 16);
#pragma unroll
      for (int q = 0; q < 8; ++q) *reinterpret_cast<__nv_bfloat16*>(s + cm_off(r + q, k)) = e[q];
    }
  }
}

template <int BN>
struct TcSmem {
  static constexpr uint32_t A_BYTES = TBM * TBK * 2;
  static constexpr uint32_t B_BYTES = BN * TBK * 2;
  static constexpr uint32_t OFF_B = 2 * A_BYTES;
  static constexpr uint32_t OFF_BAR = OFF_B + 2 * B_BYTES;
  static constexpr uint32_t BYTES = OFF_BAR + 64 + 1024;  // + barriers, slots, alignment slack
};

template <bool TA, bool TB, int EPI, int BN>
__global__ void __launch_bounds__(128) gemm_tc(int M, int N, int K, Operand A, Operand B,
                                               Epilogue ep, int* err) {
  using L = TcSmem<BN>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                           ~static_cast<uintptr_t>(1023));
  uint8_t* sA = sm;
  uint8_t* sB = sm + L::OFF_B;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::OFF_BAR);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int e = blockIdx.z;
  const int m0 = blockIdx.y * TBM, n0 = blockIdx.x * BN;
  const __nv_bfloat16* Ab = A.p + e * A.stride;
  const __nv_bfloat16* Bb = B.p + e * B.stride;

  if (warp == 0) {
    tmem_alloc(tmem_slot, BN);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int nk = (K + TBK - 1) / TBK;
  int issued = 0;  // K steps whose MMAs were issued and committed
  bool aborted = false;
  Chunks<TBM> ca;
  Chunks<BN> cb;
  load_tile<TA, TBM>(ca, A, Ab, M, K, m0, 0);
  load_tile<TB, BN>(cb, B, Bb, N, K, n0, 0);
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt & 1;
    bool bad = false;
    if (kt >= 2 && !mbar_wait_bounded(&bar[s], ((kt - 2) >> 1) & 1, kTcWaitLimit)) {
      bad = true;
      atomicExch(err, 1);
    }
    if (!bad) {
      store_tile<TA, TBM>(sA + s * L::A_BYTES, ca);
      store_tile<TB, BN>(sB + s * L::B_BYTES, cb);
    }
    fence_proxy_async_smem();
    if (__syncthreads_or(bad)) {  // a barrier whose result every thread shares
      aborted = true;
      break;
    }
    if (kt + 1 < nk) {  // the next step's loads fly while this step's MMAs are issued
      load_tile<TA, TBM>(ca, A, Ab, M, K, m0, (kt + 1) * TBK);
      load_tile<TB, BN>(cb, B, Bb, N, K, n0, (kt + 1) * TBK);
    }
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sA + s * L::A_BYTES), b0 = smem_u32(sB + s * L::B_BYTES);
#pragma unroll
      for (int j = 0; j < TBK / 16; ++j)
        umma_bf16(tmem, smem_desc(a0 + j * 256), smem_desc(b0 + j * 256), instr_desc<BN>(),
                  (kt > 0 || j > 0) ? 1u : 0u);
      umma_commit(&bar[s]);
    }
    issued = kt + 1;
  }
  // The last commit arrives once every MMA issued before it has completed.
  bool late = false;
  if (issued > 0) {
    const int last = issued - 1;
    late = !mbar_wait_bounded(&bar[last & 1], (last >> 1) & 1, kTcWaitLimit);
    if (late) atomicExch(err, 1);
  }
  late = __syncthreads_or(late);
  tc_fence_after();
  if (!late && !aborted && issued > 0) {
    // Warp w holds rows 32w..32w+31 of the tile in its TMEM lanes.  Each 32-column block goes
    // through a padded 32 x 33 shared buffer (the drained A stage) so that every store
    // instruction writes 32 consecutive columns of one row.
    float* buf = reinterpret_cast<float*>(sA) + warp * (32 * 33);
#pragma unroll 1
    for (int c0 = 0; c0 < BN && n0 + c0 < N; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 32; ++j) buf[lane * 33 + j] = __uint_as_float(v[j]);
      __syncwarp();
      const int c = n0 + c0 + lane;
#pragma unroll 4
      for (int rr = 0; rr < 32; ++rr) {
        const int row = m0 + warp * 32 + rr;
        if (row < M && c < N) epilogue_store<EPI>(ep, e, row, c, buf[rr * 33 + lane]);
      }
      __syncwarp();
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, BN);
}

template <bool TA, bool TB, int EPI, int BN>
cudaError_t launch_bn(int M, int N, int K, const Operand& A, const Operand& B, const Epilogue& ep,
                      int members, cudaStream_t st, int* err) {
  static std::atomic<unsigned long long> set_on{0};  // devices (bit per ordinal < 64) done
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (!(set_on.load() & bit) || !bit) {
    e = cudaFuncSetAttribute(gemm_tc<TA, TB, EPI, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TcSmem<BN>::BYTES);
    if (e != cudaSuccess) return e;
    set_on.fetch_or(bit);
  }
  const dim3 grid((N + BN - 1) / BN, (M + TBM - 1) / TBM, members);
  gemm_tc<TA, TB, EPI, BN><<<grid, 128, TcSmem<BN>::BYTES, st>>>(M, N, K, A, B, ep, err);
  return cudaGetLastError();
}

// ------------------------------------------------------------------- fused ensemble inference
// One CTA of 256 threads takes 256 rows (two 128-row tiles) of one member through every layer:
// the BF16 activations stay in shared memory as the next layer's A operand (one 128 x 256 K-major
// core-matrix tile per row tile, 8-row groups 4096 B apart), the weights stream through two
// 64-wide K stages (N x 64 core matrices) and each staged chunk feeds both row tiles, the FP32
// accumulators (up to 2 x 256 columns) stay in TMEM, and only the last layer's output is written
// to global memory.  Warps 0-3 run the epilogue of tile 0, warps 4-7 that of tile 1.

constexpr int FACT_K = 256;  // widest layer input held in the activation tile
constexpr int FROWS = 128;                             // rows of one tile (the MMA's M)
constexpr int FTILES = 2;                              // row tiles per CTA
constexpr int FTHREADS = 256;
constexpr uint32_t F_ACT_BYTES = FROWS * FACT_K * 2;   // 64 KB per row tile
constexpr uint32_t F_W_BYTES = 256 * TBK * 2;          // 32 KB per weight stage
constexpr uint32_t F_SMEM = FTILES * F_ACT_BYTES + 2 * F_W_BYTES + 64 + 1024;

__device__ __forceinline__ uint32_t act_off(int r, int k) {
  return (uint32_t)(((((r >> 3) * (FACT_K / 8)) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ uint64_t smem_desc_sbo(uint32_t saddr, uint32_t sbo_bytes) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(sbo_bytes >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t instr_desc_n(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(FROWS >> 4) << 24);  // M = 128 rows
}

// One thread's share of an N x 64 weight chunk (N <= 256): up to 8 chunks of 8 BF16.
struct WChunk {
  uint4 v[8];
};

__device__ __forceinline__ void load_w(WChunk& c, const __nv_bfloat16* W, int N, int K, int k0) {
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  const bool vec = (K % 8) == 0;
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int id = threadIdx.x + it * FTHREADS;
    const int n = (id >> 6) * 8 + (id & 7), k = ((id >> 3) & 7) * 8;
    if (n >= N) continue;
    const int gk = k0 + k;
    if (vec && gk + 8 <= K) {
      c.v[it] = *reinterpret_cast<const uint4*>(W + (long long)n * K + gk);
    } else {
      __nv_bfloat16 e[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) e[q] = gk + q < K ? W[(long long)n * K + gk + q] : zero;
      memcpy(&c.v[it], e, 16);
    }
  }
}

__device__ __forceinline__ void store_w(uint8_t* s, const WChunk& c, int N) {
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int id = threadIdx.x + it * FTHREADS;
    const int n = (id >> 6) * 8 + (id & 7), k = ((id >> 3) & 7) * 8;
    if (n < N) *reinterpret_cast<uint4*>(s + cm_off(n, k)) = c.v[it];
  }
}

__global__ void __launch_bounds__(FTHREADS, 1) mlp_fused_infer(FusedArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                           ~static_cast<uintptr_t>(1023));
  uint8_t* act = sm;  // [FTILES][F_ACT_BYTES]
  uint8_t* sW = sm + FTILES * F_ACT_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sW + 2 * F_W_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int e = blockIdx.y;
  const long long m0 = (long long)blockIdx.x * (FROWS * FTILES);
  const __nv_bfloat16* wbf = a.wbf + e * a.P;
  const float* prm = a.params + e * a.P;

  if (warp == 0) {
    tmem_alloc(tmem_slot, 256 * FTILES);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  // inputs (FP32 [n][in], in <= 64) -> BF16 columns 0..63 of the activation tile
  for (int q = tid; q < FTILES * FROWS * 64; q += FTHREADS) {
    const int r = q >> 6, k = q & 63;  // r: row of the CTA, tile r / FROWS
    const long long row = m0 + r;
    float v = 0.0f;
    if (row < a.n && k < a.dims[0]) v = a.x[row * a.dims[0] + k];
    *reinterpret_cast<__nv_bfloat16*>(act + (r / FROWS) * F_ACT_BYTES + act_off(r % FROWS, k)) =
        __float2bfloat16_rn(v);
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  WChunk pre;
  load_w(pre, wbf + a.w_off[0], a.dims[1], a.dims[0], 0);
  int g = 0;  // weight chunks committed so far; stage = g & 1
  bool failed = false;
  for (int l = 0; l < a.L && !failed; ++l) {
    const int K = a.dims[l], N = a.dims[l + 1];
    const int nch = (K + TBK - 1) / TBK;
    for (int c = 0; c < nch; ++c) {
      const int s = g & 1;
      bool bad = false;
      if (g >= 2 && !mbar_wait_bounded(&bar[s], ((g - 2) >> 1) & 1, kTcWaitLimit)) {
        bad = true;
        atomicExch(a.err, 1);
      }
      if (!bad) store_w(sW + s * F_W_BYTES, pre, N);
      fence_proxy_async_smem();
      if (__syncthreads_or(bad)) {
        failed = true;
        break;
      }
      if (c + 1 < nch)
        load_w(pre, wbf + a.w_off[l], N, K, (c + 1) * TBK);
      else if (l + 1 < a.L)
        load_w(pre, wbf + a.w_off[l + 1], a.dims[l + 2], a.dims[l + 1], 0);
      if (tid == 0) {
        tc_fence_after();
        const uint32_t b0 = smem_u32(sW + s * F_W_BYTES);
#pragma unroll
        for (int t = 0; t < FTILES; ++t) {
          const uint32_t a0 = smem_u32(act + t * F_ACT_BYTES);
#pragma unroll
          for (int j = 0; j < TBK / 16; ++j)
            umma_bf16(tmem + (uint32_t)(t * 256), smem_desc_sbo(a0 + (uint32_t)(c * 8 + 2 * j) * 128u,
                                                                 FACT_K / 8 * 128),
                      smem_desc_sbo(b0 + (uint32_t)j * 256u, TBK / 8 * 128), instr_desc_n(N),
                      (c > 0 || j > 0) ? 1u : 0u);
        }
        umma_commit(&bar[s]);
      }
      ++g;
    }
    if (failed) break;
    bool late = !mbar_wait_bounded(&bar[(g - 1) & 1], ((g - 1) >> 1) & 1, kTcWaitLimit);
    if (late) atomicExch(a.err, 1);
    if (__syncthreads_or(late)) {
      failed = true;
      break;
    }
    tc_fence_after();
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (rows of its tile) of tile w / 4
    const int q4 = warp & 3, t = warp >> 2;
    const int r = q4 * 32 + lane;
    const long long row = m0 + t * FROWS + r;
    uint8_t* tact = act + t * F_ACT_BYTES;
    const float* bias = prm + a.b_off[l];
    const bool last = l + 1 == a.L;
#pragma unroll 1
    for (int c0 = 0; c0 < N; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(t * 256 + c0), v);
      tmem_wait_ld();
      if (!last) {
#pragma unroll
        for (int q = 0; q < 32; q += 8) {
          __nv_bfloat16 h[8];
#pragma unroll
          for (int u = 0; u < 8; ++u)
            h[u] = __float2bfloat16_rn(gelu(__uint_as_float(v[q + u]) + bias[c0 + q + u]));
          uint4 w;
          memcpy(&w, h, 16);
          *reinterpret_cast<uint4*>(tact + act_off(r, c0 + q)) = w;
        }
      } else if (row < a.n) {
        float* o = a.out + e * a.out_stride + row * N + c0;
#pragma unroll
        for (int q = 0; q < 32; q += 4)
          *reinterpret_cast<float4*>(o + q) =
              make_float4(__uint_as_float(v[q]) + bias[c0 + q], __uint_as_float(v[q + 1]) + bias[c0 + q + 1],
                          __uint_as_float(v[q + 2]) + bias[c0 + q + 2],
                          __uint_as_float(v[q + 3]) + bias[c0 + q + 3]);
      }
    }
    fence_proxy_async_smem();  // the new activations are the next MMAs' operand
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (failed && g > 0) {  // let what was issued finish before the accumulator is released
    (void)mbar_wait_bounded(&bar[(g - 1) & 1], ((g - 1) >> 1) & 1, kTcWaitLimit);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256 * FTILES);
}

}  // namespace

template <bool TA, bool TB, int EPI>
cudaError_t launch_gemm_tc(int M, int N, int K, const Operand& A, const Operand& B,
                           const Epilogue& ep, int members, cudaStream_t st, int* err) {
  if (M < 1 || N < 1 || K < 1 || members < 1) return cudaErrorInvalidValue;
  if (N <= 64) return launch_bn<TA, TB, EPI, 64>(M, N, K, A, B, ep, members, st, err);
  return launch_bn<TA, TB, EPI, 128>(M, N, K, A, B, ep, members, st, err);
}

// The instances the MLP uses: forward (X W^T; training keeps Z, inference only the BF16
// activation), weight gradient (G^T X), input gradient (G W).
template cudaError_t launch_gemm_tc<false, false, kBiasGelu>(int, int, int, const Operand&,
                                                             const Operand&, const Epilogue&, int,
                                                             cudaStream_t, int*);
template cudaError_t launch_gemm_tc<false, false, kBiasGeluAct>(int, int, int, const Operand&,
                                                                const Operand&, const Epilogue&,
                                                                int, cudaStream_t, int*);
template cudaError_t launch_gemm_tc<false, false, kBias>(int, int, int, const Operand&,
                                                         const Operand&, const Epilogue&, int,
                                                         cudaStream_t, int*);
template cudaError_t launch_gemm_tc<true, true, kStore>(int, int, int, const Operand&,
                                                        const Operand&, const Epilogue&, int,
                                                        cudaStream_t, int*);
template cudaError_t launch_gemm_tc<false, true, kGeluBack>(int, int, int, const Operand&,
                                                            const Operand&, const Epilogue&, int,
                                                            cudaStream_t, int*);

bool mlp_fused_supported(const int* dims, int L) {
  if (L < 1 || L > kFusedMaxLayers || dims[0] < 1 || dims[0] > 64) return false;
  for (int l = 1; l <= L; ++l)
    if (dims[l] < 32 || dims[l] > FACT_K || dims[l] % 32 != 0) return false;
  return true;
}

cudaError_t launch_mlp_fused(const FusedArgs& a, int members, cudaStream_t st) {
  static std::atomic<unsigned long long> set_on{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (!(set_on.load() & bit) || !bit) {
    e = cudaFuncSetAttribute(mlp_fused_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)F_SMEM);
    if (e != cudaSuccess) return e;
    set_on.fetch_or(bit);
  }
  const dim3 grid((unsigned)((a.n + FROWS * FTILES - 1) / (FROWS * FTILES)), (unsigned)members);
  mlp_fused_infer<<<grid, FTHREADS, F_SMEM, st>>>(a);
  return cudaGetLastError();
}

}  // namespace mlp
}  // namespace fdtd
