// mlp.cu -- the spectrum surrogate: an ensemble of small MLPs trained and run on the GPU.
//
// gDiamond has no learned component; this is the extension that maps a dielectric-box
// parameterisation to a transmission spectrum, trained on spectra the batched FDTD solver
// produces, with FDTD as both the fallback and the ground truth for its error.
//
// Network per member: x -> [Linear -> GELU] x (L-1) -> Linear -> y, mean-squared-error loss.
// FP32 master weights (updated by Adam) and BF16 copies (the GEMM operands); activations that
// feed a GEMM are BF16; every GEMM accumulates in FP32 on the tensor cores.  All members of the
// ensemble run in the same launches (blockIdx.z = member), each on its own minibatch.
//
// Two GEMM paths compute the same products: tcgen05.mma with a TMEM accumulator (mlp_tc.cu) and
// the warp-level mma.sync.m16n8k16 kernel below.  The default (AUTO) runs products of >= 1024
// rows on the first and the 64-row minibatch products of training on the second;
// fdtd_mlp_set_gemm forces either (the tests cross-check them).  Inference (predict) on the
// tcgen05 path runs all layers in one fused kernel when the widths allow (mlp_tc.cu).
//
// GEMM: C[M][N] = sum_k opA(m,k) opB(n,k), opX(r,k) = TX ? X[k*ld + r] : X[r*ld + k], so one
// kernel serves the forward pass (X W^T), the input gradient (G W) and the weight gradient
// (G^T X).  mma.sync path: 64x64 CTA tiles (4 warps of 32x32), K in steps of 32 with the next
// step's tile prefetched into registers, zero fill outside the matrices.  Fused epilogues:
//   kStore      C = acc                                   (weight gradients)
//   kBias       Z = acc + b                               (output layer)
//   kBiasGelu   Z = acc + b, A = bf16(GELU(Z))            (hidden layers, training)
//   kBiasGeluAct A = bf16(GELU(acc + b))                  (hidden layers, inference)
//   kGeluBack   G = acc * GELU'(Zp), Gbf = bf16(G)        (gradient through a hidden layer)
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/fdtd_capi.h"
#include "mlp.cuh"

namespace fdtd {
namespace mlp {

constexpr int BM = 64, BN = 64, BK = 32, KP = BK + 8;  // smem row: 32 bf16 + 8 pad (80 B)
// One thread's share of a 64 x 32 tile of op(X): two 16-byte chunks of 8 elements.
struct Chunk {
  uint4 v[2];
};

template <bool T>
__device__ __forceinline__ void load_tile(Chunk& c, const Operand& X, const __nv_bfloat16* base,
                                          int R, int K, int r0, int k0) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int id = tid + it * 128;
    // !T: row r0 + id/4, k0 + (id%4)*8 .. +8;   T: k row k0 + id/8, rows r0 + (id%8)*8 .. +8
    const int gr = T ? r0 + (id & 7) * 8 : r0 + (id >> 2);
    const int gk = T ? k0 + (id >> 3) : k0 + (id & 3) * 8;
    __nv_bfloat16 e[8];
    if (!T) {
      if (X.vec && gr < R && gk + 8 <= K) {
        c.v[it] = *reinterpret_cast<const uint4*>(base + (long long)gr * X.ld + gk);
        continue;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q)
        e[q] = (gr < R && gk + q < K) ? base[(long long)gr * X.ld + gk + q]
                                      : __float2bfloat16(0.0f);
    } else {
      if (X.vec && gk < K && gr + 8 <= R) {
        c.v[it] = *reinterpret_cast<const uint4*>(base + (long long)gk * X.ld + gr);
        continue;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q)
        e[q] = (gk < K && gr + q < R) ? base[(long long)gk * X.ld + gr + q]
                                      : __float2bfloat16(0.0f);
    }
    memcpy(&c.v[it], e, 16);
  }
}

template <bool T>
__device__ __forceinline__ void store_tile(__nv_bfloat16 (*s)[KP], const Chunk& c) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int id = tid + it * 128;
    if (!T) {
      *reinterpret_cast<uint4*>(&s[id >> 2][(id & 3) * 8]) = c.v[it];
    } else {
      __nv_bfloat16 e[8];
      memcpy(e, &c.v[it], 16);
      const int kk = id >> 3, r = (id & 7) * 8;
#pragma unroll
      for (int q = 0; q < 8; ++q) s[r + q][kk] = e[q];
    }
  }
}

template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(128) gemm_bf16(int M, int N, int K, Operand A, Operand B,
                                                 Epilogue ep) {
  __shared__ __align__(16) __nv_bfloat16 sA[BM][KP];
  __shared__ __align__(16) __nv_bfloat16 sB[BN][KP];
  const int e = blockIdx.z;
  const __nv_bfloat16* Ab = A.p + e * A.stride;
  const __nv_bfloat16* Bb = B.p + e * B.stride;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int gid = lane >> 2, tig = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0f;

  Chunk ca, cb;
  load_tile<TA>(ca, A, Ab, M, K, m0, 0);
  load_tile<TB>(cb, B, Bb, N, K, n0, 0);
  for (int k0 = 0; k0 < K; k0 += BK) {
    store_tile<TA>(sA, ca);
    store_tile<TB>(sB, cb);
    __syncthreads();
    if (k0 + BK < K) {  // prefetch the next step while this one computes
      load_tile<TA>(ca, A, Ab, M, K, m0, k0 + BK);
      load_tile<TB>(cb, B, Bb, N, K, n0, k0 + BK);
    }
#pragma unroll
    for (int ks = 0; ks < BK; ks += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + gid;
        af[i][0] = *reinterpret_cast<const uint32_t*>(&sA[r][ks + tig * 2]);
        af[i][1] = *reinterpret_cast<const uint32_t*>(&sA[r + 8][ks + tig * 2]);
        af[i][2] = *reinterpret_cast<const uint32_t*>(&sA[r][ks + tig * 2 + 8]);
        af[i][3] = *reinterpret_cast<const uint32_t*>(&sA[r + 8][ks + tig * 2 + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + j * 8 + gid;
        bfr[j][0] = *reinterpret_cast<const uint32_t*>(&sB[c][ks + tig * 2]);
        bfr[j][1] = *reinterpret_cast<const uint32_t*>(&sB[c][ks + tig * 2 + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
              "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
              : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
              : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bfr[j][0]),
                "r"(bfr[j][1]));
    }
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = m0 + wm + i * 16 + gid + h * 8;
        if (r >= M) continue;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int c = n0 + wn + j * 8 + tig * 2 + q;
          if (c < N) epilogue_store<EPI>(ep, e, r, c, acc[i][j][h * 2 + q]);
        }
      }
}

// Member e's minibatch: rows perm[e][r0 .. r0+M) of X (FP32 [n][in]) as BF16 into act0 and of
// Y ([n][out]) into tgt.
__global__ void gather_batch(int M, int in, int out, long long r0, long long n, const int* perm,
                             const float* X, const float* Y, __nv_bfloat16* act0,
                             long long act0_stride, float* tgt, long long tgt_stride) {
  const int e = blockIdx.y;
  const int w = in + out;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M * w; i += gridDim.x * blockDim.x) {
    const int r = i / w, c = i % w;
    const long long src = perm[e * n + r0 + r];
    if (c < in)
      act0[e * act0_stride + (long long)r * in + c] = __float2bfloat16_rn(X[src * in + c]);
    else
      tgt[e * tgt_stride + (long long)r * out + (c - in)] = Y[src * out + (c - in)];
  }
}

// G = 2 (Y - T) / (M * N) in FP32 and BF16, and each member's summed squared error added to
// loss[e] (when given).
__global__ void mse_grad(int M, int N, const float* Y, long long y_stride, const float* T,
                         long long t_stride, float* G, __nv_bfloat16* Gbf, long long g_stride,
                         float* loss) {
  const int e = blockIdx.y;
  float s = 0.0f;
  const float scale = 2.0f / ((float)M * (float)N);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M * N; i += gridDim.x * blockDim.x) {
    const float d = Y[e * y_stride + i] - T[e * t_stride + i];
    s += d * d;
    const float g = scale * d;
    G[e * g_stride + i] = g;
    Gbf[e * g_stride + i] = __float2bfloat16_rn(g);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(&loss[e], s);
}

// db[e][c] = sum_r G[e][r][c], summed in row order (deterministic).
__global__ void col_sum(int M, int N, const float* G, long long g_stride, float* db,
                        long long db_stride) {
  const int e = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  float s = 0.0f;
  for (int r = 0; r < M; ++r) s += G[e * g_stride + (long long)r * N + c];
  db[e * db_stride + c] = s;
}

// One Adam step on every member's parameters (bias corrections c1 = 1 - b1^t, c2 = 1 - b2^t),
// refreshing the BF16 copies.
__global__ void adam_step(long long n, float* w, const float* g, float* m, float* v,
                          __nv_bfloat16* wbf, float lr, float b1, float b2, float eps, float c1,
                          float c2) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  wbf[i] = __float2bfloat16_rn(wi);
}

__global__ void to_bf16(long long n, const float* x, __nv_bfloat16* y) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

// Mean and population standard deviation over the members.
__global__ void ens_stats(long long n, int members, const float* Y, long long stride, float* mean,
                          float* sd) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.0f;
  for (int e = 0; e < members; ++e) s += Y[e * stride + i];
  const float mu = s / members;
  float q = 0.0f;
  for (int e = 0; e < members; ++e) {
    const float d = Y[e * stride + i] - mu;
    q += d * d;
  }
  mean[i] = mu;
  sd[i] = sqrtf(q / members);
}

inline unsigned nblocks(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace mlp
}  // namespace fdtd

// ============================================================================ host side

using fdtd::mlp::Epilogue;
using fdtd::mlp::Operand;

struct fdtd_mlp {
  int device = 0;
  std::vector<int> dims;  // layer widths: dims[0] inputs ... dims[L] outputs
  int L = 0, E = 1, W = 0;
  long long P = 0;                      // parameters per member
  std::vector<long long> w_off, b_off;  // offsets of W_l ([out][in], row-major) and b_l
  cudaStream_t st = nullptr;
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;  // [E][P]
  __nv_bfloat16* wbf = nullptr;                                                      // [E][P]
  long long adam_t = 0;  // Adam steps taken
  float* X = nullptr;    // training inputs [n][in]
  float* Y = nullptr;    // training targets [n][out]
  long long n = 0;
  // workspace for minibatches of up to `cap` rows per member
  long long cap = 0;
  std::vector<__nv_bfloat16*> act;  // act[l]: [E][cap][dims[l]]   (input of layer l)
  std::vector<float*> z;            // z[l]:   [E][cap][dims[l+1]] (pre-activation of layer l)
  float* g[2] = {nullptr, nullptr};           // gradients wrt a pre-activation [E][cap][W]
  __nv_bfloat16* gbf[2] = {nullptr, nullptr};  // their BF16 copies
  float* tgt = nullptr;                        // [E][cap][out]
  float* xin = nullptr;                        // FP32 input staging [cap][in]
  int gemm_kind = FDTD_MLP_GEMM_AUTO;
  mutable cudaError_t launch_err = cudaSuccess;  // first failed tcgen05 launch set-up
  int* d_err = nullptr;  // nonzero when a bounded wait in a GEMM kernel gave up
  std::string err;
};

namespace {

fdtd_status mfail(fdtd_mlp* m, fdtd_status s, const std::string& what) {
  if (m) m->err = what;
  return s;
}

#define MCUDA(m, call)                                                               \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) return mfail((m), FDTD_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

void free_workspace(fdtd_mlp* m) {
  for (auto p : m->act) cudaFree(p);
  for (auto p : m->z) cudaFree(p);
  m->act.clear();
  m->z.clear();
  for (int i = 0; i < 2; ++i) {
    cudaFree(m->g[i]);
    cudaFree(m->gbf[i]);
    m->g[i] = nullptr;
    m->gbf[i] = nullptr;
  }
  cudaFree(m->tgt);
  cudaFree(m->xin);
  m->tgt = nullptr;
  m->xin = nullptr;
  m->cap = 0;
}

fdtd_status ensure_cap(fdtd_mlp* m, long long rows) {
  if (rows <= m->cap) return FDTD_OK;
  MCUDA(m, cudaStreamSynchronize(m->st));
  free_workspace(m);
  m->act.assign(m->L + 1, nullptr);
  m->z.assign(m->L, nullptr);
  const long long E = m->E;
  for (int l = 0; l <= m->L; ++l)
    MCUDA(m, cudaMalloc(&m->act[l], E * rows * m->dims[l] * sizeof(__nv_bfloat16)));
  for (int l = 0; l < m->L; ++l)
    MCUDA(m, cudaMalloc(&m->z[l], E * rows * m->dims[l + 1] * sizeof(float)));
  for (int i = 0; i < 2; ++i) {
    MCUDA(m, cudaMalloc(&m->g[i], E * rows * m->W * sizeof(float)));
    MCUDA(m, cudaMalloc(&m->gbf[i], E * rows * m->W * sizeof(__nv_bfloat16)));
  }
  MCUDA(m, cudaMalloc(&m->tgt, E * rows * m->dims[m->L] * sizeof(float)));
  MCUDA(m, cudaMalloc(&m->xin, rows * m->dims[0] * sizeof(float)));
  m->cap = rows;
  return FDTD_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

Operand operand(const __nv_bfloat16* p, int ld, long long stride) {
  return {p, ld, stride, ld % 8 == 0 && stride % 8 == 0 && aligned16(p)};
}

template <bool TA, bool TB, int EPI>
void gemm(const fdtd_mlp* m, int M, int N, int K, const Operand& A, const Operand& B,
          const Epilogue& ep) {
  // AUTO: the tensor-memory path for tall products; the warp-level kernel for the short
  // minibatch products of training, where a 128-row tile would be half empty.
  const bool tc = m->gemm_kind == FDTD_MLP_GEMM_TCGEN05 ||
                  (m->gemm_kind == FDTD_MLP_GEMM_AUTO && M >= 1024);
  if (tc) {
    const cudaError_t e =
        fdtd::mlp::launch_gemm_tc<TA, TB, EPI>(M, N, K, A, B, ep, m->E, m->st, m->d_err);
    if (e != cudaSuccess && m->launch_err == cudaSuccess) m->launch_err = e;
    return;
  }
  const dim3 grid((N + fdtd::mlp::BN - 1) / fdtd::mlp::BN, (M + fdtd::mlp::BM - 1) / fdtd::mlp::BM,
                  m->E);
  fdtd::mlp::gemm_bf16<TA, TB, EPI><<<grid, 128, 0, m->st>>>(M, N, K, A, B, ep);
}

// After a synchronisation: launch errors and the GEMMs' device error word.
fdtd_status check_after(fdtd_mlp* m) {
  if (m->launch_err != cudaSuccess) {
    const cudaError_t le = m->launch_err;
    m->launch_err = cudaSuccess;
    return mfail(m, FDTD_ERR_CUDA, cudaGetErrorString(le));
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mfail(m, FDTD_ERR_CUDA, cudaGetErrorString(e));
  int w = 0;
  if (cudaMemcpy(&w, m->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return mfail(m, FDTD_ERR_CUDA, "reading the device error word failed");
  if (w) {
    cudaMemset(m->d_err, 0, sizeof(int));
    return mfail(m, FDTD_ERR_DEVICE_TIMEOUT,
                 "a bounded wait in a tensor-core GEMM expired; results are invalid");
  }
  return FDTD_OK;
}

// Forward pass of every member on M rows of act[0] (member stride act0_stride; 0 when all
// members see the same rows).  The output layer's result is z[L-1].
void forward(fdtd_mlp* m, int M, long long act0_stride, bool keep_z = true) {
  for (int l = 0; l < m->L; ++l) {
    const int in = m->dims[l], out = m->dims[l + 1];
    const long long sa = l == 0 ? act0_stride : m->cap * in;
    const Operand A = operand(m->act[l], in, sa);
    const Operand B = operand(m->wbf + m->w_off[l], in, m->P);
    Epilogue ep{};
    ep.out = m->z[l];
    ep.ldc = out;
    ep.stride_out = m->cap * out;
    ep.bias = m->params + m->b_off[l];
    ep.stride_bias = m->P;
    if (l + 1 < m->L) {
      ep.out_bf = m->act[l + 1];
      if (keep_z)
        gemm<false, false, fdtd::mlp::kBiasGelu>(m, M, out, in, A, B, ep);
      else
        gemm<false, false, fdtd::mlp::kBiasGeluAct>(m, M, out, in, A, B, ep);
    } else {
      gemm<false, false, fdtd::mlp::kBias>(m, M, out, in, A, B, ep);
    }
  }
}

// Backward pass after forward(): mean-squared error against tgt (member stride tgt_stride),
// every member's gradient into grads, summed squared errors added to loss[E] when given.
void backward(fdtd_mlp* m, int M, long long act0_stride, long long tgt_stride, float* loss) {
  const int out = m->dims[m->L];
  const long long gs = m->cap * m->W;
  const unsigned mb = std::min<unsigned>(fdtd::mlp::nblocks((long long)M * out), 64u);
  fdtd::mlp::mse_grad<<<dim3(mb, m->E), 256, 0, m->st>>>(M, out, m->z[m->L - 1], m->cap * out,
                                                         m->tgt, tgt_stride, m->g[0], m->gbf[0],
                                                         gs, loss);
  int cur = 0;
  for (int l = m->L - 1; l >= 0; --l) {
    const int in = m->dims[l], o = m->dims[l + 1];
    const long long sa = l == 0 ? act0_stride : m->cap * in;
    {  // dW_l [o][in] = G^T X_l
      const Operand A = operand(m->gbf[cur], o, gs);
      const Operand B = operand(m->act[l], in, sa);
      Epilogue ep{};
      ep.out = m->grads + m->w_off[l];
      ep.ldc = in;
      ep.stride_out = m->P;
      gemm<true, true, fdtd::mlp::kStore>(m, o, in, M, A, B, ep);
    }
    fdtd::mlp::col_sum<<<dim3(fdtd::mlp::nblocks(o, 128), m->E), 128, 0, m->st>>>(
        M, o, m->g[cur], gs, m->grads + m->b_off[l], m->P);
    if (l > 0) {  // G_{l-1} [M][in] = (G_l W_l) * GELU'(z[l-1])
      const Operand A = operand(m->gbf[cur], o, gs);
      const Operand B = operand(m->wbf + m->w_off[l], in, m->P);
      Epilogue ep{};
      ep.out = m->g[cur ^ 1];
      ep.out_bf = m->gbf[cur ^ 1];
      ep.zp = m->z[l - 1];
      ep.stride_zp = m->cap * in;
      ep.ldc = in;
      ep.stride_out = gs;
      gemm<false, true, fdtd::mlp::kGeluBack>(m, M, in, o, A, B, ep);
      cur ^= 1;
    }
  }
}

void destroy(fdtd_mlp* m) {
  if (m->st) cudaStreamSynchronize(m->st);
  free_workspace(m);
  cudaFree(m->params);
  cudaFree(m->grads);
  cudaFree(m->adam_m);
  cudaFree(m->adam_v);
  cudaFree(m->wbf);
  cudaFree(m->d_err);
  cudaFree(m->X);
  cudaFree(m->Y);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
}

// Runs the ensemble on n rows of FP32 inputs already on the device; mean / sd (device, n*out)
// and optionally every member's output (device, [E][n][out]).
fdtd_status predict_rows(fdtd_mlp* m, const float* x_dev, long long n, float* mean, float* sd,
                         float* per_member) {
  const int in = m->dims[0], out = m->dims[m->L];
  const long long chunk = std::min<long long>(n, 65536);
  fdtd_status s = ensure_cap(m, chunk);
  if (s != FDTD_OK) return s;
  const bool fused = m->gemm_kind != FDTD_MLP_GEMM_MMA_SYNC && m->L <= fdtd::mlp::kFusedMaxLayers &&
                     fdtd::mlp::mlp_fused_supported(m->dims.data(), m->L);
  for (long long r0 = 0; r0 < n; r0 += chunk) {
    const long long cnt = std::min<long long>(chunk, n - r0);
    if (fused) {  // every layer in one kernel: activations never leave the SM
      fdtd::mlp::FusedArgs fa{};
      fa.x = x_dev + r0 * in;
      fa.n = cnt;
      fa.L = m->L;
      for (int l = 0; l <= m->L; ++l) fa.dims[l] = m->dims[l];
      for (int l = 0; l < m->L; ++l) {
        fa.w_off[l] = m->w_off[l];
        fa.b_off[l] = m->b_off[l];
      }
      fa.wbf = m->wbf;
      fa.params = m->params;
      fa.P = m->P;
      fa.out = m->z[m->L - 1];
      fa.out_stride = m->cap * out;
      fa.err = m->d_err;
      const cudaError_t le = fdtd::mlp::launch_mlp_fused(fa, m->E, m->st);
      if (le != cudaSuccess && m->launch_err == cudaSuccess) m->launch_err = le;
    } else {
      fdtd::mlp::to_bf16<<<fdtd::mlp::nblocks(cnt * in), 256, 0, m->st>>>(
          cnt * in, x_dev + r0 * in, m->act[0]);
      forward(m, (int)cnt, 0, /*keep_z=*/false);
    }
    fdtd::mlp::ens_stats<<<fdtd::mlp::nblocks(cnt * out), 256, 0, m->st>>>(
        cnt * out, m->E, m->z[m->L - 1], m->cap * out, mean + r0 * out, sd + r0 * out);
    if (per_member)
      for (int e = 0; e < m->E; ++e)
        MCUDA(m, cudaMemcpyAsync(per_member + ((long long)e * n + r0) * out,
                                 m->z[m->L - 1] + e * m->cap * out, cnt * out * sizeof(float),
                                 cudaMemcpyDeviceToDevice, m->st));
  }
  MCUDA(m, cudaGetLastError());
  return FDTD_OK;
}

}  // namespace

extern "C" {

fdtd_status fdtd_mlp_create(const int32_t* dims, int32_t n_dims, int32_t members, uint64_t seed,
                            int32_t device, fdtd_mlp** out) {
  if (!dims || !out || n_dims < 2 || n_dims > 16 || members < 1 || members > 64)
    return FDTD_ERR_INVALID_ARG;
  for (int i = 0; i < n_dims; ++i)
    if (dims[i] < 1 || dims[i] > 8192) return FDTD_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return FDTD_ERR_CUDA;
  fdtd_mlp* m = new fdtd_mlp();
  m->device = device;
  m->dims.assign(dims, dims + n_dims);
  m->L = n_dims - 1;
  m->E = members;
  m->W = *std::max_element(m->dims.begin(), m->dims.end());
  long long off = 0;
  for (int l = 0; l < m->L; ++l) {
    m->w_off.push_back(off);
    off += (long long)dims[l] * dims[l + 1];
    off = (off + 7) / 8 * 8;  // keep every block 16-byte aligned in BF16
    m->b_off.push_back(off);
    off += dims[l + 1];
    off = (off + 7) / 8 * 8;
  }
  m->P = off;
  const long long tot = off * members;
  if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&m->params, tot * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->grads, tot * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->adam_m, tot * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->adam_v, tot * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->wbf, tot * sizeof(__nv_bfloat16)) != cudaSuccess ||
      cudaMalloc(&m->d_err, sizeof(int)) != cudaSuccess ||
      cudaMemset(m->d_err, 0, sizeof(int)) != cudaSuccess) {
    destroy(m);
    return FDTD_ERR_OOM;
  }
  // He initialisation (normal, std sqrt(2 / fan_in)), zero biases, a seed per member.
  std::vector<float> host(tot, 0.0f);
  for (int e = 0; e < members; ++e) {
    std::mt19937_64 rng(seed * 1000003ull + (uint64_t)e);
    for (int l = 0; l < m->L; ++l) {
      std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (float)dims[l]));
      float* w = host.data() + (long long)e * off + m->w_off[l];
      for (long long i = 0; i < (long long)dims[l] * dims[l + 1]; ++i) w[i] = nd(rng);
    }
  }
  bool ok = cudaMemcpy(m->params, host.data(), tot * sizeof(float), cudaMemcpyHostToDevice) ==
                cudaSuccess &&
            cudaMemset(m->grads, 0, tot * sizeof(float)) == cudaSuccess &&
            cudaMemset(m->adam_m, 0, tot * sizeof(float)) == cudaSuccess &&
            cudaMemset(m->adam_v, 0, tot * sizeof(float)) == cudaSuccess;
  if (ok) {
    fdtd::mlp::to_bf16<<<fdtd::mlp::nblocks(tot), 256, 0, m->st>>>(tot, m->params, m->wbf);
    ok = cudaStreamSynchronize(m->st) == cudaSuccess;
  }
  if (!ok) {
    destroy(m);
    return FDTD_ERR_CUDA;
  }
  *out = m;
  return FDTD_OK;
}

fdtd_status fdtd_mlp_set_gemm(fdtd_mlp* m, int32_t kind) {
  if (!m || kind < FDTD_MLP_GEMM_TCGEN05 || kind > FDTD_MLP_GEMM_AUTO)
    return FDTD_ERR_INVALID_ARG;
  m->gemm_kind = kind;
  return FDTD_OK;
}

fdtd_status fdtd_mlp_destroy(fdtd_mlp* m) {
  if (!m) return FDTD_ERR_INVALID_ARG;
  destroy(m);
  return FDTD_OK;
}

const char* fdtd_mlp_last_error(const fdtd_mlp* m) { return m ? m->err.c_str() : ""; }

fdtd_status fdtd_mlp_layout(const fdtd_mlp* m, int64_t* n_params, int64_t* w_off, int64_t* b_off) {
  if (!m || !n_params) return FDTD_ERR_INVALID_ARG;
  *n_params = m->P;
  for (int l = 0; l < m->L; ++l) {
    if (w_off) w_off[l] = m->w_off[l];
    if (b_off) b_off[l] = m->b_off[l];
  }
  return FDTD_OK;
}

fdtd_status fdtd_mlp_get_params(fdtd_mlp* m, float* out) {
  if (!m || !out) return FDTD_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  MCUDA(m, cudaStreamSynchronize(m->st));
  MCUDA(m, cudaMemcpy(out, m->params, m->E * m->P * sizeof(float), cudaMemcpyDeviceToHost));
  return FDTD_OK;
}

fdtd_status fdtd_mlp_set_params(fdtd_mlp* m, const float* in) {
  if (!m || !in) return FDTD_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  const long long tot = m->E * m->P;
  MCUDA(m, cudaStreamSynchronize(m->st));
  MCUDA(m, cudaMemcpy(m->params, in, tot * sizeof(float), cudaMemcpyHostToDevice));
  fdtd::mlp::to_bf16<<<fdtd::mlp::nblocks(tot), 256, 0, m->st>>>(tot, m->params, m->wbf);
  MCUDA(m, cudaMemsetAsync(m->adam_m, 0, tot * sizeof(float), m->st));
  MCUDA(m, cudaMemsetAsync(m->adam_v, 0, tot * sizeof(float), m->st));
  m->adam_t = 0;
  MCUDA(m, cudaStreamSynchronize(m->st));
  return FDTD_OK;
}

fdtd_status fdtd_mlp_set_data(fdtd_mlp* m, const float* x, const float* y, int64_t n) {
  if (!m || !x || !y || n < 1 || n > (int64_t)1 << 30) return FDTD_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  MCUDA(m, cudaStreamSynchronize(m->st));
  cudaFree(m->X);
  cudaFree(m->Y);
  m->X = m->Y = nullptr;
  m->n = 0;
  const int in = m->dims[0], out = m->dims[m->L];
  MCUDA(m, cudaMalloc(&m->X, n * in * sizeof(float)));
  MCUDA(m, cudaMalloc(&m->Y, n * out * sizeof(float)));
  MCUDA(m, cudaMemcpy(m->X, x, n * in * sizeof(float), cudaMemcpyHostToDevice));
  MCUDA(m, cudaMemcpy(m->Y, y, n * out * sizeof(float), cudaMemcpyHostToDevice));
  m->n = n;
  return FDTD_OK;
}

fdtd_status fdtd_mlp_grad(fdtd_mlp* m, const float* x, const float* y, int64_t n, float* loss,
                          float* grads) {
  if (!m || !x || !y || n < 1 || n > (1 << 20)) return FDTD_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  fdtd_status s = ensure_cap(m, n);
  if (s != FDTD_OK) return s;
  const int in = m->dims[0], out = m->dims[m->L];
  float* dloss = nullptr;
  MCUDA(m, cudaMalloc(&dloss, m->E * sizeof(float)));
  MCUDA(m, cudaMemsetAsync(dloss, 0, m->E * sizeof(float), m->st));
  MCUDA(m, cudaMemcpyAsync(m->xin, x, n * in * sizeof(float), cudaMemcpyHostToDevice, m->st));
  MCUDA(m, cudaMemcpyAsync(m->tgt, y, n * out * sizeof(float), cudaMemcpyHostToDevice, m->st));
  fdtd::mlp::to_bf16<<<fdtd::mlp::nblocks(n * in), 256, 0, m->st>>>(n * in, m->xin, m->act[0]);
  forward(m, (int)n, 0);
  backward(m, (int)n, 0, 0, dloss);
  std::vector<float> hl(m->E);
  cudaMemcpyAsync(hl.data(), dloss, m->E * sizeof(float), cudaMemcpyDeviceToHost, m->st);
  if (grads)
    cudaMemcpyAsync(grads, m->grads, m->E * m->P * sizeof(float), cudaMemcpyDeviceToHost, m->st);
  const cudaError_t e = cudaStreamSynchronize(m->st);
  cudaFree(dloss);
  if (e != cudaSuccess) return mfail(m, FDTD_ERR_CUDA, cudaGetErrorString(e));
  if ((s = check_after(m)) != FDTD_OK) return s;
  if (loss)
    for (int i = 0; i < m->E; ++i) loss[i] = (float)((double)hl[i] / ((double)n * out));
  return FDTD_OK;
}

fdtd_status fdtd_mlp_train(fdtd_mlp* m, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                           float* loss_out) {
  if (!m || epochs < 1 || batch < 1 || batch > (1 << 20) || !(lr > 0.0f))
    return FDTD_ERR_INVALID_ARG;
  if (!m->X) return mfail(m, FDTD_ERR_INVALID_ARG, "fdtd_mlp_train: no training data");
  MCUDA(m, cudaSetDevice(m->device));
  const int in = m->dims[0], out = m->dims[m->L];
  const long long n = m->n;
  const int mb = (int)std::min<long long>(batch, n);
  fdtd_status s = ensure_cap(m, mb);
  if (s != FDTD_OK) return s;
  int* perm = nullptr;
  float* dloss = nullptr;
  MCUDA(m, cudaMalloc(&perm, (long long)m->E * n * sizeof(int)));
  MCUDA(m, cudaMalloc(&dloss, (long long)epochs * m->E * sizeof(float)));
  MCUDA(m, cudaMemsetAsync(dloss, 0, (long long)epochs * m->E * sizeof(float), m->st));
  std::vector<int> hp((size_t)m->E * n);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  cudaError_t err = cudaSuccess;
  for (int ep = 0; ep < epochs && err == cudaSuccess; ++ep) {
    for (int e = 0; e < m->E; ++e) {  // each member its own shuffle
      int* p = hp.data() + (size_t)e * n;
      std::iota(p, p + n, 0);
      std::mt19937_64 rng(seed * 0x9E3779B97F4A7C15ull + (uint64_t)ep * 1315423911ull + e);
      std::shuffle(p, p + n, rng);
    }
    // the previous epoch's gathers are stream-ordered before this copy
    err = cudaMemcpyAsync(perm, hp.data(), hp.size() * sizeof(int), cudaMemcpyHostToDevice, m->st);
    for (long long r0 = 0; r0 < n && err == cudaSuccess; r0 += mb) {
      const int M = (int)std::min<long long>(mb, n - r0);
      fdtd::mlp::gather_batch<<<dim3(std::min<unsigned>(fdtd::mlp::nblocks((long long)M * (in + out)), 128u),
                                     m->E),
                                256, 0, m->st>>>(M, in, out, r0, n, perm, m->X, m->Y, m->act[0],
                                                 m->cap * in, m->tgt, m->cap * out);
      forward(m, M, m->cap * in);
      backward(m, M, m->cap * in, m->cap * out, dloss + (long long)ep * m->E);
      ++m->adam_t;
      const float c1 = (float)(1.0 - std::pow((double)b1, (double)m->adam_t));
      const float c2 = (float)(1.0 - std::pow((double)b2, (double)m->adam_t));
      const long long tot = m->E * m->P;
      fdtd::mlp::adam_step<<<fdtd::mlp::nblocks(tot), 256, 0, m->st>>>(
          tot, m->params, m->grads, m->adam_m, m->adam_v, m->wbf, lr, b1, b2, eps, c1, c2);
      err = cudaGetLastError();
    }
    // pageable copies are staged before returning, so hp can be refilled next epoch
  }
  std::vector<float> hl((size_t)epochs * m->E);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(hl.data(), dloss, hl.size() * sizeof(float), cudaMemcpyDeviceToHost, m->st);
  const cudaError_t e2 = cudaStreamSynchronize(m->st);
  cudaFree(perm);
  cudaFree(dloss);
  if (err != cudaSuccess) return mfail(m, FDTD_ERR_CUDA, cudaGetErrorString(err));
  if (e2 != cudaSuccess) return mfail(m, FDTD_ERR_CUDA, cudaGetErrorString(e2));
  if ((s = check_after(m)) != FDTD_OK) return s;
  if (loss_out)
    for (size_t i = 0; i < hl.size(); ++i) loss_out[i] = (float)((double)hl[i] / ((double)n * out));
  return FDTD_OK;
}

fdtd_status fdtd_mlp_predict(fdtd_mlp* m, const float* x, int64_t n, float* mean, float* sd,
                             float* per_member) {
  if (!m || !x || n < 1 || !mean || !sd) return FDTD_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  const int in = m->dims[0], out = m->dims[m->L];
  float *dx = nullptr, *dm = nullptr, *ds = nullptr, *dp = nullptr;
  MCUDA(m, cudaMalloc(&dx, n * in * sizeof(float)));
  MCUDA(m, cudaMalloc(&dm, n * out * sizeof(float)));
  MCUDA(m, cudaMalloc(&ds, n * out * sizeof(float)));
  if (per_member) MCUDA(m, cudaMalloc(&dp, m->E * n * out * sizeof(float)));
  fdtd_status s = FDTD_OK;
  cudaError_t e = cudaMemcpyAsync(dx, x, n * in * sizeof(float), cudaMemcpyHostToDevice, m->st);
  if (e == cudaSuccess) s = predict_rows(m, dx, n, dm, ds, dp);
  if (e == cudaSuccess && s == FDTD_OK) {
    cudaMemcpyAsync(mean, dm, n * out * sizeof(float), cudaMemcpyDeviceToHost, m->st);
    cudaMemcpyAsync(sd, ds, n * out * sizeof(float), cudaMemcpyDeviceToHost, m->st);
    if (per_member)
      cudaMemcpyAsync(per_member, dp, m->E * n * out * sizeof(float), cudaMemcpyDeviceToHost,
                      m->st);
  }
  const cudaError_t e2 = cudaStreamSynchronize(m->st);
  cudaFree(dx);
  cudaFree(dm);
  cudaFree(ds);
  cudaFree(dp);
  if (s != FDTD_OK) return s;
  if (e != cudaSuccess) return mfail(m, FDTD_ERR_CUDA, cudaGetErrorString(e));
  if (e2 != cudaSuccess) return mfail(m, FDTD_ERR_CUDA, cudaGetErrorString(e2));
  return check_after(m);
}

fdtd_status fdtd_mlp_predict_device(fdtd_mlp* m, const float* x_dev, int64_t n, float* mean_dev,
                                    float* sd_dev, void* stream) {
  if (!m || !x_dev || n < 1 || !mean_dev || !sd_dev) return FDTD_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  cudaEvent_t ev;
  MCUDA(m, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaEventRecord(ev, user);
  cudaStreamWaitEvent(m->st, ev, 0);
  const fdtd_status s = predict_rows(m, x_dev, n, mean_dev, sd_dev, nullptr);
  cudaEventRecord(ev, m->st);
  cudaStreamWaitEvent(user, ev, 0);
  cudaEventDestroy(ev);
  return s;
}

}  // extern "C"
