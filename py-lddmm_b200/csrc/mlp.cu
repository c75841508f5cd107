// Kernels of the learned momentum proposal: a per-vertex MLP (BF16 weights and activations, FP32 accumulation) and
// its training step, plus the nearest-target displacement feature.
//
// GEMM: C = op(A) op(B) on the tensor cores with mma.sync.m16n8k16 (bf16 x bf16 -> f32). CTA tile 64x64x32, four
// warps of 32x32; operands staged in padded shared memory (row stride +16 B: conflict-free ldmatrix), transposed
// operands read with ldmatrix.trans, so one kernel covers forward (X W), input gradient (dY W^T) and weight
// gradient (X^T dY). Epilogues fuse bias, ReLU, the ReLU-derivative mask and the BF16 / FP32 store; the weight
// gradient is split over the (long) vertex dimension and reduced in a fixed order (deterministic).
// All dimensions are padded by the caller: M, N multiples of 64, K a multiple of 32.
#include <cuda_bf16.h>

#include "../../include/lddmm_b200.h"
#include "lddmm_common.cuh"

namespace lddmm {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int BM = 64, BN = 64, BK = 32, PAD = 8, THREADS = 128;

enum Epilogue : int {
  kEpiF32 = 0,          // C (f32) = acc                      (split-K partials)
  kEpiBiasF32 = 1,      // C (f32) = acc + bias[n]
  kEpiBiasReluBf16 = 2, // C (bf16) = relu(acc + bias[n])
  kEpiBiasBf16 = 3,     // C (bf16) = acc + bias[n]
  kEpiMaskBf16 = 4,     // C (bf16) = mask[m][n] > 0 ? acc : 0  (ReLU derivative of the forward activation)
};

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const bf16* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const bf16* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Global layouts: A is [M][K] (TA = false) or stored transposed as [K][M] (TA = true);
//                 B is [K][N] (TB = false) or stored transposed as [N][K] (TB = true). C is [M][N] (+ split offset).
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(THREADS) gemm_kernel(int M, int N, int K, int k_split, const bf16* __restrict__ A,
                                                       const bf16* __restrict__ B, const float* __restrict__ bias,
                                                       const bf16* __restrict__ mask, void* __restrict__ C) {
  __shared__ __align__(16) bf16 As[TA ? BK : BM][(TA ? BM : BK) + PAD];
  __shared__ __align__(16) bf16 Bs[TB ? BN : BK][(TB ? BK : BN) + PAD];
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kb = blockIdx.z * k_split;
  const int ke = min(K, kb + k_split);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

  for (int k0 = kb; k0 < ke; k0 += BK) {
#pragma unroll
    for (int it = threadIdx.x; it < (BM * BK) / 8; it += THREADS) {
      if (!TA) {
        const int r = it / (BK / 8), c = (it % (BK / 8)) * 8;
        *reinterpret_cast<uint4*>(&As[r][c]) = *reinterpret_cast<const uint4*>(&A[(size_t)(m0 + r) * K + k0 + c]);
      } else {
        const int r = it / (BM / 8), c = (it % (BM / 8)) * 8;
        *reinterpret_cast<uint4*>(&As[r][c]) = *reinterpret_cast<const uint4*>(&A[(size_t)(k0 + r) * M + m0 + c]);
      }
    }
#pragma unroll
    for (int it = threadIdx.x; it < (BN * BK) / 8; it += THREADS) {
      if (!TB) {
        const int r = it / (BN / 8), c = (it % (BN / 8)) * 8;
        *reinterpret_cast<uint4*>(&Bs[r][c]) = *reinterpret_cast<const uint4*>(&B[(size_t)(k0 + r) * N + n0 + c]);
      } else {
        const int r = it / (BK / 8), c = (it % (BK / 8)) * 8;
        *reinterpret_cast<uint4*>(&Bs[r][c]) = *reinterpret_cast<const uint4*>(&B[(size_t)(n0 + r) * K + k0 + c]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t a[2][4], b[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int mr = wm + mt * 16;
        if (!TA)
          ldsm_x4(a[mt], &As[mr + (lane & 15)][kk + (lane >> 4) * 8]);
        else
          ldsm_x4_t(a[mt], &As[kk + (lane & 7) + (lane >> 4) * 8][mr + ((lane >> 3) & 1) * 8]);
      }
#pragma unroll
      for (int np = 0; np < 2; ++np) {
        const int nc = wn + np * 16;
        uint32_t r[4];
        if (!TB)
          ldsm_x4_t(r, &Bs[kk + (lane & 15)][nc + (lane >> 4) * 8]);
        else
          ldsm_x4(r, &Bs[nc + (lane & 7) + (lane >> 4) * 8][kk + ((lane >> 3) & 1) * 8]);
        b[2 * np][0] = r[0];
        b[2 * np][1] = r[1];
        b[2 * np + 1][0] = r[2];
        b[2 * np + 1][1] = r[3];
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], a[mt], b[nt]);
    }
    __syncthreads();
  }

  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = m0 + wm + mt * 16 + g + 8 * h;
        const int col = n0 + wn + nt * 8 + 2 * t;
        float v0 = acc[mt][nt][2 * h], v1 = acc[mt][nt][2 * h + 1];
        const size_t o = (size_t)row * N + col;
        if (EPI == kEpiF32) {
          float* Cf = reinterpret_cast<float*>(C) + (size_t)blockIdx.z * M * N;
          *reinterpret_cast<float2*>(&Cf[o]) = make_float2(v0, v1);
        } else if (EPI == kEpiBiasF32) {
          v0 += bias[col];
          v1 += bias[col + 1];
          *reinterpret_cast<float2*>(&reinterpret_cast<float*>(C)[o]) = make_float2(v0, v1);
        } else {
          if (EPI == kEpiBiasReluBf16 || EPI == kEpiBiasBf16) {
            v0 += bias[col];
            v1 += bias[col + 1];
          }
          if (EPI == kEpiBiasReluBf16) {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
          }
          if (EPI == kEpiMaskBf16) {
            const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162*>(&mask[o]);
            if (!(__bfloat162float(mk.x) > 0.f)) v0 = 0.f;
            if (!(__bfloat162float(mk.y) > 0.f)) v1 = 0.f;
          }
          *reinterpret_cast<__nv_bfloat162*>(&reinterpret_cast<bf16*>(C)[o]) = __floats2bfloat162_rn(v0, v1);
        }
      }
}

// out[i] = sum_s partials[s][i], fixed order.
__global__ void splitk_reduce_kernel(const float* __restrict__ p, int S, size_t count, float* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float s = 0.f;
  for (int k = 0; k < S; ++k) s += p[(size_t)k * count + i];
  out[i] = s;
}

// db[n] = sum_m dy[m][n] (bf16 input, f32 output), one block per 32 columns, fixed order.
__global__ void colsum_kernel(const bf16* __restrict__ dy, int M, int N, float* __restrict__ db) {
  __shared__ float red[8][33];
  const int col = blockIdx.x * 32 + (threadIdx.x & 31);
  const int ry = threadIdx.x >> 5;
  float s = 0.f;
  if (col < N)
    for (int m = ry; m < M; m += 8) s += __bfloat162float(dy[(size_t)m * N + col]);
  red[ry][threadIdx.x & 31] = s;
  __syncthreads();
  if (ry == 0 && col < N) {
    float t = 0.f;
    for (int k = 0; k < 8; ++k) t += red[k][threadIdx.x & 31];
    db[col] = t;
  }
}

// Two-stage column sums for tall matrices: stage 1, one CTA per (32 columns, kColsumRows rows) writes the chunk's
// column sums (8 row lanes x 32 columns, then the 8 lanes in order) to partial[chunk][col]; stage 2 adds the chunks
// of each column in chunk order. Deterministic; the whole GPU takes part instead of N / 32 CTAs.
constexpr int kColsumRows = 256;
__global__ void colsum_partial_kernel(const bf16* __restrict__ dy, int M, int N, float* __restrict__ partial) {
  __shared__ float red[8][33];
  const int col = blockIdx.x * 32 + (threadIdx.x & 31);
  const int ry = threadIdx.x >> 5;
  const int r0 = blockIdx.y * kColsumRows;
  const int r1 = min(M, r0 + kColsumRows);
  float s = 0.f;
  if (col < N)
    for (int m = r0 + ry; m < r1; m += 8) s += __bfloat162float(dy[(size_t)m * N + col]);
  red[ry][threadIdx.x & 31] = s;
  __syncthreads();
  if (ry == 0 && col < N) {
    float t = 0.f;
    for (int k = 0; k < 8; ++k) t += red[k][threadIdx.x & 31];
    partial[(size_t)blockIdx.y * N + col] = t;
  }
}

__global__ void colsum_final_kernel(const float* __restrict__ partial, int chunks, int N, float* __restrict__ db) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= N) return;
  float t = 0.f;
  for (int c = 0; c < chunks; ++c) t += partial[(size_t)c * N + col];
  db[col] = t;
}

// Squared-error gradient of the first `nout` output columns: dy = 2 w (y - target) for rows < valid, 0 elsewhere;
// per-row losses go to `row_loss` (FP32) for a fixed-order reduction by the host.
__global__ void mse_grad_kernel(const float* __restrict__ y, int M, int N, const float* __restrict__ target, int nout,
                                int valid, float w, bf16* __restrict__ dy, float* __restrict__ row_loss) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= M) return;
  float l = 0.f;
  for (int c = 0; c < N; ++c) {
    float g = 0.f;
    if (c < nout && r < valid) {
      const float d = y[(size_t)r * N + c] - target[(size_t)r * nout + c];
      l += d * d;
      g = 2.f * w * d;
    }
    dy[(size_t)r * N + c] = __float2bfloat16_rn(g);
  }
  row_loss[r] = l;
}

// Adam on FP32 master weights; writes the BF16 copy used by the GEMMs.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, bf16* __restrict__ pb, size_t count, float lr, float b1, float b2,
                            float eps, float c1, float c2, float wd) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i] + wd * p[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi;
  const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  const float v = p[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
  p[i] = v;
  if (pb) pb[i] = __float2bfloat16_rn(v);
}

// disp[k] = tgt[argmin_l |src_k - tgt_l|] - src_k (FP32 distances, FP64 output); ties -> lowest index.
__global__ void nearest_kernel(const double* __restrict__ src, int n, const double* __restrict__ tgt, int m,
                               double* __restrict__ disp) {
  __shared__ float4 sm[256];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int kk = k < n ? k : n - 1;
  const float y0 = (float)src[3 * kk], y1 = (float)src[3 * kk + 1], y2 = (float)src[3 * kk + 2];
  float best = 3.4e38f;
  int arg = 0;
  for (int l0 = 0; l0 < m; l0 += blockDim.x) {
    const int l = l0 + threadIdx.x;
    if (l < m) sm[threadIdx.x] = make_float4((float)tgt[3 * l], (float)tgt[3 * l + 1], (float)tgt[3 * l + 2], 0.f);
    __syncthreads();
    const int cnt = min((int)blockDim.x, m - l0);
    for (int j = 0; j < cnt; ++j) {
      const float4 q = sm[j];
      const float d0 = y0 - q.x, d1 = y1 - q.y, d2 = y2 - q.z;
      const float d = d0 * d0 + d1 * d1 + d2 * d2;
      if (d < best) {
        best = d;
        arg = l0 + j;
      }
    }
    __syncthreads();
  }
  if (k < n)
    for (int c = 0; c < 3; ++c) disp[3 * k + c] = tgt[3 * arg + c] - src[3 * k + c];
}

template <bool TA, bool TB, int EPI>
int launch_gemm(int M, int N, int K, int splits, const void* A, const void* B, const float* bias, const void* mask,
                void* C, cudaStream_t st) {
  const int k_split = ((K + splits * BK - 1) / (splits * BK)) * BK;
  const int gz = (K + k_split - 1) / k_split;
  dim3 grid(N / BN, M / BM, gz);
  gemm_kernel<TA, TB, EPI><<<grid, THREADS, 0, st>>>(M, N, K, k_split, reinterpret_cast<const bf16*>(A),
                                                     reinterpret_cast<const bf16*>(B), bias,
                                                     reinterpret_cast<const bf16*>(mask), C);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

}  // namespace mlp
}  // namespace lddmm

using namespace lddmm;
using namespace lddmm::mlp;

extern "C" {

int lddmm_bf16_gemm(int trans_a, int trans_b, int epilogue, int64_t M, int64_t N, int64_t K, const void* A,
                    const void* B, const float* bias, const void* mask, void* C, int splits, float* split_ws,
                    size_t split_ws_bytes, lddmm_stream_t stream) {
  if (M <= 0 || N <= 0 || K <= 0 || M % BM || N % BN || K % BK || M > INT32_MAX / 2 || N > 65536 || K > INT32_MAX / 2)
    return kInvalidArgument;
  if (A == nullptr || B == nullptr || C == nullptr || epilogue < 0 || epilogue > 4) return kInvalidArgument;
  if ((epilogue == kEpiBiasF32 || epilogue == kEpiBiasReluBf16 || epilogue == kEpiBiasBf16) && bias == nullptr)
    return kInvalidArgument;
  if (epilogue == kEpiMaskBf16 && mask == nullptr) return kInvalidArgument;
  if (splits < 1 || M / BM > 65535) return kInvalidArgument;
  if (splits > 1 && (epilogue != kEpiF32 || split_ws == nullptr)) return kInvalidArgument;
  cudaStream_t st = (cudaStream_t)stream;
  const int k_split = (int)(((K + splits * BK - 1) / (splits * BK)) * BK);
  const int gz = (int)((K + k_split - 1) / k_split);
  void* out = C;
  if (gz > 1) {
    if (split_ws_bytes < (size_t)gz * M * N * sizeof(float)) return kWorkspaceTooSmall;
    out = split_ws;
  }
  const int m = (int)M, n = (int)N, k = (int)K;
  int rc;
#define LDDMM_GEMM_CASE(ta, tb, epi) \
  if (trans_a == ta && trans_b == tb && epilogue == epi) rc = launch_gemm<ta, tb, epi>(m, n, k, gz, A, B, bias, mask, out, st); else
  LDDMM_GEMM_CASE(0, 0, kEpiF32) LDDMM_GEMM_CASE(0, 0, kEpiBiasF32) LDDMM_GEMM_CASE(0, 0, kEpiBiasReluBf16)
  LDDMM_GEMM_CASE(0, 0, kEpiBiasBf16) LDDMM_GEMM_CASE(0, 0, kEpiMaskBf16)
  LDDMM_GEMM_CASE(0, 1, kEpiF32) LDDMM_GEMM_CASE(0, 1, kEpiBiasF32) LDDMM_GEMM_CASE(0, 1, kEpiBiasReluBf16)
  LDDMM_GEMM_CASE(0, 1, kEpiBiasBf16) LDDMM_GEMM_CASE(0, 1, kEpiMaskBf16)
  LDDMM_GEMM_CASE(1, 0, kEpiF32) LDDMM_GEMM_CASE(1, 0, kEpiBiasF32) LDDMM_GEMM_CASE(1, 0, kEpiBiasReluBf16)
  LDDMM_GEMM_CASE(1, 0, kEpiBiasBf16) LDDMM_GEMM_CASE(1, 0, kEpiMaskBf16)
  LDDMM_GEMM_CASE(1, 1, kEpiF32) LDDMM_GEMM_CASE(1, 1, kEpiBiasF32) LDDMM_GEMM_CASE(1, 1, kEpiBiasReluBf16)
  LDDMM_GEMM_CASE(1, 1, kEpiBiasBf16) LDDMM_GEMM_CASE(1, 1, kEpiMaskBf16)
  return kInvalidArgument;
#undef LDDMM_GEMM_CASE
  if (rc != kOk) return rc;
  if (gz > 1) {
    const size_t count = (size_t)M * N;
    splitk_reduce_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(split_ws, gz, count,
                                                                          reinterpret_cast<float*>(C));
    if (cudaPeekAtLastError() != cudaSuccess) return kLaunchFailure;
  }
  return kOk;
}

int lddmm_bf16_colsum(const void* dy, int64_t M, int64_t N, float* db, float* ws, size_t ws_bytes,
                      lddmm_stream_t stream) {
  if (M < 0 || N <= 0 || dy == nullptr || db == nullptr || M > INT32_MAX || N > INT32_MAX) return kInvalidArgument;
  const int64_t chunks = (M + kColsumRows - 1) / kColsumRows;
  cudaStream_t st = (cudaStream_t)stream;
  if (ws == nullptr || chunks <= 1) {
    colsum_kernel<<<(unsigned)((N + 31) / 32), 256, 0, st>>>(reinterpret_cast<const bf16*>(dy), (int)M, (int)N, db);
  } else {
    if (ws_bytes < (size_t)chunks * (size_t)N * sizeof(float)) return kWorkspaceTooSmall;
    if (chunks > 65535) return kInvalidArgument;
    colsum_partial_kernel<<<dim3((unsigned)((N + 31) / 32), (unsigned)chunks), 256, 0, st>>>(
        reinterpret_cast<const bf16*>(dy), (int)M, (int)N, ws);
    colsum_final_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(ws, (int)chunks, (int)N, db);
  }
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

int lddmm_mse_grad(const float* y, int64_t M, int64_t N, const float* target, int64_t nout, int64_t valid, float w,
                   void* dy, float* row_loss, lddmm_stream_t stream) {
  if (M <= 0 || N <= 0 || nout < 1 || nout > N || valid < 0 || valid > M || y == nullptr || target == nullptr ||
      dy == nullptr || row_loss == nullptr || M > INT32_MAX)
    return kInvalidArgument;
  mse_grad_kernel<<<(unsigned)((M + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      y, (int)M, (int)N, target, (int)nout, (int)valid, w, reinterpret_cast<bf16*>(dy), row_loss);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

int lddmm_adam_step(float* param, const float* grad, float* m1, float* m2, void* param_bf16, int64_t count, float lr,
                    float beta1, float beta2, float eps, int64_t step, float weight_decay, lddmm_stream_t stream) {
  if (count < 0 || step < 1 || param == nullptr || grad == nullptr || m1 == nullptr || m2 == nullptr)
    return kInvalidArgument;
  if (count == 0) return kOk;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      param, grad, m1, m2, reinterpret_cast<bf16*>(param_bf16), (size_t)count, lr, beta1, beta2, eps, c1, c2,
      weight_decay);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

int lddmm_nearest_displacement(const double* src, int64_t n, const double* tgt, int64_t m, double* disp,
                               lddmm_stream_t stream) {
  if (n < 0 || m <= 0 || (n > 0 && (src == nullptr || disp == nullptr)) || tgt == nullptr || n > INT32_MAX / 4 ||
      m > INT32_MAX / 4)
    return kInvalidArgument;
  if (n == 0) return kOk;
  nearest_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(src, (int)n, tgt, (int)m, disp);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

}  // extern "C"
