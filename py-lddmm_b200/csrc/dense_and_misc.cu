// Dense-weight kernel sums (Kernel.applyK(matrixWeights=True), Kernel.applyDiffKmat) and the library-level
// C-ABI helpers (version, status strings, workspace query).
//
// The dense variants read an O(n m) weight array: they are HBM-bound streaming kernels (one warp per target row,
// coalesced row reads, FP64 arithmetic, warp-shuffle reduction), not FMA-bound pair sums.
#include "../../include/lddmm_b200.h"
#include "kernel_ops.cuh"
#include "launch_config.cuh"

namespace lddmm {

size_t kernel_sums_ws_bytes(int64_t n, int64_t m, int precision);
size_t shooting_ws_bytes(int64_t n, int precision);

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// out[k, :d] = sum_l exp(-|y_k - x_l|^2 * inv2s2) u[k, l, :d]
template <int D>
__global__ void k_mat_kernel(const double* __restrict__ y, int n, const double* __restrict__ x, int m,
                             const double* __restrict__ u, int d, double inv2s2, double* __restrict__ out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const double y0 = y[3 * warp], y1 = y[3 * warp + 1], y2 = y[3 * warp + 2];
  double acc[D > 0 ? D : 1];
  for (int c = 0; c < (D > 0 ? D : 1); ++c) acc[c] = 0.0;
  const double* row = u + (size_t)warp * (size_t)m * (size_t)d;
  for (int l = lane; l < m; l += 32) {
    const double d0 = y0 - x[3 * l], d1 = y1 - x[3 * l + 1], d2 = y2 - x[3 * l + 2];
    const double e = exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2);
    if (D > 0) {
#pragma unroll
      for (int c = 0; c < D; ++c) acc[c] += e * row[(size_t)l * D + c];
    }
  }
#pragma unroll
  for (int c = 0; c < (D > 0 ? D : 1); ++c) {
    const double v = warp_sum(acc[c]);
    if (lane == 0 && D > 0) out[(size_t)warp * D + c] = v;
  }
}

// Generic d (any width): one warp per (row, component).
__global__ void k_mat_kernel_any(const double* __restrict__ y, int n, const double* __restrict__ x, int m,
                                 const double* __restrict__ u, int d, double inv2s2, double* __restrict__ out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n * d) return;
  const int k = warp / d, c = warp - k * d;
  const double y0 = y[3 * k], y1 = y[3 * k + 1], y2 = y[3 * k + 2];
  double acc = 0.0;
  const double* row = u + (size_t)k * (size_t)m * (size_t)d;
  for (int l = lane; l < m; l += 32) {
    const double d0 = y0 - x[3 * l], d1 = y1 - x[3 * l + 1], d2 = y2 - x[3 * l + 2];
    acc += exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2) * row[(size_t)l * d + c];
  }
  acc = warp_sum(acc);
  if (lane == 0) out[(size_t)k * d + c] = acc;
}

// out[k, :] = sum_l -(y_k - x_l) inv_s2 exp(-|y_k - x_l|^2 inv_s2 / 2) beta[k, l]
__global__ void diff_k_mat_kernel(const double* __restrict__ y, int n, const double* __restrict__ x, int m,
                                  const double* __restrict__ beta, double inv_s2, double* __restrict__ out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const double y0 = y[3 * warp], y1 = y[3 * warp + 1], y2 = y[3 * warp + 2];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  const double* row = beta + (size_t)warp * (size_t)m;
  for (int l = lane; l < m; l += 32) {
    const double d0 = y0 - x[3 * l], d1 = y1 - x[3 * l + 1], d2 = y2 - x[3 * l + 2];
    const double f = exp(-0.5 * (d0 * d0 + d1 * d1 + d2 * d2) * inv_s2) * row[l];
    a0 += f * d0;
    a1 += f * d1;
    a2 += f * d2;
  }
  a0 = warp_sum(a0);
  a1 = warp_sum(a1);
  a2 = warp_sum(a2);
  if (lane == 0) {
    out[3 * warp] = -inv_s2 * a0;
    out[3 * warp + 1] = -inv_s2 * a1;
    out[3 * warp + 2] = -inv_s2 * a2;
  }
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

const char* lddmm_version(void) { return "lddmm_b200 0.1.0 (sm_100a)"; }

const char* lddmm_status_string(int status) {
  switch (status) {
    case LDDMM_OK: return "ok";
    case LDDMM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case LDDMM_ERR_LAUNCH: return "kernel launch failed";
    case LDDMM_ERR_NONFINITE: return "non-finite value detected";
    case LDDMM_ERR_WORKSPACE: return "workspace too small";
    case LDDMM_ERR_CUDA: return "CUDA runtime error";
    case LDDMM_ERR_UNSUPPORTED: return "unsupported option";
    default: return "unknown status";
  }
}

size_t lddmm_workspace_bytes(int64_t n_max, int64_t m_max, int precision) {
  if (n_max < 0 || m_max < 0 || (precision != kFP32Compensated && precision != kFP64)) return 0;
  const size_t a = kernel_sums_ws_bytes(n_max, m_max, precision);
  const int64_t nm = n_max > m_max ? n_max : m_max;
  const size_t b = shooting_ws_bytes(nm, precision);
  return a > b ? a : b;
}

int lddmm_apply_k_mat(const double* y, int64_t n, const double* x, int64_t m, const double* u, int64_t d,
                      double sigma, double* out, lddmm_stream_t stream) {
  if (n < 0 || m < 0 || d < 0 || bad_sigma(sigma) || (n > 0 && (y == nullptr || out == nullptr)) ||
      (m > 0 && x == nullptr) || (n > 0 && m > 0 && d > 0 && u == nullptr))
    return kInvalidArgument;
  if (n > INT32_MAX / 64 || m > INT32_MAX || d > 64) return kInvalidArgument;
  if (n == 0 || d == 0) return kOk;
  cudaStream_t st = (cudaStream_t)stream;
  const double inv2s2 = 0.5 / (sigma * sigma);
  const int threads = 256;
  if (m == 0) return cudaMemsetAsync(out, 0, sizeof(double) * n * d, st) == cudaSuccess ? kOk : kCudaError;
  if (d == 3) {
    const int64_t warps = n;
    k_mat_kernel<3><<<(int)((warps * 32 + threads - 1) / threads), threads, 0, st>>>(y, (int)n, x, (int)m, u, 3,
                                                                                      inv2s2, out);
  } else if (d == 1) {
    const int64_t warps = n;
    k_mat_kernel<1><<<(int)((warps * 32 + threads - 1) / threads), threads, 0, st>>>(y, (int)n, x, (int)m, u, 1,
                                                                                      inv2s2, out);
  } else {
    const int64_t warps = n * d;
    k_mat_kernel_any<<<(int)((warps * 32 + threads - 1) / threads), threads, 0, st>>>(y, (int)n, x, (int)m, u,
                                                                                       (int)d, inv2s2, out);
  }
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

int lddmm_apply_diff_k_mat(const double* y, int64_t n, const double* x, int64_t m, const double* beta, double sigma,
                           double* out, lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || (n > 0 && (y == nullptr || out == nullptr)) || (m > 0 && x == nullptr) ||
      (n > 0 && m > 0 && beta == nullptr))
    return kInvalidArgument;
  if (n > INT32_MAX / 64 || m > INT32_MAX) return kInvalidArgument;
  if (n == 0) return kOk;
  cudaStream_t st = (cudaStream_t)stream;
  if (m == 0) return cudaMemsetAsync(out, 0, sizeof(double) * n * 3, st) == cudaSuccess ? kOk : kCudaError;
  const int threads = 256;
  diff_k_mat_kernel<<<(int)((n * 32 + threads - 1) / threads), threads, 0, st>>>(y, (int)n, x, (int)m, beta,
                                                                                  1.0 / (sigma * sigma), out);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

}  // extern "C"
