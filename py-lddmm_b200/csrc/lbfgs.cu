// L-BFGS search direction in one launch: the two-loop recursion of base/bfgs.py:183-198 over the m stored pairs
// (s_k, y_k), k = 0 (oldest) .. m-1 (newest):
//   q = g;  for k = m-1 .. 0: rho_k = 1 / (y_k.s_k), alpha_k = rho_k (s_k.q), q -= alpha_k y_k
//   q *= c, c = (s_{m-1}.y_{m-1}) / (y_{m-1}.y_{m-1}) (1 when c < 1e-10)
//   for k = 0 .. m-1: beta = rho_k (y_k.q), q += (alpha_k - beta) s_k
// Every step needs a full dot product before the next update, so the recursion is 2m dependent reductions over
// n doubles. Done from the host it is ~4m small kernels and as many Python calls per BFGS iteration; here one CTA
// of 1024 threads runs the whole recursion (q lives in global memory, L1/L2-resident at the sizes this is used
// for), with block reductions in a fixed order: deterministic, no host synchronisation.
#include "../../include/lddmm_b200.h"
#include "lddmm_common.cuh"

namespace lddmm {
namespace {

constexpr int kLbfgsThreads = 1024;

struct LbfgsPairs {
  const double* s[LDDMM_LBFGS_MAX_PAIRS];
  const double* y[LDDMM_LBFGS_MAX_PAIRS];
};

// Sums of two per-thread values over the block, in a fixed order (warp shuffles, then warp 0 over the warps).
__device__ __forceinline__ void block_sum2(double& a, double& b, double (*red)[2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    red[warp][0] = a;
    red[warp][1] = b;
  }
  __syncthreads();
  if (warp == 0) {
    a = red[lane][0];
    b = red[lane][1];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
      red[0][0] = a;
      red[0][1] = b;
    }
  }
  __syncthreads();
  a = red[0][0];
  b = red[0][1];
  __syncthreads();  // red is reused by the next reduction
}

__global__ void __launch_bounds__(kLbfgsThreads) lbfgs_two_loop_kernel(const LbfgsPairs P, int m,
                                                                         const double* __restrict__ g, long long n,
                                                                         double* __restrict__ q) {
  __shared__ double red[32][2];
  __shared__ double alpha[LDDMM_LBFGS_MAX_PAIRS], rho[LDDMM_LBFGS_MAX_PAIRS];
  const long long t0 = threadIdx.x;
  for (long long i = t0; i < n; i += kLbfgsThreads) q[i] = g[i];
  __syncthreads();
  for (int k = m - 1; k >= 0; --k) {
    const double* __restrict__ s = P.s[k];
    const double* __restrict__ y = P.y[k];
    double sq = 0.0, ys = 0.0;
    for (long long i = t0; i < n; i += kLbfgsThreads) {
      const double si = s[i];
      sq = fma(si, q[i], sq);
      ys = fma(y[i], si, ys);
    }
    block_sum2(sq, ys, red);
    const double r = 1.0 / ys;
    const double al = r * sq;
    if (threadIdx.x == 0) {
      rho[k] = r;
      alpha[k] = al;
    }
    for (long long i = t0; i < n; i += kLbfgsThreads) q[i] = fma(-al, y[i], q[i]);
    __syncthreads();
  }
  {
    const double* __restrict__ s = P.s[m - 1];
    const double* __restrict__ y = P.y[m - 1];
    double sy = 0.0, yy = 0.0;
    for (long long i = t0; i < n; i += kLbfgsThreads) {
      const double yi = y[i];
      sy = fma(s[i], yi, sy);
      yy = fma(yi, yi, yy);
    }
    block_sum2(sy, yy, red);
    double c = sy / yy;
    if (c < 1e-10) c = 1.0;
    for (long long i = t0; i < n; i += kLbfgsThreads) q[i] *= c;
    __syncthreads();
  }
  for (int k = 0; k < m; ++k) {
    const double* __restrict__ s = P.s[k];
    const double* __restrict__ y = P.y[k];
    double yq = 0.0, unused = 0.0;
    for (long long i = t0; i < n; i += kLbfgsThreads) yq = fma(y[i], q[i], yq);
    block_sum2(yq, unused, red);
    const double coef = alpha[k] - rho[k] * yq;
    for (long long i = t0; i < n; i += kLbfgsThreads) q[i] = fma(coef, s[i], q[i]);
    __syncthreads();
  }
}

}  // namespace
}  // namespace lddmm

using namespace lddmm;

extern "C" int lddmm_lbfgs_direction(const double* const* s, const double* const* y, int m, const double* g,
                                     int64_t n, double* q, lddmm_stream_t stream) {
  if (m < 1 || m > LDDMM_LBFGS_MAX_PAIRS || n < 0 || s == nullptr || y == nullptr) return kInvalidArgument;
  if (n > 0 && (g == nullptr || q == nullptr)) return kInvalidArgument;
  LbfgsPairs P;
  for (int k = 0; k < m; ++k) {
    if (n > 0 && (s[k] == nullptr || y[k] == nullptr)) return kInvalidArgument;
    P.s[k] = s[k];
    P.y[k] = y[k];
  }
  for (int k = m; k < LDDMM_LBFGS_MAX_PAIRS; ++k) P.s[k] = P.y[k] = nullptr;
  if (n == 0) return kOk;
  lbfgs_two_loop_kernel<<<1, kLbfgsThreads, 0, (cudaStream_t)stream>>>(P, m, g, (long long)n, q);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}
