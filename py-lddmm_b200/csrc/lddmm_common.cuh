// Shared machinery of the all-pairs Gaussian kernel sums (sm_100a).
//
// Every hot operator of the point-set path is a map-reduce over (target k, source l) pairs:
//     out_k = epilogue_k( sum_l pair(target_k, source_l) ).
// The pair loop is FP32-FMA / MUFU bound (arithmetic intensity >> 100 flop/byte), so the design is an
// N-body tiling: a CTA owns TPB*RT targets held in registers (RT per thread), streams tiles of TPB sources
// through shared memory (every thread reads the same source record -> broadcast LDS.128), and the source
// range is split into S chunks along gridDim.y so that even mid-size problems fill all 148 SMs.
//
// Precision (FP32 path): coordinates are centred on a caller-given origin and pre-scaled by
// s = sqrt(log2(e)/2)/sigma so that exp(-|y-x|^2 / (2 sigma^2)) = 2^-(|y'-x'|^2) is one `ex2.approx.ftz`.
// Each tile is summed in plain FP32; tile sums are merged into a (hi, lo) pair by a two-sum (compensated
// accumulation across tiles). Chunk partials (hi, lo) are reduced in FP64, in fixed order, by the
// epilogue kernel, which also applies the per-target constants and writes float64 outputs (and, for the
// shooting steps, the float64 Euler update of the state).
// FP64 path ("faithful" baseline): same kernels instantiated with double, exp() and plain FP64 sums.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lddmm {

enum Status : int {
  kOk = 0,
  kInvalidArgument = 1,
  kLaunchFailure = 2,
  kNonFinite = 3,
  kWorkspaceTooSmall = 4,
  kCudaError = 5,
  kUnsupported = 6,
};

enum Precision : int { kFP32Compensated = 0, kFP64 = 1 };

template <typename R>
struct alignas(4 * sizeof(R)) V4 {
  R x, y, z, w;
};

template <typename R> struct PT;

template <> struct PT<float> {
  // sqrt(log2(e) / 2): exp(-r^2/(2 sigma^2)) == 2^-(s r)^2 with s = kScale / sigma.
  static constexpr double kScale = 0.84932180028801904272;
  using Partial = float2;  // (hi, lo) of the compensated chunk sum
  static __device__ __forceinline__ float expneg(float r2) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(-r2));
    return y;
  }
};

template <> struct PT<double> {
  static constexpr double kScale = 0.70710678118654752440;  // sqrt(1/2): exp(-(s r)^2)
  using Partial = double;
  static __device__ __forceinline__ double expneg(double r2) { return exp(-r2); }
};

// Compensated accumulator: a tile sum `t` (plain FP32) is folded into (hi, lo) by Knuth's two-sum.
template <typename R> struct Comp;
template <> struct Comp<float> {
  float hi, lo;
  __device__ __forceinline__ void zero() { hi = 0.f; lo = 0.f; }
  __device__ __forceinline__ void merge(float t) {
    float s = __fadd_rn(hi, t);
    float bp = __fsub_rn(s, hi);
    float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(t, bp));
    hi = s;
    lo = __fadd_rn(lo, err);
  }
  __device__ __forceinline__ float2 partial() const { return make_float2(hi, lo); }
};
template <> struct Comp<double> {
  double hi;
  __device__ __forceinline__ void zero() { hi = 0.0; }
  __device__ __forceinline__ void merge(double t) { hi += t; }
  __device__ __forceinline__ double partial() const { return hi; }
};

__device__ __forceinline__ double partial_value(float2 p) { return (double)p.x + (double)p.y; }
__device__ __forceinline__ double partial_value(double p) { return p; }

// Geometry shared by every op: centred, pre-scaled coordinates.
struct Frame {
  double o0, o1, o2;  // origin subtracted before scaling
  double s;           // coordinate scale (kScale / sigma)
  double kappa;       // 1 / (s sigma^2): turns a scaled difference into (y - x) / sigma^2
  double inv_s2;      // 1 / sigma^2
};

template <typename R>
__device__ __forceinline__ void load_point(const double* __restrict__ p, int i, const Frame& f, R& a, R& b, R& c) {
  a = (R)((p[3 * i + 0] - f.o0) * f.s);
  b = (R)((p[3 * i + 1] - f.o1) * f.s);
  c = (R)((p[3 * i + 2] - f.o2) * f.s);
}

template <typename R>
__device__ __forceinline__ void load_vec(const double* __restrict__ p, int i, R& a, R& b, R& c) {
  a = (R)p[3 * i + 0];
  b = (R)p[3 * i + 1];
  c = (R)p[3 * i + 2];
}

// Launch plan of one all-pairs sum: gx target blocks x S source chunks of `chunk` sources (multiple of TPB).
struct Plan {
  int gx = 0, S = 0, chunk = 0;
  size_t ws_bytes = 0;
};

int device_sm_count();

template <int TPB, int RT>
inline Plan make_plan(int64_t n, int64_t m, int na, size_t partial_bytes, int ctas_per_sm) {
  Plan p;
  if (n <= 0) return p;
  const int64_t tpb_targets = (int64_t)TPB * RT;
  p.gx = (int)((n + tpb_targets - 1) / tpb_targets);
  if (m <= 0) {
    p.S = 0;
    p.chunk = 0;
    p.ws_bytes = 0;
    return p;
  }
  const int64_t tiles = (m + TPB - 1) / TPB;
  const int64_t want = (int64_t)device_sm_count() * (ctas_per_sm > 0 ? ctas_per_sm : 1);
  int64_t S = (want + p.gx - 1) / p.gx;
  if (S < 1) S = 1;
  if (S > tiles) S = tiles;
  const int64_t tiles_per_chunk = (tiles + S - 1) / S;
  p.chunk = (int)(tiles_per_chunk * TPB);
  p.S = (int)((m + p.chunk - 1) / p.chunk);
  p.ws_bytes = (size_t)p.S * (size_t)na * (size_t)n * partial_bytes;
  return p;
}

// ---------------------------------------------------------------------------------------------------------
// Generic tiled all-pairs kernel.
//   Op::NV        number of V4<R> records per source staged in shared memory
//   Op::NA        number of scalar accumulators per target
//   Op::Tgt       per-target register state
//   Op::load_target(P, i, tgt)            (i < n)
//   Op::load_source(P, l, V4<R>* rec)     (l < m)
//   Op::pair(tgt, const V4<R>* src, R* acc)
// Output: ws[(chunk * NA + c) * n + i] = compensated partial of accumulator c of target i.
// ---------------------------------------------------------------------------------------------------------
template <class Op, typename R, int TPB, int RT>
__global__ void __launch_bounds__(TPB) pairs_kernel(const typename Op::Params P, int n, int m, int chunk,
                                                    typename PT<R>::Partial* __restrict__ ws) {
  __shared__ V4<R> sm[Op::NV][TPB];
  typename Op::Tgt tgt[RT];
  R acc[RT][Op::NA];
  Comp<R> cmp[RT][Op::NA];

  const int base = blockIdx.x * (TPB * RT) + threadIdx.x;
#pragma unroll
  for (int r = 0; r < RT; ++r) {
    const int i = base + r * TPB;
    Op::load_target(P, i < n ? i : (n - 1), tgt[r]);
#pragma unroll
    for (int c = 0; c < Op::NA; ++c) cmp[r][c].zero();
  }

  const int l_begin = blockIdx.y * chunk;
  int l_end = l_begin + chunk;
  if (l_end > m) l_end = m;

  for (int l0 = l_begin; l0 < l_end; l0 += TPB) {
    const int l = l0 + threadIdx.x;
    if (l < l_end) {
      V4<R> rec[Op::NV];
      Op::load_source(P, l, rec);
#pragma unroll
      for (int v = 0; v < Op::NV; ++v) sm[v][threadIdx.x] = rec[v];
    } else {
#pragma unroll
      for (int v = 0; v < Op::NV; ++v) sm[v][threadIdx.x] = V4<R>{R(0), R(0), R(0), R(0)};
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RT; ++r)
#pragma unroll
      for (int c = 0; c < Op::NA; ++c) acc[r][c] = R(0);
#pragma unroll 4
    for (int j = 0; j < TPB; ++j) {
      V4<R> src[Op::NV];
#pragma unroll
      for (int v = 0; v < Op::NV; ++v) src[v] = sm[v][j];
#pragma unroll
      for (int r = 0; r < RT; ++r) Op::pair(tgt[r], src, acc[r]);
    }
#pragma unroll
    for (int r = 0; r < RT; ++r)
#pragma unroll
      for (int c = 0; c < Op::NA; ++c) cmp[r][c].merge(acc[r][c]);
    __syncthreads();
  }

#pragma unroll
  for (int r = 0; r < RT; ++r) {
    const int i = base + r * TPB;
    if (i < n) {
#pragma unroll
      for (int c = 0; c < Op::NA; ++c) ws[((size_t)blockIdx.y * Op::NA + c) * (size_t)n + i] = cmp[r][c].partial();
    }
  }
}

// Epilogue: reduce the S chunk partials of target i in FP64 (fixed order) and hand them to Op::finalize.
template <class Op, typename R>
__global__ void finalize_kernel(const typename Op::Params P, int n, int S,
                                const typename PT<R>::Partial* __restrict__ ws) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc[Op::NA];
#pragma unroll
  for (int c = 0; c < Op::NA; ++c) acc[c] = 0.0;
  for (int s = 0; s < S; ++s)
#pragma unroll
    for (int c = 0; c < Op::NA; ++c) acc[c] += partial_value(ws[((size_t)s * Op::NA + c) * (size_t)n + i]);
  Op::finalize(P, i, acc);
}

// Deterministic single-block sum of `count` doubles: out[0] = (accumulate ? out[0] : 0) + scale * sum(v).
__global__ void ordered_sum_kernel(const double* __restrict__ v, int count, double scale, double* out, int accumulate);

template <class Op, typename R, int TPB, int RT>
inline int run_pairs(const typename Op::Params& P, int64_t n, int64_t m, void* ws, size_t ws_bytes,
                     cudaStream_t stream, int ctas_per_sm) {
  if (n <= 0) return kOk;
  if (n > INT32_MAX / 4 || m > INT32_MAX / 4) return kInvalidArgument;
  Plan plan = make_plan<TPB, RT>(n, m, Op::NA, sizeof(typename PT<R>::Partial), ctas_per_sm);
  if (plan.ws_bytes > ws_bytes) return kWorkspaceTooSmall;
  if (plan.ws_bytes > 0 && ws == nullptr) return kInvalidArgument;
  auto* part = reinterpret_cast<typename PT<R>::Partial*>(ws);
  if (plan.S > 0) {
    dim3 grid(plan.gx, plan.S);
    pairs_kernel<Op, R, TPB, RT><<<grid, TPB, 0, stream>>>(P, (int)n, (int)m, plan.chunk, part);
  }
  const int fb = 256;
  finalize_kernel<Op, R><<<(int)((n + fb - 1) / fb), fb, 0, stream>>>(P, (int)n, plan.S, part);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

template <class Op, typename R, int TPB, int RT>
inline size_t pairs_ws_bytes(int64_t n, int64_t m, int ctas_per_sm) {
  return make_plan<TPB, RT>(n, m, Op::NA, sizeof(typename PT<R>::Partial), ctas_per_sm).ws_bytes;
}

inline Frame make_frame(const double* origin, double sigma, double kscale) {
  Frame f;
  f.o0 = origin ? origin[0] : 0.0;
  f.o1 = origin ? origin[1] : 0.0;
  f.o2 = origin ? origin[2] : 0.0;
  f.s = kscale / sigma;
  f.kappa = 1.0 / (f.s * sigma * sigma);
  f.inv_s2 = 1.0 / (sigma * sigma);
  return f;
}

inline bool bad_sigma(double sigma) { return !(sigma > 0.0) || !(sigma < 1e300); }

}  // namespace lddmm
