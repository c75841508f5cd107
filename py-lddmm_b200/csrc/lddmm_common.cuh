// Shared machinery of the all-pairs Gaussian kernel sums (sm_100a).
//
// Every hot operator of the point-set path is a map-reduce over (target k, source l) pairs:
//     out_k = epilogue_k( sum_l pair(target_k, source_l) ).
// The pair loop is FP32-pipe / MUFU bound (arithmetic intensity >> 100 flop/byte), so the design is an N-body
// tiling: a CTA owns TPB*RT targets held in registers (RT per thread) and streams tiles of TPB sources through
// shared memory (all threads of a warp read the same source record: broadcast LDS.128). The (target block, source
// tile) units are split evenly over exactly one resident wave of CTAs (stream-K style, see SKPlan), so every
// problem size keeps all 148 SMs equally busy.
//
// FP32 path: the pair arithmetic runs on Blackwell's packed FP32 instructions (fma/add/sub/mul .f32x2): one
// instruction evaluates the same source against TWO targets of the thread, halving the issue slots of the FP32
// work. Source fields are stored duplicated ((f, f) pairs) in shared memory so that a 16-byte LDS yields two
// ready-to-use packed operands. Coordinates are centred on a caller-given origin and pre-scaled by
// s = sqrt(log2(e)/2)/sigma so that exp(-|y-x|^2/(2 sigma^2)) = 2^-(|y'-x'|^2), one `ex2.approx.ftz` (MUFU)
// per pair. Each tile is summed in plain FP32; tile sums are merged into a (hi, lo) pair by a two-sum
// (compensated accumulation across tiles). Chunk partials are reduced in FP64, in fixed order, by the epilogue
// kernel, which applies the per-target constants and writes float64 outputs (and, for shooting steps, the
// float64 Euler update of the state).
// Ops whose sum needs no coordinate differences (K a, the surface energies) run pairs_kernel_x instead: the
// squared distance expanded about the centre of each target block, three packed FMAs per pair (see there).
// FP64 path (the faithful baseline): the same pair functors instantiated with double, exp() and FP64 sums.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>

#ifndef LDDMM_MIN_CTAS
#define LDDMM_MIN_CTAS 1  // minimum resident CTAs per SM requested from ptxas (caps registers when > 1)
#endif
// per-op minimum resident CTAs (1: no register cap beyond the op's needs)
#ifndef LDDMM_SOFWD_MIN_CTAS
#define LDDMM_SOFWD_MIN_CTAS 4
#endif
#ifndef LDDMM_SOBWD_MIN_CTAS
#define LDDMM_SOBWD_MIN_CTAS 1  // at 4 targets per thread (LDDMM_RT_ADJOINT) no cap: 254 registers, 2 CTAs per SM
#endif
#ifndef LDDMM_SOBWD_SYM_MIN_CTAS
#define LDDMM_SOBWD_SYM_MIN_CTAS 2  // the symmetric adjoint step (pairs_kernel_sym)
#endif
#ifndef LDDMM_SOFWD_SYM_MIN_CTAS
#define LDDMM_SOFWD_SYM_MIN_CTAS 3  // the symmetric forward step (pairs_kernel_sym): caps it at 168 registers
#endif
#ifndef LDDMM_KSYM_MIN_CTAS
#define LDDMM_KSYM_MIN_CTAS 3  // the symmetric K(x, x) a (pairs_kernel_symx): 164 registers, 3 CTAs per SM (3% faster
                               // than 4 CTAs at 128 registers, which spill)
#endif
#ifndef LDDMM_FOBWD_SYM_MIN_CTAS
#define LDDMM_FOBWD_SYM_MIN_CTAS 2  // the symmetric first-order adjoint step (pairs_kernel_sym)
#endif
#ifndef LDDMM_FOBWD_MIN_CTAS
#define LDDMM_FOBWD_MIN_CTAS 1
#endif
#ifndef LDDMM_SURFGRAD_MIN_CTAS
#define LDDMM_SURFGRAD_MIN_CTAS 1
#endif
#ifndef LDDMM_COMP_SMEM
#define LDDMM_COMP_SMEM 1  // 0: keep every op's compensated (hi, lo) sums in registers
#endif
#ifndef LDDMM_CULL
#define LDDMM_CULL 1  // 0: no exact culling of far tile pairs (no box pre-pass)
#endif
#ifndef LDDMM_EXPAND
#define LDDMM_EXPAND 1  // 0: the Gaussian sums of ops with an expanded-distance form use the difference form
#endif
#ifndef LDDMM_SOFWD_EXPAND
#define LDDMM_SOFWD_EXPAND 1  // 0: the second-order forward step keeps the difference form
#endif
#ifndef LDDMM_SURFGRAD_EXPAND
#define LDDMM_SURFGRAD_EXPAND 1  // 0: the varifold and measure gradients keep the difference form
#endif
#ifndef LDDMM_SOURCE_UNROLL
#define LDDMM_SOURCE_UNROLL 4  // unroll depth of the per-source loop over a shared-memory tile
#endif

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

constexpr int kSourceUnroll = LDDMM_SOURCE_UNROLL;

// ---------------------------------------------------------------------------------------------------------
// Packed FP32 pair (two lanes in one 64-bit register pair) and its arithmetic (PTX .f32x2, sm_100a).
// ---------------------------------------------------------------------------------------------------------
struct F2 {
  unsigned long long v;
};

__device__ __forceinline__ F2 f2(float lo, float hi) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void split(F2 a, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
  F2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) {
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}
__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { return a = a + b; }
__device__ __forceinline__ F2 operator-(F2 a) { return f2(0.f, 0.f) - a; }

__device__ __forceinline__ float ex2neg(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(-x));
  return y;
}

// Value-type traits: V = F2 (two FP32 targets per lane group) or double (one FP64 target).
template <typename V> struct VT;
template <> struct VT<F2> {
  using Scalar = float;
  static constexpr int kLanes = 2;
  // sqrt(log2(e) / 2): exp(-r^2/(2 sigma^2)) == 2^-(s r)^2 with s = kScale / sigma.
  static constexpr double kScale = 0.84932180028801904272;
  using Partial = float2;  // (hi, lo) of the compensated chunk sum
  static __device__ __forceinline__ F2 zero() { return f2(0.f, 0.f); }
  static __device__ __forceinline__ F2 dup(double a) { return f2((float)a, (float)a); }
  static __device__ __forceinline__ F2 pack(double a, double b) { return f2((float)a, (float)b); }
  static __device__ __forceinline__ F2 expneg(F2 r2) {
    float a, b;
    split(r2, a, b);
    return f2(ex2neg(a), ex2neg(b));
  }
  static __device__ __forceinline__ double lane(F2 v, int k) {
    float a, b;
    split(v, a, b);
    return k ? (double)b : (double)a;
  }
};
template <> struct VT<double> {
  using Scalar = double;
  static constexpr int kLanes = 1;
  static constexpr double kScale = 0.70710678118654752440;  // sqrt(1/2): exp(-(s r)^2)
  using Partial = double;
  static __device__ __forceinline__ double zero() { return 0.0; }
  static __device__ __forceinline__ double dup(double a) { return a; }
  static __device__ __forceinline__ double pack(double a, double) { return a; }
  static __device__ __forceinline__ double expneg(double r2) { return exp(-r2); }
  static __device__ __forceinline__ double lane(double v, int) { return v; }
};

// Compensated accumulator: a tile sum `t` is folded into (hi, lo) by Knuth's two-sum (FP32); plain sum (FP64).
template <typename V> struct Comp;
template <> struct Comp<F2> {
  static constexpr int kWords = 2;  // (hi, lo)
  F2 hi, lo;
  __device__ __forceinline__ void zero() { hi = lo = f2(0.f, 0.f); }
  template <int TPB>
  __device__ __forceinline__ void load(const F2 (*cs)[TPB], int i, int t) { hi = cs[2 * i][t]; lo = cs[2 * i + 1][t]; }
  template <int TPB>
  __device__ __forceinline__ void store(F2 (*cs)[TPB], int i, int t) const { cs[2 * i][t] = hi; cs[2 * i + 1][t] = lo; }
  __device__ __forceinline__ void merge(F2 t) {
    const F2 s = hi + t;
    const F2 bp = s - hi;
    const F2 err = (hi - (s - bp)) + (t - bp);
    hi = s;
    lo = lo + err;
  }
  __device__ __forceinline__ float2 partial(int k) const {
    return make_float2((float)VT<F2>::lane(hi, k), (float)VT<F2>::lane(lo, k));
  }
};
template <> struct Comp<double> {
  static constexpr int kWords = 1;
  double hi;
  __device__ __forceinline__ void zero() { hi = 0.0; }
  template <int TPB>
  __device__ __forceinline__ void load(const double (*cs)[TPB], int i, int t) { hi = cs[i][t]; }
  template <int TPB>
  __device__ __forceinline__ void store(double (*cs)[TPB], int i, int t) const { cs[i][t] = hi; }
  __device__ __forceinline__ void merge(double t) { hi += t; }
  __device__ __forceinline__ double partial(int) const { return hi; }
};

// Ops whose compensated sums stay in registers (few accumulators: measured faster there) declare
// `static constexpr bool kCompInRegisters = true;`.
template <class Op, class = void>
struct CompInRegisters : std::false_type {};
template <class Op>
struct CompInRegisters<Op, std::void_t<decltype(Op::kCompInRegisters)>> : std::bool_constant<Op::kCompInRegisters> {};

__device__ __forceinline__ double partial_value(float2 p) { return (double)p.x + (double)p.y; }
__device__ __forceinline__ double partial_value(double p) { return p; }

__device__ __forceinline__ double fma(double a, double b, double c) { return ::fma(a, b, c); }

// Kernel families (the `kernel` argument of the C ABI): 0 = Gaussian, 16 + q = Laplacian (Matern) of order q <= 4,
// K(r) = P_q(r / sigma) exp(-r / sigma) (base/kernelFunctions_util.py:20-52 lapPol / lapPolDiff / lapPolDiff2).
enum KernelFamily : int { kGauss = 0, kLaplacian0 = 16, kLaplacianMax = 20 };

// Geometry shared by every op: centred, pre-scaled coordinates, and the radial profile of the kernel.
struct Frame {
  double o0, o1, o2;  // origin subtracted before scaling
  double s;           // coordinate scale (Gaussian: kScale / sigma; Laplacian: 1/sigma, times log2(e) in FP32)
  double kappa;       // 1 / (s sigma^2): turns a scaled difference into (y - x) / sigma^2
  double inv_s2;      // 1 / sigma^2
  int family;         // KernelFamily
  // Laplacian profile in the scaled radius u' = |d|: K0 = P0(u') E, K1 = P1(u') E, K2 = P2(u') E with
  // E = exp(-u') (FP64) or 2^-u' (FP32, coefficients rescaled). grad_y K = -K1 kappa d, Hessian = kappa^2 K2 d d^T
  // - K1/sigma^2 I. Row r holds the coefficients of P_r in increasing degree (zeros past the order).
  float lc[3][5];
  double dc[3][5];
};

// Radial factors of one pair: K0 (value), K1 (first-derivative factor), K2 (second-derivative factor). For the
// Gaussian all three are exp(-|d|^2); unused ones are removed by the compiler.
template <typename V>
struct KV {
  V k0, k1, k2;
};

__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// kCullR2<V>: a scaled squared distance beyond which every radial factor is exactly zero in the arithmetic of V
// (FP32: ex2.approx.ftz of an argument below -126 flushes to +0; FP64: exp below -745.2 underflows to 0), with a
// margin for the FP32 rounding of the box test that uses it.
struct Gauss {
  template <typename V>
  static __device__ __forceinline__ KV<V> eval(const Frame&, V r2) {
    const V e = VT<V>::expneg(r2);
    return {e, e, e};
  }
  template <typename V>
  static constexpr float kCullR2 = VT<V>::kLanes == 2 ? 127.0f : 746.0f;
};

struct Laplacian {
  template <typename V>
  static __device__ __forceinline__ KV<V> eval(const Frame& f, V r2);
  template <typename V>
  static constexpr float kCullR2 = VT<V>::kLanes == 2 ? 127.0f * 127.0f : 746.0f * 746.0f;  // the radius u = |d|
};

// Axis-aligned box of the scaled coordinates held by a block of threads: per-thread (lo, hi), reduced over the
// block through `red` (6 x warps floats). Every thread ends with the block's box; callers separate reuses of `red`
// by a barrier.
template <int TPB>
__device__ __forceinline__ void block_box(float lo[3], float hi[3], float (*red)[TPB / 32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[c] = fminf(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
      hi[c] = fmaxf(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      red[c][warp] = lo[c];
      red[3 + c][warp] = hi[c];
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    lo[c] = red[c][0];
    hi[c] = red[3 + c][0];
#pragma unroll
    for (int w = 1; w < TPB / 32; ++w) {
      lo[c] = fminf(lo[c], red[c][w]);
      hi[c] = fmaxf(hi[c], red[3 + c][w]);
    }
  }
}

// Squared distance between two boxes (0 when they overlap).
__device__ __forceinline__ float box_gap2(const float alo[3], const float ahi[3], const float blo[3],
                                          const float bhi[3]) {
  float d2 = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float g = fmaxf(0.f, fmaxf(blo[c] - ahi[c], alo[c] - bhi[c]));
    d2 = fmaf(g, g, d2);
  }
  return d2;
}

__device__ __forceinline__ float horner5(const float* c, float u) {
  return fmaf(fmaf(fmaf(fmaf(c[4], u, c[3]), u, c[2]), u, c[1]), u, c[0]);
}
__device__ __forceinline__ double horner5(const double* c, double u) {
  return ::fma(::fma(::fma(::fma(c[4], u, c[3]), u, c[2]), u, c[1]), u, c[0]);
}

template <>
__device__ __forceinline__ KV<F2> Laplacian::eval<F2>(const Frame& f, F2 r2) {
  float a, b;
  split(r2, a, b);
  const float ua = sqrt_approx(a), ub = sqrt_approx(b);
  const float ea = ex2neg(ua), eb = ex2neg(ub);
  KV<F2> k;
  k.k0 = f2(ea * horner5(f.lc[0], ua), eb * horner5(f.lc[0], ub));
  k.k1 = f2(ea * horner5(f.lc[1], ua), eb * horner5(f.lc[1], ub));
  k.k2 = f2(ea * horner5(f.lc[2], ua), eb * horner5(f.lc[2], ub));
  return k;
}
template <>
__device__ __forceinline__ KV<double> Laplacian::eval<double>(const Frame& f, double r2) {
  const double u = sqrt(r2), e = exp(-u);
  return {e * horner5(f.dc[0], u), e * horner5(f.dc[1], u), e * horner5(f.dc[2], u)};
}

// Shared-memory unit: two source fields (each a duplicated FP32 pair or one FP64 value), 16 bytes.
template <typename V>
struct alignas(16) Unit {
  V a, b;
};

// Per-target loaders: field values of targets i0, i1 packed into one V (V = double ignores i1).
template <typename V>
__device__ __forceinline__ V tgt_coord(const double* __restrict__ p, int i0, int i1, int c, double o, double s) {
  return VT<V>::pack((p[3 * i0 + c] - o) * s, (p[3 * i1 + c] - o) * s);
}
template <typename V>
__device__ __forceinline__ V tgt_field(const double* __restrict__ p, int stride, int i0, int i1, int c,
                                       double scale = 1.0) {
  return VT<V>::pack(scale * p[(size_t)stride * i0 + c], scale * p[(size_t)stride * i1 + c]);
}

// ---------------------------------------------------------------------------------------------------------
// Stream-K style launch plan. The work of one all-pairs sum is W = gx * TT units (gx target blocks of TPB*RT
// targets, TT source tiles of TPB sources). C = min(W, one resident wave) CTAs each take the contiguous unit range
// [start(c), start(c+1)), start(c) = floor(c W / C): every SM gets the same number of pair evaluations (to one
// tile), whatever n and m are. A CTA walks its range as segments (one target block, a run of tiles) and writes
// one compensated partial per segment; the partials of target block tb come from CTAs cta_of(tb TT) ..
// cta_of((tb+1) TT - 1) and are stored in slot (c - cta_of(tb TT)), so the epilogue reduces them in a fixed order.
// ---------------------------------------------------------------------------------------------------------
struct SKPlan {
  int gx = 0, TT = 0, C = 0, S = 0;  // S = max partial slots per target block
  long long W = 0;
  size_t box_off = 0;   // byte offset of the (gx + TT) coordinate boxes after the partial slots
  size_t ws_bytes = 0;
};

__host__ __device__ __forceinline__ long long sk_start(long long c, long long W, long long C) { return c * W / C; }

__host__ __device__ __forceinline__ int sk_cta_of(long long u, long long W, long long C) {
  long long c = ((u + 1) * C - 1) / W;
  while (c + 1 < C && sk_start(c + 1, W, C) <= u) ++c;
  while (c > 0 && sk_start(c, W, C) > u) --c;
  return (int)c;
}

int device_sm_count();

// `boxes`: reserve the coordinate boxes of exact culling (ops with Culled<Op>); other ops never read them, so their
// scratch is the partial slots alone (at most (C / gx + 2) * na * n partials, whatever m is).
template <int TPB, int RT>
inline SKPlan make_plan(int64_t n, int64_t m, int na, size_t partial_bytes, int ctas_per_sm, bool boxes = true) {
  SKPlan p;
  if (n <= 0) return p;
  const int64_t tb_targets = (int64_t)TPB * RT;
  p.gx = (int)((n + tb_targets - 1) / tb_targets);
  if (m <= 0) return p;
  p.TT = (int)((m + TPB - 1) / TPB);
  p.W = (long long)p.gx * p.TT;
  const long long wave = (long long)device_sm_count() * (ctas_per_sm > 0 ? ctas_per_sm : 1);
  p.C = (int)(p.W < wave ? p.W : wave);
  int smax = 1;
  for (int tb = 0; tb < p.gx; ++tb) {
    const int c0 = sk_cta_of((long long)tb * p.TT, p.W, p.C);
    const int c1 = sk_cta_of((long long)(tb + 1) * p.TT - 1, p.W, p.C);
    if (c1 - c0 + 1 > smax) smax = c1 - c0 + 1;
  }
  p.S = smax;
  p.box_off = ((size_t)p.S * (size_t)na * (size_t)n * partial_bytes + 255) & ~(size_t)255;
  p.ws_bytes = p.box_off + (boxes ? (size_t)(p.gx + p.TT) * 6 * sizeof(float) : 0);
  return p;
}

// ---------------------------------------------------------------------------------------------------------
// Generic tiled all-pairs kernel.
//   Op::NS         number of source fields (scalars) staged per source (NU = ceil(NS/2) 16-byte units)
//   Op::NA         number of accumulators per target
//   Op::template Tgt<V>                                  per-lane-group register state
//   Op::template load_target<V>(P, i0, i1, tgt)          (i0, i1 < n; i1 ignored for V = double)
//   Op::source_fields(P, l, double* f)                   the NS source fields of source l (l < m), FP64
//   Op::template pair<V, Fam>(const Frame&, tgt, const V* s, V* acc)   (Fam: Gauss or Laplacian)
// Output: ws[(slot * NA + c) * n + i] = compensated partial of accumulator c of target i for one segment.
// ---------------------------------------------------------------------------------------------------------
// Ops may ask for a minimum number of resident CTAs per SM (`static constexpr int kMinCtas`), which caps the
// registers the compiler may use (65536 / (TPB * kMinCtas)).
// The cap applies to the FP32 (F2) kernels only.
template <class Op, typename V, class = void>
struct MinCtas : std::integral_constant<int, LDDMM_MIN_CTAS> {};
template <class Op>
struct MinCtas<Op, F2, std::void_t<decltype(Op::kMinCtas)>> : std::integral_constant<int, Op::kMinCtas> {};

// Ops may set their own unroll depth of the per-source loop (`static constexpr int kUnroll`); the default is
// LDDMM_SOURCE_UNROLL.
template <class Op, class = void>
struct UnrollOf : std::integral_constant<int, kSourceUnroll> {};
template <class Op>
struct UnrollOf<Op, std::void_t<decltype(Op::kUnroll)>> : std::integral_constant<int, Op::kUnroll> {};

// Ops whose sums are culled declare `static constexpr bool kCull = true;`: the surface data terms, whose faces are
// stored in a spatially coherent order by mesh generators and whose widths are often small against the shape.
// Elsewhere the box pre-pass and the per-tile test cost 2-3% and seldom pay (vertex orders are less coherent, and
// deformation widths large), so the other ops evaluate every tile.
template <class Op, class = void>
struct Culled : std::false_type {};
template <class Op>
struct Culled<Op, std::void_t<decltype(Op::kCull)>> : std::bool_constant<LDDMM_CULL != 0 && Op::kCull> {};

// Ops with an expanded-distance form of their Gaussian FP32 sums (pairs_kernel_x) declare
// `static constexpr bool kExpand = true;` and provide
//   NP                                   payload fields per source (staged after the coordinates)
//   target_point(P, i, double* c)        raw (unscaled) coordinates of target i
//   source_point(P, l, double* c, double* pay)   raw coordinates and the NP payload fields of source l
//   template TgtX<V>, load_target_x<V>(P, i0, i1, TgtX&)   per-lane-group target state besides the coordinates
//   accumulate<V>(const TgtX&, V e, const V* pay, V* acc)  the pair's contribution from its kernel value e
template <class Op, class = void>
struct Expanded : std::false_type {};
template <class Op>
struct Expanded<Op, std::void_t<decltype(Op::kExpand)>> : std::bool_constant<LDDMM_EXPAND != 0 && Op::kExpand> {};
template <class Op, typename V, class Fam>
constexpr bool kUseExpanded = Expanded<Op>::value && std::is_same<V, F2>::value && std::is_same<Fam, Gauss>::value;
// pairs_kernel_x's launch shape: 8 targets per thread (4 packed lane groups per source read) with the compensated
// sums in shared memory (136 registers, 3 CTAs per SM) measured 3-6% faster than the light ops' 4 targets per thread
// with sums in registers (applyK at levels 6 and 7, varifold energy at level 6)
#ifndef LDDMM_RT_X
#define LDDMM_RT_X 8  // targets per thread of pairs_kernel_x (0: the caller's launch shape)
#endif
#ifndef LDDMM_X_COMP_SMEM
#define LDDMM_X_COMP_SMEM 1  // 0: pairs_kernel_x keeps its compensated sums in registers
#endif
// Targets per thread of the kernel that runs an op (the plan, the launch and the epilogue all use it).
// Optional members of an expanded op: kRtX (its targets per thread, default LDDMM_RT_X), NAX (accumulators of the
// expanded form, default NA) with x_partial(expand, y, sums, out) mapping them to the NA sums the epilogue reads,
// and kExpandR2 (its bound on a block's radius^2, default kExpandR2 below).
template <class Op, class = void>
struct RtXOf : std::integral_constant<int, LDDMM_RT_X> {};
template <class Op>
struct RtXOf<Op, std::void_t<decltype(Op::kRtX)>> : std::integral_constant<int, Op::kRtX> {};
template <class Op, class = void>
struct NAXOf : std::integral_constant<int, Op::NA> {};
template <class Op>
struct NAXOf<Op, std::void_t<decltype(Op::NAX)>> : std::integral_constant<int, Op::NAX> {};
template <class Op, typename V, int RT, class Fam>
constexpr int kRunRT = (kUseExpanded<Op, V, Fam> && RtXOf<Op>::value > 0) ? RtXOf<Op>::value : RT;

template <class Op, typename V, int TPB, int RT, class Fam = Gauss>
__global__ void __launch_bounds__(TPB, MinCtas<Op, V>::value)
    pairs_kernel(const typename Op::Params P, int n, int m, int TT, long long W, int C,
                 typename VT<V>::Partial* __restrict__ ws, const float* __restrict__ boxes) {
  constexpr int L = VT<V>::kLanes;
  constexpr int G = RT / L;  // lane groups per thread
  constexpr int NU = (Op::NS + 1) / 2;
  constexpr int kUnroll = UnrollOf<Op>::value;
  static_assert(RT % L == 0, "targets per thread must be a multiple of the lane count");
  __shared__ Unit<V> sm[NU][TPB];
  // The segment's compensated sums live in shared memory (one private column per thread: no barrier needed) unless
  // the op keeps them in registers; shared memory frees 2-4 registers per accumulator for more resident warps.
  constexpr bool kSm = LDDMM_COMP_SMEM && !CompInRegisters<Op>::value;
  __shared__ V cs[kSm ? G * Op::NA * Comp<V>::kWords : 1][TPB];
  // Exact culling (ops with Culled<Op>): a (target block, source tile) unit whose coordinate boxes (box_kernel) are
  // farther apart than the distance at which the kernel's radial factors are exactly zero in this arithmetic
  // contributes exactly nothing, and is skipped by the whole CTA.
  constexpr float kZeroR2 = Fam::template kCullR2<V>;
  const int gx = (n + TPB * RT - 1) / (TPB * RT);
  __shared__ float tbox[6];  // the segment's target box, in shared memory (re-read per tile, not held in registers)

  const long long u_end = sk_start(blockIdx.x + 1, W, C);
  long long u = sk_start(blockIdx.x, W, C);
  while (u < u_end) {
    const int tb = (int)(u / TT);
    const int j0 = (int)(u - (long long)tb * TT);
    const int j1 = (int)((u_end - (long long)tb * TT) < TT ? (u_end - (long long)tb * TT) : TT);
    const int slot = (int)blockIdx.x - sk_cta_of((long long)tb * TT, W, C);

    typename Op::template Tgt<V> tgt[G];
    Comp<V> cmp[G][Op::NA];   // used when !kSm
    // target of (group g, lane k): base + (g * L + k) * TPB
    const int base = tb * (TPB * RT) + threadIdx.x;
#pragma unroll
    for (int g = 0; g < G; ++g) {
      int i0 = base + (g * L) * TPB, i1 = base + (g * L + L - 1) * TPB;
      i0 = i0 < n ? i0 : n - 1;
      i1 = i1 < n ? i1 : n - 1;
      Op::template load_target<V>(P, i0, i1, tgt[g]);
#pragma unroll
      for (int c = 0; c < Op::NA; ++c) {
        cmp[g][c].zero();
        if constexpr (kSm) cmp[g][c].template store<TPB>(cs, g * Op::NA + c, threadIdx.x);
      }
    }
    if constexpr (Culled<Op>::value) {
      __syncthreads();  // the previous segment's last tile test has read tbox
      if (threadIdx.x < 6) tbox[threadIdx.x] = boxes[6 * tb + threadIdx.x];
      __syncthreads();
    }

    for (int j = j0; j < j1; ++j) {
      if constexpr (Culled<Op>::value) {
        const float* sbox = boxes + 6 * (gx + j);
        if (box_gap2(tbox, tbox + 3, sbox, sbox + 3) > kZeroR2) continue;  // uniform over the CTA
      }
      const int l = j * TPB + threadIdx.x;
      {
        double f[2 * NU];
#pragma unroll
        for (int q = 0; q < 2 * NU; ++q) f[q] = 0.0;
        if (l < m) Op::source_fields(P, l, f);
#pragma unroll
        for (int q = 0; q < NU; ++q) {
          Unit<V> w;
          w.a = VT<V>::dup(f[2 * q]);
          w.b = VT<V>::dup(f[2 * q + 1]);
          sm[q][threadIdx.x] = w;
        }
      }
      __syncthreads();
      V acc[G][Op::NA];
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int c = 0; c < Op::NA; ++c) acc[g][c] = VT<V>::zero();
#pragma unroll kUnroll
      for (int jj = 0; jj < TPB; ++jj) {
        V s[2 * NU];
#pragma unroll
        for (int q = 0; q < NU; ++q) {
          const Unit<V> w = sm[q][jj];
          s[2 * q] = w.a;
          s[2 * q + 1] = w.b;
        }
#pragma unroll
        for (int g = 0; g < G; ++g) Op::template pair<V, Fam>(P.f, tgt[g], s, acc[g]);
      }
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int c = 0; c < Op::NA; ++c) {
          if constexpr (kSm) cmp[g][c].template load<TPB>(cs, g * Op::NA + c, threadIdx.x);
          cmp[g][c].merge(acc[g][c]);
          if constexpr (kSm) cmp[g][c].template store<TPB>(cs, g * Op::NA + c, threadIdx.x);
        }
      __syncthreads();
    }

#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const int i = base + (g * L + k) * TPB;
        if (i < n) {
#pragma unroll
          for (int c = 0; c < Op::NA; ++c) {
            if constexpr (kSm) cmp[g][c].template load<TPB>(cs, g * Op::NA + c, threadIdx.x);
            ws[((size_t)slot * Op::NA + c) * (size_t)n + i] = cmp[g][c].partial(k);
          }
        }
      }
    u += j1 - j0;
  }
}

// ---------------------------------------------------------------------------------------------------------
// Expanded-distance Gaussian pair kernel (FP32; ops with Expanded<Op>).
//
// With the coordinates of a segment taken relative to the centre o of its target block (the midpoint of the
// block's coordinate box, scaled units),
//     2^-|y - x|^2 = 2^-|y|^2 * 2^-(|x|^2 - 2 y.x),
// and the bracket costs three packed FMAs per pair from the staged fields X = -2 x and q = |x|^2 (the difference
// form costs three subtractions, a multiply and two FMAs): 6 FP32 lane-ops and one ex2 per pair for K a instead
// of 9, which leaves the pair loop bound by the MUFU (ex2) pipe instead of the FP32 pipe. The factor 2^-|y|^2 is
// common to every term of a target and multiplies the segment's compensated sums once, in FP64, when they are
// written. The identity is exact for the FP32-rounded relative coordinates; the rounding of the bracket grows with
// |y|^2 and |x|^2 (far sources have a large |x|^2 but terms that are smaller still), so a block is evaluated in the
// expanded form only when its radius^2 (scaled) is at most kExpandR2, which keeps the relative L2 error of the
// sums near 1e-6 (FP32 emulation with targets in a ball of that radius: 7e-7 at 32, 1.2e-6 at 64; the difference
// form: 5e-8); other blocks (point sets in no spatial order, widths small against a block) use the difference form,
// which costs ~20% more per pair (and, stream-K balancing units rather than time, the kernel waits for the CTAs that
// drew such blocks). Both forms share the launch plan and the epilogue of pairs_kernel.
// ---------------------------------------------------------------------------------------------------------
constexpr float kExpandR2 = 64.0f;
template <class Op, class = void>
struct ExpandR2Of {
  static constexpr float value = kExpandR2;
};
template <class Op>
struct ExpandR2Of<Op, std::void_t<decltype(Op::kExpandR2)>> {
  static constexpr float value = Op::kExpandR2;
};
template <class Op, class = void>
struct HasXPartial : std::false_type {};
template <class Op>
struct HasXPartial<Op, std::void_t<decltype(&Op::x_partial)>> : std::true_type {};

template <class Op, int TPB, int RT>
__global__ void __launch_bounds__(TPB, MinCtas<Op, F2>::value)
    pairs_kernel_x(const typename Op::Params P, int n, int m, int TT, long long W, int C,
                   float2* __restrict__ ws, const float* __restrict__ boxes) {
  constexpr int L = 2;
  constexpr int G = RT / L;
  constexpr int NF = 4 + Op::NP;  // staged fields: X or x (3), q (1), payload (NP)
  constexpr int NU = (NF + 1) / 2;
  constexpr int NAX = NAXOf<Op>::value;  // accumulators of the expanded form
  constexpr int kUnroll = UnrollOf<Op>::value;
  static_assert(RT % L == 0, "targets per thread must be a multiple of the lane count");
  __shared__ Unit<F2> sm[NU][TPB];
  __shared__ float red[6][TPB / 32];
  constexpr bool kSm = LDDMM_X_COMP_SMEM != 0;
  __shared__ F2 cs[kSm ? G * NAX * 2 : 1][TPB];
  const Frame& f = P.f;
  const double fo[3] = {f.o0, f.o1, f.o2};
  const int gx = (n + TPB * RT - 1) / (TPB * RT);

  const long long u_end = sk_start(blockIdx.x + 1, W, C);
  long long u = sk_start(blockIdx.x, W, C);
  while (u < u_end) {
    const int tb = (int)(u / TT);
    const int j0 = (int)(u - (long long)tb * TT);
    const int j1 = (int)((u_end - (long long)tb * TT) < TT ? (u_end - (long long)tb * TT) : TT);
    const int slot = (int)blockIdx.x - sk_cta_of((long long)tb * TT, W, C);
    const int base = tb * (TPB * RT) + threadIdx.x;

    // the block's box and centre (every CTA working on block tb derives the same ones)
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
    for (int t = 0; t < RT; ++t) {
      int i = base + t * TPB;
      i = i < n ? i : n - 1;
      double y[3];
      Op::target_point(P, i, y);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float v = (float)((y[c] - fo[c]) * f.s);
        lo[c] = fminf(lo[c], v);
        hi[c] = fmaxf(hi[c], v);
      }
    }
    block_box<TPB>(lo, hi, red);  // its barrier also orders the previous segment's last tile reads
    float ob[3], rb2 = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ob[c] = 0.5f * (lo[c] + hi[c]);
      const float h = 0.5f * (hi[c] - lo[c]);
      rb2 = fmaf(h, h, rb2);
    }
    const bool expand = rb2 <= ExpandR2Of<Op>::value;  // uniform over the CTA

    F2 yt[G][3];  // relative scaled target coordinates, lanes = targets (g L, g L + 1) of the thread
    typename Op::template TgtX<F2> tx[G];
    Comp<F2> cmp[G][NAX];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      int i0 = base + (g * L) * TPB, i1 = base + (g * L + 1) * TPB;
      i0 = i0 < n ? i0 : n - 1;
      i1 = i1 < n ? i1 : n - 1;
      double y0[3], y1[3];
      Op::target_point(P, i0, y0);
      Op::target_point(P, i1, y1);
#pragma unroll
      for (int c = 0; c < 3; ++c)
        yt[g][c] = f2((float)((y0[c] - fo[c]) * f.s - (double)ob[c]), (float)((y1[c] - fo[c]) * f.s - (double)ob[c]));
      Op::template load_target_x<F2>(P, i0, i1, tx[g]);
#pragma unroll
      for (int c = 0; c < NAX; ++c) {
        cmp[g][c].zero();
        if constexpr (kSm) cmp[g][c].template store<TPB>(cs, g * NAX + c, threadIdx.x);
      }
    }

    for (int j = j0; j < j1; ++j) {
      if constexpr (Culled<Op>::value) {
        // the same test as pairs_kernel: every term of the unit is exactly zero in the difference form; in the
        // expanded form each would be below 2^-127 of its payload
        const float* sbox = boxes + 6 * (gx + j);
        if (box_gap2(lo, hi, sbox, sbox + 3) > Gauss::kCullR2<F2>) continue;  // uniform over the CTA
      }
      const int l = j * TPB + threadIdx.x;
      {
        double fl[2 * NU];
#pragma unroll
        for (int q = 0; q < 2 * NU; ++q) fl[q] = 0.0;
        if (l < m) {
          double xr[3], r2 = 0.0;
          Op::source_point(P, l, xr, fl + 4);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float xc = (float)((xr[c] - fo[c]) * f.s - (double)ob[c]);
            r2 += (double)xc * (double)xc;
            fl[c] = expand ? -2.0 * (double)xc : (double)xc;
          }
          fl[3] = r2;
        }
#pragma unroll
        for (int q = 0; q < NU; ++q) {
          Unit<F2> w;
          w.a = VT<F2>::dup(fl[2 * q]);
          w.b = VT<F2>::dup(fl[2 * q + 1]);
          sm[q][threadIdx.x] = w;
        }
      }
      __syncthreads();
      F2 acc[G][NAX];
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int c = 0; c < NAX; ++c) acc[g][c] = VT<F2>::zero();
      if (expand) {
#pragma unroll kUnroll
        for (int jj = 0; jj < TPB; ++jj) {
          F2 s[2 * NU];
#pragma unroll
          for (int q = 0; q < NU; ++q) {
            const Unit<F2> w = sm[q][jj];
            s[2 * q] = w.a;
            s[2 * q + 1] = w.b;
          }
#pragma unroll
          for (int g = 0; g < G; ++g) {
            F2 arg = fma(yt[g][2], s[2], s[3]);  // |x|^2 - 2 y.x
            arg = fma(yt[g][1], s[1], arg);
            arg = fma(yt[g][0], s[0], arg);
            Op::template accumulate<true>(tx[g], yt[g], VT<F2>::expneg(arg), s, acc[g]);
          }
        }
      } else {
#pragma unroll kUnroll
        for (int jj = 0; jj < TPB; ++jj) {
          F2 s[2 * NU];
#pragma unroll
          for (int q = 0; q < NU; ++q) {
            const Unit<F2> w = sm[q][jj];
            s[2 * q] = w.a;
            s[2 * q + 1] = w.b;
          }
#pragma unroll
          for (int g = 0; g < G; ++g) {
            const F2 d0 = yt[g][0] - s[0], d1 = yt[g][1] - s[1], d2 = yt[g][2] - s[2];
            Op::template accumulate<false>(tx[g], yt[g], VT<F2>::expneg(fma(d2, d2, fma(d1, d1, d0 * d0))), s, acc[g]);
          }
        }
      }
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int c = 0; c < NAX; ++c) {
          if constexpr (kSm) cmp[g][c].template load<TPB>(cs, g * NAX + c, threadIdx.x);
          cmp[g][c].merge(acc[g][c]);
          if constexpr (kSm) cmp[g][c].template store<TPB>(cs, g * NAX + c, threadIdx.x);
        }
      __syncthreads();
    }

#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const int i = base + (g * L + k) * TPB;
        if (i < n) {
          double yr[3], y2 = 0.0;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            yr[c] = VT<F2>::lane(yt[g][c], k);
            y2 += yr[c] * yr[c];
          }
          const double fac = expand ? exp2(-y2) : 1.0;
          double v[NAX], o[Op::NA];
#pragma unroll
          for (int c = 0; c < NAX; ++c) {
            if constexpr (kSm) cmp[g][c].template load<TPB>(cs, g * NAX + c, threadIdx.x);
            const float2 p = cmp[g][c].partial(k);
            v[c] = (double)p.x + (double)p.y;
          }
          if constexpr (HasXPartial<Op>::value) {
            Op::x_partial(expand, yr, v, o);
          } else {
#pragma unroll
            for (int c = 0; c < Op::NA; ++c) o[c] = v[c];
          }
#pragma unroll
          for (int c = 0; c < Op::NA; ++c) {
            const double w = o[c] * fac;
            const float h = (float)w;
            ws[((size_t)slot * Op::NA + c) * (size_t)n + i] = make_float2(h, (float)(w - (double)h));
          }
        }
      }
    u += j1 - j0;
  }
}

// Coordinate boxes for exact culling, from the same scaled coordinates the pair kernel uses: block b < gx covers
// target block b (its TPB * RT targets), block gx + j source tile j. boxes[6 b ..] = (lo xyz, hi xyz).
template <class Op, typename V, int TPB, int RT>
__global__ void __launch_bounds__(TPB) box_kernel(const typename Op::Params P, int n, int m, int gx,
                                                  float* __restrict__ boxes) {
  constexpr int L = VT<V>::kLanes;
  constexpr int G = RT / L;
  constexpr int NU = (Op::NS + 1) / 2;
  __shared__ float red[6][TPB / 32];
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  const int b = blockIdx.x;
  if (b < gx) {
    const int base = b * (TPB * RT) + threadIdx.x;
#pragma unroll
    for (int g = 0; g < G; ++g) {
      int i0 = base + (g * L) * TPB, i1 = base + (g * L + L - 1) * TPB;
      i0 = i0 < n ? i0 : n - 1;
      i1 = i1 < n ? i1 : n - 1;
      typename Op::template Tgt<V> t;
      Op::template load_target<V>(P, i0, i1, t);
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const float y[3] = {(float)VT<V>::lane(t.y0, k), (float)VT<V>::lane(t.y1, k), (float)VT<V>::lane(t.y2, k)};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          lo[c] = fminf(lo[c], y[c]);
          hi[c] = fmaxf(hi[c], y[c]);
        }
      }
    }
  } else {
    const int l = (b - gx) * TPB + threadIdx.x;
    if (l < m) {
      double f[2 * NU];
      Op::source_fields(P, l, f);
#pragma unroll
      for (int c = 0; c < 3; ++c) lo[c] = hi[c] = (float)f[c];
    }
  }
  block_box<TPB>(lo, hi, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      boxes[6 * b + c] = lo[c];
      boxes[6 * b + 3 + c] = hi[c];
    }
  }
}

// Epilogue: reduce the partial slots of target i (its block's CTAs, in CTA order) in FP64, then Op::finalize.
template <class Op, typename V>
__global__ void finalize_kernel(const typename Op::Params P, int n, int tb_targets, int TT, long long W, int C,
                                const typename VT<V>::Partial* __restrict__ ws) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc[Op::NA];
#pragma unroll
  for (int c = 0; c < Op::NA; ++c) acc[c] = 0.0;
  if (W > 0) {
    const int tb = i / tb_targets;
    const int nslot = sk_cta_of((long long)(tb + 1) * TT - 1, W, C) - sk_cta_of((long long)tb * TT, W, C) + 1;
    for (int s = 0; s < nslot; ++s)
#pragma unroll
      for (int c = 0; c < Op::NA; ++c) acc[c] += partial_value(ws[((size_t)s * Op::NA + c) * (size_t)n + i]);
  }
  Op::finalize(P, i, acc);
}

// Deterministic single-block sum of `count` doubles: out[0] = (accumulate ? out[0] : 0) + scale * sum(v).
__global__ void ordered_sum_kernel(const double* __restrict__ v, int count, double scale, double* out, int accumulate);

int resident_ctas(const void* kernel, int threads, size_t dynamic_smem = 0);

template <class Op, typename V, int TPB, int RT, class Fam = Gauss>
inline int ctas_per_sm() {
  static int cached = 0;
  if (cached == 0) {
    const void* k;
    if constexpr (kUseExpanded<Op, V, Fam>)
      k = reinterpret_cast<const void*>(&pairs_kernel_x<Op, TPB, kRunRT<Op, V, RT, Fam>>);
    else
      k = reinterpret_cast<const void*>(&pairs_kernel<Op, V, TPB, RT, Fam>);
    int c = resident_ctas(k, TPB);
    cached = c > 0 ? c : 4;
  }
  return cached;
}

template <class Op, typename V, int TPB, int RT, class Fam = Gauss>
inline int run_pairs(const typename Op::Params& P, int64_t n, int64_t m, void* ws, size_t ws_bytes,
                     cudaStream_t stream) {
  if (n <= 0) return kOk;
  if (n > INT32_MAX / 4 || m > INT32_MAX / 4) return kInvalidArgument;
  constexpr int R = kRunRT<Op, V, RT, Fam>;
  SKPlan plan = make_plan<TPB, R>(n, m, Op::NA, sizeof(typename VT<V>::Partial),
                                  ctas_per_sm<Op, V, TPB, RT, Fam>(), Culled<Op>::value);
  if (plan.ws_bytes > ws_bytes) return kWorkspaceTooSmall;
  if (plan.ws_bytes > 0 && ws == nullptr) return kInvalidArgument;
  auto* part = reinterpret_cast<typename VT<V>::Partial*>(ws);
  if (plan.W > 0) {
    float* boxes = Culled<Op>::value ? reinterpret_cast<float*>(reinterpret_cast<char*>(ws) + plan.box_off) : nullptr;
    if (Culled<Op>::value)
      box_kernel<Op, V, TPB, R><<<plan.gx + plan.TT, TPB, 0, stream>>>(P, (int)n, (int)m, plan.gx, boxes);
    if constexpr (kUseExpanded<Op, V, Fam>) {
      pairs_kernel_x<Op, TPB, R><<<plan.C, TPB, 0, stream>>>(P, (int)n, (int)m, plan.TT, plan.W, plan.C, part,
                                                              boxes);
    } else {
      pairs_kernel<Op, V, TPB, RT, Fam><<<plan.C, TPB, 0, stream>>>(P, (int)n, (int)m, plan.TT, plan.W, plan.C,
                                                                     part, boxes);
    }
  }
  const int fb = 256;
  finalize_kernel<Op, V><<<(int)((n + fb - 1) / fb), fb, 0, stream>>>(P, (int)n, TPB * R, plan.TT, plan.W, plan.C,
                                                                      part);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

template <class Op, typename V, int TPB, int RT, class Fam = Gauss>
inline size_t pairs_ws_bytes(int64_t n, int64_t m) {
  return make_plan<TPB, kRunRT<Op, V, RT, Fam>>(n, m, Op::NA, sizeof(typename VT<V>::Partial),
                                                ctas_per_sm<Op, V, TPB, RT, Fam>(), Culled<Op>::value)
      .ws_bytes;
}

// Workspace of an op for every kernel family (the larger of the Gaussian and Laplacian plans).
template <class Op, typename V, int TPB, int RT>
inline size_t pairs_ws_bytes_any(int64_t n, int64_t m) {
  const size_t a = pairs_ws_bytes<Op, V, TPB, RT, Gauss>(n, m), b = pairs_ws_bytes<Op, V, TPB, RT, Laplacian>(n, m);
  return a > b ? a : b;
}

inline bool bad_kernel(int kernel) { return !(kernel == kGauss || (kernel >= kLaplacian0 && kernel <= kLaplacianMax)); }

// Frame of one kernel width. `fp32` selects the FP32 scaling (exp2-based) or the FP64 one (exp-based).
inline Frame make_frame(const double* origin, double sigma, int kernel, bool fp32) {
  Frame f = {};
  f.family = kernel;
  f.o0 = origin ? origin[0] : 0.0;
  f.o1 = origin ? origin[1] : 0.0;
  f.o2 = origin ? origin[2] : 0.0;
  constexpr double kLog2e = 1.44269504088896340736;
  if (kernel == kGauss) {
    f.s = (fp32 ? VT<F2>::kScale : VT<double>::kScale) / sigma;
  } else {
    // P0 = lapPol of the order (Matern polynomial); P1 = (P0 - P0') / u and P2 = (P1 - P1') / u when the division
    // is exact (the constant terms cancel), else zero -- the reference's derivative tables for orders 0 and 1.
    static const double kP0[5][5] = {{1, 0, 0, 0, 0},
                                     {1, 1, 0, 0, 0},
                                     {1, 1, 1.0 / 3, 0, 0},
                                     {1, 1, 0.4, 1.0 / 15, 0},
                                     {1, 1, 3.0 / 7, 2.0 / 21, 1.0 / 105}};
    const int q = kernel - kLaplacian0;
    double c[3][5] = {};
    for (int k = 0; k < 5; ++k) c[0][k] = kP0[q][k];
    for (int r = 1; r < 3; ++r) {
      double d[5] = {};  // c[r-1] - derivative of c[r-1]
      for (int k = 0; k < 5; ++k) d[k] = c[r - 1][k] - (k + 1 < 5 ? (k + 1) * c[r - 1][k + 1] : 0.0);
      if (d[0] > -1e-12 && d[0] < 1e-12)  // exact in rationals; rounding leaves ~1e-17
        for (int k = 0; k < 4; ++k) c[r][k] = d[k + 1];
    }
    const double unit = fp32 ? kLog2e : 1.0;  // FP32 works in u' = log2(e) u so that E = 2^-u'
    f.s = unit / sigma;
    double pw = 1.0;
    for (int k = 0; k < 5; ++k) {
      for (int r = 0; r < 3; ++r) {
        f.dc[r][k] = c[r][k] * pw;
        f.lc[r][k] = (float)(c[r][k] * pw);
      }
      pw /= unit;
    }
  }
  f.kappa = 1.0 / (f.s * sigma * sigma);
  f.inv_s2 = 1.0 / (sigma * sigma);
  return f;
}

// Launch an op with the pair kernel of its frame's family (P.f.family).
template <class Op, typename V, int TPB, int RT>
inline int run_pairs_k(const typename Op::Params& P, int64_t n, int64_t m, void* ws, size_t ws_bytes,
                       cudaStream_t stream) {
  if (P.f.family == kGauss) return run_pairs<Op, V, TPB, RT, Gauss>(P, n, m, ws, ws_bytes, stream);
  return run_pairs<Op, V, TPB, RT, Laplacian>(P, n, m, ws, ws_bytes, stream);
}

inline bool bad_sigma(double sigma) { return !(sigma > 0.0) || !(sigma < 1e300); }

// Source point in the frame (FP64 before the per-path conversion).
__device__ __forceinline__ void src_point(const double* __restrict__ p, int l, const Frame& f, double* o) {
  o[0] = (p[3 * l + 0] - f.o0) * f.s;
  o[1] = (p[3 * l + 1] - f.o1) * f.s;
  o[2] = (p[3 * l + 2] - f.o2) * f.s;
}

}  // namespace lddmm
