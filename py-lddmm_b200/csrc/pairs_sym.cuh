// Symmetric all-pairs kernel for self-interaction sums (targets and sources are the same n points), FP32 only.
//
// A sum out_k = sum_l f(k, l) over the same point set evaluates every unordered pair twice in pairs_kernel. When
// f(l, k) follows from the quantities of f(k, l) (the kernel value, the dot products and the difference vector, up to
// a sign), each unordered pair can be evaluated once and credited to both points. This kernel does that:
//
//  * The points are cut into blocks of B = TPB * RT (the target blocks of pairs_kernel) and tiles of TPB (its source
//    tiles); block j holds tiles RT j .. RT j + RT - 1. A unit is (target block i, source tile t) with t in a block
//    j >= i: the upper triangle in blocks. Units with j == i ("diagonal") evaluate their ordered pairs for the rows
//    only, like pairs_kernel; units with j > i evaluate each pair once and credit the row k (registers, as in
//    pairs_kernel) and the column l.
//  * Column credit without atomics: inside a tile, warp w of the CTA takes chunk (w + phase) mod W of 32 sources in
//    phase `phase` (one barrier per phase), and lane λ processes source (λ + s) mod 32 of the chunk at step s: the 32
//    lanes read 32 different sources (conflict-free 16-byte loads of the shared tile). The lane's column sum for its
//    source (its RT targets) is added to a rotating accumulator that moves one lane down after every step (one
//    shuffle per accumulator), so it follows its source around the warp; after 32 steps lane λ holds the warp's
//    column sum of source λ of the chunk and adds it to the tile's column accumulators in shared memory. At the end
//    of the unit those hold the unit's column sums (TPB sources x NC), written as one partial per (block i, source).
//  * Stream-K over the units in row-major order (as pairs_kernel over its units): a CTA's run of units of one row i
//    is a segment with compensated row sums (one partial slot, as in pairs_kernel). Point l of block b then has the
//    row slots of block b and b column partials (one from each block i < b); the epilogue sums both in a fixed order
//    in FP64 and hands them to Op::finalize_sym. Deterministic, no atomics.
//
// Units are balanced in count, not time: a column unit costs ~1.3x a diagonal one, and diagonal units are 1 in
// (number of blocks) per row, so the imbalance is a few percent. Padded targets (past n) carry zero payload fields,
// so their column credit is zero; padded sources carry zero fields, so their row credit is zero.
//
// Op interface (besides Params, finalize_sym):
//   NSS                                  source fields staged per source (scaled coordinates 0-2 first)
//   NR, NC                               row and column accumulators per point
//   SymTgt                               per-lane-group (two targets) register state
//   load_target_sym(P, i0, i1, v0, v1, SymTgt&)     targets i0, i1 (< n); v0 / v1 false = padding (zero payload)
//   source_fields_sym(P, l, double* f)   NSS fields of source l (FP64)
//   pair_sym<COL>(const Frame&, const SymTgt&, const F2* s, F2* row, F2* col)
//   finalize_sym(P, i, const double* row, const double* col)
#pragma once
#include "lddmm_common.cuh"

#ifndef LDDMM_SYM
#define LDDMM_SYM 1  // 0: self-interaction sums evaluate every ordered pair (pairs_kernel)
#endif
#ifndef LDDMM_SYM_COMPACT
#define LDDMM_SYM_COMPACT 1  // 0: the symmetric kernels stage sources in pairs_kernel's duplicated layout (measured
                             // 3-6% slower at level 6: twice the bytes per unshared load)
#endif
#ifndef LDDMM_SYMX_COL_SPLIT
#define LDDMM_SYMX_COL_SPLIT 0  // 1: pairs_kernel_symx accumulates the column terms of even and odd lane groups apart
#endif
#ifndef LDDMM_SYMX_UNROLL
#define LDDMM_SYMX_UNROLL 8  // unroll depth of pairs_kernel_symx's source loop (8: 1% faster than 4 at level 6)
#endif
#ifndef LDDMM_SYM_UNROLL
#define LDDMM_SYM_UNROLL 4  // unroll depth of the 32-step source loop of a chunk (4: 1% faster than 2 at level 6)
#endif

namespace lddmm {

constexpr int kSymUnroll = LDDMM_SYM_UNROLL;
constexpr int kSymxUnroll = LDDMM_SYMX_UNROLL;

// Shared-memory record of a staged source tile. In the symmetric kernels the 32 lanes of a warp read 32 different
// sources at every step (no broadcast), so the record size is what the loads cost: compact records hold each field
// once in FP32 (float4 groups) and the packed (f, f) operands are formed in registers; the duplicated layout of
// pairs_kernel (Unit<F2>: one 16-byte load gives two packed operands) reads twice the bytes.
template <int NF, int TPB>
struct SymStage {
#if LDDMM_SYM_COMPACT
  static constexpr int NQ = (NF + 3) / 4;  // float4 groups
  using T = float4;
  static __device__ __forceinline__ void store(T (*sm)[TPB], int t, const double* fl) {
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      sm[q][t] = make_float4((float)fl[4 * q], (float)fl[4 * q + 1], (float)fl[4 * q + 2], (float)fl[4 * q + 3]);
  }
  static __device__ __forceinline__ void load(const T (*sm)[TPB], int src, F2* sv) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const float4 w = sm[q][src];
      sv[4 * q] = f2(w.x, w.x);
      sv[4 * q + 1] = f2(w.y, w.y);
      sv[4 * q + 2] = f2(w.z, w.z);
      sv[4 * q + 3] = f2(w.w, w.w);
    }
  }
#else
  static constexpr int NQ = (NF + 1) / 2;  // 16-byte units of two duplicated fields
  using T = Unit<F2>;
  static __device__ __forceinline__ void store(T (*sm)[TPB], int t, const double* fl) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      Unit<F2> w;
      w.a = VT<F2>::dup(fl[2 * q]);
      w.b = VT<F2>::dup(fl[2 * q + 1]);
      sm[q][t] = w;
    }
  }
  static __device__ __forceinline__ void load(const T (*sm)[TPB], int src, F2* sv) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const Unit<F2> w = sm[q][src];
      sv[2 * q] = w.a;
      sv[2 * q + 1] = w.b;
    }
  }
#endif
  static constexpr int kFields = 4 * ((NF + 3) / 4);  // size of the FP64 field buffer and of the operand array
};

// first unit of row i (rows: target blocks; row i holds the tiles RT i .. TT - 1)
__host__ __device__ __forceinline__ long long sym_row_off(long long i, long long TT, long long RT) {
  return i * TT - RT * (i * (i - 1) / 2);
}
__host__ __device__ __forceinline__ long long sym_tri(long long j) { return j * (j - 1) / 2; }

__device__ __forceinline__ int sym_row_of(long long u, int nblk, long long TT, long long RT) {
  int lo = 0, hi = nblk - 1;  // largest i with off(i) <= u
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sym_row_off(mid, TT, RT) <= u) lo = mid; else hi = mid - 1;
  }
  return lo;
}

struct SymPlan {
  int nblk = 0, TT = 0, C = 0, S = 0;
  long long U = 0;
  size_t col_off = 0, ws_bytes = 0;
};

template <int TPB, int RT>
inline SymPlan make_sym_plan(int64_t n, int nr, int nc, int ctas_per_sm) {
  SymPlan p;
  if (n <= 0) return p;
  constexpr int64_t B = (int64_t)TPB * RT;
  p.nblk = (int)((n + B - 1) / B);
  p.TT = (int)((n + TPB - 1) / TPB);
  p.U = sym_row_off(p.nblk, p.TT, RT);
  const long long wave = (long long)device_sm_count() * (ctas_per_sm > 0 ? ctas_per_sm : 1);
  p.C = (int)(p.U < wave ? p.U : wave);
  int smax = 1;
  for (int i = 0; i < p.nblk; ++i) {
    const int c0 = sk_cta_of(sym_row_off(i, p.TT, RT), p.U, p.C);
    const int c1 = sk_cta_of(sym_row_off(i + 1, p.TT, RT) - 1, p.U, p.C);
    if (c1 - c0 + 1 > smax) smax = c1 - c0 + 1;
  }
  p.S = smax;
  p.col_off = ((size_t)p.S * (size_t)nr * (size_t)n * sizeof(float2) + 255) & ~(size_t)255;
  p.ws_bytes = p.col_off + (size_t)sym_tri(p.nblk) * (size_t)nc * (size_t)B * sizeof(float);
  return p;
}

template <class Op, int TPB, int RT, bool COL, class Fam>
__device__ __forceinline__ void sym_tile(const Frame& f, const typename Op::SymTgt (&tgt)[RT / 2],
                                         const typename SymStage<Op::NSS, TPB>::T (*sm)[TPB], float (*colacc)[TPB],
                                         F2 (&acc)[RT / 2][Op::NR]) {
  using St = SymStage<Op::NSS, TPB>;
  constexpr int G = RT / 2, W = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll 1
  for (int ph = 0; ph < W; ++ph) {
    const int chunk = (warp + ph) % W;
    float cs[Op::NC];
#pragma unroll
    for (int c = 0; c < Op::NC; ++c) cs[c] = 0.f;
#pragma unroll kSymUnroll
    for (int s = 0; s < 32; ++s) {
      const int src = chunk * 32 + ((lane + s) & 31);
      F2 sv[St::kFields];
      St::load(sm, src, sv);
      if constexpr (COL) {
        F2 col[Op::NC];
#pragma unroll
        for (int c = 0; c < Op::NC; ++c) col[c] = f2(cs[c], 0.f);
#pragma unroll
        for (int g = 0; g < G; ++g) Op::template pair_sym<true, Fam>(f, tgt[g], sv, acc[g], col);
#pragma unroll
        for (int c = 0; c < Op::NC; ++c) {
          float lo, hi;
          split(col[c], lo, hi);
          cs[c] = __shfl_sync(0xffffffffu, lo + hi, (lane + 1) & 31);
        }
      } else {
#pragma unroll
        for (int g = 0; g < G; ++g) Op::template pair_sym<false, Fam>(f, tgt[g], sv, acc[g], nullptr);
      }
    }
    if constexpr (COL) {
#pragma unroll
      for (int c = 0; c < Op::NC; ++c) colacc[c][chunk * 32 + lane] += cs[c];
    }
    __syncthreads();  // the next phase hands this chunk (and its column accumulators) to another warp
  }
}

template <class Op, int TPB, int RT, class Fam = Gauss>
__global__ void __launch_bounds__(TPB, Op::kSymMinCtas)
    pairs_kernel_sym(const typename Op::Params P, int n, int nblk, int TT, long long U, int C,
                     float2* __restrict__ row_ws, float* __restrict__ col_ws) {
  using St = SymStage<Op::NSS, TPB>;
  constexpr int L = 2, G = RT / L, NR = Op::NR, NC = Op::NC;
  constexpr int B = TPB * RT;
  static_assert(TPB % 32 == 0 && RT % L == 0, "launch shape");
  __shared__ typename St::T sm[St::NQ][TPB];
  __shared__ float colacc[NC][TPB];
  // compensated row sums of the segment, one private column per thread (G * NR * 2 rows of TPB): dynamic shared
  // memory, so that 8 targets per thread may take more than the 48 KiB of static shared memory
  extern __shared__ __align__(16) unsigned char sym_dyn_smem[];
  F2 (*cs)[TPB] = reinterpret_cast<F2 (*)[TPB]>(sym_dyn_smem);
  const Frame& f = P.f;

  const long long u_end = sk_start(blockIdx.x + 1, U, C);
  long long u = sk_start(blockIdx.x, U, C);
  int i = u < u_end ? sym_row_of(u, nblk, TT, RT) : 0;
  while (u < u_end) {
    const long long off = sym_row_off(i, TT, RT);
    const int cnt = TT - RT * i;
    const int t0 = (int)(u - off);
    const int t1 = (int)((u_end - off) < cnt ? (u_end - off) : cnt);
    const int slot = (int)blockIdx.x - sk_cta_of(off, U, C);
    const int base = i * B + threadIdx.x;

    typename Op::SymTgt tgt[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int i0 = base + (g * L) * TPB, i1 = base + (g * L + 1) * TPB;
      Op::load_target_sym(P, i0 < n ? i0 : n - 1, i1 < n ? i1 : n - 1, i0 < n, i1 < n, tgt[g]);
      Comp<F2> z;
      z.zero();
#pragma unroll
      for (int c = 0; c < NR; ++c) z.template store<TPB>(cs, g * NR + c, threadIdx.x);
    }

    for (int tt = t0; tt < t1; ++tt) {
      const int t = RT * i + tt;  // absolute source tile
      const bool diag = tt < RT;  // tile of block i itself: rows only
      {
        const int l = t * TPB + threadIdx.x;
        double fl[St::kFields];
#pragma unroll
        for (int q = 0; q < St::kFields; ++q) fl[q] = 0.0;
        if (l < n) Op::source_fields_sym(P, l, fl);
        St::store(sm, threadIdx.x, fl);
#pragma unroll
        for (int c = 0; c < NC; ++c) colacc[c][threadIdx.x] = 0.f;
      }
      __syncthreads();
      F2 acc[G][NR];
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int c = 0; c < NR; ++c) acc[g][c] = VT<F2>::zero();
      if (diag)
        sym_tile<Op, TPB, RT, false, Fam>(f, tgt, sm, colacc, acc);
      else
        sym_tile<Op, TPB, RT, true, Fam>(f, tgt, sm, colacc, acc);
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int c = 0; c < NR; ++c) {
          Comp<F2> m;
          m.template load<TPB>(cs, g * NR + c, threadIdx.x);
          m.merge(acc[g][c]);
          m.template store<TPB>(cs, g * NR + c, threadIdx.x);
        }
      if (!diag) {
        // column partial of unit (block i, tile t): block j of the tile, from row block i (< j)
        const int j = t / RT;
        const size_t cb = (size_t)(sym_tri(j) + i) * NC * B + (size_t)(t - RT * j) * TPB + threadIdx.x;
#pragma unroll
        for (int c = 0; c < NC; ++c) col_ws[cb + (size_t)c * B] = colacc[c][threadIdx.x];
      }
      // the last phase barrier of sym_tile orders every read of sm and colacc before the next tile's staging
    }

#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const int idx = base + (g * L + k) * TPB;
        if (idx < n) {
#pragma unroll
          for (int c = 0; c < NR; ++c) {
            Comp<F2> m;
            m.template load<TPB>(cs, g * NR + c, threadIdx.x);
            row_ws[((size_t)slot * NR + c) * (size_t)n + idx] = m.partial(k);
          }
        }
      }
    u += t1 - t0;
    ++i;
  }
}

// Epilogue: the row slots of the point's block and its column partials, in FP64, summed by TPP threads per point
// (TPP a power of two <= 32). A CTA of kFinThreads threads takes P = kFinThreads / TPP consecutive points; thread
// (j, p) -- p = threadIdx % P, j = threadIdx / P -- sums slots j, j + TPP, ... and column partials j, j + TPP, ...
// of point p (consecutive threads read consecutive points: coalesced), and thread (0, p) adds the TPP sums in the
// order j = 0, 1, ... from shared memory and applies the op's epilogue. Every addition's order is fixed by (point,
// TPP): deterministic. With one thread per point, a point's slots and partials are one serial chain of up to tens
// of dependent loads (at 2,562 points: 11 CTAs, ~11 us, latency-bound); several threads shorten the chain and
// spread the points over more CTAs.
constexpr int kFinThreads = 256;
template <class Op, int TPB, int RT>
__global__ void __launch_bounds__(kFinThreads)
    finalize_sym_kernel(const typename Op::Params P, int n, int nblk, int TT, long long U, int C,
                        const float2* __restrict__ row_ws, const float* __restrict__ col_ws, int tpp) {
  constexpr int B = TPB * RT, NV = Op::NR + Op::NC;
  __shared__ double red[kFinThreads][NV];
  const int np = kFinThreads / tpp;
  const int p = threadIdx.x % np, j = threadIdx.x / np;
  const int idx = blockIdx.x * np + p;
  const bool live = idx < n;
  double v[NV];
#pragma unroll
  for (int c = 0; c < NV; ++c) v[c] = 0.0;
  const int b = live ? idx / B : 0, r = live ? idx - b * B : 0;
  if (live) {
    const int nslot = sk_cta_of(sym_row_off(b + 1, TT, RT) - 1, U, C) - sk_cta_of(sym_row_off(b, TT, RT), U, C) + 1;
    for (int s = j; s < nslot; s += tpp)
#pragma unroll
      for (int c = 0; c < Op::NR; ++c) v[c] += partial_value(row_ws[((size_t)s * Op::NR + c) * (size_t)n + idx]);
    for (int q = j; q < b; q += tpp) {
      const size_t cb = (size_t)(sym_tri(b) + q) * Op::NC * B + r;
#pragma unroll
      for (int c = 0; c < Op::NC; ++c) v[Op::NR + c] += (double)col_ws[cb + (size_t)c * B];
    }
  }
  if (tpp > 1) {
#pragma unroll
    for (int c = 0; c < NV; ++c) red[threadIdx.x][c] = v[c];
    __syncthreads();
    if (j == 0)
      for (int k = 1; k < tpp; ++k)
#pragma unroll
        for (int c = 0; c < NV; ++c) v[c] += red[k * np + p][c];
  }
  if (live && j == 0) Op::finalize_sym(P, idx, v, v + Op::NR);
}

// Threads per point of finalize_sym_kernel: enough to split the longest chain of slots and column partials (a row
// block's slots plus the blocks below it) into pieces of about four, at most 8.
inline int sym_finalize_tpp(const SymPlan& p) {
  const int chain = p.S + p.nblk;
  int t = 1;
  while (t < 8 && chain > 4 * t) t <<= 1;
  return t;
}

inline int sym_finalize_grid(int64_t n, int tpp, int threads) {
  const int64_t np = threads / tpp;
  return (int)((n + np - 1) / np);
}

// Dynamic shared memory of pairs_kernel_sym (its compensated row sums).
template <class Op, int TPB, int RT>
constexpr size_t sym_dyn_smem_bytes() {
  return (size_t)(RT / 2) * Op::NR * 2 * TPB * sizeof(F2);
}

// Declare the kernel's dynamic shared memory, once per device (the attribute belongs to the device's context):
// without it static + dynamic shared memory may not exceed 48 KiB. Returns false when the device refuses.
template <class Op, int TPB, int RT, class Fam = Gauss>
inline bool sym_prepare() {
  static signed char state[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (dev < 0 || dev >= 64) return false;
  if (state[dev] == 0) {
    const cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(&pairs_kernel_sym<Op, TPB, RT, Fam>),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sym_dyn_smem_bytes<Op, TPB, RT>());
    if (e != cudaSuccess) cudaGetLastError();
    state[dev] = e == cudaSuccess ? 1 : -1;
  }
  return state[dev] > 0;
}

template <class Op, int TPB, int RT, class Fam = Gauss>
inline int sym_ctas_per_sm() {
  static int cached = 0;
  if (cached == 0) {
    sym_prepare<Op, TPB, RT, Fam>();
    int c = resident_ctas(reinterpret_cast<const void*>(&pairs_kernel_sym<Op, TPB, RT, Fam>), TPB,
                          sym_dyn_smem_bytes<Op, TPB, RT>());
    cached = c > 0 ? c : 2;
  }
  return cached;
}

template <class Op, int TPB, int RT, class Fam = Gauss>
inline size_t sym_ws_bytes(int64_t n) {
  return make_sym_plan<TPB, RT>(n, Op::NR, Op::NC, sym_ctas_per_sm<Op, TPB, RT, Fam>()).ws_bytes;
}

template <class Op, int TPB, int RT, class Fam = Gauss>
inline int run_pairs_sym(const typename Op::Params& P, int64_t n, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (n <= 0) return kOk;
  if (n > INT32_MAX / 4) return kInvalidArgument;
  const SymPlan plan = make_sym_plan<TPB, RT>(n, Op::NR, Op::NC, sym_ctas_per_sm<Op, TPB, RT, Fam>());
  if (plan.ws_bytes > ws_bytes) return kWorkspaceTooSmall;
  if (ws == nullptr) return kInvalidArgument;
  if (!sym_prepare<Op, TPB, RT, Fam>()) return kLaunchFailure;
  auto* row_ws = reinterpret_cast<float2*>(ws);
  auto* col_ws = reinterpret_cast<float*>(reinterpret_cast<char*>(ws) + plan.col_off);
  pairs_kernel_sym<Op, TPB, RT, Fam><<<plan.C, TPB, sym_dyn_smem_bytes<Op, TPB, RT>(), stream>>>(
      P, (int)n, plan.nblk, plan.TT, plan.U, plan.C, row_ws, col_ws);
  const int fb = kFinThreads, tpp = sym_finalize_tpp(plan);
  finalize_sym_kernel<Op, TPB, RT><<<sym_finalize_grid(n, tpp, fb), fb, 0, stream>>>(P, (int)n, plan.nblk, plan.TT,
                                                                                      plan.U, plan.C, row_ws, col_ws,
                                                                                      tpp);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}


// ---------------------------------------------------------------------------------------------------------
// Expanded-distance form of the symmetric kernel, for sums whose pair term is the kernel value times a payload of
// the source (K a over one point set: out_k = sum_l e_kl a_l, so the mirrored term of l is e_kl a_k).
//
// As in pairs_kernel_x, the coordinates of a unit are taken relative to the centre of its row block i (box centre
// of the block's TPB * RT points, scaled): e_kl = f_k w_kl with f_k = 2^-|y_k|^2 and w_kl = 2^-(|x_l|^2 - 2 y_k.x_l),
// the bracket being three packed FMAs from the staged fields (-2 x_l, |x_l|^2). The row sums of k accumulate
// w_kl a_l and are multiplied by f_k (FP64) when the segment's partial is written; the column payload of target k is
// f_k a_k, so the column sums accumulate w_kl f_k a_k = e_kl a_k directly. 9 FP32 lane-ops and one ex2 per
// unordered pair (against 6 + 1 per ordered pair, i.e. 12 + 2, for pairs_kernel_x). Row blocks whose radius^2
// (scaled units) exceeds kExpandR2 use the difference form (e from |y - x|^2, payload a_k; 12 + 1), chosen per
// segment. Everything else -- the unit triangle, the rotating column accumulators, the stream-K split, the partial
// layouts and finalize_sym_kernel -- is pairs_kernel_sym's.
//
// Op interface: Params, NP (payload fields; NR = NC = NP), kSymMinCtas, point(P, i, double* c) (coordinates of
// point i), payload(P, i, double* p), finalize_sym(P, i, row, col).
// ---------------------------------------------------------------------------------------------------------
template <class Op, int TPB, int RT, bool COL, bool X>
__device__ __forceinline__ void symx_tile(const F2 (&yt)[RT / 2][3], const F2 (&tp)[RT / 2][Op::NP],
                                          const typename SymStage<4 + Op::NP, TPB>::T (*sm)[TPB],
                                          float (*colacc)[TPB], F2 (&acc)[RT / 2][Op::NP]) {
  using St = SymStage<4 + Op::NP, TPB>;
  constexpr int G = RT / 2, NP = Op::NP, W = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll 1
  for (int ph = 0; ph < W; ++ph) {
    const int chunk = (warp + ph) % W;
    float cs[NP];
#pragma unroll
    for (int c = 0; c < NP; ++c) cs[c] = 0.f;
#pragma unroll kSymxUnroll
    for (int s = 0; s < 32; ++s) {
      const int src = chunk * 32 + ((lane + s) & 31);
      F2 sv[St::kFields];
      St::load(sm, src, sv);
      F2 col[NP], col2[NP];
      if constexpr (COL) {
#pragma unroll
        for (int c = 0; c < NP; ++c) {
          col[c] = f2(cs[c], 0.f);
          col2[c] = VT<F2>::zero();
        }
      }
#pragma unroll
      for (int g = 0; g < G; ++g) {
        F2 arg;
        if constexpr (X) {
          arg = fma(yt[g][2], sv[2], sv[3]);  // |x|^2 - 2 y.x
          arg = fma(yt[g][1], sv[1], arg);
          arg = fma(yt[g][0], sv[0], arg);
        } else {
          const F2 d0 = yt[g][0] - sv[0], d1 = yt[g][1] - sv[1], d2 = yt[g][2] - sv[2];
          arg = fma(d2, d2, fma(d1, d1, d0 * d0));
        }
        const F2 e = VT<F2>::expneg(arg);
#pragma unroll
        for (int c = 0; c < NP; ++c) acc[g][c] = fma(e, sv[4 + c], acc[g][c]);
        if constexpr (COL) {
          if (LDDMM_SYMX_COL_SPLIT != 0 && (g & 1)) {  // resolved at compile time (the loop is unrolled)
#pragma unroll
            for (int c = 0; c < NP; ++c) col2[c] = fma(e, tp[g][c], col2[c]);
          } else {
#pragma unroll
            for (int c = 0; c < NP; ++c) col[c] = fma(e, tp[g][c], col[c]);
          }
        }
      }
      if constexpr (COL) {
#pragma unroll
        for (int c = 0; c < NP; ++c) {
          if constexpr (LDDMM_SYMX_COL_SPLIT != 0) col[c] = col[c] + col2[c];
          float lo, hi;
          split(col[c], lo, hi);
          cs[c] = __shfl_sync(0xffffffffu, lo + hi, (lane + 1) & 31);
        }
      }
    }
    if constexpr (COL) {
#pragma unroll
      for (int c = 0; c < NP; ++c) colacc[c][chunk * 32 + lane] += cs[c];
    }
    __syncthreads();  // the next phase hands this chunk (and its column accumulators) to another warp
  }
}

template <class Op, int TPB, int RT>
__global__ void __launch_bounds__(TPB, Op::kSymMinCtas)
    pairs_kernel_symx(const typename Op::Params P, int n, int nblk, int TT, long long U, int C,
                      float2* __restrict__ row_ws, float* __restrict__ col_ws) {
  using St = SymStage<4 + Op::NP, TPB>;
  constexpr int L = 2, G = RT / L, NP = Op::NP;
  constexpr int B = TPB * RT;
  static_assert(TPB % 32 == 0 && RT % L == 0, "launch shape");
  __shared__ typename St::T sm[St::NQ][TPB];
  __shared__ float colacc[NP][TPB];
  __shared__ float red[6][TPB / 32];
  extern __shared__ __align__(16) unsigned char sym_dyn_smem[];
  F2 (*cs)[TPB] = reinterpret_cast<F2 (*)[TPB]>(sym_dyn_smem);  // compensated row sums, G * NP * 2 rows
  const Frame& f = P.f;
  const double fo[3] = {f.o0, f.o1, f.o2};

  const long long u_end = sk_start(blockIdx.x + 1, U, C);
  long long u = sk_start(blockIdx.x, U, C);
  int i = u < u_end ? sym_row_of(u, nblk, TT, RT) : 0;
  while (u < u_end) {
    const long long off = sym_row_off(i, TT, RT);
    const int cnt = TT - RT * i;
    const int t0 = (int)(u - off);
    const int t1 = (int)((u_end - off) < cnt ? (u_end - off) : cnt);
    const int slot = (int)blockIdx.x - sk_cta_of(off, U, C);
    const int base = i * B + threadIdx.x;

    // box and centre of row block i (every CTA working on it derives the same ones)
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
    for (int t = 0; t < RT; ++t) {
      int k = base + t * TPB;
      k = k < n ? k : n - 1;
      double y[3];
      Op::point(P, k, y);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float v = (float)((y[c] - fo[c]) * f.s);
        lo[c] = fminf(lo[c], v);
        hi[c] = fmaxf(hi[c], v);
      }
    }
    block_box<TPB>(lo, hi, red);  // its barrier also orders the previous segment's last reads of sm and cs
    float ob[3], rb2 = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ob[c] = 0.5f * (lo[c] + hi[c]);
      const float h = 0.5f * (hi[c] - lo[c]);
      rb2 = fmaf(h, h, rb2);
    }
    const bool expand = rb2 <= kExpandR2;  // uniform over the CTA

    F2 yt[G][3], tp[G][NP];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int k0 = base + (g * L) * TPB, k1 = base + (g * L + 1) * TPB;
      double y0[3], y1[3], p0[NP], p1[NP];
      Op::point(P, k0 < n ? k0 : n - 1, y0);
      Op::point(P, k1 < n ? k1 : n - 1, y1);
      Op::payload(P, k0 < n ? k0 : n - 1, p0);
      Op::payload(P, k1 < n ? k1 : n - 1, p1);
      double q0 = 0.0, q1 = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float r0 = (float)((y0[c] - fo[c]) * f.s - (double)ob[c]);
        const float r1 = (float)((y1[c] - fo[c]) * f.s - (double)ob[c]);
        yt[g][c] = f2(r0, r1);
        q0 += (double)r0 * (double)r0;
        q1 += (double)r1 * (double)r1;
      }
      // column payload: f_k a_k (expanded form) or a_k; padded targets carry none
      const double f0 = k0 < n ? (expand ? exp2(-q0) : 1.0) : 0.0;
      const double f1 = k1 < n ? (expand ? exp2(-q1) : 1.0) : 0.0;
#pragma unroll
      for (int c = 0; c < NP; ++c) tp[g][c] = f2((float)(f0 * p0[c]), (float)(f1 * p1[c]));
      Comp<F2> z;
      z.zero();
#pragma unroll
      for (int c = 0; c < NP; ++c) z.template store<TPB>(cs, g * NP + c, threadIdx.x);
    }

    for (int tt = t0; tt < t1; ++tt) {
      const int t = RT * i + tt;  // absolute source tile
      const bool diag = tt < RT;  // tile of block i itself: rows only
      {
        const int l = t * TPB + threadIdx.x;
        double fl[St::kFields];
#pragma unroll
        for (int q = 0; q < St::kFields; ++q) fl[q] = 0.0;
        if (l < n) {
          double xr[3], r2 = 0.0;
          Op::point(P, l, xr);
          Op::payload(P, l, fl + 4);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float xc = (float)((xr[c] - fo[c]) * f.s - (double)ob[c]);
            r2 += (double)xc * (double)xc;
            fl[c] = expand ? -2.0 * (double)xc : (double)xc;
          }
          fl[3] = r2;
        }
        St::store(sm, threadIdx.x, fl);
#pragma unroll
        for (int c = 0; c < NP; ++c) colacc[c][threadIdx.x] = 0.f;
      }
      __syncthreads();
      F2 acc[G][NP];
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int c = 0; c < NP; ++c) acc[g][c] = VT<F2>::zero();
      if (expand) {
        if (diag)
          symx_tile<Op, TPB, RT, false, true>(yt, tp, sm, colacc, acc);
        else
          symx_tile<Op, TPB, RT, true, true>(yt, tp, sm, colacc, acc);
      } else {
        if (diag)
          symx_tile<Op, TPB, RT, false, false>(yt, tp, sm, colacc, acc);
        else
          symx_tile<Op, TPB, RT, true, false>(yt, tp, sm, colacc, acc);
      }
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int c = 0; c < NP; ++c) {
          Comp<F2> m;
          m.template load<TPB>(cs, g * NP + c, threadIdx.x);
          m.merge(acc[g][c]);
          m.template store<TPB>(cs, g * NP + c, threadIdx.x);
        }
      if (!diag) {
        const int j = t / RT;
        const size_t cb = (size_t)(sym_tri(j) + i) * NP * B + (size_t)(t - RT * j) * TPB + threadIdx.x;
#pragma unroll
        for (int c = 0; c < NP; ++c) col_ws[cb + (size_t)c * B] = colacc[c][threadIdx.x];
      }
      // the last phase barrier of symx_tile orders every read of sm and colacc before the next tile's staging
    }

#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const int idx = base + (g * L + k) * TPB;
        if (idx < n) {
          double y2 = 0.0;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const double yr = VT<F2>::lane(yt[g][c], k);
            y2 += yr * yr;
          }
          const double fac = expand ? exp2(-y2) : 1.0;
#pragma unroll
          for (int c = 0; c < NP; ++c) {
            Comp<F2> m;
            m.template load<TPB>(cs, g * NP + c, threadIdx.x);
            const float2 pp = m.partial(k);
            const double w = ((double)pp.x + (double)pp.y) * fac;
            const float h = (float)w;
            row_ws[((size_t)slot * NP + c) * (size_t)n + idx] = make_float2(h, (float)(w - (double)h));
          }
        }
      }
    u += t1 - t0;
    ++i;
  }
}

template <class Op, int TPB, int RT>
constexpr size_t symx_dyn_smem_bytes() {
  return (size_t)(RT / 2) * Op::NP * 2 * TPB * sizeof(F2);
}

template <class Op, int TPB, int RT>
inline bool symx_prepare() {
  static signed char state[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (dev < 0 || dev >= 64) return false;
  if (state[dev] == 0) {
    const cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(&pairs_kernel_symx<Op, TPB, RT>),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)symx_dyn_smem_bytes<Op, TPB, RT>());
    if (e != cudaSuccess) cudaGetLastError();
    state[dev] = e == cudaSuccess ? 1 : -1;
  }
  return state[dev] > 0;
}

template <class Op, int TPB, int RT>
inline int symx_ctas_per_sm() {
  static int cached = 0;
  if (cached == 0) {
    symx_prepare<Op, TPB, RT>();
    int c = resident_ctas(reinterpret_cast<const void*>(&pairs_kernel_symx<Op, TPB, RT>), TPB,
                          symx_dyn_smem_bytes<Op, TPB, RT>());
    cached = c > 0 ? c : 2;
  }
  return cached;
}

template <class Op, int TPB, int RT>
inline size_t symx_ws_bytes(int64_t n) {
  return make_sym_plan<TPB, RT>(n, Op::NP, Op::NP, symx_ctas_per_sm<Op, TPB, RT>()).ws_bytes;
}

template <class Op, int TPB, int RT>
inline int run_pairs_symx(const typename Op::Params& P, int64_t n, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (n <= 0) return kOk;
  if (n > INT32_MAX / 4) return kInvalidArgument;
  const SymPlan plan = make_sym_plan<TPB, RT>(n, Op::NP, Op::NP, symx_ctas_per_sm<Op, TPB, RT>());
  if (plan.ws_bytes > ws_bytes) return kWorkspaceTooSmall;
  if (ws == nullptr) return kInvalidArgument;
  if (!symx_prepare<Op, TPB, RT>()) return kLaunchFailure;
  auto* row_ws = reinterpret_cast<float2*>(ws);
  auto* col_ws = reinterpret_cast<float*>(reinterpret_cast<char*>(ws) + plan.col_off);
  pairs_kernel_symx<Op, TPB, RT><<<plan.C, TPB, symx_dyn_smem_bytes<Op, TPB, RT>(), stream>>>(
      P, (int)n, plan.nblk, plan.TT, plan.U, plan.C, row_ws, col_ws);
  const int fb = kFinThreads, tpp = sym_finalize_tpp(plan);
  finalize_sym_kernel<Op, TPB, RT><<<sym_finalize_grid(n, tpp, fb), fb, 0, stream>>>(P, (int)n, plan.nblk, plan.TT,
                                                                                      plan.U, plan.C, row_ws, col_ws,
                                                                                      tpp);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

}  // namespace lddmm
