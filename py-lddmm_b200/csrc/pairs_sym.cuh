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

namespace lddmm {

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

template <class Op, int TPB, int RT, bool COL>
__device__ __forceinline__ void sym_tile(const Frame& f, const typename Op::SymTgt (&tgt)[RT / 2],
                                         const Unit<F2> (*sm)[TPB], float (*colacc)[TPB], F2 (&acc)[RT / 2][Op::NR]) {
  constexpr int G = RT / 2, NU = (Op::NSS + 1) / 2, W = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll 1
  for (int ph = 0; ph < W; ++ph) {
    const int chunk = (warp + ph) % W;
    float cs[Op::NC];
#pragma unroll
    for (int c = 0; c < Op::NC; ++c) cs[c] = 0.f;
#pragma unroll 2
    for (int s = 0; s < 32; ++s) {
      const int src = chunk * 32 + ((lane + s) & 31);
      F2 sv[2 * NU];
#pragma unroll
      for (int q = 0; q < NU; ++q) {
        const Unit<F2> w = sm[q][src];
        sv[2 * q] = w.a;
        sv[2 * q + 1] = w.b;
      }
      if constexpr (COL) {
        F2 col[Op::NC];
#pragma unroll
        for (int c = 0; c < Op::NC; ++c) col[c] = f2(cs[c], 0.f);
#pragma unroll
        for (int g = 0; g < G; ++g) Op::template pair_sym<true>(f, tgt[g], sv, acc[g], col);
#pragma unroll
        for (int c = 0; c < Op::NC; ++c) {
          float lo, hi;
          split(col[c], lo, hi);
          cs[c] = __shfl_sync(0xffffffffu, lo + hi, (lane + 1) & 31);
        }
      } else {
#pragma unroll
        for (int g = 0; g < G; ++g) Op::template pair_sym<false>(f, tgt[g], sv, acc[g], nullptr);
      }
    }
    if constexpr (COL) {
#pragma unroll
      for (int c = 0; c < Op::NC; ++c) colacc[c][chunk * 32 + lane] += cs[c];
    }
    __syncthreads();  // the next phase hands this chunk (and its column accumulators) to another warp
  }
}

template <class Op, int TPB, int RT>
__global__ void __launch_bounds__(TPB, Op::kSymMinCtas)
    pairs_kernel_sym(const typename Op::Params P, int n, int nblk, int TT, long long U, int C,
                     float2* __restrict__ row_ws, float* __restrict__ col_ws) {
  constexpr int L = 2, G = RT / L, NU = (Op::NSS + 1) / 2, NR = Op::NR, NC = Op::NC;
  constexpr int B = TPB * RT;
  static_assert(TPB % 32 == 0 && RT % L == 0, "launch shape");
  __shared__ Unit<F2> sm[NU][TPB];
  __shared__ float colacc[NC][TPB];
  __shared__ F2 cs[G * NR * 2][TPB];  // compensated row sums of the segment, one private column per thread
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
        double fl[2 * NU];
#pragma unroll
        for (int q = 0; q < 2 * NU; ++q) fl[q] = 0.0;
        if (l < n) Op::source_fields_sym(P, l, fl);
#pragma unroll
        for (int q = 0; q < NU; ++q) {
          Unit<F2> w;
          w.a = VT<F2>::dup(fl[2 * q]);
          w.b = VT<F2>::dup(fl[2 * q + 1]);
          sm[q][threadIdx.x] = w;
        }
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
        sym_tile<Op, TPB, RT, false>(f, tgt, sm, colacc, acc);
      else
        sym_tile<Op, TPB, RT, true>(f, tgt, sm, colacc, acc);
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

// Epilogue: row slots of the point's block (in CTA order), then its column partials (in block order), in FP64.
template <class Op, int TPB, int RT>
__global__ void finalize_sym_kernel(const typename Op::Params P, int n, int nblk, int TT, long long U, int C,
                                    const float2* __restrict__ row_ws, const float* __restrict__ col_ws) {
  constexpr int B = TPB * RT;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  double row[Op::NR], col[Op::NC];
#pragma unroll
  for (int c = 0; c < Op::NR; ++c) row[c] = 0.0;
#pragma unroll
  for (int c = 0; c < Op::NC; ++c) col[c] = 0.0;
  const int b = idx / B, r = idx - b * B;
  const int nslot = sk_cta_of(sym_row_off(b + 1, TT, RT) - 1, U, C) - sk_cta_of(sym_row_off(b, TT, RT), U, C) + 1;
  for (int s = 0; s < nslot; ++s)
#pragma unroll
    for (int c = 0; c < Op::NR; ++c) row[c] += partial_value(row_ws[((size_t)s * Op::NR + c) * (size_t)n + idx]);
  for (int q = 0; q < b; ++q) {
    const size_t cb = (size_t)(sym_tri(b) + q) * Op::NC * B + r;
#pragma unroll
    for (int c = 0; c < Op::NC; ++c) col[c] += (double)col_ws[cb + (size_t)c * B];
  }
  Op::finalize_sym(P, idx, row, col);
}

template <class Op, int TPB, int RT>
inline int sym_ctas_per_sm() {
  static int cached = 0;
  if (cached == 0) {
    int c = resident_ctas(reinterpret_cast<const void*>(&pairs_kernel_sym<Op, TPB, RT>), TPB);
    cached = c > 0 ? c : 2;
  }
  return cached;
}

template <class Op, int TPB, int RT>
inline size_t sym_ws_bytes(int64_t n) {
  return make_sym_plan<TPB, RT>(n, Op::NR, Op::NC, sym_ctas_per_sm<Op, TPB, RT>()).ws_bytes;
}

template <class Op, int TPB, int RT>
inline int run_pairs_sym(const typename Op::Params& P, int64_t n, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (n <= 0) return kOk;
  if (n > INT32_MAX / 4) return kInvalidArgument;
  const SymPlan plan = make_sym_plan<TPB, RT>(n, Op::NR, Op::NC, sym_ctas_per_sm<Op, TPB, RT>());
  if (plan.ws_bytes > ws_bytes) return kWorkspaceTooSmall;
  if (ws == nullptr) return kInvalidArgument;
  auto* row_ws = reinterpret_cast<float2*>(ws);
  auto* col_ws = reinterpret_cast<float*>(reinterpret_cast<char*>(ws) + plan.col_off);
  pairs_kernel_sym<Op, TPB, RT><<<plan.C, TPB, 0, stream>>>(P, (int)n, plan.nblk, plan.TT, plan.U, plan.C, row_ws,
                                                            col_ws);
  const int fb = 256;
  finalize_sym_kernel<Op, TPB, RT><<<(int)((n + fb - 1) / fb), fb, 0, stream>>>(P, (int)n, plan.nblk, plan.TT, plan.U,
                                                                                 plan.C, row_ws, col_ws);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

}  // namespace lddmm
