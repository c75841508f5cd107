// Pair functors of the Gaussian kernel operators (one width sigma, KP = -1).
//
// Notation: y' = (y - o) s, x' = (x - o) s, d = y'_k - x'_l, e = expneg(|d|^2) = exp(-|y_k-x_l|^2/(2 sigma^2)),
// kappa = 1/(s sigma^2) so that (y_k - x_l)/sigma^2 = kappa d. Each functor is written once for V = F2 (two FP32
// targets per packed instruction) and V = double. Per-pair FP32 lane-op / SFU counts are listed per op (the
// figures used for the roofline; a packed instruction counts as two lane-ops).
#pragma once
#include "lddmm_common.cuh"

namespace lddmm {

template <typename V>
__device__ __forceinline__ V sqdist(V d0, V d1, V d2) {
  return fma(d2, d2, fma(d1, d1, d0 * d0));
}
template <typename V>
__device__ __forceinline__ V dot3(V a0, V a1, V a2, V b0, V b1, V b2) {
  return fma(a2, b2, fma(a1, b1, a0 * b0));
}

// K(y, x) a  -- base/kernelFunctions_util.py:451-466. 9 FP32 + 1 SFU per pair.
// Epilogue (used by the shooting drivers): out = base_sign * base + scale * K a, and optionally
// dots[i] = dotw_i . (K a)_i for FP64 energy reductions.
struct OpK {
  static constexpr int NS = 6, NA = 3;
  static constexpr bool kCompInRegisters = true;  // measured faster than shared memory for this op
  struct Params {
    const double *y, *x, *a;
    double* out;
    Frame f;
    const double* base = nullptr;
    double base_sign = 1.0;
    double scale = 1.0;
    const double* dotw = nullptr;
    double* dots = nullptr;
  };
  template <typename V> struct Tgt { V y0, y1, y2; };
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    t.y0 = tgt_coord<V>(P.y, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<V>(P.y, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<V>(P.y, i0, i1, 2, P.f.o2, P.f.s);
  }
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    src_point(P.x, l, P.f, f);
    f[3] = P.a[3 * l]; f[4] = P.a[3 * l + 1]; f[5] = P.a[3 * l + 2];
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame& f, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<V> k = Fam::template eval<V>(f, sqdist(d0, d1, d2));
    acc[0] = fma(k.k0, s[3], acc[0]);
    acc[1] = fma(k.k0, s[4], acc[1]);
    acc[2] = fma(k.k0, s[5], acc[2]);
  }
  // expanded-distance Gaussian form (pairs_kernel_x): payload a, K a accumulated from the kernel value e
  static constexpr bool kExpand = true;
  static constexpr int NP = 3;
  template <typename V> struct TgtX {};
  template <typename V>
  static __device__ __forceinline__ void load_target_x(const Params&, int, int, TgtX<V>&) {}
  static __device__ __forceinline__ void target_point(const Params& P, int i, double* c) {
    c[0] = P.y[3 * i]; c[1] = P.y[3 * i + 1]; c[2] = P.y[3 * i + 2];
  }
  static __device__ __forceinline__ void source_point(const Params& P, int l, double* c, double* f) {
    c[0] = P.x[3 * l]; c[1] = P.x[3 * l + 1]; c[2] = P.x[3 * l + 2];
    f[0] = P.a[3 * l]; f[1] = P.a[3 * l + 1]; f[2] = P.a[3 * l + 2];
  }
  // s: the staged source record (coordinates 0-2, |x|^2 3, payload from 4)
  template <bool X, typename V>
  static __device__ __forceinline__ void accumulate(const TgtX<V>&, const V*, V e, const V* s, V* acc) {
    acc[0] = fma(e, s[4], acc[0]);
    acc[1] = fma(e, s[5], acc[1]);
    acc[2] = fma(e, s[6], acc[2]);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    if (P.dots)
      P.dots[i] = P.dotw[3 * i] * acc[0] + P.dotw[3 * i + 1] * acc[1] + P.dotw[3 * i + 2] * acc[2];
    if (P.out) {
      for (int c = 0; c < 3; ++c) {
        const double b = P.base ? P.base_sign * P.base[3 * i + c] : 0.0;
        P.out[3 * i + c] = b + P.scale * acc[c];
      }
    }
  }
};

// K(x, x) a evaluated once per unordered pair (pairs_kernel_symx; Gaussian, FP32, targets == sources): the row sum
// of k takes e_kl a_l and the column sum of l takes e_kl a_k; out_k = row_k + col_k. 9 FP32 lane-ops and one ex2
// per unordered pair in the expanded-distance form. The epilogue options of OpK (base, scale, dots) apply.
struct OpKSym {
  using Params = OpK::Params;
  static constexpr int NP = 3, NR = 3, NC = 3;
  static constexpr int kSymMinCtas = LDDMM_KSYM_MIN_CTAS;
  static __device__ __forceinline__ void point(const Params& P, int i, double* c) {
    c[0] = P.x[3 * i]; c[1] = P.x[3 * i + 1]; c[2] = P.x[3 * i + 2];
  }
  static __device__ __forceinline__ void payload(const Params& P, int i, double* p) {
    p[0] = P.a[3 * i]; p[1] = P.a[3 * i + 1]; p[2] = P.a[3 * i + 2];
  }
  static __device__ __forceinline__ void finalize_sym(const Params& P, int i, const double* row, const double* col) {
    const double acc[3] = {row[0] + col[0], row[1] + col[1], row[2] + col[2]};
    OpK::finalize(P, i, acc);
  }
};

// K(x, x) a evaluated once per unordered pair in the difference form (pairs_kernel_sym), for kernel families
// without an expanded form (the Laplacian): row term k0 a_l, column term k0 a_k. The epilogue options of OpK apply.
struct OpKSymD {
  using Params = OpK::Params;
  static constexpr int NSS = 6, NR = 3, NC = 3;
  static constexpr int kSymMinCtas = LDDMM_KSYM_MIN_CTAS;
  struct SymTgt { F2 y0, y1, y2, a0, a1, a2; };
  static __device__ __forceinline__ void load_target_sym(const Params& P, int i0, int i1, bool v0, bool v1,
                                                         SymTgt& t) {
    t.y0 = tgt_coord<F2>(P.x, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<F2>(P.x, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<F2>(P.x, i0, i1, 2, P.f.o2, P.f.s);
    t.a0 = VT<F2>::pack(v0 ? P.a[3 * i0] : 0.0, v1 ? P.a[3 * i1] : 0.0);
    t.a1 = VT<F2>::pack(v0 ? P.a[3 * i0 + 1] : 0.0, v1 ? P.a[3 * i1 + 1] : 0.0);
    t.a2 = VT<F2>::pack(v0 ? P.a[3 * i0 + 2] : 0.0, v1 ? P.a[3 * i1 + 2] : 0.0);
  }
  // fields: x' (0-2), a (3-5)
  static __device__ __forceinline__ void source_fields_sym(const Params& P, int l, double* f) {
    OpK::source_fields(P, l, f);
  }
  template <bool COL, class Fam>
  static __device__ __forceinline__ void pair_sym(const Frame& f, const SymTgt& t, const F2* s, F2* row, F2* col) {
    const F2 d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<F2> k = Fam::template eval<F2>(f, sqdist(d0, d1, d2));
    row[0] = fma(k.k0, s[3], row[0]);
    row[1] = fma(k.k0, s[4], row[1]);
    row[2] = fma(k.k0, s[5], row[2]);
    if constexpr (COL) {
      col[0] = fma(k.k0, t.a0, col[0]);
      col[1] = fma(k.k0, t.a1, col[1]);
      col[2] = fma(k.k0, t.a2, col[2]);
    }
  }
  static __device__ __forceinline__ void finalize_sym(const Params& P, int i, const double* row, const double* col) {
    const double acc[3] = {row[0] + col[0], row[1] + col[1], row[2] + col[2]};
    OpK::finalize(P, i, acc);
  }
};

// DK^T(y, x; p, a) -- base/kernelFunctions_util.py:773-793 with gauss_fun_diffT (:233).
//   MODE 0 (plain): c = p_k.a_l                         13 FP32 + 1 SFU
//   MODE 1 (sym)  : c = p_k.a_l + a_k.p_l               16 FP32 + 1 SFU
//   MODE 2 (lddmm): c = p_k.a_l + a_k.(p_l - 2 w a_l)   16 FP32 + 1 SFU (source-side q_l precomputed)
// out_k = -kappa sum_l e c d.
template <int MODE>
struct OpDiffKT {
  static constexpr int NS = (MODE == 0) ? 6 : 9, NA = 3;
  struct Params {
    const double *y, *x, *p, *a;  // p: (n,3) target-indexed (and source-indexed for sym/lddmm), a: (m,3)
    double* out;
    Frame f;
    double w;  // regweight (lddmm)
  };
  template <typename V> struct Tgt { V y0, y1, y2, p0, p1, p2, a0, a1, a2; };
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    t.y0 = tgt_coord<V>(P.y, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<V>(P.y, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<V>(P.y, i0, i1, 2, P.f.o2, P.f.s);
    t.p0 = tgt_field<V>(P.p, 3, i0, i1, 0);
    t.p1 = tgt_field<V>(P.p, 3, i0, i1, 1);
    t.p2 = tgt_field<V>(P.p, 3, i0, i1, 2);
    if (MODE != 0) {
      t.a0 = tgt_field<V>(P.a, 3, i0, i1, 0);
      t.a1 = tgt_field<V>(P.a, 3, i0, i1, 1);
      t.a2 = tgt_field<V>(P.a, 3, i0, i1, 2);
    } else {
      t.a0 = t.a1 = t.a2 = VT<V>::zero();
    }
  }
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    src_point(P.x, l, P.f, f);
    for (int c = 0; c < 3; ++c) f[3 + c] = P.a[3 * l + c];
    if (MODE != 0) {
      const double k = (MODE == 2) ? 2.0 * P.w : 0.0;
      for (int c = 0; c < 3; ++c) f[6 + c] = P.p[3 * l + c] - k * P.a[3 * l + c];
    }
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame& f, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<V> k = Fam::template eval<V>(f, sqdist(d0, d1, d2));
    V c = dot3(t.p0, t.p1, t.p2, s[3], s[4], s[5]);
    if (MODE != 0) c = fma(t.a0, s[6], fma(t.a1, s[7], fma(t.a2, s[8], c)));
    const V ec = k.k1 * c;
    acc[0] = fma(ec, d0, acc[0]);
    acc[1] = fma(ec, d1, acc[1]);
    acc[2] = fma(ec, d2, acc[2]);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double k = -P.f.kappa;
    P.out[3 * i + 0] = k * acc[0];
    P.out[3 * i + 1] = k * acc[1];
    P.out[3 * i + 2] = k * acc[2];
  }
};

// DDK_{11 and 12}(x; n, a, p) -- base/kernelFunctions_util.py:1091-1129 ('11and12'), gauss_fun_ddiff (:299).
// out_k = sum_l (n_k.a_l) e [ (D.Dp) D / sigma^4 - Dp / sigma^2 ],  D = x_k - x_l, Dp = p_k - p_l
//       = kappa^2 A_k - B_k / sigma^2 with A = sum c e (d.Dp) d, B = sum c e Dp (c = n_k.a_l).
// 23 FP32 + 1 SFU per pair (the Dp components are shared by d.Dp and B).
struct OpDDiffK {
  static constexpr int NS = 9, NA = 6;
  static constexpr bool kCompInRegisters = true;  // measured faster than shared memory for this op
  struct Params {
    const double *x, *nn, *a, *p;
    double* out;
    Frame f;
  };
  template <typename V> struct Tgt { V y0, y1, y2, n0, n1, n2, p0, p1, p2; };
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    t.y0 = tgt_coord<V>(P.x, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<V>(P.x, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<V>(P.x, i0, i1, 2, P.f.o2, P.f.s);
    t.n0 = tgt_field<V>(P.nn, 3, i0, i1, 0);
    t.n1 = tgt_field<V>(P.nn, 3, i0, i1, 1);
    t.n2 = tgt_field<V>(P.nn, 3, i0, i1, 2);
    t.p0 = tgt_field<V>(P.p, 3, i0, i1, 0);
    t.p1 = tgt_field<V>(P.p, 3, i0, i1, 1);
    t.p2 = tgt_field<V>(P.p, 3, i0, i1, 2);
  }
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    src_point(P.x, l, P.f, f);
    for (int c = 0; c < 3; ++c) {
      f[3 + c] = P.a[3 * l + c];
      f[6 + c] = P.p[3 * l + c];
    }
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame& f, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<V> k = Fam::template eval<V>(f, sqdist(d0, d1, d2));
    const V q0 = t.p0 - s[6], q1 = t.p1 - s[7], q2 = t.p2 - s[8];
    const V dq = dot3(d0, d1, d2, q0, q1, q2);
    const V na = dot3(t.n0, t.n1, t.n2, s[3], s[4], s[5]);
    const V ce = k.k1 * na;
    const V ced = (k.k2 * na) * dq;  // == ce * dq for the Gaussian
    acc[0] = fma(ced, d0, acc[0]);
    acc[1] = fma(ced, d1, acc[1]);
    acc[2] = fma(ced, d2, acc[2]);
    acc[3] = fma(ce, q0, acc[3]);
    acc[4] = fma(ce, q1, acc[4]);
    acc[5] = fma(ce, q2, acc[5]);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double k2 = P.f.kappa * P.f.kappa, is2 = P.f.inv_s2;
    for (int c = 0; c < 3; ++c) P.out[3 * i + c] = k2 * acc[c] - is2 * acc[3 + c];
  }
};

// DK_{1and2}(x; a1, a2) -- base/kernelFunctions_util.py:672-675 with gauss_fun_diff (:195).
// out_k = sum_l -(D.(a1_k - a1_l))/sigma^2 e a2_l = -kappa sum_l (d.(a1_k - a1_l)) e a2_l. 16 FP32 + 1 SFU.
struct OpDiffK1and2 {
  static constexpr int NS = 9, NA = 3;
  struct Params {
    const double *x, *a1, *a2;
    double* out;
    Frame f;
  };
  template <typename V> struct Tgt { V y0, y1, y2, b0, b1, b2; };
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    t.y0 = tgt_coord<V>(P.x, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<V>(P.x, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<V>(P.x, i0, i1, 2, P.f.o2, P.f.s);
    t.b0 = tgt_field<V>(P.a1, 3, i0, i1, 0);
    t.b1 = tgt_field<V>(P.a1, 3, i0, i1, 1);
    t.b2 = tgt_field<V>(P.a1, 3, i0, i1, 2);
  }
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    src_point(P.x, l, P.f, f);
    for (int c = 0; c < 3; ++c) {
      f[3 + c] = P.a1[3 * l + c];
      f[6 + c] = P.a2[3 * l + c];
    }
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame& f, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<V> k = Fam::template eval<V>(f, sqdist(d0, d1, d2));
    const V eg = k.k1 * dot3(d0, d1, d2, t.b0 - s[3], t.b1 - s[4], t.b2 - s[5]);
    acc[0] = fma(eg, s[6], acc[0]);
    acc[1] = fma(eg, s[7], acc[1]);
    acc[2] = fma(eg, s[8], acc[2]);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double k = -P.f.kappa;
    P.out[3 * i + 0] = k * acc[0];
    P.out[3 * i + 1] = k * acc[1];
    P.out[3 * i + 2] = k * acc[2];
  }
};

// Divergence: out_k = sum_l -((y_k - x_l).a_l)/sigma^2 e = -kappa sum_l (d.a_l) e
// (base/kernelFunctions_util.py:611-626 applyDiv with gauss_fun_diff). 10 FP32 + 1 SFU.
struct OpDiv {
  static constexpr int NS = 6, NA = 1;
  struct Params {
    const double *y, *x, *a;
    double* out;
    Frame f;
  };
  template <typename V> struct Tgt { V y0, y1, y2; };
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    t.y0 = tgt_coord<V>(P.y, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<V>(P.y, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<V>(P.y, i0, i1, 2, P.f.o2, P.f.s);
  }
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    src_point(P.x, l, P.f, f);
    f[3] = P.a[3 * l]; f[4] = P.a[3 * l + 1]; f[5] = P.a[3 * l + 2];
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame& f, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<V> k = Fam::template eval<V>(f, sqdist(d0, d1, d2));
    acc[0] = fma(k.k1, dot3(d0, d1, d2, s[3], s[4], s[5]), acc[0]);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    P.out[i] = -P.f.kappa * acc[0];
  }
};

// K-tensor: out_k = sum_l e (ay_k ax_l + (by_k.bx_l)^2) (base/kernelFunctions_util.py:1475-1506).
// Accumulates A = sum e ax_l and B = sum e g^2 so that ay_k multiplies once per target. 13 FP32 + 1 SFU.
struct OpKTensor {
  static constexpr int NS = 7, NA = 2;
  struct Params {
    const double *y, *x, *ay, *ax, *by, *bx;
    double* out;
    Frame f;
  };
  template <typename V> struct Tgt { V y0, y1, y2, b0, b1, b2; };
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    t.y0 = tgt_coord<V>(P.y, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<V>(P.y, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<V>(P.y, i0, i1, 2, P.f.o2, P.f.s);
    t.b0 = tgt_field<V>(P.by, 3, i0, i1, 0);
    t.b1 = tgt_field<V>(P.by, 3, i0, i1, 1);
    t.b2 = tgt_field<V>(P.by, 3, i0, i1, 2);
  }
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    src_point(P.x, l, P.f, f);
    f[3] = P.ax[l];
    f[4] = P.bx[3 * l]; f[5] = P.bx[3 * l + 1]; f[6] = P.bx[3 * l + 2];
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame& f, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<V> k = Fam::template eval<V>(f, sqdist(d0, d1, d2));
    const V g = dot3(t.b0, t.b1, t.b2, s[4], s[5], s[6]);
    acc[0] = fma(k.k0, s[3], acc[0]);
    acc[1] = fma(k.k0, g * g, acc[1]);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    P.out[i] = P.ay[i] * acc[0] + acc[1];
  }
};

}  // namespace lddmm
