// Pair functors of the Gaussian kernel operators (one width sigma, KP = -1).
//
// Notation: y' = (y - o) s, x' = (x - o) s, d = y'_k - x'_l, e = expneg(|d|^2) = exp(-|y_k-x_l|^2/(2 sigma^2)),
// kappa = 1/(s sigma^2) so that (y_k - x_l)/sigma^2 = kappa d. Per-pair FP32/SFU work is listed per op
// (the figures used for the roofline).
#pragma once
#include "lddmm_common.cuh"

namespace lddmm {

// K(y, x) a  -- base/kernelFunctions_util.py:451-466. 9 FP32 + 1 SFU per pair.
// Epilogue (used by the shooting drivers): out = base_sign * base + scale * K a, and optionally
// dots[i] = dotw_i . (K a)_i for FP64 energy reductions.
template <typename R>
struct OpK {
  static constexpr int NV = 2, NA = 3;
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
  struct Tgt { R y0, y1, y2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    load_point(P.y, i, P.f, t.y0, t.y1, t.y2);
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_point(P.x, l, P.f, s[0].x, s[0].y, s[0].z);
    load_vec(P.a, l, s[1].x, s[1].y, s[1].z);
    s[0].w = R(0);
    s[1].w = R(0);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    acc[0] += e * s[1].x;
    acc[1] += e * s[1].y;
    acc[2] += e * s[1].z;
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

// DK^T(y, x; p, a) -- base/kernelFunctions_util.py:773-793 with gauss_fun_diffT (:233).
//   mode 0 (plain): c = p_k.a_l                         13 FP32 + 1 SFU
//   mode 1 (sym)  : c = p_k.a_l + a_k.p_l               16 FP32 + 1 SFU
//   mode 2 (lddmm): c = p_k.a_l + a_k.(p_l - 2 w a_l)   16 FP32 + 1 SFU (source-side q_l precomputed)
// out_k = -kappa sum_l e c d.
template <typename R, int MODE>
struct OpDiffKT {
  static constexpr int NV = (MODE == 0) ? 2 : 3, NA = 3;
  struct Params {
    const double *y, *x, *p, *a;  // p: (n,3) target-indexed (and source-indexed for sym/lddmm), a: (m,3)
    double* out;
    Frame f;
    double w;  // regweight (lddmm)
  };
  struct Tgt { R y0, y1, y2, p0, p1, p2, a0, a1, a2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    load_point(P.y, i, P.f, t.y0, t.y1, t.y2);
    load_vec(P.p, i, t.p0, t.p1, t.p2);
    if (MODE != 0) load_vec(P.a, i, t.a0, t.a1, t.a2);
    else { t.a0 = t.a1 = t.a2 = R(0); }
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_point(P.x, l, P.f, s[0].x, s[0].y, s[0].z);
    load_vec(P.a, l, s[1].x, s[1].y, s[1].z);
    s[0].w = R(0);
    s[1].w = R(0);
    if (MODE != 0) {
      const double k = (MODE == 2) ? 2.0 * P.w : 0.0;
      s[2].x = (R)(P.p[3 * l + 0] - k * P.a[3 * l + 0]);
      s[2].y = (R)(P.p[3 * l + 1] - k * P.a[3 * l + 1]);
      s[2].z = (R)(P.p[3 * l + 2] - k * P.a[3 * l + 2]);
      s[2].w = R(0);
    }
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    R c = t.p0 * s[1].x + t.p1 * s[1].y + t.p2 * s[1].z;
    if (MODE != 0) c += t.a0 * s[2].x + t.a1 * s[2].y + t.a2 * s[2].z;
    const R ec = e * c;
    acc[0] += ec * d0;
    acc[1] += ec * d1;
    acc[2] += ec * d2;
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
//       = kappa^2 A_k - (p_k B_k - C_k)/sigma^2 with A = sum c e (d.Dp) d, B = sum c e, C = sum c e p_l.
// 24 FP32 + 1 SFU per pair.
template <typename R>
struct OpDDiffK {
  static constexpr int NV = 3, NA = 7;
  struct Params {
    const double *x, *nn, *a, *p;
    double* out;
    Frame f;
  };
  struct Tgt { R y0, y1, y2, n0, n1, n2, p0, p1, p2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    load_point(P.x, i, P.f, t.y0, t.y1, t.y2);
    load_vec(P.nn, i, t.n0, t.n1, t.n2);
    load_vec(P.p, i, t.p0, t.p1, t.p2);
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_point(P.x, l, P.f, s[0].x, s[0].y, s[0].z);
    load_vec(P.a, l, s[1].x, s[1].y, s[1].z);
    load_vec(P.p, l, s[2].x, s[2].y, s[2].z);
    s[0].w = s[1].w = s[2].w = R(0);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    const R q0 = t.p0 - s[2].x, q1 = t.p1 - s[2].y, q2 = t.p2 - s[2].z;
    const R dq = d0 * q0 + d1 * q1 + d2 * q2;
    const R ce = e * (t.n0 * s[1].x + t.n1 * s[1].y + t.n2 * s[1].z);
    const R ced = ce * dq;
    acc[0] += ced * d0;
    acc[1] += ced * d1;
    acc[2] += ced * d2;
    acc[3] += ce;
    acc[4] += ce * s[2].x;
    acc[5] += ce * s[2].y;
    acc[6] += ce * s[2].z;
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double k2 = P.f.kappa * P.f.kappa, is2 = P.f.inv_s2;
    for (int c = 0; c < 3; ++c)
      P.out[3 * i + c] = k2 * acc[c] - is2 * (P.p[3 * i + c] * acc[3] - acc[4 + c]);
  }
};

// DK_{1and2}(x; a1, a2) -- base/kernelFunctions_util.py:672-675 with gauss_fun_diff (:195).
// out_k = sum_l -(D.(a1_k - a1_l))/sigma^2 e a2_l = -kappa sum_l (d.(a1_k - a1_l)) e a2_l. 16 FP32 + 1 SFU.
template <typename R>
struct OpDiffK1and2 {
  static constexpr int NV = 3, NA = 3;
  struct Params {
    const double *x, *a1, *a2;
    double* out;
    Frame f;
  };
  struct Tgt { R y0, y1, y2, b0, b1, b2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    load_point(P.x, i, P.f, t.y0, t.y1, t.y2);
    load_vec(P.a1, i, t.b0, t.b1, t.b2);
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_point(P.x, l, P.f, s[0].x, s[0].y, s[0].z);
    load_vec(P.a1, l, s[1].x, s[1].y, s[1].z);
    load_vec(P.a2, l, s[2].x, s[2].y, s[2].z);
    s[0].w = s[1].w = s[2].w = R(0);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    const R g = d0 * (t.b0 - s[1].x) + d1 * (t.b1 - s[1].y) + d2 * (t.b2 - s[1].z);
    const R eg = e * g;
    acc[0] += eg * s[2].x;
    acc[1] += eg * s[2].y;
    acc[2] += eg * s[2].z;
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double k = -P.f.kappa;
    P.out[3 * i + 0] = k * acc[0];
    P.out[3 * i + 1] = k * acc[1];
    P.out[3 * i + 2] = k * acc[2];
  }
};

// Divergence: out_k = sum_l -((y_k - x_l).a_l)/sigma^2 e = -kappa sum_l (d.a_l) e
// (base/kernelFunctions_util.py:611-626 applyDiv with gauss_fun_diff). 11 FP32 + 1 SFU.
template <typename R>
struct OpDiv {
  static constexpr int NV = 2, NA = 1;
  struct Params {
    const double *y, *x, *a;
    double* out;
    Frame f;
  };
  struct Tgt { R y0, y1, y2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    load_point(P.y, i, P.f, t.y0, t.y1, t.y2);
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_point(P.x, l, P.f, s[0].x, s[0].y, s[0].z);
    load_vec(P.a, l, s[1].x, s[1].y, s[1].z);
    s[0].w = s[1].w = R(0);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    acc[0] += e * (d0 * s[1].x + d1 * s[1].y + d2 * s[1].z);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    P.out[i] = -P.f.kappa * acc[0];
  }
};

// K-tensor: out_k = sum_l e (ay_k ax_l + (by_k.bx_l)^2) (base/kernelFunctions_util.py:1475-1506).
// Accumulates A = sum e ax_l and B = sum e g^2 so that ay_k multiplies once per target. 13 FP32 + 1 SFU.
template <typename R>
struct OpKTensor {
  static constexpr int NV = 2, NA = 2;
  struct Params {
    const double *y, *x, *ay, *ax, *by, *bx;
    double* out;
    Frame f;
  };
  struct Tgt { R y0, y1, y2, b0, b1, b2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    load_point(P.y, i, P.f, t.y0, t.y1, t.y2);
    load_vec(P.by, i, t.b0, t.b1, t.b2);
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_point(P.x, l, P.f, s[0].x, s[0].y, s[0].z);
    s[0].w = (R)P.ax[l];
    load_vec(P.bx, l, s[1].x, s[1].y, s[1].z);
    s[1].w = R(0);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    const R g = t.b0 * s[1].x + t.b1 * s[1].y + t.b2 * s[1].z;
    acc[0] += e * s[0].w;
    acc[1] += e * (g * g);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    P.out[i] = P.ay[i] * acc[0] + acc[1];
  }
};

}  // namespace lddmm
