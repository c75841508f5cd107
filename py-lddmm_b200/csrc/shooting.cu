// Landmark shooting and its adjoint: fused step kernels (one exp per pair shared by every sum of a step)
// with the FP64 state update done in the epilogue. Replaces base/pointEvolution.py.
#include "../../include/lddmm_b200.h"
#include "kernel_ops.cuh"
#include "launch_config.cuh"
#include "pairs_sym.cuh"

namespace lddmm {

// Second-order forward step (secondOrderEvolution loop body, base/pointEvolution.py:433-449):
//   x1 = x + dt K(x) a,   a1 = a + dt za with za = -DK^T(x; a, a) = kappa sum_l e (a_k.a_l) d.
// Accumulators: X = sum e a_l (3), A = sum e (a_k.a_l) d (3). 16 FP32 + 1 SFU per pair.
// Targets are the rows row0 .. row0+n-1 of (x, a) (row0 = 0 and n = m for a whole step; a row range for the
// sharded step), sources all m rows; outputs x1, a1 are indexed by the local target index.
struct OpSOFwd {
  static constexpr int NS = 6, NA = 6;
  static constexpr int kMinCtas = LDDMM_SOFWD_MIN_CTAS;  // 4: <= 128 registers at 128 threads, 16 warps per SM
  static constexpr int kUnroll = 8;  // measured 1.4% faster than 4 (level 6)
  struct Params {
    const double *x, *a;
    double *x1, *a1;
    Frame f;
    double dt;
    int row0 = 0;
  };
  template <typename V> struct Tgt { V y0, y1, y2, a0, a1, a2; };
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    i0 += P.row0;
    i1 += P.row0;
    t.y0 = tgt_coord<V>(P.x, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<V>(P.x, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<V>(P.x, i0, i1, 2, P.f.o2, P.f.s);
    t.a0 = tgt_field<V>(P.a, 3, i0, i1, 0);
    t.a1 = tgt_field<V>(P.a, 3, i0, i1, 1);
    t.a2 = tgt_field<V>(P.a, 3, i0, i1, 2);
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
    const V ec = k.k1 * dot3(t.a0, t.a1, t.a2, s[3], s[4], s[5]);
    acc[3] = fma(ec, d0, acc[3]);
    acc[4] = fma(ec, d1, acc[4]);
    acc[5] = fma(ec, d2, acc[5]);
  }
  // Expanded-distance form (pairs_kernel_x, Gaussian FP32): with c = a_k.a_l, the sum of e c (y - x) is written
  // y S - sum e c x with S = sum e c, and the staged X = -2 x gives sum e c x = -E/2 for E = sum e c X; no
  // difference y - x is formed (14 FP32 + 1 SFU per pair). Blocks too wide for that form (difference form) sum
  // e c (y - x) directly, without the cancellation. Radius^2 bound 32: the cancellation in y S - sum e c x grows
  // with the block radius (FP32 emulation, targets in a ball of radius^2 16: 3.7e-7 relative, against 1.2e-7 for
  // the difference form; 4.6e-7 at 64).
  static constexpr bool kExpand = LDDMM_SOFWD_EXPAND != 0;
  static constexpr int NP = 3, NAX = 7, kRtX = 4;
  static constexpr float kExpandR2 = 32.0f;
  template <typename V> struct TgtX { V a0, a1, a2; };
  template <typename V>
  static __device__ __forceinline__ void load_target_x(const Params& P, int i0, int i1, TgtX<V>& t) {
    i0 += P.row0;
    i1 += P.row0;
    t.a0 = tgt_field<V>(P.a, 3, i0, i1, 0);
    t.a1 = tgt_field<V>(P.a, 3, i0, i1, 1);
    t.a2 = tgt_field<V>(P.a, 3, i0, i1, 2);
  }
  static __device__ __forceinline__ void target_point(const Params& P, int i, double* c) {
    const int g = P.row0 + i;
    c[0] = P.x[3 * g]; c[1] = P.x[3 * g + 1]; c[2] = P.x[3 * g + 2];
  }
  static __device__ __forceinline__ void source_point(const Params& P, int l, double* c, double* f) {
    for (int k = 0; k < 3; ++k) {
      c[k] = P.x[3 * l + k];
      f[k] = P.a[3 * l + k];
    }
  }
  // s: the staged source record (X or x 0-2, |x|^2 3, a 4-6); y: the target pair's relative coordinates.
  // Sums: K a (0-2); expanded: S (3), E (4-6); difference form: sum e c d (4-6).
  template <bool X, typename V>
  static __device__ __forceinline__ void accumulate(const TgtX<V>& t, const V* y, V e, const V* s, V* acc) {
    acc[0] = fma(e, s[4], acc[0]);
    acc[1] = fma(e, s[5], acc[1]);
    acc[2] = fma(e, s[6], acc[2]);
    const V ec = e * dot3(t.a0, t.a1, t.a2, s[4], s[5], s[6]);
    if constexpr (X) {
      acc[3] = acc[3] + ec;
      acc[4] = fma(ec, s[0], acc[4]);
      acc[5] = fma(ec, s[1], acc[5]);
      acc[6] = fma(ec, s[2], acc[6]);
    } else {
      acc[4] = fma(ec, y[0] - s[0], acc[4]);
      acc[5] = fma(ec, y[1] - s[1], acc[5]);
      acc[6] = fma(ec, y[2] - s[2], acc[6]);
    }
  }
  static __device__ __forceinline__ void x_partial(bool expand, const double* y, const double* v, double* o) {
    for (int c = 0; c < 3; ++c) {
      o[c] = v[c];
      o[3 + c] = expand ? y[c] * v[3] + 0.5 * v[4 + c] : v[4 + c];
    }
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double ka = P.dt * P.f.kappa;
    const int g = P.row0 + i;
    for (int c = 0; c < 3; ++c) {
      P.x1[3 * i + c] = P.x[3 * g + c] + P.dt * acc[c];
      P.a1[3 * i + c] = P.a[3 * g + c] + ka * acc[3 + c];
    }
  }
};

// Second-order adjoint step (secondOrderCovector loop body, base/pointEvolution.py:539-546):
//   zpx = DK^T_sym(x; px, a) - DDK11and12(x; a, a, pa),   zpa = K(x) px - DK1and2(x; pa, a)
//   px_prev = px + dt zpx,  pa_prev = pa + dt zpa.
// With c1' = px'_k.a_l + a_k.px'_l (px' = -kappa px), c2'' = a''_k.a_l (a'' = -kappa^2 a), dq = d.(pa_k - pa_l)
// the accumulators are
//   G = sum e (c1' + c2'' dq) d (3), D = sum e c2'' (pa_k - pa_l) (3), E = sum e px'_l (3), F = sum e dq a_l (3)
// and zpx = G + D/(sigma^2 (-kappa^2)), zpa = E/(-kappa) + kappa F. 37 FP32 + 1 SFU per pair (the pa_k - pa_l
// components are shared by dq and D).
// Targets are rows row0 .. row0+n-1 of the state and covectors (row0 = 0 for a whole step), sources all rows;
// outputs px_prev, pa_prev are indexed by the local target index.
struct OpSOBwd {
  static constexpr int NS = 12, NA = 12;
  static constexpr int kMinCtas = LDDMM_SOBWD_MIN_CTAS;
  static constexpr bool kCompInRegisters = true;  // with 4 targets per thread: measured faster than shared memory
  static constexpr int kUnroll = 8;  // measured 1.4% faster than 4 (level 6)
  struct Params {
    const double *x, *a, *px, *pa;
    double *px_prev, *pa_prev;
    Frame f;
    double dt;
    int row0 = 0;
  };
  template <typename V> struct Tgt { V y0, y1, y2, a0, a1, a2, b0, b1, b2, p0, p1, p2, q0, q1, q2; };
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    const double k = P.f.kappa;
    i0 += P.row0;
    i1 += P.row0;
    t.y0 = tgt_coord<V>(P.x, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<V>(P.x, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<V>(P.x, i0, i1, 2, P.f.o2, P.f.s);
    t.a0 = tgt_field<V>(P.a, 3, i0, i1, 0);
    t.a1 = tgt_field<V>(P.a, 3, i0, i1, 1);
    t.a2 = tgt_field<V>(P.a, 3, i0, i1, 2);
    t.b0 = tgt_field<V>(P.a, 3, i0, i1, 0, -k * k);
    t.b1 = tgt_field<V>(P.a, 3, i0, i1, 1, -k * k);
    t.b2 = tgt_field<V>(P.a, 3, i0, i1, 2, -k * k);
    t.p0 = tgt_field<V>(P.px, 3, i0, i1, 0, -k);
    t.p1 = tgt_field<V>(P.px, 3, i0, i1, 1, -k);
    t.p2 = tgt_field<V>(P.px, 3, i0, i1, 2, -k);
    t.q0 = tgt_field<V>(P.pa, 3, i0, i1, 0);
    t.q1 = tgt_field<V>(P.pa, 3, i0, i1, 1);
    t.q2 = tgt_field<V>(P.pa, 3, i0, i1, 2);
  }
  // fields: x' (0-2), a (3-5), pa (6-8), px' = -kappa px (9-11)
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    const double k = P.f.kappa;
    src_point(P.x, l, P.f, f);
    for (int c = 0; c < 3; ++c) {
      f[3 + c] = P.a[3 * l + c];
      f[6 + c] = P.pa[3 * l + c];
      f[9 + c] = -k * P.px[3 * l + c];
    }
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame& f, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<V> k = Fam::template eval<V>(f, sqdist(d0, d1, d2));
    const V w0 = t.q0 - s[6], w1 = t.q1 - s[7], w2 = t.q2 - s[8];
    const V dq = dot3(d0, d1, d2, w0, w1, w2);
    const V c1 = fma(t.a2, s[11], fma(t.a1, s[10], fma(t.a0, s[9], dot3(t.p0, t.p1, t.p2, s[3], s[4], s[5]))));
    const V c2 = dot3(t.b0, t.b1, t.b2, s[3], s[4], s[5]);
    const V ec2 = k.k1 * c2;
    const V eg = fma(k.k2 * c2, dq, k.k1 * c1);  // Gaussian: e (c1 + c2 dq), k2 * c2 == ec2
    acc[0] = fma(eg, d0, acc[0]);
    acc[1] = fma(eg, d1, acc[1]);
    acc[2] = fma(eg, d2, acc[2]);
    acc[3] = fma(ec2, w0, acc[3]);
    acc[4] = fma(ec2, w1, acc[4]);
    acc[5] = fma(ec2, w2, acc[5]);
    acc[6] = fma(k.k0, s[9], acc[6]);
    acc[7] = fma(k.k0, s[10], acc[7]);
    acc[8] = fma(k.k0, s[11], acc[8]);
    const V edq = k.k1 * dq;
    acc[9] = fma(edq, s[3], acc[9]);
    acc[10] = fma(edq, s[4], acc[10]);
    acc[11] = fma(edq, s[5], acc[11]);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double k = P.f.kappa;
    const double cd = -1.0 / (k * k) * P.f.inv_s2;  // converts the c2''-weighted sums back, times 1/sigma^2
    const int g = P.row0 + i;
    for (int c = 0; c < 3; ++c) {
      const double pa = P.pa[3 * g + c];
      const double zpx = acc[c] + cd * acc[3 + c];
      const double zpa = -acc[6 + c] / k + k * acc[9 + c];
      P.px_prev[3 * i + c] = P.px[3 * g + c] + P.dt * zpx;
      P.pa_prev[3 * i + c] = pa + P.dt * zpa;
    }
  }
};

// The second-order forward step evaluated once per unordered pair (pairs_kernel_sym; Gaussian, FP32, whole steps):
// e and c = a_k.a_l are symmetric and d changes sign, so the row sums K a (e a_l) and A (e c d) of k mirror into
// e a_k and -e c d for l. 22 FP32 lane-ops per unordered pair (11 per ordered pair, against 14 for the expanded
// form of OpSOFwd and 16 for its difference form), one ex2.
struct OpSOFwdSym {
  using Params = OpSOFwd::Params;
  static constexpr int NSS = 6, NR = 6, NC = 6;
  static constexpr int kSymMinCtas = LDDMM_SOFWD_SYM_MIN_CTAS;
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
    OpSOFwd::source_fields(P, l, f);
  }
  // Fam: the radial factors k0 (K a) and k1 (the momentum term); both are e for the Gaussian
  template <bool COL, class Fam>
  static __device__ __forceinline__ void pair_sym(const Frame& f, const SymTgt& t, const F2* s, F2* row, F2* col) {
    const F2 d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<F2> k = Fam::template eval<F2>(f, sqdist(d0, d1, d2));
    const F2 ec = k.k1 * dot3(t.a0, t.a1, t.a2, s[3], s[4], s[5]);
    row[0] = fma(k.k0, s[3], row[0]);
    row[1] = fma(k.k0, s[4], row[1]);
    row[2] = fma(k.k0, s[5], row[2]);
    row[3] = fma(ec, d0, row[3]);
    row[4] = fma(ec, d1, row[4]);
    row[5] = fma(ec, d2, row[5]);
    if constexpr (COL) {
      col[0] = fma(k.k0, t.a0, col[0]);
      col[1] = fma(k.k0, t.a1, col[1]);
      col[2] = fma(k.k0, t.a2, col[2]);
      col[3] = fma(ec, d0, col[3]);
      col[4] = fma(ec, d1, col[4]);
      col[5] = fma(ec, d2, col[5]);
    }
  }
  // K a = row + col; sum e c d = row - col (the mirrored difference changes sign)
  static __device__ __forceinline__ void finalize_sym(const Params& P, int i, const double* row, const double* col) {
    const double ka = P.dt * P.f.kappa;
    for (int c = 0; c < 3; ++c) {
      P.x1[3 * i + c] = P.x[3 * i + c] + P.dt * (row[c] + col[c]);
      P.a1[3 * i + c] = P.a[3 * i + c] + ka * (row[3 + c] - col[3 + c]);
    }
  }
};

// The second-order adjoint step evaluated once per unordered pair (pairs_kernel_sym; Gaussian, FP32, whole steps).
// Every per-pair quantity of OpSOBwd is symmetric in (k, l) or changes sign: e, c1 = px'_k.a_l + a_k.px'_l,
// c2 = b_k.a_l (b = -kappa^2 a) and dq = d.(pa_k - pa_l) are symmetric, d and w = pa_k - pa_l change sign. With the
// four sums merged pairwise (as the epilogue of OpSOBwd combines them),
//   row px-sum of k:  v = eg d + cd ec2 w          (eg = e (c1 + c2 dq), ec2 = e c2, cd = -1/(kappa^2 sigma^2))
//   row pa-sum of k:  e px'_l - kappa^2 edq a_l    (edq = e dq)
// the mirrored contributions to l are -v and e px'_k + edq b_k. 51 FP32 lane-ops per unordered pair (25.5 per
// ordered pair, against 37 for OpSOBwd), one ex2.
struct OpSOBwdSym {
  using Params = OpSOBwd::Params;
  static constexpr int NSS = 12, NR = 6, NC = 6;
  static constexpr int kSymMinCtas = LDDMM_SOBWD_SYM_MIN_CTAS;
  struct SymTgt { F2 y0, y1, y2, a0, a1, a2, b0, b1, b2, p0, p1, p2, q0, q1, q2, cd, k2; };
  static __device__ __forceinline__ void load_target_sym(const Params& P, int i0, int i1, bool v0, bool v1,
                                                         SymTgt& t) {
    const double k = P.f.kappa;
    auto fld = [&](const double* a, int c, double sc) {
      return VT<F2>::pack(v0 ? sc * a[3 * i0 + c] : 0.0, v1 ? sc * a[3 * i1 + c] : 0.0);
    };
    t.y0 = tgt_coord<F2>(P.x, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<F2>(P.x, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<F2>(P.x, i0, i1, 2, P.f.o2, P.f.s);
    t.a0 = fld(P.a, 0, 1.0); t.a1 = fld(P.a, 1, 1.0); t.a2 = fld(P.a, 2, 1.0);
    t.b0 = fld(P.a, 0, -k * k); t.b1 = fld(P.a, 1, -k * k); t.b2 = fld(P.a, 2, -k * k);
    t.p0 = fld(P.px, 0, -k); t.p1 = fld(P.px, 1, -k); t.p2 = fld(P.px, 2, -k);
    t.q0 = fld(P.pa, 0, 1.0); t.q1 = fld(P.pa, 1, 1.0); t.q2 = fld(P.pa, 2, 1.0);
    t.cd = VT<F2>::dup(-P.f.inv_s2 / (k * k));
    t.k2 = VT<F2>::dup(-k * k);
  }
  // fields: x' (0-2), a (3-5), pa (6-8), px' = -kappa px (9-11)
  static __device__ __forceinline__ void source_fields_sym(const Params& P, int l, double* f) {
    OpSOBwd::source_fields(P, l, f);
  }
  // Fam: the radial factors k0 (the px'-sum), k1 (first-derivative terms) and k2 (the second-derivative term
  // c2 dq d); all three are e for the Gaussian, where k1 c2 and k2 c2 are one product
  template <bool COL, class Fam>
  static __device__ __forceinline__ void pair_sym(const Frame& f, const SymTgt& t, const F2* s, F2* row, F2* col) {
    const F2 d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<F2> k = Fam::template eval<F2>(f, sqdist(d0, d1, d2));
    const F2 w0 = t.q0 - s[6], w1 = t.q1 - s[7], w2 = t.q2 - s[8];
    const F2 dq = dot3(d0, d1, d2, w0, w1, w2);
    const F2 c1 = fma(t.a2, s[11], fma(t.a1, s[10], fma(t.a0, s[9], dot3(t.p0, t.p1, t.p2, s[3], s[4], s[5]))));
    const F2 c2 = dot3(t.b0, t.b1, t.b2, s[3], s[4], s[5]);
    const F2 ec2 = k.k1 * c2;
    const F2 eg = fma(k.k2 * c2, dq, k.k1 * c1);
    const F2 tw = ec2 * t.cd;
    const F2 v0 = fma(tw, w0, eg * d0), v1 = fma(tw, w1, eg * d1), v2 = fma(tw, w2, eg * d2);
    row[0] += v0;
    row[1] += v1;
    row[2] += v2;
    const F2 edq = k.k1 * dq;
    const F2 edqk = edq * t.k2;
    row[3] = fma(edqk, s[3], fma(k.k0, s[9], row[3]));
    row[4] = fma(edqk, s[4], fma(k.k0, s[10], row[4]));
    row[5] = fma(edqk, s[5], fma(k.k0, s[11], row[5]));
    if constexpr (COL) {
      col[0] += v0;
      col[1] += v1;
      col[2] += v2;
      col[3] = fma(edq, t.b0, fma(k.k0, t.p0, col[3]));
      col[4] = fma(edq, t.b1, fma(k.k0, t.p1, col[4]));
      col[5] = fma(edq, t.b2, fma(k.k0, t.p2, col[5]));
    }
  }
  // zpx = row - col (the mirrored px-sum changes sign), zpa = -(row + col) / kappa
  static __device__ __forceinline__ void finalize_sym(const Params& P, int i, const double* row, const double* col) {
    const double k = P.f.kappa;
    for (int c = 0; c < 3; ++c) {
      const double zpx = row[c] - col[c];
      const double zpa = -(row[3 + c] + col[3 + c]) / k;
      P.px_prev[3 * i + c] = P.px[3 * i + c] + P.dt * zpx;
      P.pa_prev[3 * i + c] = P.pa[3 * i + c] + P.dt * zpa;
    }
  }
};

// First-order adjoint step with the gradient of the same step (base/pointEvolution.py:186-201, :221-223;
// base/surfaceMatching.py:810, :879-891):
//   p_t = p_{t+1} + dt DK^T_lddmm(x_t; p_{t+1}, a_t) = p_{t+1} - dt kappa sum_l e (p_k.a_l + a_k.q_l) d,
//   q_l = p_l - 2 w a_l;  dat_t = K(x_t)(2 w a_t - p_{t+1}) = -sum_l e q_l (euclidean) or 2 w a_t - p_{t+1}.
// Accumulators: A = sum e c d (3), Q = sum e q_l (3). 19 FP32 + 1 SFU per pair.
struct OpFOBwd {
  static constexpr int NS = 9, NA = 6;
  static constexpr int kMinCtas = LDDMM_FOBWD_MIN_CTAS;
  static constexpr bool kCompInRegisters = true;  // measured faster than shared memory for this op
  struct Params {
    const double *x, *a, *p;
    double *p_prev, *dat;
    Frame f;
    double dt, w;
    int euclidean;
  };
  template <typename V> struct Tgt { V y0, y1, y2, p0, p1, p2, a0, a1, a2; };
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    t.y0 = tgt_coord<V>(P.x, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<V>(P.x, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<V>(P.x, i0, i1, 2, P.f.o2, P.f.s);
    t.p0 = tgt_field<V>(P.p, 3, i0, i1, 0);
    t.p1 = tgt_field<V>(P.p, 3, i0, i1, 1);
    t.p2 = tgt_field<V>(P.p, 3, i0, i1, 2);
    t.a0 = tgt_field<V>(P.a, 3, i0, i1, 0);
    t.a1 = tgt_field<V>(P.a, 3, i0, i1, 1);
    t.a2 = tgt_field<V>(P.a, 3, i0, i1, 2);
  }
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    src_point(P.x, l, P.f, f);
    for (int c = 0; c < 3; ++c) {
      f[3 + c] = P.a[3 * l + c];
      f[6 + c] = P.p[3 * l + c] - 2.0 * P.w * P.a[3 * l + c];
    }
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame& f, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<V> k = Fam::template eval<V>(f, sqdist(d0, d1, d2));
    const V c = fma(t.a2, s[8], fma(t.a1, s[7], fma(t.a0, s[6], dot3(t.p0, t.p1, t.p2, s[3], s[4], s[5]))));
    const V ec = k.k1 * c;
    acc[0] = fma(ec, d0, acc[0]);
    acc[1] = fma(ec, d1, acc[1]);
    acc[2] = fma(ec, d2, acc[2]);
    acc[3] = fma(k.k0, s[6], acc[3]);
    acc[4] = fma(k.k0, s[7], acc[4]);
    acc[5] = fma(k.k0, s[8], acc[5]);
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double k = P.dt * P.f.kappa;
    for (int c = 0; c < 3; ++c) {
      const double p = P.p[3 * i + c];
      P.p_prev[3 * i + c] = p - k * acc[c];
      P.dat[3 * i + c] = P.euclidean ? -acc[3 + c] : 2.0 * P.w * P.a[3 * i + c] - p;
    }
  }
};

// The first-order adjoint step evaluated once per unordered pair (pairs_kernel_sym; Gaussian, FP32). The coefficient
// c_kl = p_k.a_l + a_k.q_l = p_k.a_l + a_k.p_l - 2w a_k.a_l (q = p - 2w a) is symmetric in (k, l) and d changes sign,
// so the row sums A_k = sum_l e c d and Q_k = sum_l e q_l of k mirror into -e c d and e q_k for l.
// 25 FP32 lane-ops per unordered pair (12.5 per ordered pair, against 19 for OpFOBwd), one ex2.
struct OpFOBwdSym {
  using Params = OpFOBwd::Params;
  static constexpr int NSS = 9, NR = 6, NC = 6;
  static constexpr int kSymMinCtas = LDDMM_FOBWD_SYM_MIN_CTAS;
  struct SymTgt { F2 y0, y1, y2, p0, p1, p2, a0, a1, a2, q0, q1, q2; };
  static __device__ __forceinline__ void load_target_sym(const Params& P, int i0, int i1, bool v0, bool v1,
                                                         SymTgt& t) {
    auto fld = [&](const double* a, int c) {
      return VT<F2>::pack(v0 ? a[3 * i0 + c] : 0.0, v1 ? a[3 * i1 + c] : 0.0);
    };
    auto qf = [&](int c) {
      return VT<F2>::pack(v0 ? P.p[3 * i0 + c] - 2.0 * P.w * P.a[3 * i0 + c] : 0.0,
                          v1 ? P.p[3 * i1 + c] - 2.0 * P.w * P.a[3 * i1 + c] : 0.0);
    };
    t.y0 = tgt_coord<F2>(P.x, i0, i1, 0, P.f.o0, P.f.s);
    t.y1 = tgt_coord<F2>(P.x, i0, i1, 1, P.f.o1, P.f.s);
    t.y2 = tgt_coord<F2>(P.x, i0, i1, 2, P.f.o2, P.f.s);
    t.p0 = fld(P.p, 0); t.p1 = fld(P.p, 1); t.p2 = fld(P.p, 2);
    t.a0 = fld(P.a, 0); t.a1 = fld(P.a, 1); t.a2 = fld(P.a, 2);
    t.q0 = qf(0); t.q1 = qf(1); t.q2 = qf(2);
  }
  // fields: x' (0-2), a (3-5), q = p - 2 w a (6-8)
  static __device__ __forceinline__ void source_fields_sym(const Params& P, int l, double* f) {
    OpFOBwd::source_fields(P, l, f);
  }
  // Fam: k1 for the adjoint term, k0 for the Q sum (both e for the Gaussian)
  template <bool COL, class Fam>
  static __device__ __forceinline__ void pair_sym(const Frame& f, const SymTgt& t, const F2* s, F2* row, F2* col) {
    const F2 d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const KV<F2> k = Fam::template eval<F2>(f, sqdist(d0, d1, d2));
    const F2 c = fma(t.a2, s[8], fma(t.a1, s[7], fma(t.a0, s[6], dot3(t.p0, t.p1, t.p2, s[3], s[4], s[5]))));
    const F2 ec = k.k1 * c;
    row[0] = fma(ec, d0, row[0]);
    row[1] = fma(ec, d1, row[1]);
    row[2] = fma(ec, d2, row[2]);
    row[3] = fma(k.k0, s[6], row[3]);
    row[4] = fma(k.k0, s[7], row[4]);
    row[5] = fma(k.k0, s[8], row[5]);
    if constexpr (COL) {
      col[0] = fma(ec, d0, col[0]);
      col[1] = fma(ec, d1, col[1]);
      col[2] = fma(ec, d2, col[2]);
      col[3] = fma(k.k0, t.q0, col[3]);
      col[4] = fma(k.k0, t.q1, col[4]);
      col[5] = fma(k.k0, t.q2, col[5]);
    }
  }
  // A = row - col (the mirrored difference changes sign), Q = row + col
  static __device__ __forceinline__ void finalize_sym(const Params& P, int i, const double* row, const double* col) {
    const double acc[6] = {row[0] - col[0], row[1] - col[1], row[2] - col[2],
                           row[3] + col[3], row[4] + col[4], row[5] + col[5]};
    OpFOBwd::finalize(P, i, acc);
  }
};

size_t shooting_ws_bytes(int64_t n, int precision) {
  size_t b = 0;
  auto upd = [&](size_t v) { b = v > b ? v : b; };
  if (precision == kFP32Compensated) {
    if (LDDMM_SYM) {
      upd(sym_ws_bytes<OpSOBwdSym, kTpbHeavy, kRtAdjoint>(n));
      upd(sym_ws_bytes<OpSOFwdSym, kTpbLight, kRtSymFwd>(n));
      if (n <= kSymAdjSmallN) upd(sym_ws_bytes<OpSOBwdSym, kTpbHeavy, kRtSymSmall>(n));
      if (n <= kSymFwdSmallN) upd(sym_ws_bytes<OpSOFwdSym, kTpbLight, kRtSymSmall>(n));
      upd(sym_ws_bytes<OpFOBwdSym, kTpbLight, kRtFoSym>(n));
      upd(sym_ws_bytes<OpSOBwdSym, kTpbHeavy, kRtAdjointSymL, Laplacian>(n));
      upd(sym_ws_bytes<OpSOFwdSym, kTpbLight, kRtSymFwdL, Laplacian>(n));
      upd(sym_ws_bytes<OpFOBwdSym, kTpbLight, kRtFoSymL, Laplacian>(n));
      upd(symx_ws_bytes<OpKSym, kTpbKSym, kRtKSym>(n));
      upd(sym_ws_bytes<OpKSymD, kTpbLight, kRtKSymL, Laplacian>(n));
    }
    upd(pairs_ws_bytes_any<OpSOFwd, F2, kTpbLight, kRtLight>(n, n));
    upd(pairs_ws_bytes<OpSOBwd, F2, kTpbHeavy, kRtAdjoint, Gauss>(n, n));
    upd(pairs_ws_bytes<OpSOBwd, F2, kTpbHeavy, kRtHeavy, Laplacian>(n, n));
    upd(pairs_ws_bytes_any<OpFOBwd, F2, kTpbLight, kRtLight>(n, n));
    upd(pairs_ws_bytes_any<OpK, F2, kTpbLight, kRtLight>(n, n));
  } else {
    upd(pairs_ws_bytes_any<OpSOFwd, double, kTpb64, kRt64>(n, n));
    upd(pairs_ws_bytes_any<OpSOBwd, double, kTpb64, kRt64>(n, n));
    upd(pairs_ws_bytes_any<OpFOBwd, double, kTpb64, kRt64>(n, n));
    upd(pairs_ws_bytes_any<OpK, double, kTpb64, kRt64>(n, n));
  }
  // per-point dot products for the FP64 energy reductions live after the pair partials
  return ((b + 255) & ~(size_t)255) + (size_t)(n > 0 ? n : 0) * sizeof(double);
}

namespace {

// Launch shapes per precision: light (forward / first-order) ops and the second-order adjoint step.
template <typename V> struct Shape;
template <> struct Shape<F2> {
  // the adjoint step: 4 targets per thread for the Gaussian, 2 for the Laplacian (whose radial profile needs the
  // registers: 4 would spill)
  static constexpr int kTpb = kTpbLight, kRt = kRtLight, kTpbH = kTpbHeavy, kRtH = kRtAdjoint, kRtHL = kRtHeavy;
};
template <> struct Shape<double> {
  static constexpr int kTpb = kTpb64, kRt = kRt64, kTpbH = kTpb64, kRtH = kRt64, kRtHL = kRt64;
};

template <typename V>
inline Frame frame(const double* origin, double sigma, int kernel) {
  return make_frame(origin, sigma, kernel, VT<V>::kLanes == 2);
}

inline double* dots_region(void* ws, size_t pair_bytes) {
  size_t off = (pair_bytes + 255) & ~(size_t)255;
  return reinterpret_cast<double*>(reinterpret_cast<char*>(ws) + off);
}

// out = base_sign * base + scale * K(x) a, and (energy != NULL) energy = [acc ? energy : 0] + escale * sum_i dotw_i.(K a)_i
template <typename V>
int k_energy_and_update(const double* x, const double* a, int64_t n, const Frame& f, const double* base,
                        double base_sign, double scale, double* out, const double* dotw, double* energy,
                        double escale, int accumulate, void* ws, size_t wsb, cudaStream_t st) {
  constexpr int TPB = Shape<V>::kTpb, RT = Shape<V>::kRt;
  OpK::Params P;
  P.y = x; P.x = x; P.a = a; P.out = out; P.f = f;
  P.base = base; P.base_sign = base_sign; P.scale = scale;
  // K(x) a is a self-sum: FP32 sums evaluate each unordered pair once (pairs_kernel_symx for the Gaussian,
  // pairs_kernel_sym in the difference form for the Laplacian)
  constexpr bool kSymOk = std::is_same<V, F2>::value && LDDMM_SYM != 0;
  const bool gauss = f.family == kGauss;
  const size_t pb = !kSymOk ? pairs_ws_bytes_any<OpK, V, TPB, RT>(n, n)
                    : gauss ? symx_ws_bytes<OpKSym, kTpbKSym, kRtKSym>(n)
                            : sym_ws_bytes<OpKSymD, kTpbLight, kRtKSymL, Laplacian>(n);
  if (energy) {
    if (((pb + 255) & ~(size_t)255) + (size_t)n * sizeof(double) > wsb) return kWorkspaceTooSmall;
    P.dotw = dotw;
    P.dots = dots_region(ws, pb);
  }
  int rc;
  if constexpr (kSymOk) {
    rc = gauss ? run_pairs_symx<OpKSym, kTpbKSym, kRtKSym>(P, n, ws, wsb, st)
               : run_pairs_sym<OpKSymD, kTpbLight, kRtKSymL, Laplacian>(P, n, ws, wsb, st);
  } else {
    rc = run_pairs_k<OpK, V, TPB, RT>(P, n, n, ws, wsb, st);
  }
  if (rc != kOk) return rc;
  if (energy) {
    ordered_sum_kernel<<<1, 1024, 0, st>>>(P.dots, (int)n, escale, energy, accumulate);
    if (cudaPeekAtLastError() != cudaSuccess) return kLaunchFailure;
  }
  return kOk;
}

template <typename V>
int so_step(const double* x, const double* a, int64_t n, const Frame& f, double dt, double* x1, double* a1, void* ws,
            size_t wsb, cudaStream_t st, int64_t row0 = 0, int64_t nrows = -1) {
  OpSOFwd::Params P{x, a, x1, a1, f, dt, (int)row0};
  const int64_t rows = nrows < 0 ? n : nrows;
  if constexpr (std::is_same<V, F2>::value && LDDMM_SYM != 0) {
    if (row0 == 0 && rows == n) {
      if (f.family == kGauss && n <= kSymFwdSmallN)
        return run_pairs_sym<OpSOFwdSym, kTpbLight, kRtSymSmall>(P, n, ws, wsb, st);
      if (f.family == kGauss) return run_pairs_sym<OpSOFwdSym, kTpbLight, kRtSymFwd>(P, n, ws, wsb, st);
      return run_pairs_sym<OpSOFwdSym, kTpbLight, kRtSymFwdL, Laplacian>(P, n, ws, wsb, st);
    }
  }
  return run_pairs_k<OpSOFwd, V, Shape<V>::kTpb, Shape<V>::kRt>(P, rows, n, ws, wsb, st);
}

template <typename V>
int so_adjoint_step(const double* x, const double* a, const double* px, const double* pa, int64_t n, const Frame& f,
                    double dt, double* px_prev, double* pa_prev, void* ws, size_t wsb, cudaStream_t st,
                    int64_t row0 = 0, int64_t nrows = -1) {
  OpSOBwd::Params P{x, a, px, pa, px_prev, pa_prev, f, dt, (int)row0};
  const int64_t rows = nrows < 0 ? n : nrows;
  if constexpr (std::is_same<V, F2>::value && LDDMM_SYM != 0) {
    if (row0 == 0 && rows == n) {
      if (f.family == kGauss && n <= kSymAdjSmallN)
        return run_pairs_sym<OpSOBwdSym, kTpbHeavy, kRtSymSmall>(P, n, ws, wsb, st);
      if (f.family == kGauss) return run_pairs_sym<OpSOBwdSym, kTpbHeavy, kRtAdjoint>(P, n, ws, wsb, st);
      return run_pairs_sym<OpSOBwdSym, kTpbHeavy, kRtAdjointSymL, Laplacian>(P, n, ws, wsb, st);
    }
  }
  if (f.family == kGauss) return run_pairs<OpSOBwd, V, Shape<V>::kTpbH, Shape<V>::kRtH, Gauss>(P, rows, n, ws, wsb, st);
  return run_pairs<OpSOBwd, V, Shape<V>::kTpbH, Shape<V>::kRtHL, Laplacian>(P, rows, n, ws, wsb, st);
}

template <typename V>
int so_shoot(const double* x0, const double* a0, int64_t n, int64_t T, const Frame& f, double dt, double* xt,
             double* at, void* ws, size_t wsb, cudaStream_t st) {
  const size_t stride = (size_t)n * 3;
  if (cudaMemcpyAsync(xt, x0, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess) return kCudaError;
  if (cudaMemcpyAsync(at, a0, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess) return kCudaError;
  for (int64_t t = 0; t < T; ++t) {
    int rc = so_step<V>(xt + t * stride, at + t * stride, n, f, dt, xt + (t + 1) * stride, at + (t + 1) * stride, ws,
                        wsb, st);
    if (rc != kOk) return rc;
  }
  return kOk;
}

template <typename V>
int so_gradient(const double* xt, const double* at, int64_t n, int64_t T, const Frame& f, double dt,
                const double* px1, const double* pa1, double* pxt, double* pat, double* da0, void* ws, size_t wsb,
                cudaStream_t st) {
  const size_t stride = (size_t)n * 3;
  if (cudaMemcpyAsync(pxt + T * stride, px1, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return kCudaError;
  if (cudaMemcpyAsync(pat + T * stride, pa1, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return kCudaError;
  for (int64_t t = T - 1; t >= 0; --t) {
    int rc = so_adjoint_step<V>(xt + t * stride, at + t * stride, pxt + (t + 1) * stride, pat + (t + 1) * stride, n, f,
                                dt, pxt + t * stride, pat + t * stride, ws, wsb, st);
    if (rc != kOk) return rc;
  }
  if (da0) return k_energy_and_update<V>(xt, at, n, f, pat, -1.0, 1.0, da0, nullptr, nullptr, 0.0, 0, ws, wsb, st);
  return kOk;
}

template <typename V>
int fo_shoot(const double* x0, const double* at, int64_t n, int64_t T, const Frame& f, double regweight, double* xt,
             double* energy, void* ws, size_t wsb, cudaStream_t st) {
  const size_t stride = (size_t)n * 3;
  if (cudaMemcpyAsync(xt, x0, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess) return kCudaError;
  if (T == 0 && energy) {
    if (cudaMemsetAsync(energy, 0, sizeof(double), st) != cudaSuccess) return kCudaError;
  }
  const double dt = T > 0 ? 1.0 / (double)T : 0.0;
  for (int64_t t = 0; t < T; ++t) {
    const double* x = xt + t * stride;
    const double* a = at + t * stride;
    int rc = k_energy_and_update<V>(x, a, n, f, x, 1.0, dt, xt + (t + 1) * stride, a, energy, regweight * dt, t > 0,
                                    ws, wsb, st);
    if (rc != kOk) return rc;
  }
  return kOk;
}

template <typename V>
int fo_gradient(const double* xt, const double* at, int64_t n, int64_t T, const Frame& f, double regweight,
                const double* px1, int euclidean, double* pxt, double* dat, void* ws, size_t wsb, cudaStream_t st) {
  const size_t stride = (size_t)n * 3;
  if (cudaMemcpyAsync(pxt + T * stride, px1, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return kCudaError;
  const double dt = T > 0 ? 1.0 / (double)T : 0.0;
  for (int64_t t = T - 1; t >= 0; --t) {
    OpFOBwd::Params P{xt + t * stride, at + t * stride, pxt + (t + 1) * stride, pxt + t * stride, dat + t * stride,
                      f, dt, regweight, euclidean};
    int rc;
    if constexpr (std::is_same<V, F2>::value && LDDMM_SYM != 0) {
      rc = f.family == kGauss ? run_pairs_sym<OpFOBwdSym, kTpbLight, kRtFoSym>(P, n, ws, wsb, st)
                              : run_pairs_sym<OpFOBwdSym, kTpbLight, kRtFoSymL, Laplacian>(P, n, ws, wsb, st);
    } else {
      rc = run_pairs_k<OpFOBwd, V, Shape<V>::kTpb, Shape<V>::kRt>(P, n, n, ws, wsb, st);
    }
    if (rc != kOk) return rc;
  }
  return kOk;
}

bool bad(const void* p, int64_t n) { return n > 0 && p == nullptr; }

}  // namespace
}  // namespace lddmm

using namespace lddmm;

namespace {

// Runs fn(V{}, frame) with V = F2 (FP32 path) or double (FP64 path).
template <class Fn>
int by_precision(int precision, const double* origin, double sigma, int kernel, Fn&& fn) {
  if (precision == kFP32Compensated) return fn(F2{}, frame<F2>(origin, sigma, kernel));
  if (precision == kFP64) return fn(0.0, frame<double>(origin, sigma, kernel));
  return kInvalidArgument;
}

bool bad_width(double sigma, int kernel) { return bad_sigma(sigma) || bad_kernel(kernel); }

}  // namespace

extern "C" {

int lddmm_second_order_step(const double* x, const double* a, int64_t n, double sigma, int kernel, double dt,
                            const double* origin, double* x_next, double* a_next, int precision, void* ws, size_t wsb,
                            lddmm_stream_t stream) {
  if (n < 0 || bad_width(sigma, kernel) || bad(x, n) || bad(a, n) || bad(x_next, n) || bad(a_next, n))
    return kInvalidArgument;
  return by_precision(precision, origin, sigma, kernel, [&](auto v, const Frame& f) {
    return so_step<decltype(v)>(x, a, n, f, dt, x_next, a_next, ws, wsb, (cudaStream_t)stream);
  });
}

int lddmm_second_order_step_rows(const double* x, const double* a, int64_t n, int64_t row0, int64_t nrows, double sigma,
                                 int kernel, double dt, const double* origin, double* x_next_rows, double* a_next_rows,
                                 int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || row0 < 0 || nrows < 0 || row0 + nrows > n || bad_width(sigma, kernel) || bad(x, n) || bad(a, n) ||
      bad(x_next_rows, nrows) || bad(a_next_rows, nrows))
    return kInvalidArgument;
  if (nrows == 0) return kOk;
  return by_precision(precision, origin, sigma, kernel, [&](auto v, const Frame& f) {
    return so_step<decltype(v)>(x, a, n, f, dt, x_next_rows, a_next_rows, ws, wsb, (cudaStream_t)stream, row0, nrows);
  });
}

int lddmm_second_order_shoot(const double* x0, const double* a0, int64_t n, int64_t T, double sigma, int kernel,
                             double dt, const double* origin, double* xt, double* at, int precision, void* ws,
                             size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || T < 0 || bad_width(sigma, kernel) || bad(x0, n) || bad(a0, n) || bad(xt, n) || bad(at, n))
    return kInvalidArgument;
  if (n == 0) return kOk;
  return by_precision(precision, origin, sigma, kernel, [&](auto v, const Frame& f) {
    return so_shoot<decltype(v)>(x0, a0, n, T, f, dt, xt, at, ws, wsb, (cudaStream_t)stream);
  });
}

int lddmm_second_order_adjoint_step(const double* x, const double* a, const double* px, const double* pa, int64_t n,
                                    double sigma, int kernel, double dt, const double* origin, double* px_prev,
                                    double* pa_prev, int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || bad_width(sigma, kernel) || bad(x, n) || bad(a, n) || bad(px, n) || bad(pa, n) || bad(px_prev, n) ||
      bad(pa_prev, n))
    return kInvalidArgument;
  return by_precision(precision, origin, sigma, kernel, [&](auto v, const Frame& f) {
    return so_adjoint_step<decltype(v)>(x, a, px, pa, n, f, dt, px_prev, pa_prev, ws, wsb, (cudaStream_t)stream);
  });
}

int lddmm_second_order_adjoint_step_rows(const double* x, const double* a, const double* px, const double* pa,
                                         int64_t n, int64_t row0, int64_t nrows, double sigma, int kernel, double dt,
                                         const double* origin, double* px_prev_rows, double* pa_prev_rows,
                                         int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || row0 < 0 || nrows < 0 || row0 + nrows > n || bad_width(sigma, kernel) || bad(x, n) || bad(a, n) ||
      bad(px, n) || bad(pa, n) || bad(px_prev_rows, nrows) || bad(pa_prev_rows, nrows))
    return kInvalidArgument;
  if (nrows == 0) return kOk;
  return by_precision(precision, origin, sigma, kernel, [&](auto v, const Frame& f) {
    return so_adjoint_step<decltype(v)>(x, a, px, pa, n, f, dt, px_prev_rows, pa_prev_rows, ws, wsb,
                                        (cudaStream_t)stream, row0, nrows);
  });
}

int lddmm_second_order_gradient(const double* xt, const double* at, int64_t n, int64_t T, double sigma, int kernel,
                                double dt, const double* px1, const double* pa1, const double* origin, double* pxt,
                                double* pat, double* da0, int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || T < 0 || bad_width(sigma, kernel) || bad(xt, n) || bad(at, n) || bad(px1, n) || bad(pa1, n) ||
      bad(pxt, n) || bad(pat, n))
    return kInvalidArgument;
  if (n == 0) return kOk;
  return by_precision(precision, origin, sigma, kernel, [&](auto v, const Frame& f) {
    return so_gradient<decltype(v)>(xt, at, n, T, f, dt, px1, pa1, pxt, pat, da0, ws, wsb, (cudaStream_t)stream);
  });
}

int lddmm_first_order_shoot(const double* x0, const double* at, int64_t n, int64_t T, double sigma, int kernel,
                            double regweight, const double* origin, double* xt, double* energy, int precision, void* ws,
                            size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || T < 0 || bad_width(sigma, kernel) || bad(x0, n) || bad(at, n) || bad(xt, n)) return kInvalidArgument;
  if (n == 0) return kOk;
  return by_precision(precision, origin, sigma, kernel, [&](auto v, const Frame& f) {
    return fo_shoot<decltype(v)>(x0, at, n, T, f, regweight, xt, energy, ws, wsb, (cudaStream_t)stream);
  });
}

int lddmm_first_order_gradient(const double* xt, const double* at, int64_t n, int64_t T, double sigma, int kernel,
                               double regweight, const double* px1, int euclidean, const double* origin, double* pxt,
                               double* dat, int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || T < 0 || bad_width(sigma, kernel) || bad(xt, n) || bad(at, n) || bad(px1, n) || bad(pxt, n) ||
      bad(dat, n))
    return kInvalidArgument;
  if (n == 0) return kOk;
  return by_precision(precision, origin, sigma, kernel, [&](auto v, const Frame& f) {
    return fo_gradient<decltype(v)>(xt, at, n, T, f, regweight, px1, euclidean, pxt, dat, ws, wsb,
                                    (cudaStream_t)stream);
  });
}

}  // extern "C"
